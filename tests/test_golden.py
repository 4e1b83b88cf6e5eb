"""The oracle reproduces the committed golden fixtures (tests/golden/cases.json,
made by tests/golden/make_golden.py from the reference's own CPU calculators).
CPU only; the GPU parity suite checks the engine against the same fixtures."""
import json
import math
import os

import numpy as np
import pytest

import oracle as O

CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cases.json")))["cases"]


def same(a, b):
    return a == b or (isinstance(a, float) and math.isnan(a) and math.isnan(b))


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_reproduces_reference(case):
    t = np.array(case["table"], dtype=np.int32)
    if case["kind"] == "part":
        N, M = case["N"], case["M"]
        t = t.reshape(M, case["degree"])
        assert O.queue_diameter_aspl(N, M, t) == (case["ref_diameter"], case["ref_aspl"])
        assert O.queue_calc(N, M, t) == case["ref_calc"]
        r = O.bfs_pull(O.expand_part(N, M, t), np.arange(M))
    elif case["kind"] == "piece":
        Nx, Ny, Mx, My = case["dims"]
        d, a = O.piece_diameter_aspl(Nx, Ny, Mx, My, t)
        if case["ref_diameter"] == O.INT_MAX:  # cpu sentinel vs GPU-calculator sentinel
            assert (d, a) == (O.SENTINEL, float(O.SENTINEL))
        else:
            assert (d, a) == (case["ref_diameter"], case["ref_aspl"])
        r = O.bfs_pull(O.expand_piece(Nx, Ny, Mx, My, t), O.piece_reps(Nx, Ny, Mx, My))
    else:
        dims = case["dims"]
        d, a = O.box_diameter_aspl(*dims, t)
        if case["ref_diameter"] == O.INT_MAX:
            assert (d, a) == (O.SENTINEL, float(O.SENTINEL))
        else:
            assert (d, a) == (case["ref_diameter"], case["ref_aspl"])
        r = O.bfs_pull(O.expand_box(*dims, t), O.box_reps(*dims))
    assert r.total() == case["total"] and r.levels == case["levels"]
    assert r.connected == case["connected"]
