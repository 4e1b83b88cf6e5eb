"""C-ABI library checks that need no GPU: the library loads, exports every
function include/gg.h declares, rejects bad arguments, and its generators are
deterministic and produce simple connected instances."""
import ctypes
import subprocess

import numpy as np
import pytest

import graphgolf as G
from conftest import has_gpu


def test_library_exports_every_header_symbol():
    L = G.lib()
    names = G.header_functions()
    assert len(names) >= 24
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    assert set(names) <= exported


def test_abi_version_and_status_strings():
    L = G.lib()
    assert L.gg_abi_version() == 1
    for s in range(6):
        assert L.gg_status_str(s)


def test_bad_arguments_rejected_without_device():
    h = ctypes.c_void_p()
    L = G.lib()
    assert L.gg_conv_create(10, 20, 3, 0, ctypes.byref(h)) == G.GG_BAD_ARG   # M > N
    assert L.gg_graph_create(0, 3, 0, ctypes.byref(h)) == G.GG_BAD_ARG
    assert L.gg_beamer_create(2_000_000, 10, 3, 0, ctypes.byref(h)) == G.GG_BAD_ARG
    assert L.gg_piece_create(4, 4, 5, 1, 3, 0, ctypes.byref(h)) == G.GG_BAD_ARG
    assert not h.value


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU path")
def test_no_device_is_reported():
    with pytest.raises(G.GGError) as e:
        G.cudaASPLconv(64, 64, 4, 0)
    assert e.value.status == G.GG_NO_DEVICE


def _is_simple_regular_connected(adj):
    n, d = adj.shape
    for v in range(n):
        row = adj[v]
        if len(set(row.tolist())) != d or v in row:
            return False
    for v in range(n):
        for u in adj[v]:
            if v not in adj[u]:
                return False
    seen = {0}
    st = [0]
    while st:
        v = st.pop()
        for u in adj[v]:
            if int(u) not in seen:
                seen.add(int(u))
                st.append(int(u))
    return len(seen) == n


@pytest.mark.parametrize("n,d,seed", [(256, 4, 1), (1000, 3, 5), (4096, 16, 1), (3000, 4, 2)])
def test_random_regular(n, d, seed):
    a = G.random_regular(n, d, seed)
    assert _is_simple_regular_connected(a)
    assert np.array_equal(a, G.random_regular(n, d, seed))
    assert not np.array_equal(a, G.random_regular(n, d, seed + 1))


def test_random_regular_large_is_simple():
    a = G.random_regular(65536, 8, 1)
    assert a.shape == (65536, 8)
    s = np.sort(a, axis=1)
    assert not np.any(s[:, 1:] == s[:, :-1])
    assert not np.any(a == np.arange(65536)[:, None])


def test_cyclic_lift():
    N, M, diffs = G.cyclic_lift(1024, 32, 12, 1)
    assert (N, M) == (32768, 1024) and diffs.shape == (1024, 12)
    # every edge end has its reverse: u + diff lands in orbit v which holds -diff
    for u in range(M):
        for df in diffs[u]:
            v = (u + int(df)) % N % M
            assert -int(df) in diffs[v].tolist()
    N2, M2, d2 = G.cyclic_lift(1024, 32, 12, 1)
    assert np.array_equal(diffs, d2)


def test_generators_reject_bad_args():
    out = np.zeros(9, np.int32)
    assert G.lib().gg_gen_random_regular(3, 3, 1, out.ctypes.data_as(ctypes.c_void_p)) == G.GG_BAD_ARG
    assert G.lib().gg_gen_random_regular(5, 3, 1, out.ctypes.data_as(ctypes.c_void_p)) == G.GG_BAD_ARG


def test_text_formats_roundtrip():
    import io
    p = G.part.from_diffs(12, 4, [[1, -1, 4], [-1, 1, -4], [2, -2, 3], [-2, 2, -3]])
    s = io.StringIO()
    p.print(s)
    q = G.part().load(io.StringIO(s.getvalue()))
    assert (q.N, q.M, q.edges, q.regular, q.degree) == (p.N, p.M, p.edges, True, 3)
    g = G.graph().load(io.StringIO("0 1\n1 2\n2 0\n2 3\n"))
    assert g.N == 4 and g.degree_max == 3 and not g.is_regular()
    t = g.table()
    assert t.shape == (4, 3) and t[3].tolist() == [2, 3, 3]


def test_bench_input_fixtures_match_the_generator():
    """bench.py's reference arm reads these files instead of loading the engine's
    generator; they must be exactly what the generator gives for the same seeds."""
    import os
    here = os.path.join(os.path.dirname(__file__), "golden")
    for name, (n, d, seed) in (("regular_n65536_d8_seed1.npy", (65536, 8, 1)),
                               ("regular_n4096_d16_seed1.npy", (4096, 16, 1))):
        fx = np.load(os.path.join(here, name))
        assert fx.dtype == np.uint16 and fx.shape == (n, d)
        assert np.array_equal(fx.astype(np.int32), G.random_regular(n, d, seed))
