"""Autotuners and their cache file (gg_autotune, gg_batch_autotune,
gg_lift_autotune, gg_set_tune_cache).

Each tuner times the launch shapes it knows on the caller's input, keeps the
fastest and records it in the cache under (GPU, evaluator, shape).  A second
process reading the same file must plan the tuned shape without tuning, and every
shape must give the same exact results."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import graphgolf as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def second_process(code, cache):
    env = dict(os.environ, GG_TUNE_CACHE=cache)
    prog = ("import sys, json; sys.path[:0] = [%r, %r]\nimport numpy as np\nimport graphgolf as G\n" %
            (ROOT, os.path.join(ROOT, "graphgolf-cuda_b200"))) + code
    p = subprocess.run([sys.executable, "-c", prog], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_engine_tuning_persists_across_processes(tmp_path):
    cache = str(tmp_path / "tune.tsv")
    G.set_tune_cache(cache)
    try:
        adj = G.random_regular(3000, 4, 3)
        e = G.cudaASPLgraph(3000, 4, 0)
        want = e.eval(adj)
        width, ms = e.autotune(adj, trials=1)
        plan = e.plan()
        assert plan[0] == width and ms > 0
        got = e.eval(adj)
        assert (got["total"], got["levels"], got["reached"]) == (want["total"], want["levels"], want["reached"])
        text = open(cache).read()
        assert "|graph|" in text and "\t%d " % width in text
        # a new engine of the same shape in this process plans the tuned shape
        assert G.cudaASPLgraph(3000, 4, 0).plan() == plan
        # ... and so does one in another process, with the same exact counts
        other = second_process(
            "adj = G.random_regular(3000, 4, 3)\ne = G.cudaASPLgraph(3000, 4, 0)\nr = e.eval(adj)\n"
            "print(json.dumps({'plan': e.plan(), 'total': r['total'], 'levels': r['levels']}))", cache)
        assert tuple(other["plan"]) == plan
        assert (other["total"], other["levels"]) == (want["total"], want["levels"])
    finally:
        G.set_tune_cache(os.environ.get("GG_TUNE_CACHE"))


def test_batch_and_lift_tuning_persist(tmp_path):
    cache = str(tmp_path / "tune.tsv")
    G.set_tune_cache(cache)
    try:
        b = G.Batch(0)
        g = G.random_regular(1024, 6, 4)
        i = b.add_base(g)
        sw = G.gen_swaps(g, i, 256, 5)
        want = b.eval(sw)
        ms = b.autotune(sw, trials=1)
        assert ms > 0 and np.array_equal(b.eval(sw), want)
        chunk = b.chunk(i)
        N, M, D = G.cyclic_lift(256, 16, 6, 2)
        L = G.Lift(N, M, 6, 0)
        L.set_base(D)
        moves = G.gen_lift_moves(N, M, D, 24, 9)
        lw = L.eval(moves)
        grp, lms = L.autotune(moves, trials=1)
        assert L.group() == grp and np.array_equal(L.eval(moves), lw)
        other = second_process(
            "b = G.Batch(0)\ng = G.random_regular(1024, 6, 4)\ni = b.add_base(g)\n"
            "N, M, D = G.cyclic_lift(256, 16, 6, 2)\nL = G.Lift(N, M, 6, 0)\n"
            "print(json.dumps({'chunk': b.chunk(i), 'group': L.group()}))", cache)
        assert other == {"chunk": chunk, "group": grp}
    finally:
        G.set_tune_cache(os.environ.get("GG_TUNE_CACHE"))
