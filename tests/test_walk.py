"""Walk pass of the single-graph engine: levels 1..K of every source batch
computed from the walk ends of each row (bfs_batch_kernel's walk_rows) must give
exactly the counts of the level-by-level BFS, on every kind of table: random
regular graphs, self-loop padding, multigraph repeats, one-way rows, the lifted
forms (consecutive representatives and the corner tiles found through the inverse
list), batches that end inside the walk, and level caps below K.

GG_WALK_LEVELS is read when an engine plans its batches (at creation and at
set_batch_sources): 0 turns the pass off, K > 0 forces K levels.  GG_VPULL (read at
creation) chooses how the levels after the walk run: 1 (default) pulls visited sets
from two alternating copies, 0 pulls frontiers."""
import os

import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O

pytestmark = pytest.mark.gpu


def engine_with(walk, make):
    old = os.environ.get("GG_WALK_LEVELS")
    os.environ["GG_WALK_LEVELS"] = str(walk)
    try:
        return make()
    finally:
        if old is None:
            del os.environ["GG_WALK_LEVELS"]
        else:
            os.environ["GG_WALK_LEVELS"] = old


def counts(e, table, cap):
    r = e.eval(table, max_levels=cap, level_counts=True)
    return (r["total"], r["reached"], r["levels"], r["capped"], r["connected"],
            tuple(int(x) for x in r["level_counts"]))


@pytest.mark.parametrize("n,d,seed,bits", [(256, 4, 1, 0), (1000, 3, 2, 256), (2000, 6, 3, 1024),
                                           (4096, 8, 4, 4096), (3000, 8, 5, 1152), (1500, 16, 6, 512),
                                           (777, 5, 7, 384), (2048, 12, 8, 2048)])
@pytest.mark.parametrize("walk", [1, 2, 3, 4])
def test_walk_equals_level_bfs_regular(n, d, seed, bits, walk):
    if (n * d) % 2:
        n += 1
    adj = G.random_regular(n, d, seed) if d in (3, 4, 6, 8, 12, 16) else I.random_regular_np(n, d, seed)
    cap = n + 1
    off = engine_with(0, lambda: G.cudaASPLgraph(n, d, 0))
    on = engine_with(walk, lambda: G.cudaASPLgraph(n, d, 0))
    if bits:
        engine_with(0, lambda: off.set_batch_sources(bits))
        engine_with(walk, lambda: on.set_batch_sources(bits))
    want = counts(off, adj, cap)
    assert counts(on, adj, cap) == want
    o = O.bfs_pull(adj, np.arange(n))
    assert want[0] == o.total() and want[2] == o.levels


def test_walk_default_headline_shape_vs_oracle():
    """Default plan (walk on) for an 8-regular graph with 4096-source batches."""
    adj = G.random_regular(8192, 8, 11)
    e = G.cudaASPLgraph(8192, 8, 0)
    e.set_batch_sources(4096)
    r = e.eval(adj, max_levels=199, level_counts=True)
    o = O.bfs_pull(adj, np.arange(8192))
    assert r["total"] == o.total() and r["levels"] == o.levels and r["connected"]
    assert np.array_equal(r["level_counts"][:o.levels + 1], o.level_counts[:o.levels + 1])


@pytest.mark.parametrize("walk", [2, 3, 4])
def test_walk_padding_repeats_one_way(walk):
    # self-loop padding of a non-regular graph, repeated neighbours, one-way rows
    rng = np.random.default_rng(5)
    n, d = 900, 6
    adj = np.repeat(np.arange(n, dtype=np.int32)[:, None], d, axis=1)
    for v in range(n):
        k = int(rng.integers(0, d + 1))
        adj[v, :k] = rng.integers(0, n, size=k)
    for cap in (n + 1, 2, 1):
        want = counts(engine_with(0, lambda: G.cudaASPLgraph(n, d, 0)), adj, cap)
        got = counts(engine_with(walk, lambda: G.cudaASPLgraph(n, d, 0)), adj, cap)
        assert got == want, cap


@pytest.mark.parametrize("walk", [1, 3, 4])
def test_walk_batches_ending_inside_the_walk(walk):
    for adj in (np.asarray(I.complete(9), np.int32), np.zeros((1, 2), np.int32),
                np.asarray(I.cycle(5), np.int32), np.asarray(I.petersen(), np.int32),
                np.asarray(I.disjoint_union(I.cycle(10), I.cycle(12)), np.int32)):
        n, d = adj.shape
        want = counts(engine_with(0, lambda: G.cudaASPLgraph(n, d, 0)), adj, n + 1)
        assert counts(engine_with(walk, lambda: G.cudaASPLgraph(n, d, 0)), adj, n + 1) == want


@pytest.mark.parametrize("walk", [2, 3])
def test_walk_lifted_forms(walk):
    N, M, diffs = G.cyclic_lift(256, 16, 6, 3)
    want = engine_with(0, lambda: G.cudaASPLconv(N, M, 6, 0)).diameterASPL(diffs)
    assert engine_with(walk, lambda: G.cudaASPLconv(N, M, 6, 0)).diameterASPL(diffs) == want
    assert want == O.conv_diameter_aspl(N, M, diffs)
    Nx, Ny, Mx, My, vals = G.piece_lift(8, 8, 4, 4, 4, 2)
    want = engine_with(0, lambda: G.cudaASPLpiece(Nx, Ny, Mx, My, 4, 0)).diameterASPL(vals)
    assert engine_with(walk, lambda: G.cudaASPLpiece(Nx, Ny, Mx, My, 4, 0)).diameterASPL(vals) == want
    assert want == O.piece_diameter_aspl(Nx, Ny, Mx, My, vals)
    dims_rows = I.random_box(3, 2, 2, 2, 3, 2, 6, 4)
    dims, rows = dims_rows[:6], dims_rows[6]
    want = engine_with(0, lambda: G.cudaASPLbox(*dims, 6, 0)).diameterASPL(rows)
    assert engine_with(walk, lambda: G.cudaASPLbox(*dims, 6, 0)).diameterASPL(rows) == want


def circulant(n, steps):
    v = np.arange(n, dtype=np.int64)[:, None]
    s = np.asarray([x for k in steps for x in (k, -k)], np.int64)[None, :]
    return ((v + s) % n).astype(np.int32)


@pytest.mark.parametrize("n,steps,bits,walk", [(6000, (1, 7), 1024, 3), (5000, (1, 13, 97, 541), 2048, 2),
                                               (4100, (1, 3, 9), 512, 4), (9000, (1, 2), 4096, 1)])
def test_visited_pull_matches_frontier_pull(n, steps, bits, walk):
    """Long-diameter circulants: after the walk come sparse (flag-driven), dense,
    split and skip-full levels; the visited-set pull must count exactly what the
    frontier pull and the oracle count."""
    adj = circulant(n, steps)
    d = adj.shape[1]
    got = {}
    for mode in ("frontier", "visited", "visited_own"):
        env = {"GG_VPULL": "0" if mode == "frontier" else "1", "GG_OWN_SKIP": "0" if mode == "visited_own" else "1"}
        got[mode] = counts_with_env(env, walk, n, d, bits, adj)
    assert got["visited"] == got["frontier"] and got["visited_own"] == got["frontier"]
    o = O.bfs_pull(adj, np.arange(n))
    assert got["visited"][0] == o.total() and got["visited"][2] == o.levels
    assert np.array_equal(np.asarray(got["visited"][5][:o.levels + 1]), o.level_counts[:o.levels + 1])


def counts_with_env(env, walk, n, d, bits, adj):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        e = engine_with(walk, lambda: G.cudaASPLgraph(n, d, 0))
        engine_with(walk, lambda: e.set_batch_sources(bits))
        return counts(e, adj, n + 1)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("one_way", [False, True])
def test_dense_levels_without_own_chunks(one_way):
    """Dense visited-set pull levels skip their own chunks only on tables whose
    entries all list their row back (the walk index kernel's one-way flag); one
    one-way entry must bring the own reads back, with the same exact counts."""
    n, d = 12288, 8
    adj = G.random_regular(n, d, 21).copy()
    if one_way:
        v = 777
        u = int(adj[v, 0])
        w = next(x for x in range(n) if x != v and x not in adj[v] and v not in adj[x] and x != u)
        adj[v, 0] = w          # v now pulls from w; w's row does not list v
    want = counts_with_env({"GG_VPULL": "0"}, 3, n, d, 4096, adj)
    got = counts_with_env({"GG_VPULL": "1", "GG_OWN_SKIP": "1"}, 3, n, d, 4096, adj)
    assert got == want
    o = O.bfs_pull(adj, np.arange(n))
    assert got[0] == o.total() and got[2] == o.levels


@pytest.mark.parametrize("n,d,seed,walk", [(12288, 8, 31, 3), (9000, 4, 32, 3), (8200, 4, 33, 2), (8192, 8, 34, 1)])
def test_walk_all_batches_at_once(n, d, seed, walk):
    """walk_all_kernel (every batch's level-K rows built in one launch) against the
    per-batch walk pass (GG_WALK_ALL_MB=0) and the oracle, with 4096-source batches
    (the last one partial when n is not a multiple of 4096)."""
    adj = G.random_regular(n, d, seed)
    got = counts_with_env({"GG_VPULL": "1"}, walk, n, d, 4096, adj)
    per_batch = counts_with_env({"GG_VPULL": "1", "GG_WALK_ALL_MB": "0"}, walk, n, d, 4096, adj)
    assert got == per_batch
    o = O.bfs_pull(adj, np.arange(n))
    assert got[0] == o.total() and got[2] == o.levels
    assert np.array_equal(np.asarray(got[5][:o.levels + 1]), o.level_counts[:o.levels + 1])


@pytest.mark.parametrize("n,d,seed,walk,env,one_way", [
    (12288, 8, 51, 3, {}, False),
    (9000, 4, 52, 3, {}, False),
    (8192, 8, 53, 1, {}, False),
    (12288, 8, 54, 3, {}, True),
    # skip-full from the first levels on: level K+2 cannot be written whole, so
    # the batch keeps alternating with its walk slice
    (12288, 8, 55, 3, {"GG_FULL_SKIP_PPM": "1000"}, False),
    (12288, 8, 56, 2, {"GG_FULL_SKIP_PPM": "1000", "GG_SPLIT_PPM": "1000"}, False),
])
def test_walk_all_third_buffer(n, d, seed, walk, env, one_way):
    """After the walk of all batches, levels K+2.. alternate between V and a third
    buffer (level K+2 written whole) instead of the batch's walk slice; with and
    without it (GG_WALK_THIRD) the counts must equal the per-batch walk pass and
    the oracle, on one-way tables and when level K+2 is a skip-full level too."""
    adj = G.random_regular(n, d, seed).copy()
    if one_way:
        v = 901
        w = next(x for x in range(n) if x != v and x not in adj[v] and v not in adj[x] and x != int(adj[v, 0]))
        adj[v, 0] = w
    base = {"GG_VPULL": "1", **env}
    on = counts_with_env({**base, "GG_WALK_THIRD": "1"}, walk, n, d, 4096, adj)
    off = counts_with_env({**base, "GG_WALK_THIRD": "0"}, walk, n, d, 4096, adj)
    per_batch = counts_with_env({**base, "GG_WALK_ALL_MB": "0"}, walk, n, d, 4096, adj)
    assert on == off == per_batch
    o = O.bfs_pull(adj, np.arange(n))
    assert on[0] == o.total() and on[2] == o.levels
    assert np.array_equal(np.asarray(on[5][:o.levels + 1]), o.level_counts[:o.levels + 1])


@pytest.mark.parametrize("lo,hi", [(0, 8192), (4096, 12288), (1000, 9600), (300, 4500)])
def test_walk_all_source_ranges(lo, hi):
    """Source sub-ranges (not every vertex a source): walk_all_kernel counts levels
    1..K from the full vertex set of each source's walk ends; the counts must match
    the per-batch walk pass and the oracle restricted to the same sources."""
    n, d = 12288, 8
    adj = G.random_regular(n, d, 41)

    def run(env):
        old = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            e = engine_with(3, lambda: G.cudaASPLgraph(n, d, 0))
            engine_with(3, lambda: e.set_batch_sources(4096))
            r = e.eval(adj, max_levels=n + 1, src_range=(lo, hi), level_counts=True)
            return r["total"], r["levels"], tuple(int(x) for x in r["level_counts"])
        finally:
            for k, v in old.items():
                if v is None:
                    del os.environ[k]
                else:
                    os.environ[k] = v

    got = run({"GG_VPULL": "1"})
    assert got == run({"GG_VPULL": "1", "GG_WALK_ALL_MB": "0"})
    o = O.bfs_pull(adj, np.arange(lo, hi))
    assert got[0] == o.total() and got[1] == o.levels


@pytest.mark.parametrize("Mx,My,walk", [(64, 64, 3), (128, 64, -1)])
def test_walk_all_lifted_corner_tiles(Mx, My, walk):
    """walk_all_kernel on a piece lift (sources = the corner tile's vertices, found
    through the inverse list) with 4096-source batches: 4096 representatives with the
    walk forced, and 8192 with the default plan (two batches)."""
    Nx, Ny, Mx, My, vals = G.piece_lift(Mx, My, 2, 2, 8, 5)

    def run(env):
        old = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            return G.cudaASPLpiece(Nx, Ny, Mx, My, 8, 0).diameterASPL(vals)
        finally:
            for k, v in old.items():
                if v is None:
                    del os.environ[k]
                else:
                    os.environ[k] = v

    env = {} if walk < 0 else {"GG_WALK_LEVELS": str(walk)}
    got = run(env)
    assert got == run({**env, "GG_WALK_ALL_MB": "0"})
    assert got == run({"GG_WALK_LEVELS": "0"})
    assert got == O.piece_diameter_aspl(Nx, Ny, Mx, My, vals)
