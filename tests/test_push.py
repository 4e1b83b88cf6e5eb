"""Push (top-down) levels against pull levels and the oracle.

A push level ORs each frontier chunk into the neighbours' rows; on a symmetric
adjacency it reaches exactly the pairs the pull level (the reference's
formulation) reaches, so every per-level count must be identical with push
off (GG_PUSH_PPM=0), on for the sparse levels (the default) and on for every
level it can take (GG_PUSH_PPM=1000000).  Tables that are not symmetric must
fall back to pull by themselves.  The push buffers must be all zero after every
launch: repeated, interleaved, multi-batch and level-capped evaluations on one
engine check that."""
import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O

pytestmark = pytest.mark.gpu

MODES = {"pull": "0", "sparse-push": None, "all-push": "1000000"}


def engine(monkeypatch, mode, n, d):
    if MODES[mode] is None:
        monkeypatch.delenv("GG_PUSH_PPM", raising=False)
    else:
        monkeypatch.setenv("GG_PUSH_PPM", MODES[mode])
    monkeypatch.setenv("GG_PUSH_MIN_ITEMS", "0")     # push on small bitsets too
    return G.cudaASPLgraph(n, d, 0)


@pytest.mark.parametrize("n,d,seed", [(100, 3, 1), (1000, 4, 2), (4099, 6, 3), (20000, 8, 4),
                                      (3001, 5, 5), (2048, 12, 6), (777, 16, 7)])
def test_level_counts_equal_in_every_mode(monkeypatch, n, d, seed):
    if (n * d) % 2:
        n += 1
    adj = G.random_regular(n, d, seed)
    o = O.bfs_pull(adj, np.arange(n))
    for mode in MODES:
        e = engine(monkeypatch, mode, n, d)
        r = e.eval(adj, max_levels=n + 1, level_counts=True)
        assert (r["total"], r["levels"], r["reached"]) == (o.total(), o.levels, int(o.reached.sum())), mode
        assert np.array_equal(r["level_counts"][:o.levels + 1], o.level_counts[:o.levels + 1]), mode
        e.close()


@pytest.mark.parametrize("mode", list(MODES))
def test_one_way_table_falls_back_to_pull(monkeypatch, mode):
    rng = np.random.default_rng(11)
    n, d = 1500, 3
    adj = rng.integers(0, n, size=(n, d)).astype(np.int32)     # directed: u in adj[v] only
    adj[:, 0] = (np.arange(n) + 1) % n                           # keep it strongly connected
    e = engine(monkeypatch, mode, n, d)
    r = e.eval(adj, max_levels=n + 1, level_counts=True)
    o = O.bfs_pull(adj, np.arange(n))
    assert (r["total"], r["levels"], r["reached"]) == (o.total(), o.levels, int(o.reached.sum()))
    assert np.array_equal(r["level_counts"][:o.levels + 1], o.level_counts[:o.levels + 1])


@pytest.mark.parametrize("mode", list(MODES))
def test_push_buffers_stay_clean_across_launches(monkeypatch, mode):
    n, d = 5000, 6
    a1 = G.random_regular(n, d, 21)
    a2 = G.random_regular(n, d, 22)
    o1 = O.bfs_pull(a1, np.arange(n))
    o2 = O.bfs_pull(a2, np.arange(n))
    e = engine(monkeypatch, mode, n, d)
    e.set_batch_sources(384)                                    # 14 launches per evaluation
    for adj, o in ((a1, o1), (a2, o2), (a1, o1)):
        r = e.eval(adj)
        assert (r["total"], r["levels"]) == (o.total(), o.levels)
    # level caps that stop inside the push levels, then a full evaluation
    for cap in (1, 2, 3):
        r = e.eval(a1, max_levels=cap, level_counts=True)
        assert np.array_equal(r["level_counts"][:cap + 1], o1.level_counts[:cap + 1])
    r = e.eval(a2, src_range=(100, 1900))
    assert r["total"] == O.bfs_pull(a2, np.arange(100, 1900)).total()
    assert e.eval(a1)["total"] == o1.total()


def test_disconnected_and_lifted_forms_with_push(monkeypatch):
    monkeypatch.setenv("GG_PUSH_PPM", "1000000")
    monkeypatch.setenv("GG_PUSH_MIN_ITEMS", "0")
    adj = I.disjoint_union(G.random_regular(600, 4, 1), G.random_regular(400, 4, 2))
    e = G.cudaASPLgraph(1000, 4, 0)
    assert e.calc(adj) == O.graph_calc(1000, adj)
    N, M, diffs = G.cyclic_lift(256, 16, 6, 3)
    cu = G.cudaASPLconv(N, M, 6, 0)
    assert cu.diameterASPL(diffs) == O.conv_diameter_aspl(N, M, diffs)
    assert cu.WVCdiameterASPL(diffs) == O.conv_wvc(N, M, diffs)   # WVC pulls every level
    Nx, Ny, Mx, My, rows = I.random_piece(4, 3, 8, 5, 4, 3)
    assert G.cudaASPLpiece(Nx, Ny, Mx, My, 4, 0).diameterASPL(rows) == \
        O.piece_diameter_aspl(Nx, Ny, Mx, My, rows)


@pytest.mark.parametrize("n,d,seed", [(3000, 8, 1), (20000, 16, 2), (4100, 12, 3)])
def test_half_gathers_in_dense_levels(monkeypatch, n, d, seed):
    """Dense levels that gather half the neighbours first (forced on every dense
    level with GG_SPLIT_PPM=0, never with 1000001) count the same pairs."""
    adj = G.random_regular(n, d, seed)
    o = O.bfs_pull(adj, np.arange(n))
    for ppm in ("0", "1000001"):
        monkeypatch.setenv("GG_SPLIT_PPM", ppm)
        e = G.cudaASPLgraph(n, d, 0)
        r = e.eval(adj, max_levels=n + 1, level_counts=True)
        assert np.array_equal(r["level_counts"][:o.levels + 1], o.level_counts[:o.levels + 1]), ppm
        assert r["total"] == o.total()
        e.close()
