"""Incremental evaluation of 2-opt moves (gg_inc_*).
CPU: the affected-source rule, restated in numpy on full distance rows, leaves
every other source's distances unchanged (checked by brute force on the moved
graph).  GPU: every incremental result equals the oracle's full evaluation of
the moved graph -- regular and padded non-regular graphs, moves that disconnect,
graphs whose diameter exceeds the distance planes (full-evaluation fallback),
and after commits."""

import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O


def dist_rows(adj):
    """All-pairs distance matrix of a pull adjacency (-1: unreached), by BFS."""
    n = len(adj)
    nb = [sorted(set(int(u) for u in row if u != v)) for v, row in enumerate(adj)]
    D = np.full((n, n), -1, dtype=np.int64)
    for s in range(n):
        D[s, s] = 0
        frontier = [s]
        while frontier:
            nxt = []
            for v in frontier:
                for u in nb[v]:
                    if D[s, u] < 0:
                        D[s, u] = D[s, v] + 1
                        nxt.append(u)
            frontier = nxt
    return D


def affected(adj, D, s):
    """The rule of gg_inc.cu, for every source at once (D[s, v] = distance)."""
    a, b, c, d, mode = (int(s[k]) for k in ("a", "b", "c", "d", "mode"))
    p, q = (d, c) if mode else (c, d)
    aff = np.zeros(len(adj), dtype=bool)
    for x, y in ((a, b), (c, d)):
        dx, dy = D[:, x], D[:, y]
        lo_is_x = dx < dy
        for lo, hi, sel in ((x, y, lo_is_x), (y, x, dy < dx)):
            l = np.minimum(dx, dy)
            row = list(adj[hi])
            row.remove(lo)                       # the first occurrence goes
            other = np.zeros(len(adj), dtype=bool)
            for z in row:
                other |= D[:, z] == l
            aff |= sel & ~other
    aff |= (np.abs(D[:, a] - D[:, p]) >= 2) | (np.abs(D[:, b] - D[:, q]) >= 2)
    return aff


@pytest.mark.parametrize("n,d,seed", [(120, 3, 1), (300, 4, 2), (200, 6, 3)])
def test_affected_rule_keeps_other_rows(n, d, seed):
    adj = G.random_regular(n, d, seed)
    D = dist_rows(adj)
    for s in G.gen_swaps(adj, 0, 40, seed + 7):
        new = dist_rows(G.apply_swap(adj, s))
        aff = affected(adj, D, s)
        assert np.array_equal(new[~aff], D[~aff])
        assert aff.mean() < 1.0


# ---- GPU ---------------------------------------------------------------------

def check(inc, adj, s):
    got, naff = inc.eval(s)
    o = O.bfs_pull(G.apply_swap(adj, s), np.arange(len(adj)))
    assert (got["total"], got["reached"], bool(got["connected"])) == (o.total(), int(o.reached.sum()), o.connected)
    if o.connected:
        assert got["levels"] == o.levels
    return naff


@pytest.mark.gpu
@pytest.mark.parametrize("n,d,seed", [(1000, 6, 1), (3000, 8, 2), (2048, 4, 3)])
def test_incremental_equals_full_evaluation(n, d, seed):
    adj = G.random_regular(n, d, seed)
    inc = G.Incremental(n, d, 0)
    r = inc.set_graph(adj)
    o = O.bfs_pull(adj, np.arange(n))
    assert r["total"] == o.total()
    counts = [check(inc, adj, s) for s in G.gen_swaps(adj, 0, 30, seed)]
    # fewer sources are searched again; degree 4 leaves fewer alternative parents
    assert np.mean(counts) < (0.6 if d >= 6 else 0.9) * n
    # commit moves and keep going on the new current graph
    for k in range(3):
        s = G.gen_swaps(adj, 0, 1, seed + 100 + k)[0]
        r = inc.commit(s)
        adj = G.apply_swap(adj, s)
        assert r["total"] == O.bfs_pull(adj, np.arange(n)).total()
        for s2 in G.gen_swaps(adj, 0, 5, seed + 200):
            check(inc, adj, s2)
    inc.close()


@pytest.mark.gpu
def test_incremental_nonregular_and_disconnecting_move():
    adj, _ = I.random_nonregular(900, 5, 4)
    inc = G.Incremental(900, 5, 0)
    inc.set_graph(adj)
    for s in G.gen_swaps(adj, 0, 20, 9):
        check(inc, adj, s)
    # two 5-cliques joined by the edges 0-5 and 1-6: swapping those two edges
    # into 0-1 and 5-6 (both repeats) disconnects the graph
    lists = [[u for u in range(5) if u != v] for v in range(5)] + \
            [[u for u in range(5, 10) if u != v] for v in range(5, 10)]
    lists[0].append(5); lists[5].append(0); lists[1].append(6); lists[6].append(1)
    bar = O.pad_graph(10, lists, 5)
    inc2 = G.Incremental(10, 5, 0)
    inc2.set_graph(bar)
    sw = np.array([(0, 0, 5, 1, 6, 0)], dtype=G.SWAP_DTYPE)[0]
    got, _ = inc2.eval(sw)
    assert not got["connected"]
    check(inc2, bar, sw)


@pytest.mark.gpu
def test_incremental_falls_back_beyond_the_planes():
    adj = I.cycle(100)                          # diameter 50 > 15
    inc = G.Incremental(100, 2, 0)
    inc.set_graph(adj)
    for s in G.gen_swaps(adj, 0, 10, 1):
        assert check(inc, adj, s) == 100        # every source searched again


@pytest.mark.gpu
def test_incremental_one_way_table_searches_every_source():
    # a one-way entry elsewhere in the table: the distance matrix is no longer
    # symmetric, so the per-source sums cannot come from the planes' rows
    adj = G.random_regular(600, 6, 5)
    adj[10][0] = next(u for u in range(600) if u != 10 and 10 not in adj[u] and u not in adj[10])
    inc = G.Incremental(600, 6, 0)
    r = inc.set_graph(adj)
    assert r["total"] == O.bfs_pull(adj, np.arange(600)).total()
    moves = [s for s in G.gen_swaps(adj, 0, 40, 2) if 10 not in (s["a"], s["b"], s["c"], s["d"])][:8]
    for s in moves:
        assert check(inc, adj, s) == 600
    inc.close()


@pytest.mark.gpu
def test_incremental_rejects_moves_on_missing_edges():
    adj = G.random_regular(200, 4, 1)
    inc = G.Incremental(200, 4, 0)
    inc.set_graph(adj)
    non = next(u for u in range(200) if u not in adj[0] and u != 0)
    bad = np.array([(0, 0, non, int(adj[5][0]), 5, 0)], dtype=G.SWAP_DTYPE)[0]
    with pytest.raises(G.GGError) as err:
        inc.eval(bad)
    assert err.value.status == G.GG_BAD_ARG
