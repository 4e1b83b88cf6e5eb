"""Non-regular graphs (the annealingNR.cpp workload): vertices of different
degree, padded to the maximum degree with self-loops (graph form,
cudaASPLgraph.cu:149-151) or diff 0 (part form, cudaASPLconv.cu:200).  The
padding changes no distance; the proposal generator never picks a padding
slot, so every 2-opt keeps each vertex's degree."""
import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O


def real_degrees(adj):
    adj = np.asarray(adj)
    return (adj != np.arange(len(adj))[:, None]).sum(1)


def test_padding_changes_no_distance():
    adj, lists = I.random_nonregular(200, 5, 1)
    assert len(set(real_degrees(adj).tolist())) > 1
    padded = O.bfs_pull(adj, np.arange(200))
    row_ptr, col = O.lists_to_csr(lists)
    plain = O.bfs(row_ptr, col, np.arange(200))
    assert padded.total() == plain.total() and padded.levels == plain.levels


def test_swaps_on_padded_graph_keep_degrees():
    adj, _ = I.random_nonregular(300, 6, 2)
    deg = real_degrees(adj)
    sw = G.gen_swaps(adj, 0, 300, 4)
    for s in sw:
        new = G.apply_swap(adj, s)
        assert np.array_equal(real_degrees(new), deg)
        for v in range(300):
            for u in new[v]:
                assert v in new[u]


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(4))
def test_nonregular_graph_calc(seed):
    n = [257, 1000, 2500, 4100][seed]
    adj, _ = I.random_nonregular(n, 3 + seed, seed)
    assert G.cudaASPLgraph(n, adj.shape[1], 0).calc(adj) == O.graph_calc(n, adj)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(4))
def test_ragged_part_conv(seed):
    N, M, table, rows = I.ragged_part(60 + 10 * seed, 4 + seed, 4, 5 + seed, seed)
    cu = G.cudaASPLconv(N, M, 4, 0)
    assert cu.diameterASPL(table) == O.conv_diameter_aspl(N, M, table)
    assert cu.WVCdiameterASPL(table) == O.conv_wvc(N, M, table)
    # the part object with ragged rows pads the same way
    p = G.part(N=N, M=M, regular=False, degree=4, edges=rows)
    assert cu.diameterASPL(p) == O.conv_diameter_aspl(N, M, table)


@pytest.mark.gpu
def test_batch_on_nonregular_base():
    adj, _ = I.random_nonregular(1500, 6, 9)
    b = G.Batch(0)
    base = b.add_base(adj)
    sw = G.gen_swaps(adj, base, 40, 3)
    res = b.eval(sw)
    for s, r in zip(sw, res):
        o = O.bfs_pull(G.apply_swap(adj, s), np.arange(1500))
        assert (int(r["total"]), int(r["reached"]), int(r["levels"])) == (o.total(), int(o.reached.sum()), o.levels)
