"""Batched 2-opt evaluation (gg_batch_*): every candidate's exact total,
reach and diameter equal the oracle's on the edited graph.  Host logic (the
proposal generator, the edit) is checked on CPU; the kernel on the GPU."""
import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O


def exact(adj):
    r = O.bfs_pull(adj, np.arange(len(adj)))
    return r.total(), int(r.reached.sum()), r.levels, r.connected


# ---- CPU: proposals -------------------------------------------------------

def test_gen_swaps_are_valid_2opt_moves():
    adj = G.random_regular(300, 4, 3)
    sw = G.gen_swaps(adj, 0, 500, 9)
    assert len(sw) == 500 and np.all(sw["base"] == 0)
    edges = {(min(u, v), max(u, v)) for v in range(300) for u in adj[v]}
    for s in sw[:200]:
        a, b, c, d = (int(s[k]) for k in "abcd")
        assert len({a, b, c, d}) == 4
        assert (min(a, b), max(a, b)) in edges and (min(c, d), max(c, d)) in edges
        new = G.apply_swap(adj, s)
        assert np.all(np.sort(new, axis=1)[:, 1:] != np.sort(new, axis=1)[:, :-1])  # no repeats
        assert not np.any(new == np.arange(300)[:, None])                            # no loops
        for v in range(300):  # still symmetric
            for u in new[v]:
                assert v in new[u]
    assert np.array_equal(sw, G.gen_swaps(adj, 0, 500, 9))


# ---- GPU -------------------------------------------------------------------

@pytest.mark.gpu
def test_batch_mixed_bases_vs_oracle():
    b = G.Batch(0)
    g1 = G.random_regular(1024, 6, 1)
    g2 = G.random_regular(3000, 4, 1)
    g3 = I.random_regular_np(130, 3 if 130 * 3 % 2 == 0 else 4, 5)  # multigraph, ragged chunk
    ids = [b.add_base(g) for g in (g1, g2, g3)]
    sw = np.concatenate([G.gen_swaps(g1, ids[0], 24, 1), G.gen_swaps(g2, ids[1], 8, 2)])
    none = np.zeros(3, dtype=G.SWAP_DTYPE)
    none["base"] = ids
    none["a"] = -1
    sw = np.concatenate([sw, none])
    res = b.eval(sw)
    graphs = [g1, g2, g3]
    for s, r in zip(sw, res):
        want = exact(G.apply_swap(graphs[s["base"]], s))
        assert (int(r["total"]), int(r["reached"]), int(r["levels"]), bool(r["connected"])) == want
    # the same batch again (the captured graph is replayed) gives the same answers
    assert np.array_equal(b.eval(sw), res)


@pytest.mark.gpu
def test_batch_config_2048_plus_512():
    b = G.Batch(0)
    g1 = G.random_regular(1024, 6, 11)
    g2 = G.random_regular(3000, 4, 12)
    i1, i2 = b.add_base(g1), b.add_base(g2)
    sw = np.concatenate([G.gen_swaps(g1, i1, 2048, 21), G.gen_swaps(g2, i2, 512, 22)])
    res = b.eval(sw)
    assert np.all(res["connected"] == 1)
    # every one of the 2560 candidates against the oracle's BFS of its own graph
    for k, s in enumerate(sw):
        want = exact(G.apply_swap((g1, g2)[s["base"]], s))
        assert (int(res[k]["total"]), int(res[k]["reached"]), int(res[k]["levels"]), True) == want, k


@pytest.mark.gpu
def test_batch_chunk_width_invariance():
    b = G.Batch(0)
    g = G.random_regular(1000, 6, 4)
    i = b.add_base(g)
    sw = G.gen_swaps(g, i, 64, 5)
    base = b.eval(sw)
    for w in (128, 256, 512):
        b.set_chunk(i, w)
        assert np.array_equal(b.eval(sw), base)
    with pytest.raises(G.GGError):  # 2 x 1000 x 128 B of bitsets exceed the shared memory
        b.set_chunk(i, 1024)


@pytest.mark.gpu
def test_batch_rejects_bad_candidates():
    b = G.Batch(0)
    g = G.random_regular(100, 4, 4)
    i = b.add_base(g)
    sw = G.gen_swaps(g, i, 2, 5)
    sw[1]["c"] = 100
    with pytest.raises(G.GGError):
        b.eval(sw)
    sw = G.gen_swaps(g, i, 2, 5)
    sw[0]["base"] = 7
    with pytest.raises(G.GGError):
        b.eval(sw)


@pytest.mark.gpu
def test_affected_source_mode_equals_full_search(monkeypatch):
    """Default mode (each candidate searches only the sources its 2-opt can
    affect) against GG_BATCH_FULL=1 (every source), on bases that use it and on
    bases that fall back: diameter above the planes, a one-way table."""
    rng = np.random.default_rng(5)
    g_reg = G.random_regular(1024, 6, 31)
    g_sm = G.random_regular(3000, 4, 32)
    g_nr, _ = I.random_nonregular(700, 5, 33)
    g_cyc = np.asarray(I.cycle(200), dtype=np.int32)             # diameter 100
    g_dir = rng.integers(0, 300, size=(300, 3)).astype(np.int32)   # one-way entries
    g_dir[:, 0] = (np.arange(300) + 1) % 300
    bases = [g_reg, g_sm, g_nr, g_cyc, g_dir]

    def run():
        b = G.Batch(0)
        ids = [b.add_base(g) for g in bases]
        sw = [G.gen_swaps(g, i, 40, 50 + i) for g, i in zip(bases[:4], ids[:4])]
        none = np.zeros(len(ids), dtype=G.SWAP_DTYPE)
        none["base"] = ids
        none["a"] = -1
        allsw = np.concatenate(sw + [none])
        r1 = b.eval(allsw)
        # a new current graph for one base, then the same candidates again
        b.set_base(ids[0], G.apply_swap(g_reg, sw[0][0]))
        r2 = b.eval(allsw[40:])
        b.close()
        return allsw, r1, r2

    monkeypatch.delenv("GG_BATCH_FULL", raising=False)
    allsw, inc1, inc2 = run()
    monkeypatch.setenv("GG_BATCH_FULL", "1")
    _, full1, full2 = run()
    assert np.array_equal(inc1, full1) and np.array_equal(inc2, full2)
    for k in rng.choice(len(allsw), 15, replace=False):
        s = allsw[k]
        want = exact(G.apply_swap(bases[s["base"]], s))
        got = inc1[k]
        assert (int(got["total"]), int(got["reached"]), bool(got["connected"])) == (want[0], want[1], want[3])


@pytest.mark.gpu
def test_device_candidates_checked_before_use():
    """gg_batch_eval_device gets candidates the host never saw: each malformed one
    (unknown base, vertex outside the base, mode not 0/1, repeated endpoint) makes
    the launch score nothing (levels -1 everywhere) and the status call report
    GG_BAD_ARG with its index; the kernels read no base or row through it.  A good
    launch afterwards scores as the host-array call does."""
    import torch
    b = G.Batch(0)
    g = G.random_regular(200, 4, 3)
    i = b.add_base(g)
    sw = G.gen_swaps(g, i, 16, 5)
    n = len(sw)
    d_out = torch.zeros(n * G.CAND_RESULT_DTYPE.itemsize // 4, dtype=torch.int32, device="cuda")
    breakers = [("c", 5000), ("a", 200), ("base", 3), ("base", -1), ("mode", 2), ("d", None)]
    for field, value in breakers:
        bad = sw.copy()
        bad[7][field] = bad[7]["a"] if value is None else value
        d_sw = torch.from_numpy(bad.view(np.int32).copy()).cuda()
        b.eval_device(n, d_sw.data_ptr(), d_out.data_ptr())
        with pytest.raises(G.GGError) as ex:
            b.device_status()
        assert ex.value.status == G.GG_BAD_ARG and "candidate 7" in str(ex.value)
        res = d_out.cpu().numpy().view(G.CAND_RESULT_DTYPE)
        assert np.all(res["levels"] == -1) and np.all(res["total"] == 0)
    d_sw = torch.from_numpy(sw.view(np.int32).copy()).cuda()
    b.eval_device(n, d_sw.data_ptr(), d_out.data_ptr())
    b.device_status()
    res = d_out.cpu().numpy().view(G.CAND_RESULT_DTYPE)
    assert np.array_equal(res, b.eval(sw))
