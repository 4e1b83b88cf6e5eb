"""gg_graph_eval_noalloc: the evaluation entry point for callers that cannot
allocate device memory (a host whose GPU memory is owned by another framework's
pool, or a search loop that cannot pay for the device-wide synchronisation of
cudaFree).  It works in a fixed device array compiled into the library instead.

The test calls it through the C ABI with device buffers the test owns and checks
its level counts, bit for bit, against the existing engine entry point
(gg_eval on a gg_graph_create engine) on two calls in a row -- two different
graphs, then the first again -- so a result can depend neither on a fresh array
nor on what the previous call left in it.  This file is named to be collected
last; it also passes when run alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import graphgolf as G

pytestmark = pytest.mark.gpu

MAX_LEVELS = 199


def noalloc_counts(adj):
    import torch
    adj = np.ascontiguousarray(adj, dtype=np.int32)
    n, d = adj.shape
    d_adj = torch.from_numpy(adj).cuda()
    # garbage in the output buffer: the call must overwrite every entry
    out = torch.full((MAX_LEVELS + 1,), 12345, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = G.lib().gg_graph_eval_noalloc(ctypes.c_void_p(d_adj.data_ptr()), n, d, MAX_LEVELS,
                                       ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy().view(np.uint64)


def engine_counts(adj):
    n, d = adj.shape
    e = G.cudaASPLgraph(n, d, 0)
    r = e.eval(adj, max_levels=MAX_LEVELS, level_counts=True)
    e.close()
    return r["level_counts"], r


def test_noalloc_matches_engine_on_consecutive_calls():
    g1 = G.random_regular(4096, 16, 11)
    g2 = G.random_regular(1000, 3, 12)
    for adj in (g1, g2, g1):
        rc, got = noalloc_counts(adj)
        assert rc == G.GG_OK, G.lib().gg_last_error()
        want, r = engine_counts(adj)
        assert np.array_equal(got, want)
        levels = np.nonzero(got)[0]
        total = int(sum(int(L) * int(got[L]) for L in levels))
        assert total == r["total"] and int(levels.max()) == r["levels"]


@pytest.mark.parametrize("n,d,seed", [(4096, 8, 21), (2001, 5, 22), (1500, 7, 23)])
def test_noalloc_generic_degrees_and_largest_size(n, d, seed):
    """Degrees without a specialised kernel (5, 7: the run-time-degree kernel) and
    the largest size the documentation promises always fits (N = 4096)."""
    import instances as I
    if (n * d) % 2:
        n += 1
    adj = G.random_regular(n, d, seed) if d in (3, 4, 6, 8, 12, 16) else I.random_regular_np(n, d, seed)
    for _ in range(2):
        rc, got = noalloc_counts(adj)
        assert rc == G.GG_OK, G.lib().gg_last_error()
        want, _ = engine_counts(adj)
        assert np.array_equal(got, want)


def test_noalloc_rejects_an_entry_outside_the_graph():
    """An adjacency entry outside [0, N) is caught by the range check before any
    gather and returns GG_BAD_ARG; the next good call is unaffected."""
    adj = G.random_regular(512, 4, 31)
    bad = adj.copy()
    bad[100, 2] = 512
    rc, _ = noalloc_counts(bad)
    assert rc == G.GG_BAD_ARG and b"outside" in G.lib().gg_last_error()
    rc, got = noalloc_counts(adj)
    assert rc == G.GG_OK and np.array_equal(got, engine_counts(adj)[0])


def test_noalloc_rejects_sizes_beyond_its_array():
    import torch
    out = torch.zeros(MAX_LEVELS + 1, dtype=torch.int64, device="cuda")
    adj = torch.zeros((8192, 4), dtype=torch.int32, device="cuda")
    rc = G.lib().gg_graph_eval_noalloc(ctypes.c_void_p(adj.data_ptr()), 8192, 4, MAX_LEVELS,
                                       ctypes.c_void_p(out.data_ptr()), None)
    assert rc == G.GG_BAD_ARG
    assert b"scratch" in G.lib().gg_last_error()
