"""GPU parity: the CUDA engine (through the C ABI of libggb200.so) against the
oracle, the committed golden fixtures and the reference's own GPU calculators
built for sm_100a.  Integer results must be bit-exact; ASPL doubles must be
identical (they are the same integer total divided the same way)."""
import json
import math
import os

import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O

pytestmark = pytest.mark.gpu

CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cases.json")))["cases"]


def same(a, b):
    return a == b or (isinstance(a, float) and isinstance(b, float) and math.isnan(a) and math.isnan(b))


def part_adj(N, M, diffs):
    return O.expand_part(N, M, diffs)


# ---- golden fixtures -------------------------------------------------------

@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_golden(case):
    t = np.array(case["table"], dtype=np.int32)
    deg = case["degree"]
    if case["kind"] == "part":
        N, M = case["N"], case["M"]
        cu = G.cudaASPLconv(N, M, deg, 0)
        d, a = cu.diameterASPL(t)
        if case["ref_diameter"] == O.INT_MAX:
            assert (d, a) == (O.SENTINEL, float(O.SENTINEL))
            assert cu.calc(t) == 1e9
        else:
            assert (d, a) == (case["ref_diameter"], case["ref_aspl"])
            assert cu.calc(t) == case["ref_calc"]
        r = cu.eval(t)
        assert r["total"] == case["total"] and r["levels"] == case["levels"]
        assert bool(r["connected"]) == case["connected"]
        if M == N:  # plain graph: the cudaASPLgraph calculator on the same edges
            adj = part_adj(N, M, t.reshape(M, deg))
            g = G.cudaASPLgraph(N, deg, 0)
            want = (case["levels"], case["total"]) if case["connected"] else (-1, -1)
            assert g.calc(adj) == want
    elif case["kind"] == "piece":
        Nx, Ny, Mx, My = case["dims"]
        cu = G.cudaASPLpiece(Nx, Ny, Mx, My, deg, 0)
        d, a = cu.diameterASPL(t)
        want = ((O.SENTINEL, float(O.SENTINEL)) if case["ref_diameter"] == O.INT_MAX
                else (case["ref_diameter"], case["ref_aspl"]))
        assert (d, a) == want
        assert cu.eval(t)["total"] == case["total"]
    else:
        cu = G.cudaASPLbox(*case["dims"], deg, 0)
        d, a = cu.diameterASPL(t)
        want = ((O.SENTINEL, float(O.SENTINEL)) if case["ref_diameter"] == O.INT_MAX
                else (case["ref_diameter"], case["ref_aspl"]))
        assert (d, a) == want
        assert cu.eval(t)["total"] == case["total"]


# ---- closed forms through the plain-graph calculator -----------------------

@pytest.mark.parametrize("adj,kat", [
    (I.cycle(5), I.kat_cycle(5)), (I.cycle(130), I.kat_cycle(130)),
    (I.complete(9), I.kat_complete(9)), (I.hypercube(7), I.kat_hypercube(7)),
    (I.hypercube(10), I.kat_hypercube(10)), (I.petersen(), I.kat_petersen()),
    (O.pad_graph(11, I.complete_bipartite(4, 7)), I.kat_complete_bipartite(4, 7)),
])
def test_kat_graph(adj, kat):
    adj = np.asarray(adj, dtype=np.int32)
    g = G.cudaASPLgraph(len(adj), adj.shape[1], 0)
    assert g.calc(adj) == kat


# ---- random instances of every form vs the oracle --------------------------

@pytest.mark.parametrize("seed", range(10))
def test_random_parts(seed):
    rng = np.random.default_rng(1000 + seed)
    m = int(rng.integers(2, 300))
    g = int(rng.integers(1, 12))
    d = int(rng.choice([2, 3, 4, 5, 6, 8, 12, 16]))
    if (m * d) % 2:
        m += 1
    N, M, diffs = I.random_part(m, g, d, seed)
    cu = G.cudaASPLconv(N, M, d, 0)
    assert cu.diameterASPL(diffs) == O.conv_diameter_aspl(N, M, diffs)
    assert cu.calc(diffs) == O.conv_calc(N, M, diffs)
    w = cu.WVCdiameterASPL(diffs)
    assert w == O.conv_wvc(N, M, diffs)


@pytest.mark.parametrize("seed", range(6))
def test_random_pieces_boxes(seed):
    rng = np.random.default_rng(2000 + seed)
    Mx, My = int(rng.integers(1, 9)), int(rng.integers(1, 9))
    kx, ky = int(rng.integers(1, 6)), int(rng.integers(1, 6))
    d = 4
    Nx, Ny, Mx, My, rows = I.random_piece(Mx, My, kx, ky, d, seed)
    assert G.cudaASPLpiece(Nx, Ny, Mx, My, d, 0).diameterASPL(rows) == \
        O.piece_diameter_aspl(Nx, Ny, Mx, My, rows)
    M3 = [int(x) for x in rng.integers(1, 5, size=3)]
    k3 = [int(x) for x in rng.integers(1, 4, size=3)]
    dims_rows = I.random_box(*M3, *k3, 6, seed)
    dims, rows = dims_rows[:6], dims_rows[6]
    assert G.cudaASPLbox(*dims, 6, 0).diameterASPL(rows) == O.box_diameter_aspl(*dims, rows)


@pytest.mark.parametrize("n,d,seed", [(1, 2, 0), (2, 1, 0), (33, 2, 1), (127, 3, 2), (129, 5, 3),
                                      (300, 7, 4), (1000, 3, 5), (2049, 6, 6)])
def test_ragged_sizes_exact_counts(n, d, seed):
    if n == 1:
        adj = np.zeros((1, d), dtype=np.int32)
    elif n == 2:
        adj = np.array([[1], [0]], dtype=np.int32)
    else:
        if (n * d) % 2:
            n += 1
        adj = I.random_regular_np(n, d, seed)
    n = len(adj)
    e = G.cudaASPLgraph(n, adj.shape[1], 0)
    r = e.eval(adj, max_levels=n + 1, level_counts=True)
    o = O.bfs_pull(adj, np.arange(n))
    assert r["total"] == o.total() and r["levels"] == o.levels
    assert r["reached"] == int(o.reached.sum()) and bool(r["connected"]) == o.connected
    assert np.array_equal(r["level_counts"][:n], o.level_counts[:n + 1][:n])


# ---- sentinels and level caps ---------------------------------------------

def test_graph_sentinels():
    p = I.path_graph(400)
    assert G.cudaASPLgraph(400, 2, 0).calc(p) == (-2, -2)
    dis = I.disjoint_union(I.cycle(10), I.cycle(12))
    assert G.cudaASPLgraph(22, 2, 0).calc(dis) == (-1, -1)
    # disconnected AND a long component: chunk 0 decides (cudaASPLgraph.cu:158-192)
    big = I.disjoint_union(I.cycle(500), I.cycle(30))
    assert G.cudaASPLgraph(530, 2, 0).calc(big) == O.graph_calc(530, big)
    # diameter exactly 198 is still reported
    c = I.cycle(396)
    assert G.cudaASPLgraph(396, 2, 0).calc(c) == I.kat_cycle(396)


def test_conv_level_cap():
    for n in (196, 198, 199, 200, 250):
        N, M, diffs = I.plain_as_part(I.cycle(n))
        cu = G.cudaASPLconv(N, M, 2, 0)
        assert cu.diameterASPL(diffs) == O.conv_diameter_aspl(N, M, diffs)
        assert cu.calc(diffs) == O.conv_calc(N, M, diffs)
        assert cu.WVCdiameterASPL(diffs) == O.conv_wvc(N, M, diffs)


def test_disconnected_lifted():
    N, M, diffs = I.plain_as_part(I.disjoint_union(I.cycle(40), I.cycle(24)))
    cu = G.cudaASPLconv(N, M, 2, 0)
    assert cu.diameterASPL(diffs) == (O.SENTINEL, float(O.SENTINEL))
    assert cu.calc(diffs) == 1e9
    assert cu.WVCdiameterASPL(diffs) == (O.SENTINEL, O.SENTINEL, float(O.SENTINEL))


# ---- batching invariance (size-independent properties) --------------------

def test_batch_width_invariance_and_source_ranges():
    adj = G.random_regular(3000, 4, 2)
    e = G.cudaASPLgraph(3000, 4, 0)
    base = e.eval(adj)
    o = O.bfs_pull(adj, np.arange(3000))
    assert base["total"] == o.total() and base["levels"] == o.levels
    for bits in (128, 256, 640, 1024, 2944, 3000):
        e.set_batch_sources(bits)
        r = e.eval(adj)
        assert (r["total"], r["levels"], r["reached"]) == (base["total"], base["levels"], base["reached"])
    # sum over disjoint source ranges == whole (checksum of checksums)
    parts = [e.eval(adj, src_range=(a, min(a + 700, 3000)))["total"] for a in range(0, 3000, 700)]
    assert sum(parts) == base["total"]
    sub = e.eval(adj, src_range=(100, 357))
    os_ = O.bfs_pull(adj, np.arange(100, 357))
    assert sub["total"] == os_.total()


def test_autotune_keeps_results_and_is_adopted():
    adj = G.random_regular(3000, 6, 4)
    e = G.cudaASPLgraph(3000, 6, 0)
    base = e.eval(adj)
    width, ms = e.autotune(adj, trials=2)
    assert 0 < width and ms > 0
    r = e.eval(adj)
    assert (r["total"], r["levels"], r["reached"]) == (base["total"], base["levels"], base["reached"])
    # a later engine of the same shape on the same device starts from the tuned width
    e2 = G.cudaASPLgraph(3000, 6, 0)
    r2 = e2.eval(adj)
    assert r2["batches"] == r["batches"]
    assert r2["total"] == base["total"]


def test_shards_of_distributed_helper_sum_to_whole():
    import distributed as D
    adj = G.random_regular(2000, 6, 8)
    e = G.cudaASPLgraph(2000, 6, 0)
    whole = e.eval(adj)
    for world in (2, 3, 8):
        parts = [e.eval(adj, src_range=D.shard(2000, r, world)) for r in range(world)]
        assert sum(p["total"] for p in parts) == whole["total"]
        assert sum(p["reached"] for p in parts) == whole["reached"]
        assert max(p["levels"] for p in parts) == whole["levels"]


# ---- benchmark configurations ---------------------------------------------

def test_config_regular_4096_16():
    adj = G.random_regular(4096, 16, 1)
    got = G.cudaASPLgraph(4096, 16, 0).calc(adj)
    assert got == O.graph_calc(4096, adj)


def test_config_lift_32768():
    N, M, diffs = G.cyclic_lift(1024, 32, 12, 1)
    cu = G.cudaASPLconv(N, M, 12, 0)
    d, a = cu.diameterASPL(diffs)
    assert (d, a) == O.conv_diameter_aspl(N, M, diffs)
    # orbit reduction is exact: total over 1024 representatives x 32 == full 32768-source BFS
    full = G.cudaASPLgraph(N, 12, 0).calc(part_adj(N, M, diffs))
    r = cu.eval(diffs)
    assert full == (d, r["total"] * (N // M))


def test_config_regular_65536_8_full():
    """The graph the headline benchmark times: the engine's exact total and
    diameter against the oracle's BFS from every one of the 65536 sources, and
    against the reference cudaASPLgraph built for this GPU when present."""
    adj = G.random_regular(65536, 8, 1)
    got = G.cudaASPLgraph(65536, 8, 0).calc(adj)
    o = O.bfs_pull(adj, np.arange(65536))
    assert o.connected and got == (o.levels, o.total())
    if O.RefGPU.available("graph"):
        R = O.RefGPU("graph")
        R.create(65536, 8, 0)
        assert R.graph_calc(adj) == got
        R.close()


def test_config_regular_65536_8_sampled():
    adj = G.random_regular(65536, 8, 1)
    e = G.cudaASPLgraph(65536, 8, 0)
    whole = e.eval(adj, max_levels=199)
    assert whole["connected"] and not whole["capped"]
    # exact per-source totals on a sample against the oracle
    for a in (0, 31000, 65536 - 200):
        r = e.eval(adj, src_range=(a, a + 200))
        o = O.bfs_pull(adj, np.arange(a, a + 200))
        assert r["total"] == o.total() and r["levels"] == o.levels
    # batch-width invariance at full size
    e.set_batch_sources(8192)
    r = e.eval(adj, max_levels=199)
    assert (r["total"], r["levels"]) == (whole["total"], whole["levels"])
    # pair count identity: every ordered pair reached exactly once
    assert whole["reached"] == 65536 * 65536


# ---- beamer -------------------------------------------------------------------

def test_beamer_phantom_rows_and_cap():
    N, M, diffs = G.cyclic_lift(50, 20, 4, 5)   # N = 1000 < 10^6: phantom rows matter
    b = G.cudaASPLbeamer(N, M, 4, 0)
    assert b.calc(diffs) == O.beamer_calc(N, M, diffs)
    assert b.calc(diffs, regular=False) == 1e8


def test_beamer_full_domain():
    m, g = 100, 10000                            # N = 10^6 exactly
    N = m * g
    diffs = np.array([[1, -1, 100, -100, 10100, -10100]] * m, dtype=np.int32)
    b = G.cudaASPLbeamer(N, m, 6, 0)
    assert b.calc(diffs) == O.beamer_calc(N, m, diffs)


# ---- the reference's own GPU calculators on the same box -------------------

def _ref(kind):
    if not O.RefGPU.available(kind):
        pytest.skip("reference GPU build not present")
    return O.RefGPU(kind)


def test_reference_gpu_conv_and_wvc():
    R = _ref("conv")
    for seed in range(4):
        N, M, diffs = I.random_part(64 + 32 * seed, 4, 4, 50 + seed)
        R.create(N, M, 4, 0)
        cu = G.cudaASPLconv(N, M, 4, 0)
        assert cu.diameterASPL(diffs) == R.conv_diameter_aspl(N, M, diffs)
        assert cu.calc(diffs) == R.conv_calc(N, M, diffs)
        assert cu.WVCdiameterASPL(diffs) == R.conv_wvc(N, M, diffs)
        R.close()


def test_reference_gpu_graph():
    R = _ref("graph")
    adj = G.random_regular(3000, 4, 7)
    R.create(3000, 4, 0)
    assert G.cudaASPLgraph(3000, 4, 0).calc(adj) == R.graph_calc(adj)
    R.close()


def test_reference_gpu_piece_box():
    Rp = _ref("piece")
    Nx, Ny, Mx, My, rows = I.random_piece(4, 4, 5, 5, 4, 3)
    Rp.create(Nx, Ny, Mx, My, 4, 0)
    assert G.cudaASPLpiece(Nx, Ny, Mx, My, 4, 0).diameterASPL(rows) == \
        Rp.piece_diameter_aspl(Nx, Ny, Mx, My, rows)
    Rp.close()
    Rb = _ref("box")
    dims_rows = I.random_box(2, 2, 2, 3, 3, 3, 6, 4)
    Rb.create(*dims_rows[:6], 6, 0)
    assert G.cudaASPLbox(*dims_rows[:6], 6, 0).diameterASPL(dims_rows[6]) == \
        Rb.box_diameter_aspl(*dims_rows[:6], dims_rows[6])
    Rb.close()


def test_reference_gpu_beamer():
    R = _ref("beamer")
    N, M, diffs = G.cyclic_lift(50, 20, 4, 5)
    R.create(N, M, 4, 0)
    assert G.cudaASPLbeamer(N, M, 4, 0).calc(diffs) == R.beamer_calc(N, M, diffs)
    R.close()


# ---- failure paths (no GPU fault: bounded waits and host-side injection) ---

def test_bounded_barrier_wait_reports_timeout(monkeypatch):
    adj = G.random_regular(1024, 4, 3)
    e = G.cudaASPLgraph(1024, 4, 0)
    e.set_wait_limit_ms(50)
    monkeypatch.setenv("GG_FAULT_INJECT", "barrier")
    with pytest.raises(G.GGError) as err:
        e.eval(adj)
    assert err.value.status == G.GG_TIMEOUT
    monkeypatch.delenv("GG_FAULT_INJECT")
    # the context and the engine stay usable
    assert e.calc(adj) == O.graph_calc(1024, adj)


def test_injected_alloc_and_launch_failures(monkeypatch):
    monkeypatch.setenv("GG_FAULT_INJECT", "alloc")
    with pytest.raises(G.GGError) as err:
        G.cudaASPLconv(64, 64, 4, 0)
    assert err.value.status == G.GG_OUT_OF_MEMORY
    monkeypatch.delenv("GG_FAULT_INJECT")
    N, M, diffs = I.random_part(32, 2, 4, 1)
    cu = G.cudaASPLconv(N, M, 4, 0)
    monkeypatch.setenv("GG_FAULT_INJECT", "launch")
    with pytest.raises(G.GGError) as err:
        cu.diameterASPL(diffs)
    assert err.value.status == G.GG_CUDA_ERROR
    monkeypatch.delenv("GG_FAULT_INJECT")
    assert cu.diameterASPL(diffs) == O.conv_diameter_aspl(N, M, diffs)


def test_bad_graph_table_rejected():
    adj = G.random_regular(256, 4, 1).copy()
    adj[17, 2] = 256       # out of range
    e = G.cudaASPLgraph(256, 4, 0)
    with pytest.raises(G.GGError) as err:
        e.calc(adj)
    assert err.value.status == G.GG_BAD_ARG
    adj[17, 2] = -5
    with pytest.raises(G.GGError):
        e.calc(adj)


def test_replayed_evaluations_match_direct_launches(monkeypatch):
    """Repeated evaluations replay a captured CUDA graph; a sequence that changes
    the table, the source range, the level cap, the batch width and the wait limit
    between calls gives the same answers as an engine that launches directly."""
    tables = [G.random_regular(3000, 6, s) for s in (1, 2)]
    calls = [dict(t=0), dict(t=1), dict(t=0), dict(t=1, src_range=(64, 2000)), dict(t=1, src_range=(64, 2000)),
             dict(t=0, max_levels=3), dict(t=0, max_levels=3), dict(t=1, wvc=True), dict(t=0, bits=512),
             dict(t=1, bits=512), dict(t=0, wait=5000), dict(t=1)]

    def run(eng):
        out = []
        for c in calls:
            if "bits" in c:
                eng.set_batch_sources(c["bits"])
            if "wait" in c:
                eng.set_wait_limit_ms(c["wait"])
            r = eng.eval(tables[c["t"]], max_levels=c.get("max_levels", 0), src_range=c.get("src_range"),
                         want_wvc=c.get("wvc", False))
            out.append((r["total"], r["reached"], r["levels"], r["capped"], r["wvc"]))
        return out

    replay = run(G.cudaASPLgraph(3000, 6, 0))
    monkeypatch.setenv("GG_NO_GRAPH", "1")
    direct = run(G.cudaASPLgraph(3000, 6, 0))
    assert replay == direct
    o = O.bfs_pull(tables[1], np.arange(3000))
    assert replay[1][0] == o.total()
