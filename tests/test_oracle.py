"""Pin the oracle: the C restatement (oracle/gg_oracle.c + oracle/oracle.py)
against the reference's own CPU calculators compiled from its sources
(oracle/_ref/libref_cpu.so: cpuASPLqueue / cpuASPLpiece / cpuASPLbox) and
against closed-form known answers.  CPU only."""
import math

import numpy as np
import pytest

import instances as I
import oracle as O

needs_ref = pytest.mark.skipif(not O.RefCPU.available(),
                               reason="reference CPU build (oracle/_ref) not present")


def rows_of(table):
    return [list(map(int, np.asarray(r).reshape(-1))) for r in table]


@pytest.fixture(scope="module")
def ref():
    return O.RefCPU()


# ---- closed forms ---------------------------------------------------------

@pytest.mark.parametrize("n", [3, 4, 5, 8, 9, 64, 101])
def test_kat_cycle(n):
    r = O.bfs_pull(I.cycle(n), np.arange(n))
    assert (r.levels, r.total()) == I.kat_cycle(n) and r.connected


@pytest.mark.parametrize("n", [2, 3, 5, 17])
def test_kat_complete(n):
    r = O.bfs_pull(I.complete(n), np.arange(n))
    assert (r.levels, r.total()) == I.kat_complete(n)


@pytest.mark.parametrize("k", [1, 2, 3, 6, 9])
def test_kat_hypercube(k):
    n = 1 << k
    r = O.bfs_pull(I.hypercube(k), np.arange(n))
    assert (r.levels, r.total()) == I.kat_hypercube(k)


def test_kat_petersen():
    r = O.bfs_pull(I.petersen(), np.arange(10))
    assert (r.levels, r.total()) == I.kat_petersen()


@pytest.mark.parametrize("a,b", [(1, 1), (2, 3), (4, 7)])
def test_kat_complete_bipartite(a, b):
    t = O.pad_graph(a + b, I.complete_bipartite(a, b))
    r = O.bfs_pull(t, np.arange(a + b))
    assert (r.levels, r.total()) == I.kat_complete_bipartite(a, b)


def test_cycle_as_part_matches_reference_value():
    # C8 -> diameter 4, ASPL 16/7 (value recorded from the reference cpuASPLqueue<1024>)
    N, M, diffs = I.plain_as_part(I.cycle(8))
    d, a = O.queue_diameter_aspl(N, M, diffs)
    assert d == 4 and a == pytest.approx(16 / 7, abs=0)


# ---- the restatement against the reference CPU build ----------------------

@needs_ref
@pytest.mark.parametrize("seed", range(12))
def test_queue_random_parts(ref, seed):
    rng = np.random.default_rng(seed)
    m = int(rng.integers(2, 40))
    g = int(rng.integers(1, 9))
    d = int(rng.choice([2, 3, 4]))
    if (m * d) % 2:
        m += 1
    N, M, diffs = I.random_part(m, g, d, seed)
    want = ref.queue_diameter_aspl(N, M, rows_of(diffs))
    got = O.queue_diameter_aspl(N, M, diffs)
    assert got[0] == want[0]
    assert got[1] == want[1] or (math.isnan(got[1]) and math.isnan(want[1]))
    assert O.queue_calc(N, M, diffs) == ref.queue_calc(N, M, rows_of(diffs))


@needs_ref
@pytest.mark.parametrize("n,d,seed", [(256, 4, 1), (100, 3, 2), (500, 5, 3), (64, 2, 4)])
def test_queue_plain_graphs(ref, n, d, seed):
    N, M, diffs = I.plain_as_part(I.random_regular_np(n, d, seed))
    assert O.queue_diameter_aspl(N, M, diffs) == ref.queue_diameter_aspl(N, M, rows_of(diffs))


@needs_ref
def test_queue_disconnected(ref):
    adj = I.disjoint_union(I.cycle(10), I.petersen()[:, :2])
    N, M, diffs = I.plain_as_part(adj)
    got = O.queue_diameter_aspl(N, M, diffs)
    assert got == ref.queue_diameter_aspl(N, M, rows_of(diffs))
    assert got[0] == O.INT_MAX
    assert O.queue_calc(N, M, diffs) == ref.queue_calc(N, M, rows_of(diffs)) == 1e9


@needs_ref
def test_queue_nonregular(ref):
    # rows of different length: the reference pads nothing on the CPU side
    rows = [[1, -1, 3], [-1, 1], [1, -1, 2], [-1, -3, 1], [1, -1], [-2, 1, -1]]
    N = M = 6
    want = ref.queue_diameter_aspl(N, M, rows)
    width = max(map(len, rows))
    # pad with diff 0 (self loop), which leaves every distance unchanged
    table = np.array([r + [0] * (width - len(r)) for r in rows], dtype=np.int32)
    assert O.queue_diameter_aspl(N, M, table) == want


@needs_ref
@pytest.mark.parametrize("seed", range(8))
def test_piece_random(ref, seed):
    rng = np.random.default_rng(100 + seed)
    Mx, My = int(rng.integers(1, 5)), int(rng.integers(1, 5))
    kx, ky = int(rng.integers(1, 5)), int(rng.integers(1, 5))
    d = 4 if (Mx * My) % 2 else int(rng.choice([3, 4]))
    Nx, Ny, Mx, My, rows = I.random_piece(Mx, My, kx, ky, d, seed)
    want = ref.piece_diameter_aspl(Nx, Ny, Mx, My, rows_of(rows))
    got = O.piece_diameter_aspl(Nx, Ny, Mx, My, rows)
    # cudaASPLpiece and cpuASPLpiece agree except for their disconnection sentinel
    if want[0] == O.INT_MAX:
        assert got == (O.SENTINEL, float(O.SENTINEL))
    else:
        assert got == want


@needs_ref
@pytest.mark.parametrize("seed", range(8))
def test_box_random(ref, seed):
    rng = np.random.default_rng(200 + seed)
    Mx, My, Mz = (int(x) for x in rng.integers(1, 4, size=3))
    kx, ky, kz = (int(x) for x in rng.integers(1, 4, size=3))
    d = 4
    Nx, Ny, Nz, Mx, My, Mz, rows = I.random_box(Mx, My, Mz, kx, ky, kz, d, seed)
    want = ref.box_diameter_aspl(Nx, Ny, Nz, Mx, My, Mz, rows_of(rows))
    got = O.box_diameter_aspl(Nx, Ny, Nz, Mx, My, Mz, rows)
    if want[0] == O.INT_MAX:
        assert got == (O.SENTINEL, float(O.SENTINEL))
    else:
        assert got == want


# ---- internal consistency of the restated conventions ---------------------

def test_exact_total_matches_reference_double():
    N, M, diffs = I.random_part(64, 8, 4, 7)
    r = O.bfs_pull(O.expand_part(N, M, diffs), np.arange(M))
    _, a = O.queue_diameter_aspl(N, M, diffs)
    assert round(a * N * (N - 1)) == r.total() * (N // M)


def test_conv_diameter_cap_partial_total():
    # cycle of 250 vertices: diameter 125 >= 99 -> (1e8, ASPL of levels <= 99)
    n = 250
    N, M, diffs = I.plain_as_part(I.cycle(n))
    d, a = O.conv_diameter_aspl(N, M, diffs)
    assert d == O.SENTINEL
    part_total = n * 2 * sum(range(1, 100))
    assert a == float(part_total) / (N * (N - 1))


def test_graph_calc_sentinels():
    assert O.graph_calc(400, I.path_graph(400)) == (-2, -2)
    assert O.graph_calc(20, I.disjoint_union(I.cycle(10), I.cycle(10))) == (-1, -1)
    assert O.graph_calc(64, I.cycle(64)) == I.kat_cycle(64)


def test_wvc_simple():
    # cycle C_n as a part (M = N): every source has eccentricity n//2, so every
    # lane position j < min(32, n) completes at the last level
    for n in (8, 40, 70):
        N, M, diffs = I.plain_as_part(I.cycle(n))
        w, d, a = O.conv_wvc(N, M, diffs)
        assert d == n // 2 and w == min(32, n)


def test_beamer_within_domain_equals_capped_bfs():
    # for N = 10^6 the beamer kernel scans exactly the real vertices
    N, M = O.BEAMER_N, 10
    diffs = np.array([[1, -1, 1000, -1000]] * M, dtype=np.int32)
    a = O.beamer_calc(N, M, diffs)
    r = O.bfs_pull(O.expand_part(N, M, diffs), np.arange(M))
    assert a == float(r.total(cap=7) * (N // M)) / (N * (N - 1))
