"""Batched evaluation of cyclic-lift candidates (gg_lift_*) and the lift moves
(gg_gen_lift_moves).

CPU: every move keeps the lift symmetric and simple, moves only non-padding
slots, draws shift moves only when N/M > 1, and is reproducible from its seed.
GPU: every candidate's exact counts equal the oracle's BFS from the M orbit
vertices of its own lift, in one round or many, at every group size, with a
level cap, on a disconnected base, and the reference ASPL equals the
cudaASPLconv calculator's."""

import numpy as np
import pytest

import graphgolf as G
import oracle as O


def lift_ok(N, M, diffs):
    """The lift of `diffs` is symmetric (each edge at both ends) and simple."""
    adj = O.expand_part(N, M, diffs)
    pad = np.asarray(diffs).reshape(M, -1)[np.arange(N) % M] % N == 0
    for v in range(N):
        row = [int(u) for u, p in zip(adj[v], pad[v]) if not p]
        if v in row or len(set(row)) != len(row):
            return False
        for u in row:
            back = [int(x) for x, p in zip(adj[u], pad[u]) if not p]
            if v not in back:
                return False
    return True


@pytest.mark.parametrize("m,g,d,seed", [(64, 8, 6, 3), (40, 5, 4, 1), (96, 1, 5, 2)])
def test_lift_moves_keep_the_lift_simple(m, g, d, seed):
    N, M, D = G.cyclic_lift(m, g, d, seed)
    moves = G.gen_lift_moves(N, M, D, 60, seed + 11)
    assert set(np.unique(moves["count"])) <= ({2, 4} if g > 1 else {4})
    for e in moves:
        t = G.apply_lift_edit(D, e)
        assert lift_ok(N, M, t)
        assert (t != D).sum() <= e["count"]
    if g > 1:
        assert (moves["count"] == 2).any() and (moves["count"] == 4).any()


def test_lift_moves_are_reproducible_and_skip_padding():
    N, M, D = G.cyclic_lift(48, 4, 6, 7)
    a = G.gen_lift_moves(N, M, D, 30, 99)
    b = G.gen_lift_moves(N, M, D, 30, 99)
    c = G.gen_lift_moves(N, M, D, 30, 100)
    assert a.tobytes() == b.tobytes() and a.tobytes() != c.tobytes()
    # a 5-regular lift padded to degree 6: slot 5 of every row is padding (diff 0)
    N2, M2, D5 = G.cyclic_lift(48, 4, 5, 7)
    P = np.concatenate([D5, np.zeros((M2, 1), np.int32)], axis=1)
    for e in G.gen_lift_moves(N2, M2, P, 40, 3):
        assert all(int(e["slot"][j]) != 5 for j in range(int(e["count"])))
        assert lift_ok(N2, M2, G.apply_lift_edit(P, e))


def test_lift_moves_bad_arguments():
    N, M, D = G.cyclic_lift(16, 4, 4, 1)
    with pytest.raises(G.GGError):
        G.gen_lift_moves(N + 1, M, D, 4, 1)        # M does not divide N


# ---- GPU ---------------------------------------------------------------------

def oracle_counts(N, M, t):
    r = O.bfs_pull(O.expand_part(N, M, t), np.arange(M))
    return r.total(), int(r.reached.sum()), r.levels, int(r.connected)


def check_all(L, N, M, D, moves, res):
    for e, got in zip(moves, res):
        want = oracle_counts(N, M, G.apply_lift_edit(D, e))
        assert (int(got["total"]), int(got["reached"]), int(got["connected"])) == (want[0], want[1], want[3])
        if want[3]:
            assert int(got["levels"]) == want[2]


@pytest.mark.gpu
@pytest.mark.parametrize("m,g,d,seed", [(256, 8, 6, 1), (100, 12, 4, 2), (130, 3, 5, 3)])
def test_lift_candidates_equal_the_oracle(m, g, d, seed):
    N, M, D = G.cyclic_lift(m, g, d, seed)
    L = G.Lift(N, M, d, 0)
    L.set_base(D)
    moves = np.concatenate([np.zeros(1, dtype=G.LIFT_EDIT_DTYPE), G.gen_lift_moves(N, M, D, 45, seed)])
    res = L.eval(moves)
    check_all(L, N, M, D, moves, res)
    # the same through every group size: one candidate per round, odd, automatic
    for grp in (1, 3, 0):
        L.set_group(grp)
        again = L.eval(moves)
        assert again.tobytes() == res.tobytes()
    # the reference ASPL of the base equals the cudaASPLconv calculator's
    c = G.cudaASPLconv(N, M, d, 0)
    diam, aspl = c.diameterASPL(D)
    assert L.aspl(res[:1])[0] == aspl and int(res[0]["levels"]) == diam
    L.close()


@pytest.mark.gpu
def test_lift_level_cap_and_disconnected_base():
    N, M, D = G.cyclic_lift(200, 6, 4, 5)
    L = G.Lift(N, M, 4, 0)
    L.set_base(D)
    moves = G.gen_lift_moves(N, M, D, 10, 1)
    full = L.eval(moves)
    capped = L.eval(moves, max_levels=3)
    assert (capped["connected"] == 0).all() and (capped["levels"] == 3).all()
    for a, b in zip(full, capped):
        assert int(b["reached"]) < int(a["reached"])
    # two disjoint cycles of length N/2 (orbit diffs +-2): disconnected
    N2, M2 = 64, 8
    T = np.zeros((M2, 2), np.int32)
    T[:, 0], T[:, 1] = 2, -2
    L2 = G.Lift(N2, M2, 2, 0)
    L2.set_base(T)
    base = np.zeros(1, dtype=G.LIFT_EDIT_DTYPE)
    r = L2.eval(base)
    want = oracle_counts(N2, M2, T)
    assert int(r[0]["connected"]) == 0 == want[3]
    assert (int(r[0]["total"]), int(r[0]["reached"])) == (want[0], want[1])
    L.close()
    L2.close()


@pytest.mark.gpu
def test_lift_many_rounds():
    N, M, D = G.cyclic_lift(512, 4, 8, 9)
    L = G.Lift(N, M, 8, 0)
    L.set_base(D)
    L.set_group(2)
    moves = G.gen_lift_moves(N, M, D, 21, 4)       # 11 rounds, the last one half full
    check_all(L, N, M, D, moves, L.eval(moves))
    assert L.last_ms() > 0
    L.close()


@pytest.mark.gpu
def test_lift_annealing_improves_and_reports_exact_aspl():
    import anneal as A
    N, M, D = G.cyclic_lift(64, 8, 4, 2)
    start = O.conv_diameter_aspl(N, M, D)[1]
    best, tr = A.anneal_lift(N, M, D, 80, seed=3, exact=16)
    assert tr.steps == 80 and tr.accepted > 0 and tr.exact_evals == 80 * 16
    assert lift_ok(N, M, best)
    diam, aspl = O.conv_diameter_aspl(N, M, best)
    assert aspl == tr.final_best and aspl < start
    assert all(b >= c for b, c in zip(tr.best, tr.best[1:]))


# ---- 2-D and 3-D torus lifts (piece, box) ------------------------------------

import instances as I


def graph_ok(adj, pad):
    """Pull adjacency `adj` with padding mask `pad`: simple and symmetric."""
    n = len(adj)
    rows = [[int(u) for u, p in zip(adj[v], pad[v]) if not p] for v in range(n)]
    for v in range(n):
        if v in rows[v] or len(set(rows[v])) != len(rows[v]):
            return False
        if any(v not in rows[u] for u in rows[v]):
            return False
    return True


def simple_piece(Mx, My, kx, ky, d, seed):
    for s in range(seed, seed + 200):
        Nx, Ny, _, _, T = I.random_piece(Mx, My, kx, ky, d, s)
        if graph_ok(O.expand_piece(Nx, Ny, Mx, My, T), np.zeros((Nx * Ny, d), bool)):
            return Nx, Ny, T
    raise AssertionError("no simple piece")


def simple_box(Mx, My, Mz, kx, ky, kz, d, seed):
    for s in range(seed, seed + 200):
        Nx, Ny, Nz, _, _, _, T = I.random_box(Mx, My, Mz, kx, ky, kz, d, s)
        if graph_ok(O.expand_box(Nx, Ny, Nz, Mx, My, Mz, T), np.zeros((Nx * Ny * Nz, d), bool)):
            return Nx, Ny, Nz, T
    raise AssertionError("no simple box")


def test_piece_and_box_moves_keep_the_lift_simple():
    Nx, Ny, T = simple_piece(6, 4, 3, 2, 4, 1)
    moves = G.gen_piece_moves(Nx, Ny, 6, 4, T, 40, 5)
    assert (moves["count"] == 2).any() and (moves["count"] == 4).any()
    for e in moves:
        t = G.apply_lift_edit(T, e)
        assert graph_ok(O.expand_piece(Nx, Ny, 6, 4, t), np.zeros((Nx * Ny, 4), bool))
        assert (e["diff"][:, 2] == 0).all()
    Nx, Ny, Nz, B = simple_box(3, 2, 2, 2, 2, 3, 4, 1)
    moves = G.gen_box_moves(Nx, Ny, Nz, 3, 2, 2, B, 40, 6)
    for e in moves:
        t = G.apply_lift_edit(B, e)
        assert graph_ok(O.expand_box(Nx, Ny, Nz, 3, 2, 2, t), np.zeros((Nx * Ny * Nz, 4), bool))
    a = G.gen_box_moves(Nx, Ny, Nz, 3, 2, 2, B, 10, 7)
    assert a.tobytes() == G.gen_box_moves(Nx, Ny, Nz, 3, 2, 2, B, 10, 7).tobytes()


@pytest.mark.gpu
def test_piece_candidates_equal_the_oracle():
    Mx, My = 16, 10
    Nx, Ny, T = simple_piece(Mx, My, 4, 3, 4, 2)
    L = G.Lift.piece(Nx, Ny, Mx, My, 4, 0)
    L.set_base(T)
    moves = np.concatenate([np.zeros(1, dtype=G.LIFT_EDIT_DTYPE), G.gen_piece_moves(Nx, Ny, Mx, My, T, 30, 3)])
    res = L.eval(moves)
    reps = O.piece_reps(Nx, Ny, Mx, My)
    for e, got in zip(moves, res):
        r = O.bfs_pull(O.expand_piece(Nx, Ny, Mx, My, G.apply_lift_edit(T, e)), reps)
        assert (int(got["total"]), int(got["reached"]), int(got["connected"])) == \
            (r.total(), int(r.reached.sum()), int(r.connected))
        if r.connected:
            assert int(got["levels"]) == r.levels
    L.set_group(1)
    assert L.eval(moves).tobytes() == res.tobytes()
    diam, aspl = G.cudaASPLpiece(Nx, Ny, Mx, My, 4, 0).diameterASPL(T)
    assert L.aspl(res[:1])[0] == aspl and int(res[0]["levels"]) == diam
    L.close()


@pytest.mark.gpu
def test_box_candidates_equal_the_oracle():
    Mx, My, Mz = 6, 5, 4
    Nx, Ny, Nz, B = simple_box(Mx, My, Mz, 2, 3, 2, 6, 3)
    L = G.Lift.box(Nx, Ny, Nz, Mx, My, Mz, 6, 0)
    L.set_base(B)
    moves = np.concatenate([np.zeros(1, dtype=G.LIFT_EDIT_DTYPE),
                            G.gen_box_moves(Nx, Ny, Nz, Mx, My, Mz, B, 30, 4)])
    res = L.eval(moves)
    reps = O.box_reps(Nx, Ny, Nz, Mx, My, Mz)
    for e, got in zip(moves, res):
        r = O.bfs_pull(O.expand_box(Nx, Ny, Nz, Mx, My, Mz, G.apply_lift_edit(B, e)), reps)
        assert (int(got["total"]), int(got["reached"]), int(got["connected"])) == \
            (r.total(), int(r.reached.sum()), int(r.connected))
        if r.connected:
            assert int(got["levels"]) == r.levels
    diam, aspl = G.cudaASPLbox(Nx, Ny, Nz, Mx, My, Mz, 6, 0).diameterASPL(B)
    assert L.aspl(res[:1])[0] == aspl and int(res[0]["levels"]) == diam
    L.close()


@pytest.mark.gpu
def test_piece_annealing_and_box_hill_climb_report_exact_aspl():
    import anneal as A
    Mx, My = 8, 6
    Nx, Ny, T = simple_piece(Mx, My, 3, 2, 4, 5)
    start = O.piece_diameter_aspl(Nx, Ny, Mx, My, T)[1]
    best, tr = A.anneal_piece(Nx, Ny, Mx, My, T, 60, seed=2, exact=16)
    assert tr.accepted > 0 and O.piece_diameter_aspl(Nx, Ny, Mx, My, best)[1] == tr.final_best < start
    assert graph_ok(O.expand_piece(Nx, Ny, Mx, My, best), np.zeros((Nx * Ny, 4), bool))
    Nx, Ny, Nz, B = simple_box(3, 2, 2, 2, 2, 3, 4, 1)
    start = O.box_diameter_aspl(Nx, Ny, Nz, 3, 2, 2, B)[1]
    best, tr = A.anneal_box(Nx, Ny, Nz, 3, 2, 2, B, 40, seed=3, exact=16)
    got = O.box_diameter_aspl(Nx, Ny, Nz, 3, 2, 2, best)[1]
    assert got == tr.final_best <= start
    # a hill climb never accepts a worse total
    assert all(b >= c for b, c in zip(tr.best, tr.best[1:]))


def test_piece_lift_generator_is_simple_and_connected():
    Nx, Ny, Mx, My, T = G.piece_lift(8, 6, 4, 3, 4, 3)
    assert (Nx, Ny, T.shape) == (32, 18, (48, 4, 2))
    adj = O.expand_piece(Nx, Ny, Mx, My, T)
    assert graph_ok(adj, np.zeros((Nx * Ny, 4), bool))
    assert O.bfs_pull(adj, np.arange(Nx * Ny)).connected
    again = G.piece_lift(8, 6, 4, 3, 4, 3)[4]
    assert again.tobytes() == T.tobytes()


@pytest.mark.gpu
def test_lift_diameter_beyond_the_first_count_rows():
    # a cycle of 600 as a part with 2 orbits: diameter 300, past the 256 count rows a
    # launch starts with, so the population runs again with rows for the full cap
    N, M = 600, 2
    T = np.array([[1, -1], [1, -1]], np.int32)
    L = G.Lift(N, M, 2, 0)
    L.set_base(T)
    base = np.zeros(2, dtype=G.LIFT_EDIT_DTYPE)
    want = oracle_counts(N, M, T)
    r = L.eval(base)
    assert want[2] == 300 and want[3] == 1
    for x in r:
        assert (int(x["total"]), int(x["reached"]), int(x["levels"]), int(x["connected"])) == want
    capped = L.eval(base, max_levels=280)
    assert (capped["connected"] == 0).all() and (capped["levels"] == 280).all()
    L.close()


def test_piece_and_box_moves_without_copies_are_all_2opt_and_bad_sizes_fail():
    # a tile that is the whole torus (one copy): no lift shift to redraw
    Nx, Ny, Mx, My, T = G.piece_lift(6, 5, 1, 1, 4, 2)
    moves = G.gen_piece_moves(Nx, Ny, Mx, My, T, 20, 1)
    assert (moves["count"] == 4).all()
    with pytest.raises(G.GGError):
        G.gen_piece_moves(Nx + 1, Ny, Mx, My, T, 2, 1)          # 7 is no multiple of 6
    Nx, Ny, Nz, B = simple_box(3, 2, 2, 2, 2, 3, 4, 1)
    with pytest.raises(G.GGError):
        G.gen_box_moves(Nx, Ny, Nz + 1, 3, 2, 2, B, 2, 1)
