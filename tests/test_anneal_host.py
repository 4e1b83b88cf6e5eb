"""Host-side parts of the annealers (no GPU): the rank correlation, and the
lifted annealing loop driven by an oracle-backed stand-in for the GPU lift
evaluator (acceptance, hill-climb order, exact reported ASPL, target stop)."""
import numpy as np
import pytest

import anneal as A


def test_rank_correlation_matches_scipy():
    from scipy.stats import spearmanr
    rng = np.random.default_rng(4)
    x = rng.normal(size=200)
    y = x + rng.normal(size=200)
    y[::7] = y[0]                        # ties
    assert abs(A.rank_correlation(x, y) - spearmanr(x, y).correlation) < 1e-12
    assert A.rank_correlation(x, -x) == -1.0


# ---- the lifted annealing loop, driven by an oracle-backed stand-in -----------

import graphgolf as G
import oracle as O


class OracleLift:
    """Stand-in for G.Lift (part form): the same set_base / eval interface, exact
    counts from the oracle; records every base the loop installs."""

    def __init__(self, N, M):
        self.N, self.M = N, M
        self.bases = []

    def set_base(self, table):
        self.base = np.array(table, dtype=np.int32, copy=True)
        self.bases.append(self.base)

    def eval(self, edits):
        out = np.zeros(len(edits), dtype=G.CAND_RESULT_DTYPE)
        for i, e in enumerate(edits):
            r = O.bfs_pull(O.expand_part(self.N, self.M, G.apply_lift_edit(self.base, e)), np.arange(self.M))
            out[i] = (r.total(), int(r.reached.sum()), r.levels, int(r.connected))
        return out


def _key(N, M, table):
    r = O.bfs_pull(O.expand_part(N, M, table), np.arange(M))
    return r.levels, r.total()


def test_lifted_hill_climb_never_worsens_and_reports_exact_aspl():
    N, M, D = G.cyclic_lift(24, 4, 4, 2)
    L = OracleLift(N, M)
    gen = lambda t, c, s: G.gen_lift_moves(N, M, t, c, s)  # noqa: E731
    best, tr = A._anneal_table(L, gen, D, 25, seed=4, exact=8, t0_frac=0.0, t_end=1e-6, target=None,
                               time_limit=None)
    keys = [_key(N, M, b) for b in L.bases]
    assert all(k2 <= k1 for k1, k2 in zip(keys, keys[1:]))       # (diameter, total) never rises
    assert tr.accepted == len(L.bases) - 1 and tr.exact_evals == 25 * 8
    assert O.conv_diameter_aspl(N, M, best)[1] == tr.final_best
    assert tr.final_best <= O.conv_diameter_aspl(N, M, D)[1]


def test_lifted_annealing_stops_at_the_target():
    N, M, D = G.cyclic_lift(24, 4, 4, 2)
    gen = lambda t, c, s: G.gen_lift_moves(N, M, t, c, s)  # noqa: E731
    _, full = A._anneal_table(OracleLift(N, M), gen, D, 25, seed=4, exact=8, t0_frac=0.0, t_end=1e-6,
                              target=None, time_limit=None)
    assert len(full.best) >= 3                                   # this start improves several times
    target = full.best[2]
    _, tr = A._anneal_table(OracleLift(N, M), gen, D, 25, seed=4, exact=8, t0_frac=0.0, t_end=1e-6,
                            target=target, time_limit=None)
    assert tr.hit_time is not None and tr.final_best <= target and tr.steps == tr.hit_step


class OraclePiece:
    """Stand-in for G.Lift.piece: exact counts over the corner tile by the oracle."""

    def __init__(self, Nx, Ny, Mx, My):
        self.dims = (Nx, Ny, Mx, My)
        self.reps = O.piece_reps(Nx, Ny, Mx, My)

    def set_base(self, table):
        self.base = np.array(table, dtype=np.int32, copy=True)

    def eval(self, edits):
        out = np.zeros(len(edits), dtype=G.CAND_RESULT_DTYPE)
        for i, e in enumerate(edits):
            r = O.bfs_pull(O.expand_piece(*self.dims, G.apply_lift_edit(self.base, e)), self.reps)
            out[i] = (r.total(), int(r.reached.sum()), r.levels, int(r.connected))
        return out


def test_piece_initial_temperature_from_exact_uphill_moves():
    import math
    Nx, Ny, Mx, My, d = 16, 12, 4, 3, 4
    it = A.initial_temperature_piece(Nx, Ny, Mx, My, d, graphs=3, neighbours=12, seed=2,
                                     make_lift=lambda: OraclePiece(Nx, Ny, Mx, My))
    # the same quantity from the reference's ASPL values (cudaASPLpiece-style, over
    # the tile, scaled by N/M), restated here directly
    N, scale = Nx * Ny, (Nx * Ny) // (Mx * My)
    ups = []
    for k in range(3):
        T = G.piece_lift(Mx, My, Nx // Mx, Ny // My, d, 2 * 1000003 + k)[4]
        fx = O.piece_diameter_aspl(Nx, Ny, Mx, My, T)[1]
        for e in G.gen_piece_moves(Nx, Ny, Mx, My, T, 12, (2 << 20) ^ k):
            diam, fy = O.piece_diameter_aspl(Nx, Ny, Mx, My, G.apply_lift_edit(T, e))
            if diam < 10 ** 8 and fy > fx:
                ups.append((fy - fx) * N * (N - 1))
    assert it.uphill == len(ups) and it.proposals == 36
    assert abs(it.avg - sum(ups) / len(ups)) < 1e-6 * it.avg
    assert abs(it.temp + it.avg / math.log(0.4)) < 1e-9 * it.temp
    assert scale == 16


@pytest.mark.parametrize("t0", [0.2, 0.0])
def test_lifted_annealing_resumes_from_a_checkpoint(tmp_path, t0):
    # 20 steps in one go against the same run resumed from its checkpoint after
    # step 9: the same tables, counts and trace
    N, M, D = G.cyclic_lift(24, 4, 4, 2)
    gen = lambda t, c, s: G.gen_lift_moves(N, M, t, c, s)  # noqa: E731
    # one proposal per step and a warm start: the run accepts uphill moves, so the
    # resumed random stream must continue where it stopped
    kw = dict(seed=5, exact=1, t0_frac=t0, t_end=1e-6, target=None)
    full_L = OracleLift(N, M)
    best, tr = A._anneal_table(full_L, gen, D, 20, time_limit=None, **kw)
    ck = str(tmp_path / "run_{step}.npz")
    A._anneal_table(OracleLift(N, M), gen, D, 20, time_limit=None, checkpoint=ck, checkpoint_every=9, **kw)
    assert (tmp_path / "run_9.npz").exists() and (tmp_path / "run_18.npz").exists()
    L2 = OracleLift(N, M)
    best2, tr2 = A._anneal_table(L2, gen, None, 20, time_limit=None, resume=str(tmp_path / "run_9.npz"), **kw)
    assert np.array_equal(best2, best) and np.array_equal(L2.base, full_L.base)
    assert (tr2.steps, tr2.accepted, tr2.exact_evals) == (tr.steps, tr.accepted, tr.exact_evals)
    assert tr2.best == tr.best and tr2.final_best == tr.final_best
    if t0 > 0:
        keys = [_key(N, M, b) for b in L2.bases]
        assert any(b > a for a, b in zip(keys, keys[1:]))      # an uphill move after the resume


def test_lifted_annealing_log_lines(tmp_path):
    import json
    N, M, D = G.cyclic_lift(24, 4, 4, 2)
    gen = lambda t, c, s: G.gen_lift_moves(N, M, t, c, s)  # noqa: E731
    log = tmp_path / "run.jsonl"
    _, tr = A._anneal_table(OracleLift(N, M), gen, D, 15, seed=5, exact=4, t0_frac=0.05, t_end=1e-6,
                            target=None, time_limit=None, log=str(log))
    lines = [json.loads(x) for x in log.read_text().splitlines()]
    assert 0 < len(lines) <= tr.accepted
    assert [x["step"] for x in lines] == sorted(x["step"] for x in lines)
    assert min(x["best_aspl"] for x in lines) == tr.final_best
    assert all(x["best_aspl"] <= x["aspl"] for x in lines)


def test_checkpoint_resume_keeps_wall_time_and_hit(tmp_path):
    """A snapshot is written atomically (temporary file renamed into place), takes
    the path with or without ".npz", records the elapsed wall time and the
    time-to-target state, and a resumed run that had already reached its target
    stops at once; a snapshot of another lift's shape is refused."""
    N, M, D = G.cyclic_lift(24, 4, 4, 2)
    gen = lambda t, c, s: G.gen_lift_moves(N, M, t, c, s)  # noqa: E731
    kw = dict(seed=5, exact=4, t0_frac=0.05, t_end=1e-6, time_limit=None)
    ck = str(tmp_path / "snap")          # no suffix: written as snap.npz
    _, tr = A._anneal_table(OracleLift(N, M), gen, D, 12, target=10.0, checkpoint=ck, **kw)
    assert tr.hit_step == 1 and (tmp_path / "snap.npz").exists()
    assert not list(tmp_path.glob("*.tmp.npz"))
    z = np.load(tmp_path / "snap.npz")
    assert float(z["elapsed"]) >= 0.0 and int(z["hit_step"]) == 1
    for name in (ck, ck + ".npz"):
        L2 = OracleLift(N, M)
        _, tr2 = A._anneal_table(L2, gen, None, 12, target=10.0, resume=name, **kw)
        assert tr2.hit_step == 1 and tr2.steps == tr.steps and len(L2.bases) == 1
        assert tr2.wall >= float(z["elapsed"])
    N2, M2, D2 = G.cyclic_lift(30, 4, 4, 2)
    with pytest.raises(ValueError):
        A._anneal_table(OracleLift(N2, M2), lambda t, c, s: G.gen_lift_moves(N2, M2, t, c, s), D2, 12,
                        target=None, resume=ck, **kw)
