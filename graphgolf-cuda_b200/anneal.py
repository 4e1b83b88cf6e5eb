"""Batched simulated annealing of a regular graph, with or without the surrogate.

The reference's annealer proposes one move, scores it with one calculator call
and accepts it by Metropolis (cppcode/annealing.cpp:397-443).  Here every step
scores a batch of 2-opt proposals exactly in one launch (gg_batch_eval):

  plain      `exact` uniform random proposals;
  surrogate  `pool` uniform random proposals ranked by the surrogate network;
             the `exact - explore` best-ranked plus `explore` random ones of the
             rest are scored exactly.  The exact results train the network online
             (one Adam step per annealing step), so it learns on the annealer's
             own (swap, exact ΔASPL) pairs.

Acceptance uses only exact values: the best proposal of the step (smallest
diameter, then smallest total) replaces the current graph if it lowers the
diameter, or keeps it and lowers the total, or else with probability
exp(-ΔASPL / T); a larger diameter is never accepted (cppcode/annealing.cpp:407-412).
T follows a geometric schedule from T0 = t0_frac * ASPL(start) to t_end.
"""
from __future__ import annotations

import json
import os
import math
import time
from dataclasses import dataclass, field

import numpy as np

import graphgolf as G

HIST_K = 4


def features(batch, bid):
    """Per-vertex inputs of the surrogate: the distance histogram to depth 4,
    standardised over the graph, and a constant."""
    h = batch.vertex_hist(bid, HIST_K).astype(np.float64)
    h = (h - h.mean(0)) / (h.std(0) + 1e-6)
    return np.concatenate([h, np.ones((len(h), 1))], axis=1).astype(np.float32)


@dataclass
class Trace:
    times: list = field(default_factory=list)      # wall seconds at each improvement of the best
    best: list = field(default_factory=list)       # best ASPL after each improvement
    steps: int = 0
    accepted: int = 0
    exact_evals: int = 0
    train_pairs: int = 0
    wall: float = 0.0
    final_best: float = math.inf
    hit_time: float | None = None                  # wall seconds when best <= target
    hit_step: int | None = None
    hit_train_pairs: int | None = None             # pairs the network had trained on at the hit
    spearman: float | None = None                  # surrogate: rank correlation on a fresh sample


def rank_correlation(x, y):
    """Spearman rank correlation (average ranks for ties)."""
    def ranks(v):
        v = np.asarray(v, dtype=np.float64)
        order = np.argsort(v, kind="stable")
        r = np.empty(len(v))
        r[order] = np.arange(len(v), dtype=np.float64)
        _, inv, cnt = np.unique(v, return_inverse=True, return_counts=True)
        sums = np.bincount(inv, weights=r)
        return (sums / cnt)[inv]
    rx, ry = ranks(x), ranks(y)
    rx -= rx.mean()
    ry -= ry.mean()
    den = math.sqrt(float((rx * rx).sum() * (ry * ry).sum()))
    return float((rx * ry).sum() / den) if den > 0 else 0.0


def anneal(adj0, steps, *, seed=1, exact=32, pool=4096, explore=8, surrogate=False, t0_frac=1e-3,
           t_end=1e-6, target=None, time_limit=None, lr=2e-3, feature_every=32, train_every=2,
           device=0, spearman_sample=0, min_train_pairs=0):
    """Anneal from `adj0` (n x d simple regular graph).  Returns (best_adj, Trace).
    With a `target`, the run stops at the first step after which the best ASPL is
    at or below it and the network has trained on at least `min_train_pairs` pairs;
    that step and its wall time are the hit.
    With the surrogate, the adjacency it passes messages over follows every
    accepted move; its distance-histogram features are recomputed every
    `feature_every` accepted moves (one 2-opt changes them only locally)."""
    adj = np.array(adj0, dtype=np.int32, copy=True)
    n, d = adj.shape
    npairs = n * (n - 1)
    b = G.Batch(device)
    bid = b.add_base(adj)
    me = np.array([(bid, -1, -1, -1, -1, 0)], dtype=G.SWAP_DTYPE)
    r0 = b.eval(me)[0]
    if not r0["connected"]:
        raise ValueError("start graph is disconnected")
    cur_total, cur_diam = int(r0["total"]), int(r0["levels"])
    best_aspl, best_adj = cur_total / npairs, adj.copy()
    T0 = t0_frac * best_aspl
    rng = np.random.default_rng(seed)
    net = None
    scale = None
    feats = None
    pending = []
    if surrogate:
        net = G.Surrogate(n, d, HIST_K + 1, seed=seed)
        feats = features(b, bid)
        net.set_graph(adj, feats)
    tr = Trace()
    t_start = time.perf_counter()
    tr.times.append(0.0)
    tr.best.append(best_aspl)
    for i in range(steps):
        T = T0 * (t_end / T0) ** (i / max(steps - 1, 1))
        step_seed = (seed << 32) ^ i
        if net is None:
            props = G.gen_swaps(adj, bid, exact, step_seed)
        else:
            cand = G.gen_swaps(adj, bid, pool, step_seed)
            pred = net.predict(cand)
            order = np.argsort(pred, kind="stable")
            top = order[:exact - explore]
            rest = order[exact - explore:]
            pick = np.concatenate([top, rng.choice(rest, explore, replace=False)])
            props = cand[pick]
        res = b.eval(props)
        tr.exact_evals += len(props)
        ok = res["connected"] == 1
        totals = res["total"].astype(np.int64)
        if net is not None:
            # label the exact results and train every `train_every` steps on the
            # pairs gathered since the last update (one backward over the graph)
            delta = (totals - cur_total).astype(np.float64) / npairs
            if scale is None and ok.any():
                scale = max(float(np.std(delta[ok])), 1e-12)
            pending.append((props, (delta / scale).astype(np.float32), ok.astype(np.int32)))
            if len(pending) >= train_every:
                net.train(np.concatenate([p[0] for p in pending]), np.concatenate([p[1] for p in pending]),
                          lr=lr, mask=np.concatenate([p[2] for p in pending]))
                tr.train_pairs += int(sum(p[2].sum() for p in pending))
                pending.clear()
        if ok.any():
            key = np.where(ok, res["levels"].astype(np.int64) * (1 << 40) + totals, np.iinfo(np.int64).max)
            k = int(np.argmin(key))
            dy, ty = int(res["levels"][k]), int(totals[k])
            dA = (ty - cur_total) / npairs
            accept = dy < cur_diam or (dy == cur_diam and (dA < 0 or rng.random() < math.exp(-dA / T)))
            if dy > cur_diam:
                accept = False
            if accept:
                adj = G.apply_swap(adj, props[k])
                b.set_base(bid, adj)
                cur_total, cur_diam = ty, dy
                tr.accepted += 1
                if net is not None:
                    if tr.accepted % feature_every == 0:
                        feats = features(b, bid)
                    net.set_graph(adj, feats)
                aspl = cur_total / npairs
                if aspl < best_aspl:
                    best_aspl, best_adj = aspl, adj.copy()
                    tr.times.append(time.perf_counter() - t_start)
                    tr.best.append(best_aspl)
        tr.steps = i + 1
        # the target counts as reached once the best is at or below it AND the
        # network has trained on at least min_train_pairs exact pairs
        if (target is not None and tr.hit_time is None and best_aspl <= target and
                tr.train_pairs >= min_train_pairs):
            tr.hit_time, tr.hit_step = time.perf_counter() - t_start, i + 1
            tr.hit_train_pairs = tr.train_pairs
            break
        if time_limit is not None and time.perf_counter() - t_start > time_limit:
            break
    tr.wall = time.perf_counter() - t_start
    tr.final_best = best_aspl
    if net is not None and spearman_sample > 0:
        # after the timed run: predicted vs exact change of the total on a fresh
        # uniform sample of proposals of the final graph
        cand = G.gen_swaps(adj, bid, spearman_sample, (seed << 32) ^ 0x5eed)
        pred = net.predict(cand)
        r = b.eval(cand)
        ok = r["connected"] == 1
        if ok.sum() > 2:
            tr.spearman = rank_correlation(pred[ok], r["total"][ok].astype(np.float64) - cur_total)
    b.close()
    if net is not None:
        net.close()
    return best_adj, tr


def npz_path(path):
    """Checkpoint file name: `path` with ".npz" appended unless it ends so already
    (np.savez would append it anyway; resume= then takes either spelling)."""
    return path if path.endswith(".npz") else path + ".npz"


def save_checkpoint(path, *, table, best, cur_total, cur_diam, best_aspl, T0, step, rng, tr, elapsed):
    """Snapshot of a lifted annealing run after `step` steps (an .npz): current and
    best tables, exact counts, start temperature, RNG state, trace, the run's wall
    seconds so far and its time-to-target state.  Written to a temporary file and
    renamed into place, so a crash mid-write leaves the previous snapshot intact."""
    final = npz_path(path)
    tmp = final[:-4] + ".tmp.npz"
    np.savez(tmp, table=table, best=best, cur_total=np.int64(cur_total), cur_diam=np.int64(cur_diam),
             best_aspl=np.float64(best_aspl), T0=np.float64(T0), step=np.int64(step),
             rng=np.array(json.dumps(rng.bit_generator.state)), times=np.array(tr.times, dtype=np.float64),
             best_trace=np.array(tr.best, dtype=np.float64), accepted=np.int64(tr.accepted),
             exact_evals=np.int64(tr.exact_evals), elapsed=np.float64(elapsed),
             hit_time=np.float64(-1.0 if tr.hit_time is None else tr.hit_time),
             hit_step=np.int64(-1 if tr.hit_step is None else tr.hit_step))
    os.replace(tmp, final)


def _anneal_table(L, gen, table0, steps, *, seed, exact, t0_frac, t_end, target, time_limit, checkpoint=None,
                  checkpoint_every=0, resume=None, log=None):
    """Batched annealing of one lift table with handle L (a G.Lift) and move
    generator gen(table, count, seed).  t0_frac == 0: hill climbing (only moves
    that lower the diameter, or keep it and lower the total).  `checkpoint`: a path
    written every `checkpoint_every` steps and at the end ("{step}" in it is replaced
    by the step count); `resume`: a checkpoint to continue from (the same seed,
    schedule and step count continue the same run).  `log`: a path that gets one
    JSON line per accepted move that changes the ASPL or the diameter (step, best
    ASPL, current ASPL, diameter, temperature, wall seconds), the fields of the reference's
    --log lines (cppcode/annealing.cpp:323-326, 424)."""
    scale, npairs = L.N // L.M, L.N * (L.N - 1)
    tr = Trace()
    rng = np.random.default_rng(seed)
    first = 0
    elapsed0 = 0.0
    if resume is not None:
        ck = np.load(npz_path(resume), allow_pickle=False)
        table, best = np.array(ck["table"], dtype=np.int32), np.array(ck["best"], dtype=np.int32)
        # the snapshot must fit this run's lift handle (and its start table, if given)
        if table0 is not None:
            want = np.asarray(table0).shape
        elif hasattr(L, "degree"):
            ax = getattr(L, "axes", 1)
            want = (L.M, L.degree) if ax == 1 else (L.M, L.degree, ax)
        else:
            want = (L.M,) + table.shape[1:]
        if table.shape != want or best.shape != want:
            raise ValueError(f"checkpoint tables have shape {table.shape}, this run's tables {want}")
        cur_total, cur_diam = int(ck["cur_total"]), int(ck["cur_diam"])
        best_aspl, T0, first = float(ck["best_aspl"]), float(ck["T0"]), int(ck["step"])
        rng.bit_generator.state = json.loads(str(ck["rng"]))
        tr.times, tr.best = list(ck["times"]), list(ck["best_trace"])
        tr.accepted, tr.exact_evals, tr.steps = int(ck["accepted"]), int(ck["exact_evals"]), first
        elapsed0 = float(ck["elapsed"]) if "elapsed" in ck.files else (tr.times[-1] if tr.times else 0.0)
        if "hit_step" in ck.files and int(ck["hit_step"]) >= 0:
            tr.hit_time, tr.hit_step = float(ck["hit_time"]), int(ck["hit_step"])
        L.set_base(table)
    else:
        table = np.array(table0, dtype=np.int32, copy=True)
        L.set_base(table)
        r0 = L.eval(np.zeros(1, dtype=G.LIFT_EDIT_DTYPE))[0]
        if not r0["connected"]:
            raise ValueError("start lift is disconnected")
        cur_total, cur_diam = int(r0["total"]), int(r0["levels"])
        best_aspl, best = cur_total * scale / npairs, table.copy()
        T0 = t0_frac * best_aspl
        tr.times.append(0.0)
        tr.best.append(best_aspl)
    # wall time continues from the snapshot's elapsed seconds
    t_start = time.perf_counter() - elapsed0

    def snapshot(step):
        if checkpoint is not None:
            save_checkpoint(checkpoint.format(step=step), table=table, best=best, cur_total=cur_total, cur_diam=cur_diam,
                            best_aspl=best_aspl, T0=T0, step=step, rng=rng, tr=tr,
                            elapsed=time.perf_counter() - t_start)

    # a run resumed after it had already reached its target stops at once
    done = target is not None and tr.hit_time is not None
    for i in range(first, steps if not done else first):
        T = T0 * (t_end / T0) ** (i / max(steps - 1, 1)) if T0 > 0 else 0.0
        moves = gen(table, exact, (seed << 32) ^ i)
        res = L.eval(moves)
        tr.exact_evals += len(moves)
        ok = res["connected"] == 1
        if ok.any():
            totals = res["total"].astype(np.int64)
            key = np.where(ok, res["levels"].astype(np.int64) * (1 << 40) + totals, np.iinfo(np.int64).max)
            k = int(np.argmin(key))
            dy, ty = int(res["levels"][k]), int(totals[k])
            dA = (ty - cur_total) * scale / npairs
            accept = dy < cur_diam or (dy == cur_diam and (dA < 0 or (T > 0 and rng.random() < math.exp(-dA / T))))
            if accept:
                table = G.apply_lift_edit(table, moves[k])
                L.set_base(table)
                changed = ty != cur_total or dy != cur_diam
                cur_total, cur_diam = ty, dy
                tr.accepted += 1
                aspl = cur_total * scale / npairs
                if aspl < best_aspl:
                    best_aspl, best = aspl, table.copy()
                    tr.times.append(time.perf_counter() - t_start)
                    tr.best.append(best_aspl)
                    if target is not None and tr.hit_time is None and best_aspl <= target:
                        tr.hit_time, tr.hit_step = tr.times[-1], i + 1
                if log is not None and changed:
                    with open(log, "a") as f:
                        f.write(json.dumps({"step": i + 1, "best_aspl": best_aspl, "aspl": aspl, "diameter": dy,
                                            "temp": T, "wall_s": time.perf_counter() - t_start}) + "\n")
        tr.steps = i + 1
        if checkpoint_every and tr.steps % checkpoint_every == 0:
            snapshot(tr.steps)
        if target is not None and tr.hit_time is not None:
            break
        if time_limit is not None and time.perf_counter() - t_start > time_limit:
            break
    snapshot(tr.steps)
    tr.wall = time.perf_counter() - t_start
    tr.final_best = best_aspl
    return best, tr


def anneal_lift(N, M, diffs0, steps, *, seed=1, exact=32, t0_frac=1e-3, t_end=1e-6, target=None,
                time_limit=None, device=0, **ck):
    """Anneal a cyclic lift in part form (the reference's main annealer,
    cppcode/annealing.cpp:396-443, on the moves of :112-197).  Every step draws
    `exact` moves (gg_gen_lift_moves: new lift shifts and orbit 2-opts) and scores
    them all in one launch (gg_lift_eval); the best (smallest diameter, then
    smallest total) goes through the same acceptance rule as anneal().  ASPL is the
    reference's total * (N/M) / (N(N-1)).  t0_frac = 0 climbs (HillClimb.cpp).
    Keyword `checkpoint`, `checkpoint_every`, `resume`: snapshots of the run (the
    reference keeps only its best solution, cppcode/annealing.cpp:431-452); `log`: a
    JSON-lines progress log (see _anneal_table).
    Returns (best_diffs, Trace)."""
    diffs = np.asarray(diffs0, dtype=np.int32).reshape(M, -1)
    L = G.Lift(N, M, diffs.shape[1], device)
    try:
        return _anneal_table(L, lambda t, c, s: G.gen_lift_moves(N, M, t, c, s), diffs, steps, seed=seed,
                             exact=exact, t0_frac=t0_frac, t_end=t_end, target=target, time_limit=time_limit, **ck)
    finally:
        L.close()


def anneal_piece(Nx, Ny, Mx, My, vals0, steps, *, seed=1, exact=32, t0_frac=1e-3, t_end=1e-6, target=None,
                 time_limit=None, device=0, **ck):
    """The same for a 2-D torus lift (cppcode/pieceannealing.cpp; vals [Mx*My, d, 2]);
    t0_frac = 0 is the hill climb of pieceHillClimb.cpp."""
    vals = np.asarray(vals0, dtype=np.int32).reshape(Mx * My, -1, 2)
    L = G.Lift.piece(Nx, Ny, Mx, My, vals.shape[1], device)
    try:
        return _anneal_table(L, lambda t, c, s: G.gen_piece_moves(Nx, Ny, Mx, My, t, c, s), vals, steps,
                             seed=seed, exact=exact, t0_frac=t0_frac, t_end=t_end, target=target,
                             time_limit=time_limit, **ck)
    finally:
        L.close()


def anneal_box(Nx, Ny, Nz, Mx, My, Mz, vals0, steps, *, seed=1, exact=32, t0_frac=0.0, t_end=1e-6,
               target=None, time_limit=None, device=0, **ck):
    """The same for a 3-D torus lift (vals [Mx*My*Mz, d, 3]); the default t0_frac = 0
    is the hill climb of cppcode/boxHillClimb.cpp."""
    vals = np.asarray(vals0, dtype=np.int32).reshape(Mx * My * Mz, -1, 3)
    L = G.Lift.box(Nx, Ny, Nz, Mx, My, Mz, vals.shape[1], device)
    try:
        return _anneal_table(L, lambda t, c, s: G.gen_box_moves(Nx, Ny, Nz, Mx, My, Mz, t, c, s), vals, steps,
                             seed=seed, exact=exact, t0_frac=t0_frac, t_end=t_end, target=target,
                             time_limit=time_limit, **ck)
    finally:
        L.close()


def time_to(trace, target):
    """Wall seconds at which a finished trace's best first reached `target`."""
    for t, v in zip(trace.times, trace.best):
        if v <= target:
            return t
    return None


@dataclass
class InitTemp:
    temp: float           # T0 in the reference's unit: a change of the total distance (ΔASPL * N(N-1))
    temp_aspl: float      # the same T0 as a change of ASPL (the unit anneal() uses)
    avg: float            # mean uphill change of the total distance
    uphill: int           # proposals that raised the total (connected ones only)
    proposals: int
    ms: float             # device time of the batched evaluation


def initial_temperature(n, d, *, graphs=100, neighbours=100, seed=1, accept=0.4, device=0, bases=None):
    """Initial annealing temperature, restating cppcode/initTemp.cpp:399-430 on the
    batched evaluator: for `graphs` random d-regular graphs and `neighbours` 2-opt
    proposals of each, the mean increase of the total distance over the proposals
    that are connected and uphill, avg; T0 = -avg / ln(accept) (the reference
    prints -avg/log(0.4), initTemp.cpp:425-430).  The reference sums ASPL
    differences and multiplies by N(N-1); here the same quantity is summed exactly
    as integer totals.  All base graphs and proposals go through one batched
    evaluation instead of graphs * (neighbours + 1) calculator calls.

    `bases` replaces the random graphs (each an n x d adjacency)."""
    if bases is None:
        bases = [G.random_regular(n, d, seed * 1000003 + k) for k in range(graphs)]
    b = G.Batch(device)
    try:
        ids = [b.add_base(a) for a in bases]
        none = np.zeros(len(ids), dtype=G.SWAP_DTYPE)
        none["base"] = ids
        none["a"] = -1
        props = [G.gen_swaps(a, i, neighbours, (seed << 20) ^ k) for k, (a, i) in enumerate(zip(bases, ids))]
        res = b.eval(np.concatenate([none] + props))
        ms = b.last_ms()
    finally:
        b.close()
    k = len(ids)
    base_total = res["total"][:k].astype(np.int64)
    base_ok = res["connected"][:k] == 1
    cand = res[k:]
    owner = np.repeat(np.arange(k), neighbours)
    delta = cand["total"].astype(np.int64) - base_total[owner]
    up = (cand["connected"] == 1) & base_ok[owner] & (delta > 0)
    cnt = int(up.sum())
    if cnt == 0:
        raise ValueError("no connected uphill proposal")
    avg = int(delta[up].sum()) / cnt
    temp = -avg / math.log(accept)
    npairs = n * (n - 1)
    return InitTemp(temp=temp, temp_aspl=temp / npairs, avg=avg, uphill=cnt, proposals=len(cand), ms=ms)


def initial_temperature_piece(Nx, Ny, Mx, My, d, *, graphs=100, neighbours=100, seed=1, accept=0.4, device=0,
                              bases=None, make_lift=None):
    """Initial temperature for 2-D torus lifts, restating cppcode/pieceinitTemp.cpp:211-260
    on the batched lift evaluator: for `graphs` random pieces (tile Mx x My, lifted
    Nx x Ny, degree d) and `neighbours` lift moves of each (gg_gen_piece_moves, the
    moves of :113-209), the mean increase of the total distance over the connected
    uphill moves; T0 = -avg / ln(accept) (:253-258).  Each piece and its moves are one
    launch.  The reference's filter `fy != 1e9` (:249) does not catch
    cudaASPLpiece's disconnected sentinel 1e8, so it counts disconnected neighbours
    as uphill moves of about 1e8; here, as in initial_temperature, only connected
    neighbours of connected pieces count.  The totals are exact integers (ASPL
    differences times N(N-1) in the reference).

    `bases` replaces the random pieces (each a [Mx*My, d, 2] table); `make_lift`
    replaces the evaluator factory (G.Lift.piece)."""
    N = Nx * Ny
    if bases is None:
        bases = [G.piece_lift(Mx, My, Nx // Mx, Ny // My, d, seed * 1000003 + k)[4] for k in range(graphs)]
    if make_lift is None:
        make_lift = lambda: G.Lift.piece(Nx, Ny, Mx, My, d, device)  # noqa: E731
    L = make_lift()
    deltas, proposals, ms = [], 0, 0.0
    try:
        for k, T in enumerate(bases):
            L.set_base(T)
            moves = G.gen_piece_moves(Nx, Ny, Mx, My, T, neighbours, (seed << 20) ^ k)
            res = L.eval(np.concatenate([np.zeros(1, dtype=G.LIFT_EDIT_DTYPE), moves]))
            ms += L.last_ms() if hasattr(L, "last_ms") else 0.0
            proposals += len(moves)
            if not res["connected"][0]:
                continue
            cand = res[1:]
            delta = cand["total"].astype(np.int64) - int(res["total"][0])
            deltas.append(delta[(cand["connected"] == 1) & (delta > 0)])
    finally:
        if hasattr(L, "close"):
            L.close()
    up = np.concatenate(deltas) if deltas else np.zeros(0, dtype=np.int64)
    if len(up) == 0:
        raise ValueError("no connected uphill proposal")
    # the totals are over the M representatives: scale to all N sources
    avg = int(up.sum()) * (N // (Mx * My)) / len(up)
    temp = -avg / math.log(accept)
    return InitTemp(temp=temp, temp_aspl=temp / (N * (N - 1)), avg=avg, uphill=len(up), proposals=proposals, ms=ms)
