"""Work split over the ranks of a torch.distributed group.

One evaluation: the sources of an evaluation are independent (each BFS column
of the bitset is its own search), so a graph's all-pairs total is the sum of the
totals of any partition of its sources.  Each rank evaluates a contiguous source
range with gg_eval (gg_eval_opts.src_begin/src_end) and one all-reduce combines
the exact counts: total, reached (sum), levels (max), capped (max).

A population of candidates: candidates are independent graphs, so each rank
scores a contiguous slice with a batched evaluator (gg_batch_eval,
gg_lift_eval) and one all-gather gives every rank all results in order.

On GPUs the group is NCCL over NVLink; the same code runs on CPU ranks with gloo.
"""
from __future__ import annotations


def shard(n_sources, rank, world, align=32):
    """Contiguous source range of `rank` (starts aligned to `align`, so that the
    WVC bit positions of every shard match the unsplit evaluation)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    blocks = (n_sources + align - 1) // align
    b0 = blocks * rank // world
    b1 = blocks * (rank + 1) // world
    return min(b0 * align, n_sources), min(b1 * align, n_sources)


def combine(part, pairs, group=None):
    """All-reduce the exact counts of one rank's part (a gg_eval result dict)."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    s = torch.tensor([part["total"], part["reached"], part["level_steps"]], dtype=torch.int64, device=dev)
    m = torch.tensor([part["levels"], part["capped"]], dtype=torch.int64, device=dev)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    total, reached, steps = (int(x) for x in s.tolist())
    levels, capped = (int(x) for x in m.tolist())
    return {"total": total, "reached": reached, "pairs": pairs, "levels": levels, "capped": capped,
            "connected": int(not capped and reached == pairs), "level_steps": steps}


def eval_sharded(engine, table, n_sources, n_vertices, max_levels=0, group=None):
    """Evaluate `table` on `engine` with this rank's share of the sources and
    combine over `group`.  Returns the combined exact counts."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard(n_sources, rank, world)
    if hi > lo:
        part = engine.eval(table, max_levels=max_levels, src_range=(lo, hi))
    else:
        part = {"total": 0, "reached": 0, "levels": 0, "capped": 0, "level_steps": 0}
    return combine(part, n_sources * n_vertices, group)


def eval_candidates_sharded(evaluator, cands, group=None):
    """Score `cands` (an array of candidate records) split over the ranks of
    `group`: this rank calls `evaluator` (e.g. Batch.eval or Lift.eval) on its
    contiguous slice, and one all-gather returns every candidate's result
    (CAND_RESULT_DTYPE records, in the order of `cands`) on every rank."""
    import numpy as np
    import torch
    import torch.distributed as dist
    from graphgolf import CAND_RESULT_DTYPE
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n = len(cands)
    bounds = [(n * r // world, n * (r + 1) // world) for r in range(world)]
    lo, hi = bounds[rank]
    width = max(h - l for l, h in bounds)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    buf = torch.full((max(width, 1), 4), -1, dtype=torch.int64, device=dev)
    if hi > lo:
        mine = np.asarray(evaluator(cands[lo:hi]), dtype=CAND_RESULT_DTYPE)
        rows = np.stack([mine["total"].astype(np.int64), mine["reached"].astype(np.int64),
                         mine["levels"].astype(np.int64), mine["connected"].astype(np.int64)], axis=1)
        buf[:hi - lo] = torch.from_numpy(rows).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.zeros(n, dtype=CAND_RESULT_DTYPE)
    for (l, h), part in zip(bounds, parts):
        rows = part[:h - l].cpu().numpy()
        out["total"][l:h] = rows[:, 0].astype(np.uint64)
        out["reached"][l:h] = rows[:, 1].astype(np.uint64)
        out["levels"][l:h] = rows[:, 2]
        out["connected"][l:h] = rows[:, 3]
    return out
