#!/usr/bin/env python
"""Throughput of the exact ASPL/diameter engine (ASPL evaluations per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one exact all-pairs evaluation (uint64 total distance + diameter) of
one graph.  Default workload: a seeded random simple connected 8-regular graph
on n = 65536 vertices (int32 adjacency), evaluated through the plain-graph
calculator with the reference's level cap of 199 (cudaASPLgraph.cu:163).

* value      evals/s with the adjacency resident in HBM (gg_eval_device),
             device-timed with CUDA events on the launching stream, K steps,
             max over ranks.  A 256 MiB write flushes the L2 before every timed
             step (the engine keeps each 4096-source batch's bitsets, 96 MiB, in
             the L2 by design, so the flush is what makes steps independent).
* e2e        the same metric through the reference-facing C-ABI call
             gg_graph_calc with a host adjacency: H2D of the table, the
             evaluation, D2H of the level counters, every step.
* parity     rank 0 compares the timed result with the oracle's BFS from every
             source of the same graph (the cpu_baseline run) and fails on any
             difference; the line says "parity": "exact".
* roofline   bound "hbm": DRAM bytes one evaluation moves (ncu dram__bytes of its
             launches, profiles/traffic.json) / the evaluation's CUDA-event time,
             against MEASURED_PEAKS.json hbm_gbs.  Beside it: "l2_gather", the
             live ceiling of the kernel's access pattern (gg_gather_peak: random
             512-byte row gathers from L2-resident arrays, one dense BFS level per
             pass), and "algorithmic", the bytes-per-level count N*d*4 + N*(d+2)*S/8.
* cpu_baseline  the oracle port (oracle/gg_oracle.c, a restatement of
             cpuASPLqueue) over all host cores; rank 0, N = 1.

Multi-GPU: `--gpus N` without torchrun starts N ranks itself (torch.distributed.run,
NCCL).  Default workload: weak scaling, every rank evaluates its own graph (seed +
rank), one MAX all-reduce of the timings.  `regular_n65536_d8_sharded`: strong
scaling, the ranks split the sources of the one graph and one NCCL all-reduce
combines the exact counts every step (graphgolf-cuda_b200/distributed.py).
``--impl reference`` times the CPU reference path on rank 0 and, beside it, the
reference's own cudaASPLgraph built for this GPU (oracle/_ref), on the same graph
read from tests/golden (no engine library loaded).
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "graphgolf-cuda_b200")]

WORKLOADS = {
    "regular_n65536_d8": dict(form="graph", n=65536, d=8, seed=1),
    # strong scaling: the sources of the one graph split over the ranks, exact
    # counts combined by an NCCL all-reduce every step
    "regular_n65536_d8_sharded": dict(form="graph", n=65536, d=8, seed=1, sharded=True),
    "regular_n4096_d16": dict(form="graph", n=4096, d=16, seed=1),
    "lift_m1024_g32_d12": dict(form="part", m=1024, g=32, d=12, seed=1),
    # batched 2-opt candidates: 2048 on a 6-regular n=1024 base + 512 on a
    # 4-regular n=3000 base, one launch per step
    "batch_2opt_2048x1024d6_512x3000d4": dict(form="batch", seed=11),
    # surrogate-ranked vs plain batched annealing: random 8-regular n=4096 start,
    # geometric schedule 1e-3*ASPL -> 1e-6 over 1e5 steps, 32 exact scores per step
    "anneal_n4096_d8_time_to_target": dict(form="anneal", n=4096, d=8, seed=1, steps=100000),
    # one 2-opt move of a random 8-regular n=65536 graph per step, scored exactly by
    # searching again only from the affected sources (gg_inc_eval)
    "incremental_n65536_d8": dict(form="incremental", n=65536, d=8, seed=1),
    # 256 shift / orbit 2-opt moves of a random cyclic lift (m=1024 orbits, g=32,
    # degree 12, N=32768) per step, all scored in one launch (gg_lift_eval)
    "lift_moves_256_m1024_g32_d12": dict(form="liftbatch", m=1024, g=32, d=12, seed=1, cands=256),
    # the same for a 2-D torus lift (piece form): tile 32 x 32, lifted 256 x 128
    # (N=32768), degree 8
    "piece_moves_256_32x32_x8x4_d8": dict(form="liftbatch", kind="piece", Mx=32, My=32, kx=8, ky=4, d=8, seed=1,
                                          cands=256),
}
METRIC = "ASPL evals/s"
UNIT = "evals/s"


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        j = json.load(open(p))
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


GOLDEN = os.path.join(ROOT, "tests", "golden")


def fixture_of(w, seed):
    """Committed input graph of a plain-graph workload (tests/golden), or None."""
    if w["form"] != "graph":
        return None
    p = os.path.join(GOLDEN, f"regular_n{w['n']}_d{w['d']}_seed{seed}.npy")
    if not os.path.exists(p):
        return None
    import numpy as np
    return np.load(p).astype(np.int32)


L2_NOTE = "GPU steps: a 256 MiB write flushes the L2 before every timed step"


def graph_config(workload):
    """`config` of the plain-graph workloads, the same dict in both arms."""
    w = WORKLOADS[workload]
    return {"workload": workload, "n": w["n"], "degree": w["d"], "seed": w["seed"],
            "input": f"tests/golden/regular_n{w['n']}_d{w['d']}_seed{w['seed']}.npy", "l2": L2_NOTE}


def make_workload(name, rank):
    import graphgolf as G
    w = WORKLOADS[name]
    seed = w["seed"] + (0 if w.get("sharded") else 1000 * rank)
    if w["form"] == "graph":
        adj = G.random_regular(w["n"], w["d"], seed)
        fx = fixture_of(w, seed)
        if fx is not None and not (fx.shape == adj.shape and (fx == adj).all()):
            raise SystemExit(f"generator output differs from the committed fixture for seed {seed}")
        return dict(form="graph", N=w["n"], d=w["d"], table=adj, S=w["n"], M=w["n"])
    N, M, diffs = G.cyclic_lift(w["m"], w["g"], w["d"], seed)
    return dict(form="part", N=N, d=w["d"], table=diffs, S=M, M=M)


def algorithmic_bytes(wl, res, batch_bits):
    """sum over batches and executed levels of N*d*4 + N*(d+2)*S_b/8."""
    N, d = wl["N"], wl["d"]
    n_src = res["n_sources"]
    nb = res["batches"]
    per_level_adj = N * d * 4
    # equal-width batches except the last; level_steps is summed over batches,
    # so use the mean width per executed level
    mean_bits = n_src / nb
    return res["level_steps"] * (per_level_adj + N * (d + 2) * mean_bits / 8.0)


class Clocks:
    """nvidia-smi sampler for the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = open(os.devnull, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.15)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.12)
        self.proc.terminate()
        try:
            text, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            text = ""
        rows = [r for r in csv.reader(io.StringIO(text)) if len(r) >= 8]
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if "Active" in r[4 + k] and "Not" not in r[4 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def gpu_uuid(dev):
    import torch
    try:
        u = torch.cuda.get_device_properties(dev).uuid
        s = str(u)
        return s if s.startswith("GPU-") else "GPU-" + s
    except Exception:
        return dev


def cpu_sample(wl, target_s=8.0, threads=0, full=False):
    """Oracle port over all host cores -> (evals/s record, the oracle's BFS or None).
    full: BFS from every source (one whole evaluation, also the parity check);
    else a bounded source sample of about target_s seconds, scaled."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    if wl["form"] == "graph":
        adj = wl["table"]
    else:
        adj = O.expand_part(wl["N"], wl["M"], wl["table"])
    rp, col = O.pull_to_push_csr(adj)
    n_src_all = wl["S"]
    threads = threads or os.cpu_count() or 1
    s = n_src_all if full else min(n_src_all, max(threads, 32))
    while True:
        t0 = time.perf_counter()
        r = O.bfs(rp, col, np.arange(s), threads=threads)
        dt = time.perf_counter() - t0
        if dt >= target_s * 0.5 or s >= n_src_all:
            break
        s = min(n_src_all, int(s * max(2.0, target_s / max(dt, 1e-3) * 0.9)))
    per_eval = dt * n_src_all / s
    what = (f"one whole evaluation: BFS from all {n_src_all} sources ({dt:.2f} s)" if s == n_src_all else
            f"BFS from {s} of {n_src_all} sources ({dt:.2f} s), scaled to one evaluation")
    rec = {"value": 1.0 / per_eval, "unit": UNIT, "cores": threads, "kind": "port", "sample": what}
    return rec, (r if s == n_src_all else None)


def reference_gpu_graph(adj, steps=5):
    """The reference's own cudaASPLgraph::calc (cudacode/cudaASPLgraph.cu:141-199),
    compiled from the reference sources for this GPU into oracle/_ref, on `adj`:
    host clock around each blocking call, after one warm-up call."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.RefGPU.available("graph"):
        return {"unavailable": "oracle/_ref/libref_graph.so not built (make -C oracle ref)"}
    import torch
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    n, d = adj.shape
    R = O.RefGPU("graph").create(n, d, 0)
    try:
        res = R.graph_calc(adj)
        ts = []
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        for _ in range(steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r2 = R.graph_calc(adj)
            ts.append(time.perf_counter() - t0)
            if r2 != res:
                raise SystemExit("reference cudaASPLgraph is not deterministic")
    finally:
        R.close()
    ms = 1000.0 * statistics.median(ts)
    return {"value": 1000.0 / ms, "unit": UNIT, "ms_per_eval": ms, "calls": steps,
            "result": {"diameter": res[0], "total": res[1]},
            "what": "reference cudaASPLgraph::calc built for sm_100a from the reference source "
                    "(oracle/_ref/libref_graph.so), host clock around each blocking call, L2 flushed "
                    "before each"}


def run_reference(args):
    """CPU reference path: each timed step is one whole evaluation of the
    workload's graph by the oracle port of cpuASPLqueue (BFS from every source,
    all host threads).  The graph comes from the committed fixture, so this arm
    never loads the engine library.  Beside it, the reference cudaASPLgraph on
    the same graph (reference_gpu)."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]
    adj = fixture_of(w, w["seed"])
    if adj is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"no committed input fixture for workload {args.workload} (plain-graph workloads only)"}),
              flush=True)
        return 0
    wl = dict(form="graph", N=w["n"], d=w["d"], table=adj, S=w["n"], M=w["n"])
    for _ in range(args.warmup):
        cpu_sample(wl, target_s=0.5)
    vals, rec, first = [], None, None
    t_all = time.perf_counter()
    for _ in range(args.steps):
        rec, r = cpu_sample(wl, full=True)
        vals.append(rec["value"])
        if first is None:
            first = r
    elapsed = time.perf_counter() - t_all
    v = args.steps / elapsed
    cb = dict(rec)
    cb["value"] = v
    cb["sample"] = f"{args.steps} whole evaluations (BFS from all {w['n']} sources each), {elapsed:.1f} s"
    ref_gpu = reference_gpu_graph(adj)
    oracle_res = {"diameter": first.levels if first.connected else -1, "total": first.total()}
    if "result" in ref_gpu and ref_gpu["result"] != oracle_res:
        raise SystemExit(f"reference GPU {ref_gpu['result']} != oracle {oracle_res}")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "impl": "reference",
            "config": graph_config(args.workload),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "result": oracle_res,
            "reference_gpu": ref_gpu,
            "wall_s": elapsed,
            "note": "the reference cpuASPLqueue is single-threaded (cpuASPLqueue.cpp:64) and evaluates "
                    "all sources in one call; each step runs its restatement (oracle/gg_oracle.c) over "
                    "all host threads"}
    print(json.dumps(line), flush=True)
    return 0


def timed(fn, steps, sync):
    sync()
    t0 = time.perf_counter()
    for _ in range(steps):
        fn()
    sync()
    return time.perf_counter() - t0


def traffic_of(workload):
    """DRAM bytes of one evaluation (all its launches) from the committed ncu capture, or None."""
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(tp):
        return None, None
    tj = json.load(open(tp)).get(workload)
    if not tj:
        return None, None
    return tj.get("dram_bytes_per_eval"), tj.get("note")


def run_ours(args):
    import numpy as np
    import torch
    import graphgolf as G

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w = WORKLOADS[args.workload]
    sharded = bool(w.get("sharded")) and world > 1
    wl = make_workload(args.workload, rank)
    if wl["form"] == "graph":
        eng = G.cudaASPLgraph(wl["N"], wl["d"], local)
        max_levels = 199
    else:
        eng = G.cudaASPLconv(wl["N"], wl["M"], wl["d"], local)
        max_levels = 99
    if args.batch_sources:
        eng.set_batch_sources(args.batch_sources)
    src_range = None
    if sharded:
        import distributed as D
        src_range = D.shard(wl["S"], rank, world)
    table_dev = torch.from_numpy(np.ascontiguousarray(wl["table"])).cuda()
    # an explicit stream: the engine runs on it, and the events and the L2
    # flush are recorded on it (the legacy default stream has the handle 0,
    # which the engine reads as "use your own stream")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    def step():
        r = eng.eval_device(table_dev.data_ptr(), max_levels=max_levels, stream=sptr, src_range=src_range)
        if sharded:
            # the exact counts of the whole graph: one all-reduce of the shards'
            # sums and maxima (distributed.combine, the function the gloo tests run)
            c = D.combine(r, wl["S"] * wl["N"])
            c.update(n_sources=wl["S"], batches=r["batches"])
            return c
        return r

    def combined(r):
        return dict(r)

    res = None
    for _ in range(max(args.warmup, 0)):
        res = step()
    if res is None:
        res = step()
    assert res["connected"] or sharded, res

    clocks = Clocks(gpu_uuid(local))

    # L2 flush between timed steps: a 256 MiB write (twice the 126 MB L2),
    # outside each step's own event pair.
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def measure():
        dev_ms, launches, step_ms = [], 0, []
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        r = None
        for _ in range(args.steps):
            flush.fill_(1)
            es, ee = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            es.record(stream)
            r = step()
            ee.record(stream)
            step_ms.append((es, ee))
            dev_ms.append(eng.last_device_ms())
            launches += eng.last_launches()
        ev1.record(stream)
        torch.cuda.synchronize()
        ck = clocks.stop()
        if dist:
            dist.barrier()
        steps_total = sum(a.elapsed_time(b) for a, b in step_ms)
        ck["bracket_ms_incl_flush"] = ev0.elapsed_time(ev1)
        return steps_total, dev_ms, launches, ck, combined(r)

    elapsed_ms, dev_ms, launches, ck, r = measure()
    bad = {"hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"}
    if set(ck.get("reasons", [])) & bad:
        elapsed_ms, dev_ms, launches, ck, r = measure()
    if dist:
        t = torch.tensor([elapsed_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    assert r["connected"] and not r["capped"], r

    # end to end through the C ABI with a host adjacency
    host_table = np.ascontiguousarray(wl["table"])
    if wl["form"] == "graph" and not sharded:
        e2e_fn = lambda: eng.calc(host_table)  # noqa: E731
    elif wl["form"] == "graph":
        e2e_fn = lambda: eng.eval(host_table, max_levels=199, src_range=src_range)  # noqa: E731
    else:
        e2e_fn = lambda: eng.diameterASPL(host_table)  # noqa: E731
    e2e_first = e2e_fn()
    if wl["form"] == "graph" and not sharded:
        assert e2e_first == (r["levels"], r["total"]), (e2e_first, r)
    e2e_steps = max(3, min(args.steps, 20))
    e2e_s = 0.0
    for _ in range(e2e_steps):  # each call is blocking; L2 flushed before each
        flush.fill_(2)
        torch.cuda.synchronize()
        e2e_s += timed(e2e_fn, 1, lambda: None)
    h2d, d2h = eng.last_transfer_bytes()
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    # whole-job throughput: evaluations of whole graphs per second
    evals = args.steps * (1 if sharded else world)
    value = evals / (elapsed_ms / 1000.0)
    kern_ms = statistics.mean(dev_ms)
    alg = algorithmic_bytes(wl, r, eng.table_shape)
    peak, peak_kind = peaks()
    traffic, traffic_note = traffic_of(args.workload)
    if sharded:
        traffic = None    # the committed capture is of one whole evaluation on one GPU
    roof = {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
            "traffic": traffic, "peak_source": peak_kind, "kernel_ms": kern_ms,
            "achieved_from": "DRAM bytes of one evaluation's launches (traffic, ncu) / the "
                             "evaluation's mean CUDA-event time (kernel_ms)",
            "traffic_source": traffic_note}
    if traffic:
        roof["achieved"] = traffic / (kern_ms / 1000.0) / 1e9
        roof["frac"] = roof["achieved"] / peak
    l2 = None
    if rank == 0 and not args.no_gather_peak:
        gp, gms = G.gather_peak(rows=wl["N"], degree=wl["d"], iters=20, device=local)
        # per-level device timestamps of batch 0 (one more evaluation, outside the timed steps)
        lv = eng.eval_device(table_dev.data_ptr(), max_levels=max_levels, stream=sptr, level_ns=True,
                             src_range=src_range)["level_ns"].astype(np.int64)
        level_us = [round((int(lv[i]) - int(lv[i - 1])) / 1000.0, 2) for i in range(1, len(lv)) if lv[i]]
        # a dense visited-set pull level moves d + 1 row transfers per row (d gathers, one
        # write: no own row on a table without one-way entries); the gather pass moves
        # d + 2: its time x (d + 1) / (d + 2) is the dense level's floor at this rate
        floor_us = 1000.0 * gms * (wl["d"] + 1) / (wl["d"] + 2)
        # the dense levels: past the first (the walk pass, or level 1), within 30 % of the slowest
        rest = level_us[1:]
        dense = [t for t in rest if t >= 0.7 * max(rest)] if rest else []
        l2 = {"gather_peak_gbs": gp, "gather_pass_ms": gms,
              "what": f"gg_gather_peak: {wl['N']} rows x ({wl['d']} random + 1 own) 512-byte row reads + "
                      "1 row write per pass, the access pattern of one dense BFS level of one source "
                      "batch, arrays L2-resident",
              "levels_batch0_us": level_us,
              "dense_level_floor_us": floor_us,
              "dense_level_frac": (floor_us / statistics.median(dense)) if dense else None,
              "kernel_ms_in_gather_passes": kern_ms / gms,
              "level_steps": r["level_steps"]}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic",
            "config": (graph_config(args.workload) if wl["form"] == "graph" else
                       {"workload": args.workload, "n": wl["N"], "degree": wl["d"], "l2": L2_NOTE}),
            "run": {"sources": wl["S"], "batches": r["batches"],
                    "level_steps": r["level_steps"], "diameter": r["levels"],
                    "parallelism": (f"source-sharded{world}" if sharded else
                                    (f"replicas{world}" if world > 1 else "single")),
                    "batch_sources": -(-wl["S"] // max(1, r["batches"])) if not sharded else None,
                    "bit_edge_traversals_per_s": bit_edges_per_eval(wl, r) * evals / (elapsed_ms / 1000.0),
                    "timing": "each step timed by its own CUDA event pair on the launching stream"},
            "e2e": {"value": (1 if sharded else world) * e2e_steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roof,
            "l2_gather": l2,
            "algorithmic": {"bytes": alg, "gbs": alg / (kern_ms / 1000.0) / 1e9,
                            "definition": "per executed level N*d*4 + N*(d+2)*S/8 bytes (S = sources of "
                                          "the batch), summed over batches; counts gathers the kernel "
                                          "skips or the L2 serves, so it is no DRAM figure"},
            "gpu_launches": launches,
            "clocks": ck,
            "result": {"diameter": r["levels"], "total": r["total"]}}
    if rank == 0 and world == 1 and not args.no_cpu:
        cb, o = cpu_sample(wl, full=True)
        line["cpu_baseline"] = cb
        if o is not None:
            want_total = o.total()
            if not (o.connected and want_total == r["total"] and o.levels == r["levels"]):
                raise SystemExit(f"PARITY FAILURE: engine {r['levels']},{r['total']} vs oracle "
                                 f"{o.levels},{want_total}")
            line["parity"] = f"exact: equals the oracle BFS from all {wl['S']} sources"
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


def spawn_ranks(args):
    """`--gpus N` outside torchrun: run this script as N ranks on this node."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd, timeout=3600).returncode


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="regular_n65536_d8")
    ap.add_argument("--batch-sources", type=int, default=0)
    ap.add_argument("--cpu-s", type=float, default=10.0)
    ap.add_argument("--ref-step-s", type=float, default=4.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-gather-peak", action="store_true")
    ap.add_argument("--anneal-steps", type=int, default=0, help="annealing schedule length (time-to-target workload)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args)
    if args.impl == "reference":
        return run_reference(args)
    if WORKLOADS[args.workload]["form"] == "batch":
        return run_batch(args)
    if WORKLOADS[args.workload]["form"] == "anneal":
        return run_anneal(args)
    if WORKLOADS[args.workload]["form"] == "incremental":
        return run_incremental(args)
    if WORKLOADS[args.workload]["form"] == "liftbatch":
        return run_lift_batch(args)
    return run_ours(args)


def run_anneal(args):
    """Time-to-target: plain batched annealing runs its whole schedule; its final
    best ASPL is the target; the surrogate-ranked annealer (same seed, same
    schedule) runs until it reaches that exact-verified ASPL and has trained on at
    least 200k (swap, exact change) pairs.  value = plain wall time to its final
    best / surrogate wall time to the same ASPL (its first hit)."""
    import torch
    import graphgolf as G
    import anneal as A
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    steps = args.anneal_steps or w["steps"]
    adj = G.random_regular(w["n"], w["d"], w["seed"] + 1000 * rank)
    A.anneal(adj, 50, seed=w["seed"])                      # warm-up (graphs, caches)
    A.anneal(adj, 50, seed=w["seed"], surrogate=True)
    _, plain = A.anneal(adj, steps, seed=w["seed"], exact=32, device=local)
    target = plain.final_best
    t_plain = A.time_to(plain, target)
    _, sur = A.anneal(adj, steps, seed=w["seed"], exact=32, surrogate=True, target=target, device=local,
                      spearman_sample=2048, min_train_pairs=200_000)
    line = {"metric": "ASPL time-to-target, plain / surrogate", "value":
            (t_plain / sur.hit_time) if sur.hit_time else None, "unit": "x", "n_gpus": world,
            "steps": steps, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32 exact BFS; bf16/fp32 surrogate", "data": "synthetic",
            "config": {"workload": args.workload, "n": w["n"], "degree": w["d"], "exact_per_step": 32,
                       "surrogate_pool": 4096, "schedule": "geometric 1e-3*ASPL -> 1e-6"},
            "plain": {"wall_s": plain.wall, "time_to_final_s": t_plain, "steps": plain.steps,
                      "start_aspl": plain.best[0], "final_aspl": target, "ms_per_step": 1000 * plain.wall / plain.steps},
            "surrogate": {"hit_s": sur.hit_time, "hit_step": sur.hit_step, "final_aspl": sur.final_best,
                          "train_pairs": sur.train_pairs, "train_pairs_at_hit": sur.hit_train_pairs,
                          "steps": sur.steps, "ms_per_step": 1000 * sur.wall / max(sur.steps, 1),
                          "spearman_predicted_vs_exact": sur.spearman,
                          "spearman_sample": "2048 uniform 2-opt proposals of the final graph, after the run"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def bit_edges_per_eval(wl, r):
    """Bit-edge traversals: sum over executed levels of N * d * S (S = sources of the
    batch), for an evaluation with all batches of equal width."""
    S = -(-r["n_sources"] // r["batches"])
    return r["level_steps"] * wl["N"] * wl["d"] * S


def run_incremental(args):
    """One exact 2-opt move evaluation per step (gg_inc_eval: affected-source test
    with the cached per-source sums, search from the affected sources).
    The call is blocking and reads a count back halfway, so a step is timed by the
    host clock around the call (L2 flushed and the device idle before each step);
    that is also the end-to-end figure.  The full calculator call on the same moved
    graphs is timed the same way for comparison."""
    import numpy as np
    import torch
    import graphgolf as G
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    adj = G.random_regular(w["n"], w["d"], w["seed"] + 1000 * rank)
    inc = G.Incremental(w["n"], w["d"], local)
    inc.set_graph(adj)
    sw = G.gen_swaps(adj, 0, args.steps + args.warmup, w["seed"] + 7)
    for s in sw[:max(args.warmup, 1)]:
        inc.eval(s)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    clocks = Clocks(gpu_uuid(local))
    clocks.start()
    t, aff = 0.0, 0
    for s in sw[args.warmup:]:
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, a = inc.eval(s)
        t += time.perf_counter() - t0
        aff += a
    ck = clocks.stop()
    full = G.cudaASPLgraph(w["n"], w["d"], local)
    full.calc(G.apply_swap(adj, sw[0]))
    tf, nf = 0.0, min(args.steps, 10)
    for s in sw[args.warmup:args.warmup + nf]:
        moved = G.apply_swap(adj, s)
        flush.fill_(2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        full.calc(moved)
        tf += time.perf_counter() - t0
    value = world * args.steps / t
    line = {"metric": "2-opt move evals/s", "value": value, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": args.workload, "n": w["n"], "degree": w["d"],
                       "affected_sources_mean": aff / args.steps,
                       "timed": "host clock around each blocking call; L2 flushed before each step",
                       "full_calc_ms": 1000 * tf / nf},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 24,
                    "d2h_bytes_per_step": 24},
            "gpu_launches": 5 * args.steps, "clocks": ck}
    if rank == 0:
        print(json.dumps(line), flush=True)
    inc.close()
    full.close()
    return 0


def lift_bitset_rate(res, group, N, M, d, ms):
    """Bitset GB/s of one lift launch: the algorithmic bytes of a BFS level over a
    batch of S sources, N*d*4 + N*(d+2)*S/8, for each candidate of a round at
    each of the round's levels (its candidates' largest eccentricity), over the
    device time; against the measured HBM copy bandwidth."""
    per_level = N * d * 4 + N * (d + 2) * M / 8
    levels = [int(res["levels"][i:i + group].max()) for i in range(0, len(res), group)]
    nbytes = sum(L * min(group, len(res) - r * group) * per_level for r, L in enumerate(levels))
    peak, src = peaks()
    gbs = nbytes / (ms * 1e-3) / 1e9
    return {"algorithmic_bytes": nbytes, "gbs": gbs, "peak_gbs": peak, "frac": gbs / peak,
            "peak_source": src + " HBM copy"}


def run_lift_batch(args):
    """Batched lifted candidates: every step scores the same population of moves
    of one cyclic lift with one blocking gg_lift_eval call (edits in, counts out).
    value = candidates per second of device time (CUDA events around the table
    build and the BFS launch, L2 flushed before each step); e2e = the same over the
    host clock around the call.  Beside it, the reference-style path: one
    cudaASPLconv::diameterASPL call per candidate on this engine (its table built
    on the host), timed on a sample of the candidates."""
    import numpy as np
    import torch
    import graphgolf as G
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    if w.get("kind") == "piece":
        Nx, Ny, Mx, My, D = G.piece_lift(w["Mx"], w["My"], w["kx"], w["ky"], w["d"], w["seed"] + 1000 * rank)
        N, M = Nx * Ny, Mx * My
        L = G.Lift.piece(Nx, Ny, Mx, My, w["d"], local)
        moves = G.gen_piece_moves(Nx, Ny, Mx, My, D, w["cands"], w["seed"] + 5)
        conv = G.cudaASPLpiece(Nx, Ny, Mx, My, w["d"], local)
        what = "gg_piece_diameter_aspl per candidate table, host clock"
    else:
        N, M, D = G.cyclic_lift(w["m"], w["g"], w["d"], w["seed"] + 1000 * rank)
        L = G.Lift(N, M, w["d"], local)
        moves = G.gen_lift_moves(N, M, D, w["cands"], w["seed"] + 5)
        conv = G.cudaASPLconv(N, M, w["d"], local)
        what = "gg_conv_diameter_aspl per candidate table, host clock"
    L.set_base(D)
    n = len(moves)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(max(args.warmup, 1)):
        res = L.eval(moves)
    clocks = Clocks(gpu_uuid(local))
    clocks.start()
    dev_ms, host_s = 0.0, 0.0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = L.eval(moves)
        host_s += time.perf_counter() - t0
        dev_ms += L.last_ms()
    ck = clocks.stop()
    # one calculator call per candidate, as the reference scores them
    sample = min(n, 32)
    tabs = [G.apply_lift_edit(D, e) for e in moves[:sample]]
    conv.diameterASPL(tabs[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    single = [conv.diameterASPL(t) for t in tabs]
    per_call_ms = 1000.0 * (time.perf_counter() - t0) / sample
    aspl = L.aspl(res[:sample])
    assert all(a == s[1] for a, s in zip(aspl, single) if np.isfinite(a))
    conv.close()
    line = {"metric": METRIC, "value": world * n * args.steps / (dev_ms / 1000.0), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": args.workload, "N": N, "M": M, "degree": w["d"], "candidates_per_step": n,
                       "moves": {"shift": int((moves["count"] == 2).sum()),
                                 "orbit_2opt": int((moves["count"] == 4).sum())},
                       "group": L.group(), "l2": "flushed (256 MiB write) before every timed step"},
            "e2e": {"value": world * n * args.steps / host_s, "unit": UNIT,
                    "h2d_bytes_per_step": int(moves.nbytes),
                    # the control block, then the per-level count rows 0..diameter+1
                    "d2h_bytes_per_step": int(256 + (int(res["levels"].max()) + 2) * n * 8)},
            "single_call": {"ms_per_candidate": per_call_ms, "sample": sample, "what": what},
            "bitset": lift_bitset_rate(res, L.group(), N, M, w["d"], dev_ms / args.steps),
            "gpu_launches": (2 if w.get("kind") != "piece" else 3) * args.steps, "clocks": ck}
    if rank == 0:
        print(json.dumps(line), flush=True)
    L.close()
    return 0


def run_batch(args):
    """Batched 2-opt scoring: value = candidates scored per second with the
    candidates resident on the device (gg_batch_eval_device, CUDA events on the
    launching stream, L2 flushed before each step); e2e = the host-array call
    gg_batch_eval (H2D of the swaps, the launch, D2H of the results)."""
    import numpy as np
    import torch
    import graphgolf as G
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    seed = WORKLOADS[args.workload]["seed"] + 1000 * rank
    b = G.Batch(local)
    g1, g2 = G.random_regular(1024, 6, seed), G.random_regular(3000, 4, seed + 1)
    i1, i2 = b.add_base(g1), b.add_base(g2)
    sw = np.concatenate([G.gen_swaps(g1, i1, 2048, seed + 2), G.gen_swaps(g2, i2, 512, seed + 3)])
    n = len(sw)
    d_sw = torch.from_numpy(sw.view(np.int32).copy()).cuda()
    d_out = torch.zeros(n * G.CAND_RESULT_DTYPE.itemsize // 4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()  # explicit: the launch, the events and the flush share it
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(max(args.warmup, 1)):
        b.eval_device(n, d_sw.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    clocks = Clocks(gpu_uuid(local))
    clocks.start()
    pairs = []
    for _ in range(args.steps):
        flush.fill_(1)
        es, ee = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        es.record(stream)
        b.eval_device(n, d_sw.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
        ee.record(stream)
        pairs.append((es, ee))
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = sum(a.elapsed_time(c) for a, c in pairs)
    res = d_out.cpu().numpy().view(G.CAND_RESULT_DTYPE)
    assert np.all(res["connected"] == 1)
    b.eval(sw)
    e2e_s = 0.0
    for _ in range(max(3, min(args.steps, 20))):
        flush.fill_(2)
        torch.cuda.synchronize()
        e2e_s += timed(lambda: b.eval(sw), 1, lambda: None)
    e2e_steps = max(3, min(args.steps, 20))
    line = {"metric": METRIC, "value": world * n * args.steps / (ms / 1000.0), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": args.workload, "candidates_per_step": n,
                       "bases": ["random 6-regular n=1024", "random 4-regular n=3000"],
                       "l2": "flushed (256 MiB write) before every timed step"},
            "e2e": {"value": world * n * e2e_steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": int(sw.nbytes), "d2h_bytes_per_step": int(res.nbytes)},
            "gpu_launches": 3 * args.steps, "clocks": ck}
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
