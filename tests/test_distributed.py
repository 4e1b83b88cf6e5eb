"""Sharded work over torch.distributed, two gloo ranks on CPU.

Source-sharded evaluation: the ranks run the sharding and the all-reduce of
distributed.py; each rank's share is computed by an oracle-backed stand-in
engine (the GPU engine does the same through gg_eval with a source range,
tests/test_parity_gpu.py checks that), and the combined counts must equal the
unsplit evaluation.  Candidate-sharded scoring: each rank scores its slice of a
population of lift moves with an oracle-backed stand-in for Lift.eval, and the
gathered results must equal the unsplit scoring on both ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import distributed as D
import instances as I
import oracle as O


def test_shard_covers_all_sources_once():
    for n in (1, 31, 32, 33, 1000, 4096):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                lo, hi = D.shard(n, r, world)
                assert lo % 32 == 0 or lo == n
                got.extend(range(lo, hi))
            assert got == list(range(n))


class OracleEngine:
    """Stand-in with the Engine.eval signature, computed by the oracle."""

    def __init__(self, adj):
        self.adj = adj

    def eval(self, table, max_levels=0, src_range=None):
        lo, hi = src_range
        r = O.bfs_pull(self.adj, np.arange(lo, hi))
        return {"total": r.total(), "reached": int(r.reached.sum()), "levels": r.levels,
                "capped": 0, "level_steps": r.levels + 1}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, adj, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = D.eval_sharded(OracleEngine(adj), adj, len(adj), len(adj))
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("adj", [I.random_regular_np(300, 4, 1), I.disjoint_union(I.cycle(40), I.cycle(50))])
def test_two_gloo_ranks_combine_exactly(adj):
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, adj, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    whole = O.bfs_pull(adj, np.arange(len(adj)))
    for r in range(2):
        res = out[r]
        assert res["total"] == whole.total()
        assert res["reached"] == int(whole.reached.sum())
        assert res["levels"] == whole.levels
        assert bool(res["connected"]) == whole.connected


def lift_oracle_eval(N, M, T):
    """Stand-in for Lift.eval: exact counts of each edit by the oracle."""
    import graphgolf as G

    def ev(edits):
        out = np.zeros(len(edits), dtype=G.CAND_RESULT_DTYPE)
        for i, e in enumerate(edits):
            r = O.bfs_pull(O.expand_part(N, M, G.apply_lift_edit(T, e)), np.arange(M))
            out[i] = (r.total(), int(r.reached.sum()), r.levels, int(r.connected))
        return out
    return ev


def _cand_worker(rank, world, port, N, M, T, moves, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = D.eval_candidates_sharded(lift_oracle_eval(N, M, T), moves).tobytes()
    finally:
        dist.destroy_process_group()



@pytest.mark.parametrize("count", [9, 1])
def test_two_gloo_ranks_gather_candidate_results(count):
    import graphgolf as G
    N, M, T = G.cyclic_lift(40, 4, 4, 3)
    moves = G.gen_lift_moves(N, M, T, count, 5)
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_cand_worker, args=(r, 2, port, N, M, T, moves, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    whole = lift_oracle_eval(N, M, T)(moves).tobytes()
    assert out[0] == whole and out[1] == whole


def test_bench_gpus_flag_starts_one_rank_per_gpu(monkeypatch):
    """`bench.py --gpus N` outside torchrun re-runs itself as N ranks with
    torch.distributed.run on 127.0.0.1, passing every argument through."""
    import sys
    import types
    import bench
    calls = []

    def fake_run(cmd, timeout):
        calls.append(cmd)
        return types.SimpleNamespace(returncode=0)

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "4", "--steps", "3", "--workload",
                                      "regular_n65536_d8_sharded"])
    assert bench.main() == 0
    cmd = calls[0]
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd and "--nnodes=1" in cmd
    assert cmd[-6:] == ["--gpus", "4", "--steps", "3", "--workload", "regular_n65536_d8_sharded"]
