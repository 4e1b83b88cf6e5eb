"""Source-sharded evaluation over torch.distributed: two gloo ranks on CPU run
the sharding and the all-reduce of distributed.py; each rank's share is
computed by an oracle-backed stand-in engine (the GPU engine does the same
through gg_eval with a source range, tests/test_parity_gpu.py checks that), and
the combined counts must equal the unsplit evaluation."""
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
