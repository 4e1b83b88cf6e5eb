"""Microbenchmarks of the dense level's access pattern: gg_gather_peak (random
512-byte row gathers) and gg_level_probe (the dense level loop with its counts,
flag words and grid barrier, outside the engine).

CPU: argument checks, which return before any device call.  GPU: small runs give
positive, finite rates and reject nothing they should accept.
"""
import math

import pytest

import graphgolf as G


@pytest.mark.parametrize("kw", [
    dict(rows=32),                    # below 64 rows
    dict(rows=1 << 19),               # above 262144 rows
    dict(chunks=8),                   # only 16 or 32 chunks a row
    dict(rows=65, chunks=16),         # 16-chunk rows come in pairs
    dict(levels=11),                  # the first 10 levels are warm-up
    dict(levels=1025),
    dict(variant=2),
])
def test_level_probe_rejects_bad_arguments(kw):
    with pytest.raises(G.GGError) as e:
        G.level_probe(**kw)
    assert e.value.status == G.GG_BAD_ARG


@pytest.mark.parametrize("kw", [dict(rows=0), dict(degree=0), dict(degree=65), dict(iters=0)])
def test_gather_peak_rejects_bad_arguments(kw):
    with pytest.raises(G.GGError) as e:
        G.gather_peak(**kw)
    assert e.value.status == G.GG_BAD_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("chunks,variant", [(32, 0), (32, 1), (16, 0), (16, 1)])
def test_level_probe_runs(chunks, variant):
    us = G.level_probe(rows=4096, chunks=chunks, levels=16, variant=variant)
    assert math.isfinite(us) and 0.0 < us < 10000.0


@pytest.mark.gpu
def test_gather_peak_runs():
    gbs, ms = G.gather_peak(rows=4096, degree=8, iters=3)
    assert math.isfinite(gbs) and gbs > 0.0 and ms > 0.0
