"""Write the input graphs of the single-graph benchmark workloads as fixtures.

    python tests/golden/make_bench_inputs.py

bench.py's reference arm reads these files, so that timing the reference path
never loads the engine library (its generator is the engine's
gg_gen_random_regular); the engine arm regenerates each graph from its seed and
checks that it equals the fixture.  Stored as uint16 (every vertex id < 65536),
rows as the generator returns them (sorted ascending):
  regular_n65536_d8_seed1.npy    random simple connected 8-regular graph, n = 65536, seed 1
  regular_n4096_d16_seed1.npy    random simple connected 16-regular graph, n = 4096, seed 1
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "graphgolf-cuda_b200")]

import graphgolf as G  # noqa: E402

INPUTS = {"regular_n65536_d8_seed1.npy": (65536, 8, 1), "regular_n4096_d16_seed1.npy": (4096, 16, 1)}


def main():
    for name, (n, d, seed) in INPUTS.items():
        adj = G.random_regular(n, d, seed)
        assert adj.min() >= 0 and adj.max() < 65536
        np.save(os.path.join(HERE, name), adj.astype(np.uint16))
        print(name, adj.shape)


if __name__ == "__main__":
    main()
