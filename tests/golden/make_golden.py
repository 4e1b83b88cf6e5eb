"""Generate tests/golden/cases.json from the reference's own CPU calculators.

    make -C oracle ref            # builds oracle/_ref/libref_cpu.so from the reference sources
    python tests/golden/make_golden.py

Each case stores its input table and what the reference returned for it:
  part  : cpuASPLqueue<cap>::diameterASPL and ::calc   (cppcode/cpuASPLqueue.cpp:11-96)
  piece : cpuASPLpiece<cap>::diameterASPL              (cppcode/cpuASPLpiece.cpp:12-63)
  box   : cpuASPLbox<cap>::diameterASPL                (cppcode/cpuASPLbox.cpp:12-66)
plus the exact integer total distance (over the representative sources, before
the N/M scale) that the oracle computes, cross-checked here against the
reference's double: round(aspl * N * (N-1)) == total * (N // M).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"),
                os.path.join(ROOT, "graphgolf-cuda_b200")]

import instances as I  # noqa: E402
import oracle as O  # noqa: E402


def rows_of(t):
    return [list(map(int, np.asarray(r).reshape(-1))) for r in t]


def part_case(name, N, M, diffs, ref):
    diffs = np.asarray(diffs, dtype=np.int32)
    d, a = ref.queue_diameter_aspl(N, M, rows_of(diffs))
    calc = ref.queue_calc(N, M, rows_of(diffs))
    r = O.bfs_pull(O.expand_part(N, M, diffs), np.arange(M))
    if d != O.INT_MAX:
        assert round(a * N * (N - 1)) == r.total() * (N // M), name
    return {"name": name, "kind": "part", "N": N, "M": M, "degree": int(diffs.shape[1]),
            "table": diffs.reshape(-1).tolist(), "ref_diameter": d, "ref_aspl": a,
            "ref_calc": calc, "total": r.total(), "levels": r.levels,
            "connected": r.connected}


def piece_case(name, Nx, Ny, Mx, My, rows, ref):
    rows = np.asarray(rows, dtype=np.int32)
    d, a = ref.piece_diameter_aspl(Nx, Ny, Mx, My, rows_of(rows))
    r = O.bfs_pull(O.expand_piece(Nx, Ny, Mx, My, rows), O.piece_reps(Nx, Ny, Mx, My))
    return {"name": name, "kind": "piece", "dims": [Nx, Ny, Mx, My], "degree": int(rows.shape[1]),
            "table": rows.reshape(-1).tolist(), "ref_diameter": d, "ref_aspl": a,
            "total": r.total(), "levels": r.levels, "connected": r.connected}


def box_case(name, dims, rows, ref):
    rows = np.asarray(rows, dtype=np.int32)
    d, a = ref.box_diameter_aspl(*dims, rows_of(rows))
    r = O.bfs_pull(O.expand_box(*dims, rows), O.box_reps(*dims))
    return {"name": name, "kind": "box", "dims": list(dims), "degree": int(rows.shape[1]),
            "table": rows.reshape(-1).tolist(), "ref_diameter": d, "ref_aspl": a,
            "total": r.total(), "levels": r.levels, "connected": r.connected}


def main():
    import graphgolf as G
    ref = O.RefCPU()
    cases = []
    # the single-graph oracle configuration: random 4-regular, n = 256, seed 1
    adj = G.random_regular(256, 4, 1)
    cases.append(part_case("regular_n256_d4_seed1", *I.plain_as_part(adj), ref))
    cases.append(part_case("regular_n512_d6_seed2", *I.plain_as_part(G.random_regular(512, 6, 2)), ref))
    cases.append(part_case("cycle8", *I.plain_as_part(I.cycle(8)), ref))
    cases.append(part_case("cycle33", *I.plain_as_part(I.cycle(33)), ref))
    cases.append(part_case("petersen", *I.plain_as_part(I.petersen()), ref))
    cases.append(part_case("hypercube5", *I.plain_as_part(I.hypercube(5)), ref))
    cases.append(part_case("complete6", *I.plain_as_part(I.complete(6)), ref))
    cases.append(part_case("disconnected_c10_c12",
                           *I.plain_as_part(I.disjoint_union(I.cycle(10), I.cycle(12))), ref))
    for i, (m, g, d) in enumerate([(16, 4, 3), (40, 8, 4), (64, 16, 6), (100, 3, 5), (33, 7, 4)]):
        if (m * d) % 2:
            m += 1
        cases.append(part_case(f"random_part_{m}x{g}_d{d}", *I.random_part(m, g, d, 10 + i), ref))
    N, M, diffs = G.cyclic_lift(32, 8, 4, 3)
    cases.append(part_case("cyclic_lift_m32_g8_d4_seed3", N, M, diffs, ref))
    for i, (Mx, My, kx, ky, d) in enumerate([(2, 2, 3, 3, 4), (3, 4, 2, 3, 3), (4, 4, 4, 2, 4)]):
        cases.append(piece_case(f"random_piece_{i}", *I.random_piece(Mx, My, kx, ky, d, 20 + i), ref))
    for i, (M3, k3, d) in enumerate([((2, 2, 2), (2, 2, 2), 4), ((1, 2, 3), (3, 2, 2), 4),
                                     ((2, 3, 2), (2, 2, 3), 6)]):
        Nx, Ny, Nz, Mx, My, Mz, rows = I.random_box(*M3, *k3, d, 30 + i)
        cases.append(box_case(f"random_box_{i}", (Nx, Ny, Nz, Mx, My, Mz), rows, ref))
    out = os.path.join(HERE, "cases.json")
    with open(out, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference": "cpuASPLqueue / cpuASPLpiece / cpuASPLbox built from the reference sources",
                   "cases": cases}, f, indent=0)
    print(f"wrote {len(cases)} cases to {out}")


if __name__ == "__main__":
    main()
