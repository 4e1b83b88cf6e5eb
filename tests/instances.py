"""Small seeded test instances (numpy RNG) in the packed table formats of the
reference calculators, plus closed-form known answers.

These are test inputs only; the benchmark workloads come from the engine's own
generators (gg_gen_random_regular / gg_gen_cyclic_lift)."""
from __future__ import annotations

import itertools

import numpy as np


def plain_as_part(adj):
    """A plain graph as a part with M = N: row v holds diffs (u - v)."""
    adj = np.asarray(adj, dtype=np.int64)
    n = len(adj)
    return n, n, (adj - np.arange(n)[:, None]).astype(np.int32)


def cycle(n):
    v = np.arange(n)
    return np.stack([(v - 1) % n, (v + 1) % n], axis=1).astype(np.int32)


def path_graph(n):
    """Path 0-1-...-(n-1), padded to degree 2 with self-loops at the ends."""
    v = np.arange(n)
    a = np.stack([np.maximum(v - 1, 0), np.minimum(v + 1, n - 1)], axis=1)
    return a.astype(np.int32)


def complete(n):
    return np.array([[u for u in range(n) if u != v] for v in range(n)], dtype=np.int32)


def hypercube(k):
    n = 1 << k
    return np.array([[v ^ (1 << b) for b in range(k)] for v in range(n)], dtype=np.int32)


def petersen():
    outer = [(i, (i + 1) % 5) for i in range(5)]
    spokes = [(i, i + 5) for i in range(5)]
    inner = [(5 + i, 5 + (i + 2) % 5) for i in range(5)]
    adj = [[] for _ in range(10)]
    for a, b in outer + spokes + inner:
        adj[a].append(b)
        adj[b].append(a)
    return np.array([sorted(r) for r in adj], dtype=np.int32)


def complete_bipartite(a, b):
    adj = [list(range(a, a + b)) if v < a else list(range(a)) for v in range(a + b)]
    return adj  # ragged when a != b


# closed forms: (diameter, total over ordered pairs)
def kat_cycle(n):
    return n // 2, n * (n * n // 4)


def kat_complete(n):
    return (1 if n > 1 else 0), n * (n - 1)


def kat_hypercube(k):
    n = 1 << k
    return k, n * k * (1 << (k - 1))


def kat_petersen():
    return 2, 10 * 15


def kat_complete_bipartite(a, b):
    return (2 if max(a, b) > 1 else 1), a * (b + 2 * (a - 1)) + b * (a + 2 * (b - 1))


def random_regular_np(n, d, seed):
    """Random d-regular multigraph by stub pairing (loops/multi-edges allowed)."""
    rng = np.random.default_rng(seed)
    stubs = np.repeat(np.arange(n), d)
    rng.shuffle(stubs)
    rows = [[] for _ in range(n)]
    for a, b in stubs.reshape(-1, 2):
        rows[a].append(int(b))
        rows[b].append(int(a))
    return np.array(rows, dtype=np.int32)


def random_part(m, g, d, seed):
    """Random cyclic lift in part form (N = m*g, M = m), diff = (b-a) + m*k as in
    the reference's own generator encoding (cppcode/initTemp.cpp:399-405)."""
    rng = np.random.default_rng(seed)
    stubs = np.repeat(np.arange(m), d)
    rng.shuffle(stubs)
    rows = [[] for _ in range(m)]
    for a, b in stubs.reshape(-1, 2):
        a, b = (int(a), int(b)) if a <= b else (int(b), int(a))
        diff = (b - a) + m * int(rng.integers(0, g))
        rows[a].append(diff)
        rows[b].append(-diff)
    return m * g, m, np.array(rows, dtype=np.int32)


def random_piece(Mx, My, kx, ky, d, seed):
    """Random 2-D torus lift: N = (Mx*kx) x (My*ky); rows [Mx*My, d, 2]."""
    rng = np.random.default_rng(seed)
    M = Mx * My
    stubs = np.repeat(np.arange(M), d)
    rng.shuffle(stubs)
    rows = [[] for _ in range(M)]
    for a, b in stubs.reshape(-1, 2):
        ax, ay, bx, by = a // My, a % My, b // My, b % My
        dx = (bx - ax) + Mx * int(rng.integers(0, kx))
        dy = (by - ay) + My * int(rng.integers(0, ky))
        rows[a].append((dx, dy))
        rows[b].append((-dx, -dy))
    return Mx * kx, My * ky, Mx, My, np.array(rows, dtype=np.int32)


def random_box(Mx, My, Mz, kx, ky, kz, d, seed):
    """Random 3-D torus lift; rows [Mx*My*Mz, d, 3]."""
    rng = np.random.default_rng(seed)
    M = Mx * My * Mz
    stubs = np.repeat(np.arange(M), d)
    rng.shuffle(stubs)
    rows = [[] for _ in range(M)]

    def xyz(i):
        return i // (My * Mz), (i // Mz) % My, i % Mz

    for a, b in stubs.reshape(-1, 2):
        (ax, ay, az), (bx, by, bz) = xyz(a), xyz(b)
        dx = (bx - ax) + Mx * int(rng.integers(0, kx))
        dy = (by - ay) + My * int(rng.integers(0, ky))
        dz = (bz - az) + Mz * int(rng.integers(0, kz))
        rows[a].append((dx, dy, dz))
        rows[b].append((-dx, -dy, -dz))
    return (Mx * kx, My * ky, Mz * kz, Mx, My, Mz, np.array(rows, dtype=np.int32))


def disjoint_union(adj_a, adj_b):
    """Two graphs of equal degree side by side (disconnected)."""
    a = np.asarray(adj_a)
    b = np.asarray(adj_b) + len(a)
    return np.concatenate([a, b]).astype(np.int32)


def all_subsets(n):
    return itertools.chain.from_iterable(itertools.combinations(range(n), k) for k in range(n + 1))


def random_nonregular(n, dmax, seed, extra=1.5):
    """Connected simple graph with degrees in [1, dmax] (a random spanning tree
    plus random extra edges), padded to [n, dmax] with self-loops as the
    reference pads missing edges (cudaASPLgraph.cu:149-151)."""
    rng = np.random.default_rng(seed)
    lists = [[] for _ in range(n)]
    order = rng.permutation(n)
    for i in range(1, n):
        v = int(order[i])
        for _ in range(64):
            u = int(order[rng.integers(0, i)])
            if len(lists[u]) < dmax:
                break
        else:
            u = next(int(order[j]) for j in range(i) if len(lists[int(order[j])]) < dmax)
        lists[u].append(v)
        lists[v].append(u)
    for _ in range(int(extra * n)):
        a, b = (int(x) for x in rng.integers(0, n, size=2))
        if a != b and b not in lists[a] and len(lists[a]) < dmax and len(lists[b]) < dmax:
            lists[a].append(b)
            lists[b].append(a)
    t = np.repeat(np.arange(n, dtype=np.int32)[:, None], dmax, axis=1)
    for v, l in enumerate(lists):
        t[v, :len(l)] = l
    return t, lists


def ragged_part(m, g, d, drop, seed):
    """A cyclic lift whose orbit rows have different lengths: random_part with
    `drop` orbit edges removed (both ends), rows padded with diff 0."""
    N, M, rows = random_part(m, g, d, seed)
    rows = [list(map(int, r)) for r in rows]
    rng = np.random.default_rng(seed + 7)
    for _ in range(drop):
        a = int(rng.integers(0, m))
        if not rows[a]:
            continue
        diff = rows[a].pop(int(rng.integers(0, len(rows[a]))))
        b = (a + diff) % m
        rows[b].remove(-diff)
    t = np.zeros((m, d), dtype=np.int32)
    for i, r in enumerate(rows):
        t[i, :len(r)] = r
    return N, M, t, rows
