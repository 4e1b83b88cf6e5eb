"""CPU oracle for the bit-parallel all-pairs BFS -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this module.  The product
(the CUDA engine behind ``include/gg.h``) never calls it.

Layers
------
* ``liboracle.so`` (``oracle/gg_oracle.c``): queue BFS per source, a restatement
  of ``cppcode/cpuASPLqueue.cpp:54-96`` that returns exact per-level pair
  counts, per-source eccentricity and per-source reach.
* This module: the adjacency expansions of every calculator form, and every
  return convention of the reference calculators (sentinels, N/M scaling,
  level caps), recomputed exactly from those counts:

  =====================  ==============================================
  function               reference it restates
  =====================  ==============================================
  ``queue_diameter_aspl``  ``cppcode/cpuASPLqueue.cpp:54-96``
  ``queue_calc``           ``cppcode/cpuASPLqueue.cpp:11-53``
  ``conv_diameter_aspl``   ``cudacode/cudaASPLconv.cu:197-243``
  ``conv_calc``            ``cudacode/cudaASPLconv.cu:151-196``
  ``conv_wvc``             ``cudacode/cudaASPLconv.cu:244-308``
  ``graph_calc``           ``cudacode/cudaASPLgraph.cu:141-199``
  ``piece_diameter_aspl``  ``cudacode/cudaASPLpiece.cu:159-216`` (= cpuASPLpiece)
  ``box_diameter_aspl``    ``cudacode/cudaASPLbox.cu:166-226`` (= cpuASPLbox)
  ``beamer_calc``          ``cudacode/cudaASPLbeamer.cu:7-84``
  =====================  ==============================================

* ``RefCPU``: ctypes access to the reference's own CPU calculators compiled
  from the reference sources into ``oracle/_ref/libref_cpu.so`` (see
  ``oracle/Makefile``); used to pin this restatement.

Parity is pinned by (i) the reference's own CPU calculators run on the same
inputs (``tests/test_oracle.py``) and (ii) closed-form known answers (cycles,
complete graphs, hypercubes, the Petersen graph).  The reference ships no test
vectors of its own.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
INT_MAX = 2**31 - 1
SENTINEL = 100000000          # cudaASPLconv.cu:207,229,257,293
BEAMER_N = 1000000            # cudaASPLbeamer.cu:10-12 (31250 words x 32 bits)
BEAMER_LEVELS = 7             # cudaASPLbeamer.cu:17

_lib = None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    lib = ctypes.CDLL(path)
    lib.ggo_bfs.restype = ctypes.c_int
    lib.ggo_bfs.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p]
    _lib = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------
# Adjacency expansions.  Each returns the *pull* table adj[v, i] (the vertex v
# ORs the bits of adj[v, i]), which is what the GPU calculators gather
# (cudaASPLconv.cu:41-44, cudaASPLpiece.cu:41-50, cudaASPLbox.cu:44-57,
# cudaASPLgraph.cu:33-35).  For an undirected (symmetric) description it equals
# the out-list table of the CPU calculators (cpuASPLqueue.cpp:57-62).
# --------------------------------------------------------------------------

def pmod(a, n):
    """Mathematical modulo; equals C's (n + a) % n whenever n + a >= 0, the only
    case in which the reference's own index arithmetic is defined."""
    return np.mod(a, n)


def expand_part(N, M, diffs, n_rows=None):
    """Part/cyclic lift: vertex v has neighbours (v + diffs[v % M, i]) mod N.
    ``diffs`` is the padded [M, degree] table (padding = diff 0, cudaASPLconv.cu:200).
    ``n_rows`` > N adds the phantom rows the beamer kernel scans (cudaASPLbeamer.cu:38-50)."""
    diffs = np.asarray(diffs, dtype=np.int64).reshape(M, -1)
    rows = N if n_rows is None else n_rows
    v = np.arange(rows, dtype=np.int64)
    return pmod(v[:, None] + diffs[v % M], N).astype(np.int32)


def expand_piece(Nx, Ny, Mx, My, vals):
    """2-D torus lift (cpuASPLpiece.cpp:184-196): vertex x*Ny+y, diff table
    [Mx*My, degree, 2] (padding (0,0), cudaASPLpiece.cu:168-176)."""
    vals = np.asarray(vals, dtype=np.int64).reshape(Mx * My, -1, 2)
    x = np.repeat(np.arange(Nx), Ny)
    y = np.tile(np.arange(Ny), Nx)
    t = vals[(x % Mx) * My + (y % My)]
    tx = pmod(x[:, None] + t[:, :, 0], Nx)
    ty = pmod(y[:, None] + t[:, :, 1], Ny)
    return (tx * Ny + ty).astype(np.int32)


def expand_box(Nx, Ny, Nz, Mx, My, Mz, vals):
    """3-D torus lift (cpuASPLbox.cpp:115-130): vertex x*Ny*Nz+y*Nz+z, diff table
    [Mx*My*Mz, degree, 3] (padding (0,0,0), cudaASPLbox.cu:170-183)."""
    vals = np.asarray(vals, dtype=np.int64).reshape(Mx * My * Mz, -1, 3)
    v = np.arange(Nx * Ny * Nz)
    x, y, z = v // (Ny * Nz), (v // Nz) % Ny, v % Nz
    t = vals[((x % Mx) * My + (y % My)) * Mz + (z % Mz)]
    tx = pmod(x[:, None] + t[:, :, 0], Nx)
    ty = pmod(y[:, None] + t[:, :, 1], Ny)
    tz = pmod(z[:, None] + t[:, :, 2], Nz)
    return ((tx * Ny + ty) * Nz + tz).astype(np.int32)


def piece_reps(Nx, Ny, Mx, My):
    """Representatives = corner tile x<Mx, y<My (cpuASPLpiece.cpp:199-200)."""
    return np.array([x * Ny + y for x in range(Mx) for y in range(My)], dtype=np.int32)


def box_reps(Nx, Ny, Nz, Mx, My, Mz):
    """Representatives = corner tile (cpuASPLbox.cpp:133-134)."""
    return np.array([(x * Ny + y) * Nz + z for x in range(Mx) for y in range(My)
                     for z in range(Mz)], dtype=np.int32)


def pad_graph(N, lists, degree_max=None):
    """Adjacency lists -> [N, degree_max] table padded with self-loops
    (cudaASPLgraph.cu:144-153)."""
    dm = max((len(l) for l in lists), default=0) if degree_max is None else degree_max
    t = np.empty((N, max(dm, 1)), dtype=np.int32)
    for v in range(N):
        t[v, :] = v
        t[v, :len(lists[v])] = lists[v]
    return t[:, :dm] if dm else t[:, :0]


def pull_to_push_csr(adj):
    """CSR of the edges u -> v for every v and u in adj[v] (transpose of the pull
    table), so that the push BFS of gg_oracle.c explores what the GPU pull
    gathers explore.  Rows keep ascending v order within each u."""
    adj = np.asarray(adj, dtype=np.int64)
    n_rows, d = adj.shape
    if d == 0:
        return np.zeros(n_rows + 1, np.int32), np.zeros(0, np.int32)
    u = adj.reshape(-1)
    v = np.repeat(np.arange(n_rows, dtype=np.int64), d)
    order = np.lexsort((v, u))
    col = v[order].astype(np.int32)
    counts = np.bincount(u, minlength=n_rows)
    row_ptr = np.zeros(n_rows + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return row_ptr.astype(np.int32), col


def lists_to_csr(lists):
    """Out-list CSR straight from adjacency lists (cpuASPLqueue.cpp:57-62 order)."""
    row_ptr = np.zeros(len(lists) + 1, np.int64)
    np.cumsum([len(l) for l in lists], out=row_ptr[1:])
    col = np.array([u for l in lists for u in l], dtype=np.int32)
    return row_ptr.astype(np.int32), col


# --------------------------------------------------------------------------
# BFS
# --------------------------------------------------------------------------

@dataclass
class BFS:
    n: int                     # vertices
    sources: np.ndarray        # source vertex ids
    level_counts: np.ndarray   # uint64[n]: pairs at distance L (L=0: the sources)
    ecc: np.ndarray            # per-source eccentricity within its component
    reached: np.ndarray        # per-source reach (itself included)

    @property
    def levels(self):
        """max eccentricity = last level with pairs."""
        return int(self.ecc.max()) if len(self.ecc) else 0

    def total(self, cap=None):
        """sum over levels L <= cap of L * pairs(L), as an exact Python int."""
        c = self.level_counts
        top = len(c) - 1 if cap is None else min(cap, len(c) - 1)
        return sum(int(L) * int(c[L]) for L in range(1, top + 1) if c[L])

    @property
    def connected(self):
        return bool(np.all(self.reached == self.n))


def bfs(row_ptr, col, sources, threads=0):
    """All-pairs BFS (gg_oracle.c) from ``sources`` over the push CSR."""
    lib = _load()
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    src = np.ascontiguousarray(sources, dtype=np.int32)
    n = len(row_ptr) - 1
    lc = np.zeros(n, dtype=np.uint64)
    ecc = np.zeros(len(src), dtype=np.int32)
    reached = np.zeros(len(src), dtype=np.int64)
    rc = lib.ggo_bfs(n, _ptr(row_ptr), _ptr(col if len(col) else np.zeros(1, np.int32)),
                     len(src), _ptr(src if len(src) else np.zeros(1, np.int32)), threads,
                     _ptr(lc), _ptr(ecc), _ptr(reached))
    if rc != 0:
        raise ValueError("oracle BFS rejected its input")
    return BFS(n, src, lc, ecc, reached)


def bfs_pull(adj, sources, threads=0):
    rp, col = pull_to_push_csr(adj)
    return bfs(rp, col, sources, threads)


# --------------------------------------------------------------------------
# Reference return conventions, recomputed from exact counts.
# --------------------------------------------------------------------------

def _aspl(total_reps, N, M):
    """total *= N/M (integer division); double(total)/(int64(N)*(N-1))
    (cudaASPLconv.cu:241-242, cpuASPLqueue.cpp:93-94)."""
    total = total_reps * (N // M)
    den = N * (N - 1)
    return float(total) / den if den else float("nan")


def queue_diameter_aspl(N, M, diffs, threads=0):
    """cpuASPLqueue<cap>::diameterASPL (cpuASPLqueue.cpp:54-96):
    (INT_MAX if any source misses a vertex else max eccentricity, ASPL)."""
    r = bfs_pull(expand_part(N, M, diffs), np.arange(M), threads)
    diam = INT_MAX if not r.connected else r.levels
    return diam, _aspl(r.total(), N, M)


def queue_calc(N, M, diffs, threads=0):
    """cpuASPLqueue<cap>::calc (cpuASPLqueue.cpp:11-53): 1e9 if disconnected."""
    r = bfs_pull(expand_part(N, M, diffs), np.arange(M), threads)
    return 1e9 if not r.connected else _aspl(r.total(), N, M)


def _level_loop(r: BFS, last_step):
    """The level loop `for step=1..last_step` of the GPU calculators: returns
    ('done', diameter) when a step finds no new pair (then the AND test runs),
    or ('cap', None) when every step up to last_step found new pairs."""
    E = r.levels
    if E + 1 <= last_step:
        return ("done", E)
    return ("cap", None)


def conv_diameter_aspl(N, M, diffs, *, reps=None, adj=None, threads=0):
    """cudaASPLconv::diameterASPL (cudaASPLconv.cu:197-243); also the piece and
    box calculators (cudaASPLpiece.cu:159-216, cudaASPLbox.cu:166-226), which
    differ only in the expansion and the representatives."""
    if adj is None:
        adj = expand_part(N, M, diffs)
    if reps is None:
        reps = np.arange(M)
    r = bfs_pull(adj, reps, threads)
    kind, E = _level_loop(r, 99)
    if kind == "done":
        if not r.connected:
            return SENTINEL, float(SENTINEL)
        return E, _aspl(r.total(), N, M)
    return SENTINEL, _aspl(r.total(cap=99), N, M)


def conv_calc(N, M, diffs, threads=0):
    """cudaASPLconv::calc (cudaASPLconv.cu:151-196): 1e9 if disconnected."""
    r = bfs_pull(expand_part(N, M, diffs), np.arange(M), threads)
    kind, _ = _level_loop(r, 99)
    if kind == "done":
        return 1e9 if not r.connected else _aspl(r.total(), N, M)
    return _aspl(r.total(cap=99), N, M)


def wvc_from(r: BFS, M):
    """Lane-aggregated completion count of cudaASPLconv.cu:258-285: bit j of the
    AND over all visited words is set when every source s<M with s%32==j has
    reached every vertex.  At the last updating level E the count is the number
    of bit positions j whose latest-completing source completes exactly at E."""
    E = r.levels
    latest = {}
    for s in range(M):
        latest[s % 32] = max(latest.get(s % 32, 0), int(r.ecc[s]))
    return sum(1 for j, e in latest.items() if e == E)


def conv_wvc(N, M, diffs, threads=0):
    """cudaASPLconv::WVCdiameterASPL (cudaASPLconv.cu:244-308) ->
    (WVC, diameter, ASPL); (1e8, 1e8, 1e8) if disconnected or the level loop
    reaches step 100 with new pairs."""
    r = bfs_pull(expand_part(N, M, diffs), np.arange(M), threads)
    E = r.levels
    if E + 1 > 100:
        return SENTINEL, SENTINEL, float(SENTINEL)
    if not r.connected:
        return SENTINEL, SENTINEL, float(SENTINEL)
    return wvc_from(r, M), E, _aspl(r.total(), N, M)


def graph_calc(N, adj, threads=0, chunk=1024):
    """cudaASPLgraph::calc (cudaASPLgraph.cu:141-199) on the padded table
    ``adj`` [N, degree_max] -> (diameter, total over all ordered pairs).
    Sources go in chunks of 1024 (:158); the first chunk whose level loop
    reaches step 199 with new pairs returns (-2,-2) (:187-190), the first chunk
    that ends disconnected returns (-1,-1) (:179-182)."""
    r = bfs_pull(adj, np.arange(N), threads)
    diameter = 0
    for off in range(0, N, chunk):
        e = r.ecc[off:off + chunk]
        ok = r.reached[off:off + chunk] == N
        if int(e.max()) >= 199:
            return -2, -2
        if not ok.all():
            return -1, -1
        diameter = max(diameter, int(e.max()))
    return diameter, r.total()


def piece_diameter_aspl(Nx, Ny, Mx, My, vals, threads=0):
    N, M = Nx * Ny, Mx * My
    return conv_diameter_aspl(N, M, None, reps=piece_reps(Nx, Ny, Mx, My),
                              adj=expand_piece(Nx, Ny, Mx, My, vals), threads=threads)


def box_diameter_aspl(Nx, Ny, Nz, Mx, My, Mz, vals, threads=0):
    N, M = Nx * Ny * Nz, Mx * My * Mz
    return conv_diameter_aspl(N, M, None, reps=box_reps(Nx, Ny, Nz, Mx, My, Mz),
                              adj=expand_box(Nx, Ny, Nz, Mx, My, Mz, vals), threads=threads)


def beamer_calc(N, M, diffs, regular=True, threads=0):
    """cudaASPLbeamer::calc (cudaASPLbeamer.cu:71-84): 1e8 for non-regular
    input (:72).  The kernel (:7-53) scans the fixed 10^6-vertex bitset, so rows
    v >= N (pulling from (v + diff) mod N) are reached too, and it stops after 7
    levels; no connectivity test."""
    if not regular:
        return float(SENTINEL)
    adj = expand_part(N, M, diffs, n_rows=max(N, BEAMER_N))
    r = bfs_pull(adj, np.arange(M), threads)
    return _aspl(r.total(cap=BEAMER_LEVELS), N, M)


# --------------------------------------------------------------------------
# The reference's own CPU calculators (compiled from the reference sources).
# --------------------------------------------------------------------------

class RefCPU:
    """ctypes access to oracle/_ref/libref_cpu.so (built by ``make -C oracle ref``)."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "_ref", "libref_cpu.so")
        self.lib = ctypes.CDLL(path)
        I, P, D = ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        IP = ctypes.POINTER(ctypes.c_int)
        self.lib.ggr_queue_diameter_aspl.argtypes = [I, I, P, P, IP, D]
        self.lib.ggr_queue_calc.argtypes = [I, I, P, P, D]
        self.lib.ggr_piece_diameter_aspl.argtypes = [I, I, I, I, P, P, IP, D]
        self.lib.ggr_box_diameter_aspl.argtypes = [I, I, I, I, I, I, P, P, IP, D]

    @staticmethod
    def available(path=None):
        return os.path.exists(path or os.path.join(HERE, "_ref", "libref_cpu.so"))

    @staticmethod
    def _rows(rows, width=1):
        deg = np.array([len(r) // width for r in rows], dtype=np.int32)
        flat = np.array([x for r in rows for x in r] or [0], dtype=np.int32)
        return deg, flat

    def queue_diameter_aspl(self, N, M, rows):
        deg, flat = self._rows(rows)
        d, a = ctypes.c_int(), ctypes.c_double()
        if self.lib.ggr_queue_diameter_aspl(N, M, _ptr(deg), _ptr(flat), ctypes.byref(d),
                                            ctypes.byref(a)):
            raise ValueError("N above the largest instantiated capacity")
        return d.value, a.value

    def queue_calc(self, N, M, rows):
        deg, flat = self._rows(rows)
        a = ctypes.c_double()
        if self.lib.ggr_queue_calc(N, M, _ptr(deg), _ptr(flat), ctypes.byref(a)):
            raise ValueError("N above the largest instantiated capacity")
        return a.value

    def piece_diameter_aspl(self, Nx, Ny, Mx, My, rows):
        deg, flat = self._rows(rows, 2)
        d, a = ctypes.c_int(), ctypes.c_double()
        self.lib.ggr_piece_diameter_aspl(Nx, Ny, Mx, My, _ptr(deg), _ptr(flat),
                                         ctypes.byref(d), ctypes.byref(a))
        return d.value, a.value

    def box_diameter_aspl(self, Nx, Ny, Nz, Mx, My, Mz, rows):
        deg, flat = self._rows(rows, 3)
        d, a = ctypes.c_int(), ctypes.c_double()
        self.lib.ggr_box_diameter_aspl(Nx, Ny, Nz, Mx, My, Mz, _ptr(deg), _ptr(flat),
                                       ctypes.byref(d), ctypes.byref(a))
        return d.value, a.value


class RefGPU:
    """ctypes access to the reference GPU calculators compiled for sm_100a from
    the reference sources (oracle/_ref/libref_{graph,conv,piece,box,beamer}.so).
    Test and baseline infrastructure: used to pin the WVC convention and to time
    the reference GPU path on the same B200."""

    def __init__(self, kind):
        self.kind = kind
        self.lib = ctypes.CDLL(os.path.join(HERE, "_ref", f"libref_{kind}.so"))
        L = self.lib
        I, P, D = ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        IP = ctypes.POINTER(ctypes.c_int)
        getattr(L, f"ggrg_{kind}_create").restype = P
        getattr(L, f"ggrg_{kind}_destroy").argtypes = [P]
        if kind == "graph":
            L.ggrg_graph_create.argtypes = [I, I, I]
            L.ggrg_graph_calc.argtypes = [P, I, P, P, IP, ctypes.POINTER(ctypes.c_int64)]
        elif kind == "conv":
            L.ggrg_conv_create.argtypes = [I, I, I, I]
            L.ggrg_conv_calc.argtypes = [P, I, I, P, P, D]
            L.ggrg_conv_diameter_aspl.argtypes = [P, I, I, P, P, IP, D]
            L.ggrg_conv_wvc.argtypes = [P, I, I, P, P, IP, IP, D]
        elif kind == "beamer":
            L.ggrg_beamer_create.argtypes = [I, I, I, I]
            L.ggrg_beamer_calc.argtypes = [P, I, I, P, P, D]
        elif kind == "piece":
            L.ggrg_piece_create.argtypes = [I] * 6
            L.ggrg_piece_diameter_aspl.argtypes = [P, I, I, I, I, P, P, IP, D]
        elif kind == "box":
            L.ggrg_box_create.argtypes = [I] * 8
            L.ggrg_box_diameter_aspl.argtypes = [P, I, I, I, I, I, I, P, P, IP, D]
        self.h = None

    @staticmethod
    def available(kind):
        return os.path.exists(os.path.join(HERE, "_ref", f"libref_{kind}.so"))

    def create(self, *args):
        self.h = getattr(self.lib, f"ggrg_{self.kind}_create")(*args)
        return self

    def close(self):
        if self.h:
            getattr(self.lib, f"ggrg_{self.kind}_destroy")(self.h)
            self.h = None

    @staticmethod
    def _flat(table, rows):
        t = np.ascontiguousarray(np.asarray(table, dtype=np.int32).reshape(rows, -1))
        per = t.shape[1]
        return t, per

    def graph_calc(self, adj):
        adj = np.ascontiguousarray(np.asarray(adj, dtype=np.int32))
        N = len(adj)
        deg = np.full(N, adj.shape[1], dtype=np.int32)
        d, tot = ctypes.c_int(), ctypes.c_int64()
        self.lib.ggrg_graph_calc(self.h, N, _ptr(deg), _ptr(adj), ctypes.byref(d), ctypes.byref(tot))
        return d.value, tot.value

    def _part_args(self, N, M, diffs):
        t = np.ascontiguousarray(np.asarray(diffs, dtype=np.int32).reshape(M, -1))
        deg = np.full(M, t.shape[1], dtype=np.int32)
        return t, deg

    def conv_calc(self, N, M, diffs):
        t, deg = self._part_args(N, M, diffs)
        a = ctypes.c_double()
        self.lib.ggrg_conv_calc(self.h, N, M, _ptr(deg), _ptr(t), ctypes.byref(a))
        return a.value

    def conv_diameter_aspl(self, N, M, diffs):
        t, deg = self._part_args(N, M, diffs)
        d, a = ctypes.c_int(), ctypes.c_double()
        self.lib.ggrg_conv_diameter_aspl(self.h, N, M, _ptr(deg), _ptr(t), ctypes.byref(d),
                                         ctypes.byref(a))
        return d.value, a.value

    def conv_wvc(self, N, M, diffs):
        t, deg = self._part_args(N, M, diffs)
        w, d, a = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self.lib.ggrg_conv_wvc(self.h, N, M, _ptr(deg), _ptr(t), ctypes.byref(w), ctypes.byref(d),
                               ctypes.byref(a))
        return w.value, d.value, a.value

    def beamer_calc(self, N, M, diffs):
        t, deg = self._part_args(N, M, diffs)
        a = ctypes.c_double()
        self.lib.ggrg_beamer_calc(self.h, N, M, _ptr(deg), _ptr(t), ctypes.byref(a))
        return a.value

    def piece_diameter_aspl(self, Nx, Ny, Mx, My, vals):
        t = np.ascontiguousarray(np.asarray(vals, dtype=np.int32).reshape(Mx * My, -1))
        deg = np.full(Mx * My, t.shape[1] // 2, dtype=np.int32)
        d, a = ctypes.c_int(), ctypes.c_double()
        self.lib.ggrg_piece_diameter_aspl(self.h, Nx, Ny, Mx, My, _ptr(deg), _ptr(t),
                                          ctypes.byref(d), ctypes.byref(a))
        return d.value, a.value

    def box_diameter_aspl(self, Nx, Ny, Nz, Mx, My, Mz, vals):
        M = Mx * My * Mz
        t = np.ascontiguousarray(np.asarray(vals, dtype=np.int32).reshape(M, -1))
        deg = np.full(M, t.shape[1] // 3, dtype=np.int32)
        d, a = ctypes.c_int(), ctypes.c_double()
        self.lib.ggrg_box_diameter_aspl(self.h, Nx, Ny, Nz, Mx, My, Mz, _ptr(deg), _ptr(t),
                                        ctypes.byref(d), ctypes.byref(a))
        return d.value, a.value
