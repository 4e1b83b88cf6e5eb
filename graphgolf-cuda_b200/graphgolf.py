"""graphgolf -- Python mirror of the reference calculator API over libggb200.so.

The reference (C++) exposes calculators constructed from the graph dimensions
and called once per candidate (cudacode/cudaASPL*.hpp).  This module keeps
those names, constructor arguments, method names and return conventions:

=========================  ===========================================  =====================
Python                     reference                                    C ABI (include/gg.h)
=========================  ===========================================  =====================
``graph``                  ``graphgolf::graph`` (cppcode/graph.hpp)     --
``part``                   ``graphgolf::part`` (cppcode/part.hpp)       --
``piece``                  ``graphgolf::piece`` (cppcode/piece.hpp)     --
``box``                    ``graphgolf::box`` (cppcode/box.hpp)         --
``cudaASPLgraph``          cudacode/cudaASPLgraph.hpp:14-18             ``gg_graph_*``
``cudaASPLconv``           cudacode/cudaASPLconv.hpp:16-22              ``gg_conv_*``
``cudaASPLpiece``          cudacode/cudaASPLpiece.hpp:16-20             ``gg_piece_*``
``cudaASPLbox``            cudacode/cudaASPLbox.hpp:16-20               ``gg_box_*``
``cudaASPLbeamer``         cudacode/cudaASPLbeamer.hpp:12-16            ``gg_beamer_*``
=========================  ===========================================  =====================

Every calculator call runs on the GPU through the C ABI.  There is no CPU
fallback: if the library cannot be loaded, or no GPU is present, the calls
raise ``GGError``.
"""
from __future__ import annotations

import ctypes
import os
import re
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libggb200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "gg.h")

GG_OK, GG_BAD_ARG, GG_CUDA_ERROR, GG_TIMEOUT, GG_OUT_OF_MEMORY, GG_NO_DEVICE = range(6)
STATUS_NAMES = {0: "GG_OK", 1: "GG_BAD_ARG", 2: "GG_CUDA_ERROR", 3: "GG_TIMEOUT",
                4: "GG_OUT_OF_MEMORY", 5: "GG_NO_DEVICE"}


class GGError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Result(ctypes.Structure):
    """gg_result (include/gg.h)."""
    _fields_ = [("total", ctypes.c_uint64), ("reached", ctypes.c_uint64),
                ("pairs", ctypes.c_uint64), ("scale", ctypes.c_uint64),
                ("levels", ctypes.c_int32), ("capped", ctypes.c_int32),
                ("connected", ctypes.c_int32), ("wvc", ctypes.c_int32),
                ("n_sources", ctypes.c_int32), ("batches", ctypes.c_int32),
                ("level_steps", ctypes.c_int32), ("reserved", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EvalOpts(ctypes.Structure):
    """gg_eval_opts (include/gg.h)."""
    _fields_ = [("max_levels", ctypes.c_int32), ("src_begin", ctypes.c_int32),
                ("src_end", ctypes.c_int32), ("want_wvc", ctypes.c_int32),
                ("level_counts", ctypes.c_void_p), ("level_ns", ctypes.c_void_p)]


_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)
_EPP = ctypes.POINTER(ctypes.c_void_p)

_SIGS = {
    "gg_graph_create": [_I, _I, _I, _EPP],
    "gg_graph_calc": [_P, _P, _IP, ctypes.POINTER(ctypes.c_int64)],
    "gg_conv_create": [_I, _I, _I, _I, _EPP],
    "gg_conv_calc": [_P, _P, _DP],
    "gg_conv_diameter_aspl": [_P, _P, _IP, _DP],
    "gg_conv_wvc_diameter_aspl": [_P, _P, _IP, _IP, _DP],
    "gg_piece_create": [_I, _I, _I, _I, _I, _I, _EPP],
    "gg_piece_diameter_aspl": [_P, _P, _IP, _DP],
    "gg_box_create": [_I, _I, _I, _I, _I, _I, _I, _I, _EPP],
    "gg_box_diameter_aspl": [_P, _P, _IP, _DP],
    "gg_beamer_create": [_I, _I, _I, _I, _EPP],
    "gg_beamer_calc": [_P, _P, _I, _DP],
    "gg_eval": [_P, _P, ctypes.POINTER(EvalOpts), ctypes.POINTER(Result)],
    "gg_eval_device": [_P, _P, ctypes.POINTER(EvalOpts), ctypes.POINTER(Result), _P],
    "gg_last_device_ms": [_P, _DP],
    "gg_last_launches": [_P, _IP],
    "gg_last_batch_ns": [_P, _P, _I],
    "gg_last_transfer_bytes": [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)],
    "gg_set_batch_sources": [_P, _I],
    "gg_autotune": [_P, _P, _I, _IP, _DP],
    "gg_set_wait_limit_ms": [_P, _I],
    "gg_gather_peak": [_I, _I, _I, _I, _DP, _DP],
    "gg_level_probe": [_I, _I, _I, _I, _I, _DP],
    "gg_engine_plan": [_P, _IP, _IP, _IP],
    "gg_set_tune_cache": [ctypes.c_char_p],
    "gg_batch_autotune": [_P, _I, _P, _I, _DP],
    "gg_batch_chunk": [_P, _I, _IP],
    "gg_lift_autotune": [_P, _I, _P, _I, _I, _IP, _DP],
    "gg_destroy": [_P],
    "gg_graph_eval_noalloc": [_P, _I, _I, _I, _P, _P],
    "gg_batch_create": [_I, _EPP],
    "gg_batch_add_base": [_P, _I, _I, _P, _IP],
    "gg_batch_set_chunk": [_P, _I, _I],
    "gg_batch_set_base": [_P, _I, _P],
    "gg_batch_vertex_hist": [_P, _I, _I, _P],
    "gg_batch_eval": [_P, _I, _P, _P],
    "gg_batch_eval_device": [_P, _I, _P, _P, _P],
    "gg_batch_device_status": [_P, _P, _IP],
    "gg_batch_last_ms": [_P, _DP],
    "gg_batch_destroy": [_P],
    "gg_gen_swaps": [_I, _I, _P, _I, _I, ctypes.c_uint64, _P],
    "gg_surrogate_create": [_I, _I, _I, _I, ctypes.c_uint64, _EPP],
    "gg_surrogate_set_graph": [_P, _P, _P],
    "gg_surrogate_predict": [_P, _I, _P, _P],
    "gg_surrogate_train": [_P, _I, _P, _P, _P, ctypes.c_float, ctypes.POINTER(ctypes.c_float)],
    "gg_surrogate_param_count": [_P, _IP],
    "gg_surrogate_get_params": [_P, _P],
    "gg_surrogate_set_params": [_P, _P],
    "gg_surrogate_grad": [_P, _I, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_float)],
    "gg_surrogate_destroy": [_P],
    "gg_gen_random_regular": [_I, _I, ctypes.c_uint64, _P],
    "gg_inc_create": [_I, _I, _I, _EPP],
    "gg_inc_set_graph": [_P, _P, _P],
    "gg_inc_eval": [_P, _P, _P, _IP],
    "gg_inc_commit": [_P, _P, _P],
    "gg_inc_destroy": [_P],
    "gg_gen_cyclic_lift": [_I, _I, _I, ctypes.c_uint64, _P],
    "gg_gen_piece_lift": [_I, _I, _I, _I, _I, ctypes.c_uint64, _P],
    "gg_lift_create": [_I, _I, _I, _I, _EPP],
    "gg_lift_create_piece": [_I, _I, _I, _I, _I, _I, _EPP],
    "gg_lift_create_box": [_I, _I, _I, _I, _I, _I, _I, _I, _EPP],
    "gg_gen_piece_moves": [_I, _I, _I, _I, _I, _P, _I, ctypes.c_uint64, _P],
    "gg_gen_box_moves": [_I, _I, _I, _I, _I, _I, _I, _P, _I, ctypes.c_uint64, _P],
    "gg_lift_set_base": [_P, _P],
    "gg_lift_eval": [_P, _I, _P, _I, _P],
    "gg_lift_set_group": [_P, _I],
    "gg_lift_group": [_P, _IP],
    "gg_lift_last_ms": [_P, _DP],
    "gg_lift_set_half_ppm": [_P, _I],
    "gg_lift_last_level_ns": [_P, _P, _I],
    "gg_lift_destroy": [_P],
    "gg_gen_lift_moves": [_I, _I, _I, _P, _I, ctypes.c_uint64, _P],
}


def lib():
    """Load libggb200.so (built in-tree by graphgolf-cuda_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GGError(GG_CUDA_ERROR, f"{LIB_PATH} is missing: run graphgolf-cuda_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.gg_status_str.restype = ctypes.c_char_p
    L.gg_status_str.argtypes = [_I]
    L.gg_last_error.restype = ctypes.c_char_p
    L.gg_abi_version.restype = ctypes.c_int
    _lib = L
    return L


def header_functions(path=HEADER):
    """Names of every function declared in include/gg.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gg_[a-z0-9_]+)\s*\(", text)))


def _check(status):
    if status != GG_OK:
        raise GGError(status, lib().gg_last_error().decode())


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ----------------------------------------------------------------------------
# Generators (host, deterministic)
# ----------------------------------------------------------------------------

def random_regular(n, d, seed):
    """Simple connected random d-regular graph -> int32 adjacency [n, d]."""
    out = np.empty((n, d), dtype=np.int32)
    _check(lib().gg_gen_random_regular(n, d, seed, _ptr(out)))
    return out


def cyclic_lift(m, g, d, seed):
    """Simple connected random cyclic lift in part form -> (N, M, diffs [m, d])."""
    out = np.empty((m, d), dtype=np.int32)
    _check(lib().gg_gen_cyclic_lift(m, g, d, seed, _ptr(out)))
    return m * g, m, out


def piece_lift(Mx, My, kx, ky, d, seed):
    """Simple connected random 2-D torus lift -> (Nx, Ny, Mx, My, vals [Mx*My, d, 2])."""
    out = np.empty((Mx * My, d, 2), dtype=np.int32)
    _check(lib().gg_gen_piece_lift(Mx, My, kx, ky, d, seed, _ptr(out)))
    return Mx * kx, My * ky, Mx, My, out


# ----------------------------------------------------------------------------
# Data model (cppcode/graph.hpp, part.hpp, piece.hpp, box.hpp) and text formats
# ----------------------------------------------------------------------------

@dataclass
class graph:
    """Edge-list graph (cppcode/graph.hpp:11-52).  load() reads "u v" lines;
    N = max id + 1, each edge is stored at both ends."""
    edges: List[List[int]] = field(default_factory=list)
    N: int = 0
    degree_max: int = 0

    def load(self, ist):
        pairs = []
        n = 0
        for line in ist.read().splitlines() if hasattr(ist, "read") else ist:
            parts = line.split()
            if len(parts) < 2:
                continue
            u, v = int(parts[0]), int(parts[1])
            pairs.append((u, v))
            n = max(n, u, v)
        self.N = n + 1
        self.edges = [[] for _ in range(self.N)]
        for u, v in pairs:
            self.edges[u].append(v)
            self.edges[v].append(u)
        self.degree_max = max((len(e) for e in self.edges), default=0)
        return self

    def is_regular(self):
        return all(len(e) == self.degree_max for e in self.edges)

    def print(self, ost):
        for v, lst in enumerate(self.edges):
            for u in lst:
                if u < v:
                    ost.write(f"{u} {v}\n")

    @classmethod
    def from_adjacency(cls, adj):
        adj = np.asarray(adj)
        g = cls(edges=[list(map(int, r)) for r in adj], N=len(adj), degree_max=adj.shape[1])
        return g

    @classmethod
    def from_pairs(cls, pairs):
        """The graph load() makes from these "u v" lines, in order."""
        pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
        return cls().load(f"{u} {v}" for u, v in pairs.tolist())

    def table(self, degree_max=None):
        """N x degree_max int32, padded with self-loops (cudaASPLgraph.cu:144-153)."""
        dm = self.degree_max if degree_max is None else degree_max
        t = np.repeat(np.arange(self.N, dtype=np.int32)[:, None], max(dm, 0), axis=1)
        for v, lst in enumerate(self.edges):
            k = min(len(lst), dm)
            t[v, :k] = lst[:k]
        return t


@dataclass
class part:
    """Cyclic lift (cppcode/part.hpp:6-44): N vertices, M orbit rows of diffs."""
    N: int = 0
    M: int = 0
    regular: bool = True
    degree: int = 0
    edges: List[List[int]] = field(default_factory=list)

    def load(self, ist):
        tok = (ist.read() if hasattr(ist, "read") else ist).split()
        it = iter(tok)
        self.N, self.M = int(next(it)), int(next(it))
        self.edges = []
        self.degree, self.regular = 0, True
        for _ in range(self.M):
            E = int(next(it))
            if not self.degree:
                self.degree = E
            elif self.degree != E:
                self.regular = False
                self.degree = max(self.degree, E)
            self.edges.append([int(next(it)) for _ in range(E)])
        return self

    def print(self, ost):
        ost.write(f"{self.N} {self.M}\n")
        for row in self.edges:
            ost.write(" ".join([str(len(row))] + [str(x) for x in row]) + "\n")

    @classmethod
    def from_diffs(cls, N, M, diffs):
        rows = [list(map(int, r)) for r in np.asarray(diffs).reshape(M, -1)]
        return cls(N=N, M=M, regular=True, degree=len(rows[0]) if rows else 0, edges=rows)

    def table(self, degree):
        """M x degree int32, padding diff 0 (cudaASPLconv.cu:199-201)."""
        t = np.zeros((self.M, degree), dtype=np.int32)
        for i, row in enumerate(self.edges):
            k = min(len(row), degree)
            t[i, :k] = row[:k]
        return t


@dataclass
class piece:
    """2-D torus lift (cppcode/piece.hpp:7-53): edges[x][y] = [(dx, dy), ...]."""
    Nx: int = 0
    Ny: int = 0
    Mx: int = 0
    My: int = 0
    regular: bool = True
    degree: int = 0
    edges: list = field(default_factory=list)

    def load(self, ist):
        tok = (ist.read() if hasattr(ist, "read") else ist).split()
        it = iter(tok)
        self.Nx, self.Ny, self.Mx, self.My = (int(next(it)) for _ in range(4))
        self.degree, self.regular = 0, True
        self.edges = [[[] for _ in range(self.My)] for _ in range(self.Mx)]
        for x in range(self.Mx):
            for y in range(self.My):
                E = int(next(it))
                if not self.degree:
                    self.degree = E
                elif self.degree != E:
                    self.regular = False
                self.edges[x][y] = [(int(next(it)), int(next(it))) for _ in range(E)]
        return self

    def print(self, ost):
        ost.write(f"{self.Nx} {self.Ny} {self.Mx} {self.My}\n")
        for x in range(self.Mx):
            for y in range(self.My):
                row = self.edges[x][y]
                ost.write(" ".join([str(len(row))] + [f"{a} {b}" for a, b in row]) + "\n")

    @classmethod
    def from_table(cls, Nx, Ny, Mx, My, vals):
        """The piece of a table [Mx*My, d, 2] (e.g. an annealer's result)."""
        t = np.asarray(vals).reshape(Mx * My, -1, 2)
        edges = [[[(int(a), int(b)) for a, b in t[x * My + y]] for y in range(My)] for x in range(Mx)]
        return cls(Nx=Nx, Ny=Ny, Mx=Mx, My=My, regular=True, degree=t.shape[1], edges=edges)

    def table(self, degree):
        """Mx*My*degree*2 int32, padding (0,0) (cudaASPLpiece.cu:166-176)."""
        t = np.zeros((self.Mx * self.My, degree, 2), dtype=np.int32)
        for x in range(self.Mx):
            for y in range(self.My):
                for e, (a, b) in enumerate(self.edges[x][y][:degree]):
                    t[x * self.My + y, e] = (a, b)
        return t


@dataclass
class box:
    """3-D torus lift (cppcode/box.hpp:6-81): edges[x][y][z] = [(dx, dy, dz), ...]."""
    Nx: int = 0
    Ny: int = 0
    Nz: int = 0
    Mx: int = 0
    My: int = 0
    Mz: int = 0
    regular: bool = True
    degree: int = 0
    edges: list = field(default_factory=list)

    @property
    def N(self):
        return self.Nx * self.Ny * self.Nz

    @property
    def M(self):
        return self.Mx * self.My * self.Mz

    def load(self, ist):
        tok = (ist.read() if hasattr(ist, "read") else ist).split()
        it = iter(tok)
        self.Nx, self.Ny, self.Nz, self.Mx, self.My, self.Mz = (int(next(it)) for _ in range(6))
        self.regular = True
        self.edges = [[[[] for _ in range(self.Mz)] for _ in range(self.My)] for _ in range(self.Mx)]
        for x in range(self.Mx):
            for y in range(self.My):
                for z in range(self.Mz):
                    E = int(next(it))
                    if not self.degree:
                        self.degree = E
                    elif self.degree != E:
                        self.regular = False
                    self.edges[x][y][z] = [(int(next(it)), int(next(it)), int(next(it)))
                                           for _ in range(E)]
        return self

    def print(self, ost):
        ost.write(f"{self.Nx} {self.Ny} {self.Nz} {self.Mx} {self.My} {self.Mz}\n")
        for x in range(self.Mx):
            for y in range(self.My):
                for z in range(self.Mz):
                    row = self.edges[x][y][z]
                    ost.write(" ".join([str(len(row))] + [f"{a} {b} {c}" for a, b, c in row]) + "\n")

    @classmethod
    def from_table(cls, Nx, Ny, Nz, Mx, My, Mz, vals):
        """The box of a table [Mx*My*Mz, d, 3] (e.g. an annealer's result)."""
        t = np.asarray(vals).reshape(Mx * My * Mz, -1, 3)
        edges = [[[[tuple(int(c) for c in e) for e in t[(x * My + y) * Mz + z]] for z in range(Mz)]
                  for y in range(My)] for x in range(Mx)]
        return cls(Nx=Nx, Ny=Ny, Nz=Nz, Mx=Mx, My=My, Mz=Mz, regular=True, degree=t.shape[1], edges=edges)

    def table(self, degree):
        """Mx*My*Mz*degree*3 int32, padding (0,0,0) (cudaASPLbox.cu:170-184)."""
        t = np.zeros((self.M, degree, 3), dtype=np.int32)
        for x in range(self.Mx):
            for y in range(self.My):
                for z in range(self.Mz):
                    for e, tr in enumerate(self.edges[x][y][z][:degree]):
                        t[(x * self.My + y) * self.Mz + z, e] = tr
        return t


# ----------------------------------------------------------------------------
# Form -> plain graph converters (cppcode/piece2graph.cpp:84-103,
# cppcode/box2graph.cpp:86-106): every vertex's lifted edges, each pair written
# once as (min, max), sorted, duplicates dropped.
# ----------------------------------------------------------------------------

def _unique_pairs(a, b):
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    if lo.size == 0:
        return np.zeros((0, 2), dtype=np.int64)
    return np.unique(np.stack([lo, hi], axis=1), axis=0)


def part_pairs(p: part):
    """Edge list of a cyclic lift: vertex v has edges v -> (v + diff) mod N for
    the diffs of orbit row v mod M (cudaASPLconv.cu:35-48 applies the same rule)."""
    a, b = [], []
    for r, row in enumerate(p.edges):
        if not row:
            continue
        v = np.arange(r, p.N, p.M, dtype=np.int64)
        for e in row:
            a.append(v)
            b.append((v + e) % p.N)
    if not a:
        return _unique_pairs(np.zeros(0, np.int64), np.zeros(0, np.int64))
    return _unique_pairs(np.concatenate(a), np.concatenate(b))


def piece_pairs(p: piece):
    """piece2graph: vertex x*Ny + y, neighbour ((x+dx) mod Nx)*Ny + (y+dy) mod Ny,
    diffs of tile (x mod Mx, y mod My)."""
    a, b = [], []
    for tx in range(p.Mx):
        for ty in range(p.My):
            xs = np.arange(tx, p.Nx, p.Mx, dtype=np.int64)[:, None]
            ys = np.arange(ty, p.Ny, p.My, dtype=np.int64)[None, :]
            for dx, dy in p.edges[tx][ty]:
                a.append((xs * p.Ny + ys).ravel())
                b.append((((xs + dx) % p.Nx) * p.Ny + (ys + dy) % p.Ny).ravel())
    if not a:
        return _unique_pairs(np.zeros(0, np.int64), np.zeros(0, np.int64))
    return _unique_pairs(np.concatenate(a), np.concatenate(b))


def box_pairs(p: box):
    """box2graph: vertex (x*Ny + y)*Nz + z (box.hpp xyz2id), neighbour at the
    wrapped (x+dx, y+dy, z+dz), diffs of tile (x mod Mx, y mod My, z mod Mz)."""
    a, b = [], []
    for tx in range(p.Mx):
        for ty in range(p.My):
            for tz in range(p.Mz):
                xs = np.arange(tx, p.Nx, p.Mx, dtype=np.int64)[:, None, None]
                ys = np.arange(ty, p.Ny, p.My, dtype=np.int64)[None, :, None]
                zs = np.arange(tz, p.Nz, p.Mz, dtype=np.int64)[None, None, :]
                for dx, dy, dz in p.edges[tx][ty][tz]:
                    a.append(((xs * p.Ny + ys) * p.Nz + zs).ravel())
                    b.append(((((xs + dx) % p.Nx) * p.Ny + (ys + dy) % p.Ny) * p.Nz
                              + (zs + dz) % p.Nz).ravel())
    if not a:
        return _unique_pairs(np.zeros(0, np.int64), np.zeros(0, np.int64))
    return _unique_pairs(np.concatenate(a), np.concatenate(b))


def to_graph(p):
    """Any form as the plain graph its edge list loads into."""
    if isinstance(p, graph):
        return p
    fn = {part: part_pairs, piece: piece_pairs, box: box_pairs}[type(p)]
    return graph.from_pairs(fn(p))


def write_pairs(pairs, ost):
    """"a b" lines, as piece2graph/box2graph print them."""
    for a, b in np.asarray(pairs).tolist():
        ost.write(f"{a} {b}\n")


# ----------------------------------------------------------------------------
# Engine handle
# ----------------------------------------------------------------------------

class Engine:
    """One gg_engine.  Use the calculator classes below for the reference API;
    this class adds the raw exact counts (gg_eval)."""

    def __init__(self, handle, table_shape):
        self._h = handle
        self.table_shape = table_shape

    def _table(self, t):
        t = _i32(t)
        if t.size != int(np.prod(self.table_shape)):
            raise GGError(GG_BAD_ARG, f"table has {t.size} entries, expected {self.table_shape}")
        return t

    def eval(self, table, max_levels=0, src_range=None, want_wvc=False, level_counts=False):
        t = self._table(table)
        o = EvalOpts()
        o.max_levels = max_levels
        if src_range is not None:
            o.src_begin, o.src_end = src_range
        o.want_wvc = int(want_wvc)
        lc = None
        if level_counts:
            if max_levels <= 0:
                raise GGError(GG_BAD_ARG, "level_counts needs max_levels > 0")
            lc = np.zeros(max_levels + 1, dtype=np.uint64)
            o.level_counts = lc.ctypes.data
        r = Result()
        _check(lib().gg_eval(self._h, _ptr(t), ctypes.byref(o), ctypes.byref(r)))
        d = r.as_dict()
        if lc is not None:
            d["level_counts"] = lc
        return d

    def eval_device(self, dev_ptr, max_levels=0, stream=0, level_ns=False, src_range=None):
        o = EvalOpts()
        o.max_levels = max_levels
        if src_range is not None:
            o.src_begin, o.src_end = src_range
        ns = None
        if level_ns:
            if max_levels <= 0:
                raise GGError(GG_BAD_ARG, "level_ns needs max_levels > 0")
            ns = np.zeros(max_levels + 1, dtype=np.uint64)
            o.level_ns = ns.ctypes.data
        r = Result()
        _check(lib().gg_eval_device(self._h, ctypes.c_void_p(dev_ptr), ctypes.byref(o),
                                    ctypes.byref(r), ctypes.c_void_p(stream)))
        d = r.as_dict()
        if ns is not None:
            d["level_ns"] = ns
        return d

    def last_device_ms(self):
        ms = ctypes.c_double()
        _check(lib().gg_last_device_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def last_launches(self):
        n = ctypes.c_int()
        _check(lib().gg_last_launches(self._h, ctypes.byref(n)))
        return n.value

    def last_batch_ns(self, n):
        """(start, end) device-clock ns of each source batch of the last evaluation."""
        out = np.zeros(2 * n, dtype=np.uint64)
        _check(lib().gg_last_batch_ns(self._h, _ptr(out), n))
        return out.reshape(n, 2)

    def last_transfer_bytes(self):
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().gg_last_transfer_bytes(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_batch_sources(self, bits):
        _check(lib().gg_set_batch_sources(self._h, bits))

    def autotune(self, table, trials=3):
        """Pick the fastest source-batch width for this table; returns (sources, ms)."""
        t = self._table(table)
        w, ms = ctypes.c_int(), ctypes.c_double()
        _check(lib().gg_autotune(self._h, _ptr(t), trials, ctypes.byref(w), ctypes.byref(ms)))
        return w.value, ms.value

    def set_wait_limit_ms(self, ms):
        _check(lib().gg_set_wait_limit_ms(self._h, ms))

    def plan(self):
        """(sources per batch, resident blocks per SM, walk levels) of the current plan."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().gg_engine_plan(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def close(self):
        if self._h:
            lib().gg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _create(fn, *args):
    h = ctypes.c_void_p()
    _check(getattr(lib(), fn)(*args, ctypes.byref(h)))
    return h


# ----------------------------------------------------------------------------
# Calculators (reference API)
# ----------------------------------------------------------------------------

class cudaASPLgraph(Engine):
    """cudaASPLgraph(N, degree_max, device); calc(graph) -> (diameter, total)
    with (-1,-1) disconnected, (-2,-2) diameter >= 199 (cudaASPLgraph.cu:141-199)."""

    def __init__(self, N, degree_max, device=0):
        super().__init__(_create("gg_graph_create", N, degree_max, device), (N, degree_max))
        self.N, self.degree_max, self.device = N, degree_max, device

    def calc(self, g):
        t = self._table(g.table(self.degree_max) if isinstance(g, graph) else g)
        d, tot = ctypes.c_int(), ctypes.c_int64()
        _check(lib().gg_graph_calc(self._h, _ptr(t), ctypes.byref(d), ctypes.byref(tot)))
        return d.value, tot.value


class cudaASPLconv(Engine):
    """cudaASPLconv(N, M, degree, device) (cudaASPLconv.hpp:16-22)."""

    def __init__(self, N, M, degree, device=0):
        super().__init__(_create("gg_conv_create", N, M, degree, device), (M, degree))
        self.N, self.M, self.degree, self.device = N, M, degree, device

    def _t(self, p):
        return self._table(p.table(self.degree) if isinstance(p, part) else p)

    def calc(self, p):
        t, a = self._t(p), ctypes.c_double()
        _check(lib().gg_conv_calc(self._h, _ptr(t), ctypes.byref(a)))
        return a.value

    def diameterASPL(self, p):
        t, d, a = self._t(p), ctypes.c_int(), ctypes.c_double()
        _check(lib().gg_conv_diameter_aspl(self._h, _ptr(t), ctypes.byref(d), ctypes.byref(a)))
        return d.value, a.value

    def WVCdiameterASPL(self, p):
        t, w, d, a = self._t(p), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(lib().gg_conv_wvc_diameter_aspl(self._h, _ptr(t), ctypes.byref(w), ctypes.byref(d),
                                               ctypes.byref(a)))
        return w.value, d.value, a.value


class cudaASPLpiece(Engine):
    """cudaASPLpiece(Nx, Ny, Mx, My, degree, device) (cudaASPLpiece.hpp:16-20)."""

    def __init__(self, Nx, Ny, Mx, My, degree, device=0):
        super().__init__(_create("gg_piece_create", Nx, Ny, Mx, My, degree, device),
                         (Mx * My, degree, 2))
        self.Nx, self.Ny, self.Mx, self.My, self.degree = Nx, Ny, Mx, My, degree

    def diameterASPL(self, p):
        t = self._table(p.table(self.degree) if isinstance(p, piece) else p)
        d, a = ctypes.c_int(), ctypes.c_double()
        _check(lib().gg_piece_diameter_aspl(self._h, _ptr(t), ctypes.byref(d), ctypes.byref(a)))
        return d.value, a.value


class cudaASPLbox(Engine):
    """cudaASPLbox(Nx, Ny, Nz, Mx, My, Mz, degree, device) (cudaASPLbox.hpp:16-20)."""

    def __init__(self, Nx, Ny, Nz, Mx, My, Mz, degree, device=0):
        super().__init__(_create("gg_box_create", Nx, Ny, Nz, Mx, My, Mz, degree, device),
                         (Mx * My * Mz, degree, 3))
        self.degree = degree

    def diameterASPL(self, p):
        t = self._table(p.table(self.degree) if isinstance(p, box) else p)
        d, a = ctypes.c_int(), ctypes.c_double()
        _check(lib().gg_box_diameter_aspl(self._h, _ptr(t), ctypes.byref(d), ctypes.byref(a)))
        return d.value, a.value


class cudaASPLbeamer(Engine):
    """cudaASPLbeamer(N, M, degree, device) (cudaASPLbeamer.hpp:12-16)."""

    def __init__(self, N, M, degree, device=0):
        super().__init__(_create("gg_beamer_create", N, M, degree, device), (M, degree))
        self.N, self.M, self.degree = N, M, degree

    def calc(self, p, regular=None):
        if isinstance(p, part):
            regular = p.regular if regular is None else regular
            t = self._table(p.table(self.degree))
        else:
            t = self._table(p)
            regular = True if regular is None else regular
        a = ctypes.c_double()
        _check(lib().gg_beamer_calc(self._h, _ptr(t), int(bool(regular)), ctypes.byref(a)))
        return a.value


# ----------------------------------------------------------------------------
# Batched candidate evaluation (gg_batch_* in include/gg.h)
# ----------------------------------------------------------------------------

SWAP_DTYPE = np.dtype([("base", np.int32), ("a", np.int32), ("b", np.int32), ("c", np.int32),
                       ("d", np.int32), ("mode", np.int32)])
CAND_RESULT_DTYPE = np.dtype([("total", np.uint64), ("reached", np.uint64), ("levels", np.int32),
                              ("connected", np.int32)])


def gen_swaps(adj, base_id, count, seed):
    """Uniform random 2-opt proposals (no loops, no repeated edges) -> SWAP_DTYPE array."""
    adj = _i32(adj)
    n, d = adj.shape
    out = np.zeros(count, dtype=SWAP_DTYPE)
    _check(lib().gg_gen_swaps(n, d, _ptr(adj), base_id, count, seed, _ptr(out)))
    return out


def set_tune_cache(path):
    """Tuning cache file of every autotuner (gg_set_tune_cache); None or "": none."""
    _check(lib().gg_set_tune_cache(path.encode() if path else None))


def gather_peak(rows=65536, degree=8, iters=20, device=0):
    """Ceiling of a dense BFS level (gg_gather_peak): -> (GB/s, ms per pass) of
    rows x (degree + 1) random 512-byte row reads and one row write."""
    g, ms = ctypes.c_double(), ctypes.c_double()
    _check(lib().gg_gather_peak(device, rows, degree, iters, ctypes.byref(g), ctypes.byref(ms)))
    return g.value, ms.value


def level_probe(rows=65536, chunks=32, levels=40, variant=0, device=0):
    """Dense level loop outside the engine (gg_level_probe): -> microseconds a
    level for rows of `chunks` x 16 bytes (32: 4096 sources, 16: 2048), 8 gathers
    a row, counts, flag words and the grid barrier; variant 1 keeps a second row
    in flight a warp through cp.async."""
    us = ctypes.c_double()
    _check(lib().gg_level_probe(device, rows, chunks, levels, variant, ctypes.byref(us)))
    return us.value


def apply_swap(adj, s):
    """Host copy of the edit the batch kernel applies (first occurrence replaced)."""
    adj = np.array(adj, dtype=np.int32, copy=True)
    if s["a"] < 0:
        return adj
    a, b, c, d = int(s["a"]), int(s["b"]), int(s["c"]), int(s["d"])
    to = (c, d, a, b) if s["mode"] == 0 else (d, c, b, a)
    for row, frm, t in zip((a, b, c, d), (b, a, d, c), to):
        j = int(np.nonzero(adj[row] == frm)[0][0])
        adj[row, j] = t
    return adj


class Surrogate:
    """ΔASPL ranker (gg_surrogate_*): message passing over the current graph,
    bf16 products with fp32 accumulation, Adam on fp32 master weights."""

    def __init__(self, n, degree, in_features, seed=0, device=0):
        self._h = _create("gg_surrogate_create", device, n, degree, in_features, seed)
        self.n, self.degree, self.in_features = n, degree, in_features

    def set_graph(self, adj, features):
        adj = _i32(adj)
        f = np.ascontiguousarray(features, dtype=np.float32)
        _check(lib().gg_surrogate_set_graph(self._h, _ptr(adj), _ptr(f)))

    def predict(self, swaps):
        swaps = np.ascontiguousarray(swaps, dtype=SWAP_DTYPE)
        out = np.zeros(len(swaps), dtype=np.float32)
        _check(lib().gg_surrogate_predict(self._h, len(swaps), _ptr(swaps), _ptr(out)))
        return out

    def _common(self, swaps, target, mask):
        swaps = np.ascontiguousarray(swaps, dtype=SWAP_DTYPE)
        t = np.ascontiguousarray(target, dtype=np.float32)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
        return swaps, t, m

    def train(self, swaps, target, lr=1e-3, mask=None):
        swaps, t, m = self._common(swaps, target, mask)
        loss = ctypes.c_float()
        _check(lib().gg_surrogate_train(self._h, len(swaps), _ptr(swaps), _ptr(t),
                                        None if m is None else _ptr(m), lr, ctypes.byref(loss)))
        return loss.value

    def grad(self, swaps, target, mask=None):
        swaps, t, m = self._common(swaps, target, mask)
        g = np.zeros(self.param_count(), dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().gg_surrogate_grad(self._h, len(swaps), _ptr(swaps), _ptr(t),
                                       None if m is None else _ptr(m), _ptr(g), ctypes.byref(loss)))
        return g, loss.value

    def param_count(self):
        c = ctypes.c_int()
        _check(lib().gg_surrogate_param_count(self._h, ctypes.byref(c)))
        return c.value

    def get_params(self):
        p = np.zeros(self.param_count(), dtype=np.float32)
        _check(lib().gg_surrogate_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib().gg_surrogate_set_params(self._h, _ptr(p)))

    def close(self):
        if self._h:
            lib().gg_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Scores many 2-opt candidates of registered base graphs in one launch."""

    def __init__(self, device=0):
        self._h = _create("gg_batch_create", device)
        self.bases = []

    def add_base(self, adj):
        adj = _i32(adj)
        n, d = adj.shape
        bid = ctypes.c_int()
        _check(lib().gg_batch_add_base(self._h, n, d, _ptr(adj), ctypes.byref(bid)))
        self.bases.append(adj)
        return bid.value

    def set_chunk(self, base_id, sources):
        _check(lib().gg_batch_set_chunk(self._h, base_id, sources))

    def set_base(self, base_id, adj):
        adj = _i32(adj)
        _check(lib().gg_batch_set_base(self._h, base_id, _ptr(adj)))
        self.bases[base_id] = adj

    def vertex_hist(self, base_id, K):
        """[n, K] uint32: vertices at distance 1..K from each vertex of the base."""
        n = len(self.bases[base_id])
        out = np.zeros((n, K), dtype=np.uint32)
        _check(lib().gg_batch_vertex_hist(self._h, base_id, K, _ptr(out)))
        return out

    def eval(self, swaps):
        swaps = np.ascontiguousarray(swaps, dtype=SWAP_DTYPE)
        out = np.zeros(len(swaps), dtype=CAND_RESULT_DTYPE)
        _check(lib().gg_batch_eval(self._h, len(swaps), _ptr(swaps), _ptr(out)))
        return out

    def eval_device(self, n, d_swaps, d_out, stream=0):
        _check(lib().gg_batch_eval_device(self._h, n, ctypes.c_void_p(d_swaps), ctypes.c_void_p(d_out),
                                          ctypes.c_void_p(stream)))

    def autotune(self, swaps, trials=3):
        """Tune each used base's chunk width on these candidates (gg_batch_autotune);
        returns the fastest launch in ms."""
        swaps = np.ascontiguousarray(swaps, dtype=SWAP_DTYPE)
        ms = ctypes.c_double()
        _check(lib().gg_batch_autotune(self._h, len(swaps), _ptr(swaps), trials, ctypes.byref(ms)))
        return ms.value

    def chunk(self, base_id):
        s = ctypes.c_int()
        _check(lib().gg_batch_chunk(self._h, base_id, ctypes.byref(s)))
        return s.value

    def device_status(self, stream=0):
        """Wait for `stream`; raise GGError(GG_BAD_ARG) if the last device launch
        rejected a candidate (gg_batch_device_status)."""
        first = ctypes.c_int()
        _check(lib().gg_batch_device_status(self._h, ctypes.c_void_p(stream), ctypes.byref(first)))

    def last_ms(self):
        ms = ctypes.c_double()
        _check(lib().gg_batch_last_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if self._h:
            lib().gg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


LIFT_EDIT_DTYPE = np.dtype([("count", np.int32), ("row", np.int32, 4), ("slot", np.int32, 4),
                            ("diff", np.int32, (4, 3))])


def gen_lift_moves(N, M, diffs, count, seed):
    """Random shift / orbit 2-opt moves of a cyclic lift (gg_gen_lift_moves) ->
    LIFT_EDIT_DTYPE array."""
    diffs = _i32(diffs).reshape(M, -1)
    out = np.zeros(count, dtype=LIFT_EDIT_DTYPE)
    _check(lib().gg_gen_lift_moves(N, M, diffs.shape[1], _ptr(diffs), count, seed, _ptr(out)))
    return out


def gen_piece_moves(Nx, Ny, Mx, My, vals, count, seed):
    """The same moves for a 2-D torus lift (vals [Mx*My, d, 2])."""
    vals = _i32(vals).reshape(Mx * My, -1, 2)
    out = np.zeros(count, dtype=LIFT_EDIT_DTYPE)
    _check(lib().gg_gen_piece_moves(Nx, Ny, Mx, My, vals.shape[1], _ptr(vals), count, seed, _ptr(out)))
    return out


def gen_box_moves(Nx, Ny, Nz, Mx, My, Mz, vals, count, seed):
    """The same moves for a 3-D torus lift (vals [Mx*My*Mz, d, 3])."""
    vals = _i32(vals).reshape(Mx * My * Mz, -1, 3)
    out = np.zeros(count, dtype=LIFT_EDIT_DTYPE)
    _check(lib().gg_gen_box_moves(Nx, Ny, Nz, Mx, My, Mz, vals.shape[1], _ptr(vals), count, seed, _ptr(out)))
    return out


def apply_lift_edit(table, e):
    """Host copy of a lift edit: the table (part [M, d], piece [M, d, 2], box
    [M, d, 3]) with the edit's slots replaced."""
    t = np.array(table, dtype=np.int32, copy=True)
    for j in range(int(e["count"])):
        r, k = int(e["row"][j]), int(e["slot"][j])
        if t.ndim == 2:
            t[r, k] = int(e["diff"][j][0])
        else:
            t[r, k, :] = e["diff"][j][:t.shape[2]]
    return t


class Lift:
    """Scores many edits of one cyclic-lift diff table in one launch (gg_lift_*).
    Results are over the M orbit sources: ASPL = total * (N // M) / (N * (N - 1))."""

    def __init__(self, N, M, degree, device=0, _handle=None, _axes=1):
        self.N, self.M, self.degree, self.axes = N, M, degree, _axes
        self._h = _handle if _handle is not None else _create("gg_lift_create", N, M, degree, device)

    @classmethod
    def piece(cls, Nx, Ny, Mx, My, degree, device=0):
        """Candidates of a 2-D torus lift (the cudaASPLpiece form)."""
        h = _create("gg_lift_create_piece", Nx, Ny, Mx, My, degree, device)
        return cls(Nx * Ny, Mx * My, degree, device, _handle=h, _axes=2)

    @classmethod
    def box(cls, Nx, Ny, Nz, Mx, My, Mz, degree, device=0):
        """Candidates of a 3-D torus lift (the cudaASPLbox form)."""
        h = _create("gg_lift_create_box", Nx, Ny, Nz, Mx, My, Mz, degree, device)
        return cls(Nx * Ny * Nz, Mx * My * Mz, degree, device, _handle=h, _axes=3)

    def set_base(self, table):
        shape = (self.M, self.degree) if self.axes == 1 else (self.M, self.degree, self.axes)
        self.base = _i32(table).reshape(shape)
        _check(lib().gg_lift_set_base(self._h, _ptr(self.base)))

    def eval(self, edits, max_levels=0):
        edits = np.ascontiguousarray(edits, dtype=LIFT_EDIT_DTYPE)
        out = np.zeros(len(edits), dtype=CAND_RESULT_DTYPE)
        _check(lib().gg_lift_eval(self._h, len(edits), _ptr(edits), max_levels, _ptr(out)))
        return out

    def aspl(self, res):
        """The reference's ASPL of each result (cudaASPLconv.cu:241-242); inf when
        disconnected."""
        tot = res["total"].astype(np.float64) * (self.N // self.M)
        return np.where(res["connected"] == 1, tot / (self.N * (self.N - 1)), np.inf)

    def set_group(self, group):
        _check(lib().gg_lift_set_group(self._h, group))

    def autotune(self, edits, max_levels=0, trials=3):
        """Tune the group size on these edits (gg_lift_autotune) -> (group, ms)."""
        edits = np.ascontiguousarray(edits, dtype=LIFT_EDIT_DTYPE)
        g, ms = ctypes.c_int(), ctypes.c_double()
        _check(lib().gg_lift_autotune(self._h, len(edits), _ptr(edits), max_levels, trials, ctypes.byref(g),
                                      ctypes.byref(ms)))
        return g.value, ms.value

    def group(self):
        g = ctypes.c_int()
        _check(lib().gg_lift_group(self._h, ctypes.byref(g)))
        return g.value

    def set_half_ppm(self, half_ppm=850000):
        _check(lib().gg_lift_set_half_ppm(self._h, half_ppm))

    def last_level_us(self, n=64):
        """Microseconds of each level of the last evaluation's first round (level 1
        includes the reset of the round's bitsets)."""
        ns = np.zeros(n, dtype=np.uint64)
        _check(lib().gg_lift_last_level_ns(self._h, _ptr(ns), n))
        k = int(np.count_nonzero(ns))
        return np.diff(ns[:k].astype(np.int64)) / 1000.0

    def last_ms(self):
        ms = ctypes.c_double()
        _check(lib().gg_lift_last_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if self._h:
            lib().gg_lift_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Incremental:
    """Exact evaluation of 2-opt moves on one current graph, searching again only
    from the sources a move can affect (gg_inc_*)."""

    def __init__(self, n, degree, device=0):
        self.n, self.d = n, degree
        self._h = _create("gg_inc_create", n, degree, device)

    def set_graph(self, adj):
        r = Result()
        _check(lib().gg_inc_set_graph(self._h, _ptr(_i32(adj)), ctypes.byref(r)))
        return r.as_dict()

    def eval(self, swap):
        """(result dict, sources searched again) of the current graph with `swap` applied."""
        sw = np.ascontiguousarray(np.asarray(swap, dtype=SWAP_DTYPE).reshape(1))
        out = np.zeros(1, dtype=CAND_RESULT_DTYPE)
        aff = ctypes.c_int()
        _check(lib().gg_inc_eval(self._h, _ptr(sw), _ptr(out), ctypes.byref(aff)))
        o = out[0]
        return {"total": int(o["total"]), "reached": int(o["reached"]), "levels": int(o["levels"]),
                "connected": int(o["connected"])}, aff.value

    def commit(self, swap):
        sw = np.ascontiguousarray(np.asarray(swap, dtype=SWAP_DTYPE).reshape(1))
        r = Result()
        _check(lib().gg_inc_commit(self._h, _ptr(sw), ctypes.byref(r)))
        return r.as_dict()

    def close(self):
        if self._h:
            lib().gg_inc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

