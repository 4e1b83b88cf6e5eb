"""Build the engine's shared libraries in-tree (sm_100a).

    python graphgolf-cuda_b200/build.py          # engine + reference shim (+ oracle)

Outputs (git-ignored, but shipped with the working tree):
  graphgolf-cuda_b200/libggb200.so      C ABI of include/gg.h (CUDA engine)
  graphgolf-cuda_b200/libgg_refshim.so  the reference calculator classes defined on
                                        top of the C ABI (needs the reference headers
                                        at build time; skipped when they are absent)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The reference tree (read-only; only its headers and sources are read, never
# copied): GG_REFERENCE_TREE, else the `reference` directory beside this repository.
REF = os.environ.get("GG_REFERENCE_TREE", os.path.join(os.path.dirname(ROOT), "reference"))

ENGINE_SRC = ["gg_engine.cu", "gg_batch.cu", "gg_surrogate.cu", "gg_noalloc.cu", "gg_inc.cu", "gg_lift.cu", "gg_probe.cu", "gg_gen.cpp", "gg_tune.cpp"]
ENGINE_LIB = os.path.join(PKG, "libggb200.so")
SHIM_LIB = os.path.join(PKG, "libgg_refshim.so")


def nvcc():
    for p in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if p and os.path.exists(p):
            return p
    raise RuntimeError("nvcc not found")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_engine(force=False, extra=()):
    srcs = [os.path.join(CSRC, s) for s in ENGINE_SRC]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(INC, "gg.h"))
    if not force and not _stale(ENGINE_LIB, deps):
        return ENGINE_LIB
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O3,-fopenmp",
           "-shared", "-I", INC, "-I", CSRC, "-o", ENGINE_LIB, *srcs, *extra, "-lgomp"]
    _run(cmd)
    return ENGINE_LIB


def build_shim(force=False):
    """libgg_refshim.so: compiled against the reference headers in place."""
    src = os.path.join(CSRC, "refshim.cpp")
    hdr = os.path.join(REF, "cudacode", "cudaASPLconv.hpp")
    if not os.path.exists(src) or not os.path.exists(hdr):
        return None
    if not force and not _stale(SHIM_LIB, [src, ENGINE_LIB]):
        return SHIM_LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared",
           "-I", INC, "-I", os.path.join(REF, "cudacode"), "-I", os.path.join(REF, "cppcode"),
           "-o", SHIM_LIB, src, "-L", PKG, "-lggb200", "-Wl,-rpath,$ORIGIN"]
    _run(cmd)
    return SHIM_LIB


DRIVER_SRC = os.path.join(ROOT, "tests", "shim_driver.cpp")
DRIVER_BIN = os.path.join(ROOT, "tests", "_bin", "shim_driver")


def build_driver(force=False):
    """tests/_bin/shim_driver: the reference-style caller of libgg_refshim.so
    (compiled against the reference headers; skipped when they are absent)."""
    hdr = os.path.join(REF, "cudacode", "cudaASPLconv.hpp")
    if not os.path.exists(hdr) or not os.path.exists(SHIM_LIB):
        return None
    if not force and not _stale(DRIVER_BIN, [DRIVER_SRC, SHIM_LIB]):
        return DRIVER_BIN
    os.makedirs(os.path.dirname(DRIVER_BIN), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(REF, "cudacode"),
           "-I", os.path.join(REF, "cppcode"), "-o", DRIVER_BIN, DRIVER_SRC,
           "-L", PKG, "-lgg_refshim", "-lggb200",
           "-Wl,-rpath,$ORIGIN/../../graphgolf-cuda_b200"]
    _run(cmd)
    return DRIVER_BIN


# The reference's own command-line drivers, compiled unchanged from the reference
# tree, each twice: "<name>_shim" linked against libgg_refshim.so (this engine
# behind the reference classes) and "<name>_orig" against the reference's own
# calculators built for this GPU (oracle/_ref/libref_<calc>.so).  Boost is not in
# this image; tests/boost_stub holds test-only stand-ins of the two Boost headers
# they include.  Test infrastructure: tests/test_ref_drivers.py runs both.
REF_DRIVERS = {"aspl_cuda": "graph", "piece2aspl": "piece", "box2aspl": "box", "main": "conv",
               "annealing": "conv"}
STUB = os.path.join(ROOT, "tests", "boost_stub")
BIN = os.path.join(ROOT, "tests", "_bin")


def build_reference_drivers(force=False):
    if not os.path.isdir(os.path.join(REF, "cppcode")) or not os.path.exists(SHIM_LIB):
        return []
    os.makedirs(BIN, exist_ok=True)
    stubs = [os.path.join(STUB, "boost", f) for f in os.listdir(os.path.join(STUB, "boost"))]
    inc = ["-I", STUB, "-I", os.path.join(REF, "cudacode"), "-I", os.path.join(REF, "cppcode")]
    out = []
    for name, calc in REF_DRIVERS.items():
        src = os.path.join(REF, "cppcode", name + ".cpp")
        shim_bin = os.path.join(BIN, f"ref_{name}_shim")
        if force or _stale(shim_bin, [src, SHIM_LIB, *stubs]):
            _run(["g++", "-O2", "-std=c++17", *inc, "-o", shim_bin, src, "-L", PKG, "-lgg_refshim", "-lggb200",
                  "-Wl,-rpath,$ORIGIN/../../graphgolf-cuda_b200"])
        out.append(shim_bin)
        ref_lib = os.path.join(ROOT, "oracle", "_ref", f"libref_{calc}.so")
        if os.path.exists(ref_lib):
            orig_bin = os.path.join(BIN, f"ref_{name}_orig")
            if force or _stale(orig_bin, [src, ref_lib, *stubs]):
                _run(["g++", "-O2", "-std=c++17", *inc, "-o", orig_bin, src, "-L",
                      os.path.join(ROOT, "oracle", "_ref"), f"-lref_{calc}", "-Wl,-rpath,$ORIGIN/../../oracle/_ref"])
            out.append(orig_bin)
    return out


def build_oracle():
    """The oracle (test infrastructure) and, when the reference tree is here,
    the reference's own calculators in oracle/_ref/."""
    od = os.path.join(ROOT, "oracle")
    _run(["make", "-s", "-C", od, "liboracle.so"])
    if os.path.isdir(os.path.join(REF, "cppcode")):
        _run(["make", "-s", "-C", od, f"REF={REF}", "ref"])


def build_all(force=False):
    build_engine(force)
    build_shim(force)
    build_driver(force)
    build_oracle()
    build_reference_drivers(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
