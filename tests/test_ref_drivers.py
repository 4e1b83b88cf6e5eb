"""The reference's own command-line programs, linked against this engine.

cppcode/aspl_cuda.cpp (cudaASPLgraph), piece2aspl.cpp (cudaASPLpiece),
box2aspl.cpp (cudaASPLbox), main.cpp (cudaASPLconv::WVCdiameterASPL) and the
annealer annealing.cpp (cudaASPLconv::diameterASPL in its accept loop,
cppcode/annealing.cpp:396-443) are compiled unchanged from the reference tree
(graphgolf-cuda_b200/build.py, build_reference_drivers), each twice: against
libgg_refshim.so (the reference classes defined on this engine) and against the
reference's own calculators built for this GPU.  Both builds get the same input
file and arguments; everything they print and write must be identical except
the wall-clock lines.  For the annealer that covers the whole trajectory: its
log has one line per accepted move, and its output file is the best solution.

CPU: the programs load (both libraries resolve) and parse their options with the
test-only Boost stand-in (tests/boost_stub): --help, and an unknown option."""
import io
import os
import re
import subprocess

import numpy as np
import pytest

import graphgolf as G
import instances as I

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "_bin")
NAMES = ["aspl_cuda", "piece2aspl", "box2aspl", "main", "annealing"]


def binary(name, kind):
    p = os.path.join(BIN, f"ref_{name}_{kind}")
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (needs the reference tree at build time)")
    return p


def run(path, args, cwd):
    p = subprocess.run([path, *args], capture_output=True, text=True, timeout=600, cwd=cwd)
    return p.returncode, p.stdout, p.stderr


def without_reference_diagnostics(text):
    """The reference calculators print diagnostics the shim leaves out: the launch
    shape from their constructors ("width: W nBlock: B", cudaASPLconv.cu:125,
    cudaASPLbox.cu:140, cudaASPLpiece.cu) and cudaASPLgraph's per-chunk progress
    "offset/N", each after a cursor-up/erase sequence but the first
    (cudaASPLgraph.cu:159-160), and the erase sequence after its last chunk
    (cudaASPLgraph.cu:194).  Remove exactly those from the reference build's output."""
    text = re.sub(r"^width: \d+ nBlock: \d+\n", "", text, flags=re.M)
    text = re.sub(r"(?:\x1b\[F\x1b\[E\x1b\[K)?\d+/\d+(?=\x1b\[F|Diameter: )", "", text)
    return re.sub(r"\x1b\[F\x1b\[E\x1b\[K(?=Diameter: )", "", text)


def timeless(text):
    """Drop the wall-clock parts: 'TIME: ...' lines and ' time: ...ms' progress."""
    keep = []
    for line in text.replace("\x1b[F", "\n").replace("\x1b[E", "").replace("\x1b[K", "").splitlines():
        if line.startswith("TIME:") or line.startswith("total elapsed time"):
            continue
        if " time: " in line:
            line = line[:line.index(" time: ")]
        keep.append(line)
    return "\n".join(keep)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("kind", ["shim", "orig"])
def test_driver_loads_and_parses_options(name, kind, tmp_path):
    path = binary(name, kind)
    rc, out, _ = run(path, ["--help"], tmp_path)
    assert rc == 0 and "--input" in out and "-i" in out
    rc, out, _ = run(path, ["--no-such-option"], tmp_path)
    assert rc == 1 and "no-such-option" in out


def write(tmp_path, name, obj):
    f = tmp_path / name
    buf = io.StringIO()
    obj.print(buf)
    f.write_text(buf.getvalue())
    return str(f)


def both(name, args, tmp_path):
    outs = []
    for kind in ("shim", "orig"):
        d = tmp_path / kind
        d.mkdir(exist_ok=True)
        rc, out, err = run(binary(name, kind), args, d)
        assert rc == 0, (kind, err)
        if kind == "orig":
            out = without_reference_diagnostics(out)
        files = {p.name: p.read_text() for p in sorted(d.iterdir())}
        outs.append((timeless(out), {k: timeless(v) for k, v in files.items()}))
    return outs


@pytest.mark.gpu
def test_aspl_cuda_same_as_reference_build(tmp_path):
    adj = G.random_regular(3000, 4, 7)
    src = write(tmp_path, "g.txt", G.graph.from_adjacency(adj))
    (s_out, s_files), (o_out, o_files) = both("aspl_cuda", ["-i", src, "-o", "res.txt"], tmp_path)
    assert s_out == o_out and s_files == o_files
    assert "Diameter:" in s_out and "ASPL:" in s_files["res.txt"]
    # a non-regular graph (self-loop padding inside the calculator)
    _, lists = I.random_nonregular(700, 5, 3)
    pairs = [(u, v) for v, row in enumerate(lists) for u in row if u < v]
    src2 = write(tmp_path, "g2.txt", G.graph.from_pairs(pairs))
    (s_out, s_files), (o_out, o_files) = both("aspl_cuda", ["-i", src2, "-o", "res2.txt"], tmp_path)
    assert s_out == o_out and s_files == o_files


@pytest.mark.gpu
def test_piece2aspl_and_box2aspl_same_as_reference_build(tmp_path):
    Nx, Ny, Mx, My, vals = G.piece_lift(8, 8, 4, 4, 4, 2)
    src = write(tmp_path, "p.txt", G.piece.from_table(Nx, Ny, Mx, My, vals))
    (s_out, s_files), (o_out, o_files) = both("piece2aspl", ["-i", src, "-o", "res.txt"], tmp_path)
    assert s_out == o_out and s_files == o_files and "ASPL:" in s_out
    dims_rows = I.random_box(3, 2, 2, 2, 3, 2, 6, 4)
    dims, rows = dims_rows[:6], dims_rows[6]
    src = write(tmp_path, "b.txt", G.box.from_table(*dims, rows))
    (s_out, s_files), (o_out, o_files) = both("box2aspl", ["-i", src, "-o", "res.txt"], tmp_path)
    assert s_out == o_out and s_files == o_files and "ASPL:" in s_out


@pytest.mark.gpu
def test_main_wvc_same_as_reference_build(tmp_path):
    for seed, (m, g, d) in enumerate([(64, 4, 4), (200, 8, 6), (96, 1, 4)]):
        N, M, diffs = I.random_part(m, g, d, 40 + seed)
        src = write(tmp_path, f"q{seed}.txt", G.part.from_diffs(N, M, diffs))
        (s_out, s_files), (o_out, o_files) = both("main", ["-i", src, "-o", f"res{seed}.txt"], tmp_path)
        assert s_out == o_out and s_files == o_files and "WVC:" in s_out


@pytest.mark.gpu
def test_annealing_trajectory_same_as_reference_build(tmp_path):
    """The reference annealer, 400 iterations from the same start and seed: every
    accepted move (log), the best solution (output file) and the console lines."""
    N, M, diffs = G.cyclic_lift(64, 8, 4, 3)
    src = write(tmp_path, "start.txt", G.part.from_diffs(N, M, diffs))
    args = ["-i", src, "-o", "best.txt", "-l", "run.log", "-s", "7", "-c", "400", "-t", "0.5"]
    (s_out, s_files), (o_out, o_files) = both("annealing", args, tmp_path)
    assert s_files == o_files and s_out == o_out
    log = s_files["run.log"].splitlines()
    assert len([l for l in log if not l.startswith("#")]) > 2      # moves were accepted
    best = G.part().load(io.StringIO(s_files["best.txt"]))
    assert best.N == N and best.M == M


def test_reference_diagnostics_are_the_only_lines_removed():
    esc = "\x1b[F\x1b[E\x1b[K"
    raw = ("Nodes: 3000 Degrees_max: 4\n0/3000" + esc + "1024/3000" + esc + "2048/3000" + esc + "Diameter: 10\n"
           "ASPL: 6.6235365122 (29795979/4498500)\nwidth: 2 nBlock: 1\nASPL: 5.0\n")
    assert without_reference_diagnostics(raw) == ("Nodes: 3000 Degrees_max: 4\nDiameter: 10\n"
                                                  "ASPL: 6.6235365122 (29795979/4498500)\nASPL: 5.0\n")
