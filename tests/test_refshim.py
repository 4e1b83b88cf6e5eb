"""The drop-in layer: libgg_refshim.so defines the reference calculator classes
(cudacode/cudaASPL*.hpp) on the engine, and tests/_bin/shim_driver -- written
like the reference CLIs, compiled against the reference headers -- runs them.

CPU: the library exports every member the reference headers declare.
GPU: the driver reproduces the golden fixtures (reference CPU results) and the
oracle's return conventions on instances written in the reference's own text
formats (cppcode/{graph,part,piece,box}.hpp print/load)."""
import io
import json
import os
import subprocess

import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "graphgolf-cuda_b200", "libgg_refshim.so")
DRIVER = os.path.join(ROOT, "tests", "_bin", "shim_driver")
CASES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cases.json")))["cases"]

needs_shim = pytest.mark.skipif(not os.path.exists(SHIM), reason="shim not built (needs the reference headers)")

EXPECTED_SYMBOLS = [
    "graphgolf::cudaASPLgraph::cudaASPLgraph(int, int, int)",
    "graphgolf::cudaASPLgraph::~cudaASPLgraph()",
    "graphgolf::cudaASPLgraph::calc(graphgolf::graph&)",
    "graphgolf::cudaASPLconv::cudaASPLconv(int, int, int, int)",
    "graphgolf::cudaASPLconv::~cudaASPLconv()",
    "graphgolf::cudaASPLconv::calc(graphgolf::part&)",
    "graphgolf::cudaASPLconv::diameterASPL(graphgolf::part&)",
    "graphgolf::cudaASPLconv::WVCdiameterASPL(graphgolf::part&)",
    "graphgolf::cudaASPLpiece::cudaASPLpiece(int, int, int, int, int, int)",
    "graphgolf::cudaASPLpiece::~cudaASPLpiece()",
    "graphgolf::cudaASPLpiece::diameterASPL(graphgolf::piece&)",
    "graphgolf::cudaASPLbox::cudaASPLbox(int, int, int, int, int, int, int, int)",
    "graphgolf::cudaASPLbox::~cudaASPLbox()",
    "graphgolf::cudaASPLbox::diameterASPL(graphgolf::box&)",
    "graphgolf::cudaASPLbeamer::cudaASPLbeamer(int, int, int, int)",
    "graphgolf::cudaASPLbeamer::~cudaASPLbeamer()",
    "graphgolf::cudaASPLbeamer::calc(graphgolf::part&)",
]


@needs_shim
def test_shim_exports_reference_members():
    out = subprocess.run(["nm", "-DC", "--defined-only", SHIM], capture_output=True, text=True,
                         check=True).stdout
    have = {l.split(" ", 2)[2] for l in out.splitlines() if " T " in l}
    missing = [s for s in EXPECTED_SYMBOLS if s not in have]
    assert not missing, missing


def run_driver(kind, text):
    p = subprocess.run([DRIVER, kind], input=text, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    line = [l for l in p.stdout.splitlines() if "=" in l][-1]
    return {k: v for k, v in (t.split("=") for t in line.split())}


def part_text(N, M, table):
    s = io.StringIO()
    G.part.from_diffs(N, M, table).print(s)
    return s.getvalue()


def graph_text(adj):
    s = io.StringIO()
    G.graph.from_adjacency(adj).print(s)
    return s.getvalue()


def piece_text(Nx, Ny, Mx, My, rows):
    rows = np.asarray(rows).reshape(Mx * My, -1, 2)
    p = G.piece(Nx=Nx, Ny=Ny, Mx=Mx, My=My)
    p.edges = [[[tuple(map(int, e)) for e in rows[x * My + y]] for y in range(My)] for x in range(Mx)]
    s = io.StringIO()
    p.print(s)
    return s.getvalue()


def box_text(dims, rows):
    Nx, Ny, Nz, Mx, My, Mz = dims
    rows = np.asarray(rows).reshape(Mx * My * Mz, -1, 3)
    b = G.box(Nx=Nx, Ny=Ny, Nz=Nz, Mx=Mx, My=My, Mz=Mz)
    b.edges = [[[[tuple(map(int, e)) for e in rows[(x * My + y) * Mz + z]] for z in range(Mz)]
                for y in range(My)] for x in range(Mx)]
    s = io.StringIO()
    b.print(s)
    return s.getvalue()


@pytest.mark.gpu
@needs_shim
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_driver_reproduces_golden(case):
    if not os.path.exists(DRIVER):
        pytest.skip("driver not built")
    t = np.array(case["table"], dtype=np.int32)
    if case["kind"] == "part":
        N, M, deg = case["N"], case["M"], case["degree"]
        t = t.reshape(M, deg)
        r = run_driver("part", part_text(N, M, t))
        if case["ref_diameter"] == O.INT_MAX:
            assert int(r["diameter"]) == O.SENTINEL and float(r["calc"]) == 1e9
        else:
            assert int(r["diameter"]) == case["ref_diameter"]
            assert float(r["aspl"]) == case["ref_aspl"] and float(r["calc"]) == case["ref_calc"]
        assert (int(r["wvc"]), int(r["wvc_diameter"]), float(r["wvc_aspl"])) == O.conv_wvc(N, M, t)
        if M == N and case["connected"]:
            g = run_driver("graph", graph_text(O.expand_part(N, M, t)))
            assert (int(g["diameter"]), int(g["total"])) == (case["levels"], case["total"])
    elif case["kind"] == "piece":
        Nx, Ny, Mx, My = case["dims"]
        r = run_driver("piece", piece_text(Nx, Ny, Mx, My, t))
        assert (int(r["diameter"]), float(r["aspl"])) == O.piece_diameter_aspl(Nx, Ny, Mx, My, t)
    else:
        r = run_driver("box", box_text(case["dims"], t))
        assert (int(r["diameter"]), float(r["aspl"])) == O.box_diameter_aspl(*case["dims"], t)


@pytest.mark.gpu
@needs_shim
def test_driver_beamer():
    if not os.path.exists(DRIVER):
        pytest.skip("driver not built")
    N, M, diffs = G.cyclic_lift(50, 20, 4, 5)
    r = run_driver("beamer", part_text(N, M, diffs))
    assert float(r["aspl"]) == O.beamer_calc(N, M, diffs)
