"""Text formats and form -> plain graph converters (cppcode/piece2graph.cpp,
cppcode/box2graph.cpp).  CPU: the converters against the oracle's expansion
of the same tables, and print/load round trips.  GPU: each form's calculator
against cudaASPLgraph on the converted graph (the cross-check the converters
exist for)."""
import io

import numpy as np
import pytest

import graphgolf as G
import instances as I
import oracle as O


def make_piece(Nx, Ny, Mx, My, rows):
    p = G.piece(Nx=Nx, Ny=Ny, Mx=Mx, My=My, degree=rows.shape[1])
    p.edges = [[[tuple(map(int, e)) for e in rows[x * My + y]] for y in range(My)] for x in range(Mx)]
    return p


def make_box(Nx, Ny, Nz, Mx, My, Mz, rows):
    b = G.box(Nx=Nx, Ny=Ny, Nz=Nz, Mx=Mx, My=My, Mz=Mz, degree=rows.shape[1])
    b.edges = [[[[tuple(map(int, e)) for e in rows[(x * My + y) * Mz + z]] for z in range(Mz)]
                for y in range(My)] for x in range(Mx)]
    return b


def oracle_pairs(adj):
    adj = np.asarray(adj, dtype=np.int64)
    v = np.repeat(np.arange(len(adj)), adj.shape[1])
    u = adj.ravel()
    return np.unique(np.stack([np.minimum(u, v), np.maximum(u, v)], 1), axis=0)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_piece_pairs_match_oracle_expansion(seed):
    Nx, Ny, Mx, My, rows = I.random_piece(3, 4, 5, 3, 4, seed)
    p = make_piece(Nx, Ny, Mx, My, rows)
    got = G.piece_pairs(p)
    assert np.array_equal(got, oracle_pairs(O.expand_piece(Nx, Ny, Mx, My, rows)))
    assert (got[:, 0] <= got[:, 1]).all()


@pytest.mark.parametrize("seed", [1, 2])
def test_box_pairs_match_oracle_expansion(seed):
    Nx, Ny, Nz, Mx, My, Mz, rows = I.random_box(2, 3, 2, 3, 2, 4, 4, seed)
    b = make_box(Nx, Ny, Nz, Mx, My, Mz, rows)
    assert np.array_equal(G.box_pairs(b), oracle_pairs(O.expand_box(Nx, Ny, Nz, Mx, My, Mz, rows)))


def test_part_pairs_match_oracle_expansion():
    N, M, diffs = I.random_part(40, 8, 4, 5)
    p = G.part.from_diffs(N, M, diffs)
    assert np.array_equal(G.part_pairs(p), oracle_pairs(O.expand_part(N, M, diffs)))


def test_to_graph_and_text_round_trips():
    Nx, Ny, Mx, My, rows = I.random_piece(2, 2, 4, 4, 3, 7)
    p = make_piece(Nx, Ny, Mx, My, rows)
    s = io.StringIO()
    p.print(s)
    q = G.piece().load(io.StringIO(s.getvalue()))
    assert (q.Nx, q.Ny, q.Mx, q.My, q.degree, q.edges) == (p.Nx, p.Ny, p.Mx, p.My, p.degree, p.edges)
    g = G.to_graph(p)
    assert g.N == Nx * Ny and g.is_regular() and g.degree_max == 3
    # edge list -> graph.load -> print gives the same pairs back
    s = io.StringIO()
    G.write_pairs(G.piece_pairs(p), s)
    g2 = G.graph().load(io.StringIO(s.getvalue()))
    out = io.StringIO()
    g2.print(out)
    back = np.array([list(map(int, l.split())) for l in out.getvalue().splitlines()])
    assert np.array_equal(np.unique(back, axis=0), G.piece_pairs(p))


def test_tables_round_trip_through_the_text_formats():
    # an annealer's result table -> form -> text -> form -> the same table
    Nx, Ny, Mx, My, rows = I.random_piece(3, 2, 2, 3, 4, 5)
    p = G.piece.from_table(Nx, Ny, Mx, My, rows)
    assert p.edges == make_piece(Nx, Ny, Mx, My, rows).edges
    s = io.StringIO()
    p.print(s)
    assert np.array_equal(G.piece().load(io.StringIO(s.getvalue())).table(4), rows)
    Nx, Ny, Nz, Mx, My, Mz, rows = I.random_box(2, 2, 3, 2, 1, 2, 4, 6)
    b = G.box.from_table(Nx, Ny, Nz, Mx, My, Mz, rows)
    assert b.edges == make_box(Nx, Ny, Nz, Mx, My, Mz, rows).edges
    s = io.StringIO()
    b.print(s)
    assert np.array_equal(G.box().load(io.StringIO(s.getvalue())).table(4), rows)
    N, M, D = G.cyclic_lift(12, 3, 4, 2)
    s = io.StringIO()
    G.part.from_diffs(N, M, D).print(s)
    assert np.array_equal(G.part().load(io.StringIO(s.getvalue())).table(4), D)


def test_converter_drops_repeated_lifted_edges():
    # a 1x1 tile whose two diffs lift to the same edges: (1,0) and (-1,0) on Nx=2
    p = G.piece(Nx=2, Ny=1, Mx=1, My=1, degree=2)
    p.edges = [[[(1, 0), (-1, 0)]]]
    assert G.piece_pairs(p).tolist() == [[0, 1]]


def check(d_form, a_form, d_graph, total, N):
    if d_graph == -1:                      # disconnected: each calculator's own sentinel
        assert (d_form, a_form) == (O.SENTINEL, float(O.SENTINEL))
    else:
        assert d_form == d_graph
        assert a_form == total / (N * (N - 1))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_forms_equal_their_plain_graphs_on_gpu(seed):
    Nx, Ny, Mx, My, rows = I.random_piece(4, 4, 6, 5, 4, seed)
    p = make_piece(Nx, Ny, Mx, My, rows)
    g = G.to_graph(p)
    d_p, a_p = G.cudaASPLpiece(Nx, Ny, Mx, My, 4, 0).diameterASPL(p)
    d_g, total = G.cudaASPLgraph(g.N, g.degree_max, 0).calc(g)
    check(d_p, a_p, d_g, total, g.N)
    Nx, Ny, Nz, Mx, My, Mz, rows = I.random_box(2, 2, 3, 4, 5, 3, 4, seed)
    b = make_box(Nx, Ny, Nz, Mx, My, Mz, rows)
    g = G.to_graph(b)
    d_b, a_b = G.cudaASPLbox(Nx, Ny, Nz, Mx, My, Mz, 4, 0).diameterASPL(b)
    d_g, total = G.cudaASPLgraph(g.N, g.degree_max, 0).calc(g)
    check(d_b, a_b, d_g, total, g.N)
