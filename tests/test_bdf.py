"""CPU: BDF mesh input/output (GRID + CQUAD4/9/16/25), gmsh -> tensor node order."""
import numpy as np
import pytest


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("order", ["tensor", "gmsh"])
def test_round_trip(fem, tmp_path, p, order):
    m = fem.square_mesh(4, 3, p, 2.0, 1.0, 0.15, seed=p)
    path = str(tmp_path / f"m{p}.bdf")
    fem.write_bdf(m, path, node_order=order)
    r = fem.read_bdf(path, node_order=order, E=m.E, nu=m.nu)
    assert r.order == p and r.num_elements == m.num_elements
    assert np.array_equal(r.conn, m.conn) and np.array_equal(r.conn_ptr, m.conn_ptr)
    assert np.array_equal(r.coords, m.coords)


def test_gmsh_permutation_structure(fem):
    for p in range(1, 5):
        perm = fem.gmsh_to_tensor(p)
        assert sorted(perm.tolist()) == list(range((p + 1) ** 2))
        n = p + 1
        # gmsh lists the four corners first, counter-clockwise from (0, 0)
        corners_tensor = [0, p, n * n - 1, n * p]
        assert [int(perm[c]) for c in corners_tensor] == [0, 1, 2, 3]
    # the 9-node quad: edge midpoints 4..7 (bottom, right, top, left), centre 8
    assert fem.gmsh_to_tensor(2).tolist() == [0, 4, 1, 7, 8, 5, 3, 6, 2]


def test_small_field_cards_with_continuations(fem, orc, tmp_path):
    """A gmsh/fixGmshBDF-style file: 8-character fields, continuation lines,
    Nastran short exponents."""
    txt = """$ two CQUAD9 elements
BEGIN BULK
GRID           1       0      0.      0.      0.
GRID           2       0     0.5      0.      0.
GRID           3       0     1.0      0.      0.
GRID           4       0     1.5      0.      0.
GRID           5       0     2.0      0.      0.
GRID           6       0      0.     0.5      0.
GRID           7       0     0.5     0.5      0.
GRID           8       0     1.0     0.5      0.
GRID           9       0     1.5     0.5      0.
GRID          10       0     2.0     0.5      0.
GRID          11       0      0.   1.0+0      0.
GRID          12       0     0.5     1.0      0.
GRID          13       0     1.0     1.0      0.
GRID          14       0     1.5     1.0      0.
GRID          15       0     2.0     1.0      0.
CQUAD9         1       1       1       2       3       6       7       8
              11      12      13
CQUAD9         2       1       3       4       5       8       9      10
              13      14      15
ENDDATA
"""
    path = tmp_path / "two.bdf"
    path.write_text(txt)
    m = fem.read_bdf(str(path))
    assert m.order == 2 and m.num_elements == 2 and m.num_nodes == 15
    assert np.allclose(m.coords[10], [0.0, 1.0])
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    assert cols.size == 9 * 9 + 9 * 9 - 3 * 3
    m.states = np.random.default_rng(0).uniform(-1e-3, 1e-3, m.coords.shape)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, 9, rowp, cols)
    R, A = orc.assemble(m, mp, cols.size)
    assert np.abs(orc.bsr_spmv(rowp, cols, A, m.states.reshape(-1)) - R).max() <= 1e-12 * np.abs(R).max()
