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


def _gmsh_card(eid, nodes, tag):
    """gmsh's raw small-field CQUAD output: the element name without its node count,
    eight fields per line and '+' continuation markers in field 10 of the parent line
    and field 1 of the continuation (the form the reference's fixGmshBDF reflows)."""
    fields = [f"{x}" for x in [eid, 1] + list(nodes)]
    lines, cur = [], "CQUAD".ljust(8)
    k = 0
    for f in fields:
        if k == 8:
            lines.append(cur + f"+{tag}{len(lines)}".ljust(8))
            cur = f"+{tag}{len(lines) - 1}".ljust(8)
            k = 0
        cur += f.rjust(8)
        k += 1
    lines.append(cur)
    return "\n".join(lines)


@pytest.mark.parametrize("p", [2, 3])
def test_raw_gmsh_output_in_gmsh_node_order(fem, orc, tmp_path, p):
    """Elements written the way gmsh writes them -- corners counter-clockwise from
    (0, 0), then each edge's interior nodes along the edge (bottom, right, top,
    left), then the interior recursively -- read with node_order="gmsh" give the
    tensor-order connectivity of the same mesh, and the same assembly."""
    n = p + 1
    nx = 2  # two elements side by side on a (2p+1) x (p+1) node grid
    W = nx * p + 1
    gid = lambda ix, iy: 1 + iy * W + ix  # noqa: E731
    rng = np.random.default_rng(p)
    grids = []
    for iy in range(n):
        for ix in range(W):
            x = ix / p + (0.05 * rng.uniform(-1, 1) if 0 < ix < W - 1 and 0 < iy < n - 1 else 0.0)
            grids.append(f"GRID".ljust(8) + f"{gid(ix, iy)}".rjust(8) + "0".rjust(8) + f"{x:.5f}".rjust(8)[:8]
                         + f"{iy / p:.5f}".rjust(8)[:8] + "0.".rjust(8))

    def gmsh_nodes(e):
        x0 = e * p
        seq = []

        def ring(lo, hi):
            if hi < lo:
                return
            if hi == lo:
                seq.append((lo, lo))
                return
            seq.extend([(lo, lo), (hi, lo), (hi, hi), (lo, hi)])
            seq.extend((i, lo) for i in range(lo + 1, hi))
            seq.extend((hi, j) for j in range(lo + 1, hi))
            seq.extend((i, hi) for i in range(hi - 1, lo, -1))
            seq.extend((lo, j) for j in range(hi - 1, lo, -1))
            ring(lo + 1, hi - 1)

        ring(0, p)
        return [gid(x0 + ix, iy) for ix, iy in seq]

    cards = [_gmsh_card(e + 1, gmsh_nodes(e), chr(ord("A") + e)) for e in range(nx)]
    path = tmp_path / "gmsh_raw.bdf"
    path.write_text("$ gmsh output\nBEGIN BULK\n" + "\n".join(grids + cards) + "\nENDDATA\n")
    m = fem.read_bdf(str(path), node_order="gmsh")
    assert m.order == p and m.num_elements == nx
    # tensor order: local a = ay * (p + 1) + ax of element e is grid node (e p + ax, ay)
    want = np.array([[gid(e * p + a % n, a // n) - 1 for a in range(n * n)] for e in range(nx)], dtype=np.int32)
    assert np.array_equal(m.conn.reshape(nx, -1), want)
    # the assembly equals that of the tensor-order mesh written and read back
    m.states = rng.uniform(-1e-3, 1e-3, m.coords.shape)
    tpath = str(tmp_path / "tensor.bdf")
    fem.write_bdf(m, tpath, node_order="tensor")
    t = fem.read_bdf(tpath, node_order="tensor")
    assert np.array_equal(t.conn, m.conn) and np.array_equal(t.coords, m.coords)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, n * n, rowp, cols)
    R, A = orc.assemble(m, mp, cols.size)
    assert np.abs(orc.bsr_spmv(rowp, cols, A, m.states.reshape(-1)) - R).max() <= 1e-12 * np.abs(R).max()
