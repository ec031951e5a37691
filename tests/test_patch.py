"""Row-complete patches (CPU): the helper behind the full-size parity tests.

For the nodes S of a few core elements, the patch of every element touching S
must assemble S's residual entries and matrix rows exactly as the whole mesh
does: same columns, and (the oracle scatters in element order) the same bits."""
import numpy as np
import pytest


@pytest.mark.parametrize("kind", ["square_p3", "annulus_p2_seam"])
def test_patch_rows_equal_full_mesh_rows(fem, orc, kind):
    if kind == "square_p3":
        m = fem.square_mesh(12, 10, 3, 10.0, 10.0, 0.2, seed=0x640)
        core = [9 * 12 + 10, 9 * 12 + 11, 4 * 12 + 5]
    else:
        m = fem.annulus_mesh(4, 12, 2, seed=0x641)
        core = [11 * 4 + 0, 0 * 4 + 0, 11 * 4 + 3]  # both sides of the theta = 0 seam
    rowp, cols = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    R, A = orc.assemble(m, orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols), cols.size)
    patch, S, loc = fem.mesh.row_complete_patch(m, core)
    assert patch.num_elements < m.num_elements
    prow, pcol = orc.bsr_pattern(patch.num_nodes, patch.conn_ptr, patch.conn)
    pR, pA = orc.assemble(patch, orc.element_bsr_map(patch.conn_ptr, patch.conn, patch.nodes_per_element, prow, pcol),
                          pcol.size)
    for r, l in zip(S, loc):
        assert np.array_equal(cols[rowp[r]:rowp[r + 1]], patch.global_nodes[pcol[prow[l]:prow[l + 1]]])
        assert np.array_equal(R[2 * r:2 * r + 2], pR[2 * l:2 * l + 2])
        assert np.array_equal(A[4 * rowp[r]:4 * rowp[r + 1]], pA[4 * prow[l]:4 * prow[l + 1]])


def test_extended_j_matches_plain_on_small_meshes(fem, orc):
    """Away from large coordinates the long-double J changes nothing measurable."""
    m = fem.square_mesh(6, 5, 3, 1.0, 1.0, 0.2, seed=0x642)
    rowp, cols = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    R0, A0 = orc.assemble(m, mp, cols.size)
    orc.set_extended_j(True)
    try:
        R1, A1 = orc.assemble(m, mp, cols.size)
    finally:
        orc.set_extended_j(False)
    assert np.abs(R1 - R0).max() <= 1e-14 * np.abs(R0).max()
    assert np.abs(A1 - A0).max() <= 1e-14 * np.abs(A0).max()
