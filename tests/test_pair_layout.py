"""CPU: the pair layout of orders 2-4 (fem_pair_layout, the element order of the
fragment kernel's single-mesh plan launches).  Checks that the list is a
permutation, that each listed pair shares its edge node for node (the first
element's right edge is the second's left edge), that the units of a colour share
no node, and replays the write protocol of the code records: in list order,
colour after colour, every block and residual row is stored exactly once, by its
first contributor, before any element adds to it."""
import numpy as np
import pytest


def _check(fem, mesh, expect_pairs=None, expect_colours=None):
    P = mesh.order
    P1 = P + 1
    nn = P1 * P1
    cp, conn = mesh.conn_ptr, mesh.conn
    elist, cptr, npairs, codes = fem.pair_layout(P, mesh.num_nodes, cp, conn, codes=True)
    ne = mesh.num_elements
    assert cptr.size >= 2 and cptr[0] == 0 and cptr[-1] == ne
    assert np.array_equal(np.sort(elist), np.arange(ne))
    if expect_pairs is not None:
        assert npairs == expect_pairs
    if expect_colours is not None:
        assert cptr.size - 1 == expect_colours
    nodes = lambda e: conn[cp[e]:cp[e + 1]]
    rowp, cols = fem.build_bsr_pattern(mesh.num_nodes, cp, conn)
    written = np.zeros(cols.size, bool)
    res_written = np.zeros(mesh.num_nodes, bool)
    seen_pairs = 0
    for c in range(cptr.size - 1):
        b, e_ = int(cptr[c]), int(cptr[c + 1])
        # pairs first: a position pair is a pair when the two share the edge
        units, k = [], b
        while k < e_:
            if k + 1 < e_:
                e0, e1 = elist[k], elist[k + 1]
                n0, n1 = nodes(e0).reshape(P1, P1), nodes(e1).reshape(P1, P1)  # [ly][lx]
                if np.array_equal(n0[:, P], n1[:, 0]):
                    units.append((k, k + 1))
                    k += 2
                    seen_pairs += 1
                    continue
            units.append((k,))
            k += 1
        used = set()
        for u in units:
            un = set()
            for k in u:
                un |= set(nodes(elist[k]).tolist())
            assert not (un & used), (c, u)
            used |= un
        for u in units:
            for k in u:
                en = nodes(elist[k])
                rec = codes[k]
                for a in range(nn):
                    r = en[a]
                    first = bool(rec[nn * nn + a])
                    assert first == (not res_written[r])
                    res_written[r] = True
                    row = cols[rowp[r]:rowp[r + 1]]
                    for bb in range(nn):
                        code = int(rec[a * nn + bb])
                        rank = code & 0x7F
                        assert row[rank] == en[bb]
                        blk = rowp[r] + rank
                        assert bool(code & 0x80) == (not written[blk])
                        written[blk] = True
    assert seen_pairs == npairs
    assert written.all() and res_written.all()


@pytest.mark.parametrize("order", [2, 3, 4])
def test_pair_layout_square(fem, order):
    m = fem.square_mesh(8, 6, order, seed=5)
    _check(fem, m, expect_pairs=6 * 4, expect_colours=4)


def test_pair_layout_odd_rows_and_scrambled(fem):
    m = fem.square_mesh(7, 5, 3, seed=2)
    _check(fem, m, expect_pairs=5 * 3)
    # scrambled element order and node numbering: pairs are found by shared edges
    rng = np.random.default_rng(0)
    perm_e = rng.permutation(m.num_elements)
    perm_n = rng.permutation(m.num_nodes)
    nn = (m.order + 1) ** 2
    conn = perm_n[m.conn.reshape(-1, nn)[perm_e]].reshape(-1).astype(np.int32)
    m2 = fem.Mesh(m.order, np.zeros((m.num_nodes, 2)), np.arange(0, conn.size + 1, nn, dtype=np.int32), conn,
                  np.zeros((m.num_nodes, 2)), m.E, m.nu, m.t)
    _check(fem, m2)


def test_pair_layout_annulus(fem):
    m = fem.annulus_mesh(6, 24, 2)
    _check(fem, m)
