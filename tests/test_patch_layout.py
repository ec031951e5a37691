"""CPU tests of the order-3 patch layout (fem_patch_layout, the tables that
fem_plan_create_ex(FEM_PLAN_PATCHES) uploads).

The patch kernel's write protocol is replayed here on the host with integer
contributions (exact in FP64, so any order of summation gives the same bits):
per patch colour, per patch, phase 0 positions store their blocks and residual
rows into the patch copy, phase 1 positions store or add as their codes say,
then the segments are stored or added into the matrix and the residual rows
into the residual.  The result must equal the direct scatter through the
reference element map (generateElementBCSRMap, verification/TACSHelpers.h:138-182),
every block and row must be stored exactly once before any add, and the slot
and node budgets must hold."""
import numpy as np
import pytest

NN = 16
SLOTS, NODES = 2560, 128


def _meshes(fem):
    out = [("strip_24x5", fem.square_mesh(24, 5, 3, seed=3)),
           ("odd_13x7", fem.square_mesh(13, 7, 3, 2.0, 1.0, 0.1, seed=4)),
           ("annulus_3x10", fem.annulus_mesh(3, 10, 3, seed=5)),
           ("one_el", fem.square_mesh(1, 1, 3, seed=6))]
    # scrambled element order and node numbering: patches of unrelated elements
    m = fem.square_mesh(9, 8, 3, seed=7)
    rng = np.random.default_rng(7)
    perm = rng.permutation(m.num_nodes)
    inv = np.argsort(perm)
    conn = inv[m.conn].reshape(-1, NN)[rng.permutation(m.num_elements)].reshape(-1)
    m.conn = np.ascontiguousarray(conn.astype(np.int32))
    m.coords = np.ascontiguousarray(m.coords[perm])
    m.states = np.ascontiguousarray(m.states[perm])
    out.append(("scrambled_9x8", m))
    return out


def _replay(L, conn, rowp, num_nodes, ke, re):
    """The patch kernel's writes, in order, with exactness checks."""
    nnzb = int(rowp[-1])
    mat = np.zeros((nnzb, 4))
    res = np.zeros((num_nodes, 2))
    mat_set = np.zeros(nnzb, bool)
    res_set = np.zeros(num_nodes, bool)
    cp = L["colour_ptr"]
    for c in range(cp.size - 1):
        for q in range(cp[c], cp[c + 1]):
            buf = {}
            rbuf = {}
            for phase in (0, 1):
                for j in range(phase, 8, 2):
                    e = L["elem"][q, j]
                    if e < 0:
                        continue
                    code, sb = L["code"][q, j], L["slot_base"][q, j]
                    en = conn[e]
                    for a in range(NN):
                        loc = sb[a] & 255
                        assert 0 <= loc < NODES
                        if code[NN * NN + a]:
                            assert phase == 1 and loc in rbuf
                            rbuf[loc] = rbuf[loc] + re[e, a]
                        else:
                            assert loc not in rbuf, "a residual slot is stored twice"
                            rbuf[loc] = re[e, a].copy()
                        for b in range(NN):
                            k = int(code[a * NN + b]) & 0x7F
                            slot = (int(sb[a]) >> 8) + k
                            assert 0 <= slot < SLOTS
                            assert 0 <= k < rowp[en[a] + 1] - rowp[en[a]]
                            if code[a * NN + b] & 0x80:
                                assert phase == 1 and slot in buf
                                buf[slot] = buf[slot] + ke[e, a, b]
                            else:
                                assert slot not in buf, "a slot is stored twice"
                                buf[slot] = ke[e, a, b].copy()
            covered = set()
            for i in range(L["seg_ptr"][q], L["seg_ptr"][q + 1]):
                g0, w = int(L["seg"][i, 0]), int(np.uint32(L["seg"][i, 1]))
                s0, n, add = w & 0xFFFF, (w >> 16) & 0x7FFF, w >> 31
                assert n >= 1 and s0 + n <= SLOTS
                for u in range(n):
                    v = buf[s0 + u]
                    covered.add(s0 + u)
                    if add:
                        assert mat_set[g0 + u], "added before it was stored"
                        mat[g0 + u] += v
                    else:
                        assert not mat_set[g0 + u], "stored twice"
                        mat[g0 + u] = v
                        mat_set[g0 + u] = True
            assert covered == set(buf), "segments must cover exactly the patch's blocks"
            n0, n1 = L["node_ptr"][q], L["node_ptr"][q + 1]
            assert set(range(n1 - n0)) == set(rbuf)
            for i in range(n0, n1):
                v = int(L["node"][i])
                r, add = v & 0x7FFFFFFF, v < 0
                if add:
                    assert res_set[r]
                    res[r] += rbuf[i - n0]
                else:
                    assert not res_set[r]
                    res[r] = rbuf[i - n0]
                    res_set[r] = True
    assert mat_set.all() and res_set.all(), "a block or residual row was never written"
    return mat, res


@pytest.mark.parametrize("idx", range(5))
def test_patch_layout_replay_bit_exact(fem, idx):
    name, m = _meshes(fem)[idx]
    L = fem.patch_layout(3, m.num_nodes, m.conn_ptr, m.conn)
    ne = m.num_elements
    conn = m.conn.reshape(ne, NN)
    # every element sits at exactly one position; phase-mates share no node
    el = L["elem"]
    assert sorted(el[el >= 0].tolist()) == list(range(ne))
    for q in range(el.shape[0]):
        for ph in (0, 1):
            nodes = [n for e in el[q, ph::2] if e >= 0 for n in conn[e]]
            assert len(nodes) == len(set(nodes)), (name, q, ph)
    # patches of one colour share no node
    cp = L["colour_ptr"]
    for c in range(cp.size - 1):
        seen = set()
        for q in range(cp[c], cp[c + 1]):
            nodes = {int(n) for e in el[q] if e >= 0 for n in conn[e]}
            assert not (nodes & seen)
            seen |= nodes
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, NN, rowp, cols).reshape(ne, NN, NN) // 4
    rng = np.random.default_rng(idx)
    ke = rng.integers(-1000, 1000, size=(ne, NN, NN, 4)).astype(np.float64)
    re = rng.integers(-1000, 1000, size=(ne, NN, 2)).astype(np.float64)
    mat, res = _replay(L, conn, rowp, m.num_nodes, ke, re)
    ref = np.zeros_like(mat)
    np.add.at(ref, mp.reshape(-1), ke.reshape(-1, 4))
    rref = np.zeros_like(res)
    np.add.at(rref, conn.reshape(-1), re.reshape(-1, 2))
    assert np.array_equal(mat, ref) and np.array_equal(res, rref), name


def test_patch_strips_on_structured_mesh(fem):
    """A 32x6 grid: every patch is a full strip of 8 consecutive elements, 4 colours,
    and most blocks leave in segments longer than one element row run (4 blocks)."""
    m = fem.square_mesh(32, 6, 3, seed=9)
    L = fem.patch_layout(3, m.num_nodes, m.conn_ptr, m.conn)
    assert L["elem"].shape[0] == 32 * 6 // 8
    assert (L["elem"] >= 0).all()
    assert L["colour_ptr"].size - 1 == 4
    w = L["seg"][:, 1].view(np.uint32)
    n = (w >> 16) & 0x7FFF
    assert n.sum() == int(fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)[0][-1]) + int(n[(w >> 31) == 1].sum())
    assert n[n > 4].sum() > 0.8 * n.sum()


def test_patch_layout_rejects_other_orders(fem):
    m = fem.square_mesh(3, 3, 2, seed=1)
    with pytest.raises(fem.FemError):
        fem.patch_layout(2, m.num_nodes, m.conn_ptr, m.conn)
