"""CPU check of the launch order of fem_plan_assemble_host (the host-buffer call
that splits colour launches into element bands to overlap the copies).

Restated rule: elements in colour order (greedy colouring, ascending ids per
colour), bands k = element-id ranges [k nE/B, (k+1) nE/B), band node span = the
smallest and largest node of its elements; step t(k, 0) = k and
t(k, c) = max(k, t(k', c - 1) + 1) over the bands k' whose span overlaps band k's;
launches run by step, and one launch may take several ranges of the same step.
The property that makes the result equal the colour-ordered plan's: two elements
sharing a node are in different colours and the one of the lower colour runs at a
strictly earlier step (so its store precedes the other's add), on structured,
wrapping and scrambled numbering and for any band count."""
import numpy as np
import pytest


def _schedule(conn, num_nodes, colour, nc, B):
    ne = conn.shape[0]
    B = min(B, max(1, min(num_nodes, ne)))
    band = (np.arange(ne, dtype=np.int64) * 0)
    edges = [(k * ne) // B for k in range(B + 1)]
    for k in range(B):
        band[edges[k]:edges[k + 1]] = k
    lo, hi = conn.min(1), conn.max(1)
    blo = np.full(B, np.iinfo(np.int64).max)
    bhi = np.full(B, -1)
    for k in range(B):
        sel = band == k
        if sel.any():
            blo[k], bhi[k] = lo[sel].min(), hi[sel].max()
    t = np.zeros((B, nc), np.int64)
    t[:, 0] = np.arange(B)
    for c in range(1, nc):
        for k in range(B):
            tk = k
            for k2 in range(B):
                if bhi[k2] >= 0 and bhi[k] >= 0 and blo[k2] <= bhi[k] and blo[k] <= bhi[k2]:
                    tk = max(tk, t[k2, c - 1] + 1)
            t[k, c] = tk
    return t[band, colour]


def _meshes(fem):
    out = [fem.square_mesh(24, 16, 3, seed=1), fem.square_mesh(13, 7, 2, seed=2), fem.square_mesh(40, 40, 1, seed=3),
           fem.annulus_mesh(5, 30, 2, seed=4)]
    m = fem.square_mesh(11, 9, 3, seed=5)
    rng = np.random.default_rng(5)
    perm = rng.permutation(m.num_nodes)
    conn = perm[m.conn.reshape(-1, 16)][rng.permutation(m.num_elements)]
    m.conn = np.ascontiguousarray(conn.reshape(-1)).astype(np.int32)
    out.append(m)
    return out


@pytest.mark.parametrize("idx", range(5))
@pytest.mark.parametrize("B", [1, 3, 8, 32])
def test_sharing_elements_run_in_colour_order(fem, idx, B):
    m = _meshes(fem)[idx]
    n = m.nodes_per_element
    conn = m.conn.reshape(-1, n)
    colour, nc = fem.colour_elements(m.num_nodes, m.conn_ptr, m.conn)
    step = _schedule(conn, m.num_nodes, colour, nc, B)
    # node -> elements
    order = np.argsort(conn.reshape(-1), kind="stable")
    nodes = conn.reshape(-1)[order]
    elems = order // n
    starts = np.flatnonzero(np.r_[True, nodes[1:] != nodes[:-1]])
    ends = np.r_[starts[1:], nodes.size]
    for s0, s1 in zip(starts, ends):
        es = np.unique(elems[s0:s1])
        for i in range(es.size):
            for j in range(i + 1, es.size):
                a, b = es[i], es[j]
                assert colour[a] != colour[b]
                lo_e, hi_e = (a, b) if colour[a] < colour[b] else (b, a)
                assert step[lo_e] < step[hi_e], (idx, B, a, b)
