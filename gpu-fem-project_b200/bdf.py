"""Nastran BDF mesh input/output for CQUAD4/9/16/25 meshes.

The reference drives its kernels with gmsh-generated BDF files read through
TACS (verification/TACSHelpers.h:35-129, meshes/GmshUtils.py:118-196): GRID
cards carry the nodes, CQUADn cards (renamed from gmsh's CQUAD/CQUAD4 output by
fixGmshBDF) carry elements of (p+1)^2 nodes.  The assembly kernels expect the
tensor-product local order a = ay*(p+1) + ax (element/FEKernels.h:136,452).
gmsh writes high-order quads in its own order (corners counter-clockwise, then
the nodes of each edge, then the interior recursively); `node_order="gmsh"`
converts that to tensor order, `node_order="tensor"` keeps the file's order.

Small-field (8-character) and free-field (comma-separated) cards are accepted,
with continuation lines that start with '+', '*' or blanks.
"""
from __future__ import annotations

import numpy as np

from .mesh import Mesh


def gmsh_to_tensor(p: int) -> np.ndarray:
    """perm such that tensor_local[a] = gmsh_local[perm[a]] for an order-p quad."""
    # gmsh's recursive ordering, built on the (p+1)x(p+1) grid of (ix, iy)
    order = []

    def ring(lo, hi):
        if hi < lo:
            return
        if hi == lo:
            order.append((lo, lo))
            return
        # corners counter-clockwise from (lo, lo)
        order.extend([(lo, lo), (hi, lo), (hi, hi), (lo, hi)])
        # edge interiors: 0->1, 1->2, 2->3, 3->0
        order.extend((i, lo) for i in range(lo + 1, hi))
        order.extend((hi, j) for j in range(lo + 1, hi))
        order.extend((i, hi) for i in range(hi - 1, lo, -1))
        order.extend((lo, j) for j in range(hi - 1, lo, -1))
        ring(lo + 1, hi - 1)

    ring(0, p)
    pos = {xy: k for k, xy in enumerate(order)}
    return np.array([pos[(ax, ay)] for ay in range(p + 1) for ax in range(p + 1)], dtype=np.int64)


def _fields_small(line: str):
    body = line.rstrip("\n")
    return [body[i:i + 8].strip() for i in range(0, min(len(body), 72), 8)]


def _cards(lines):
    """Yield cards as lists of fields (name first), joining continuation lines."""
    cur = None
    for raw in lines:
        line = raw.rstrip("\n")
        if not line.strip() or line.lstrip().startswith("$"):
            continue
        free = "," in line
        first = line.split(",")[0] if free else line[:8]
        is_cont = first.strip() == "" or first.strip().startswith("+") or first.strip().startswith("*")
        fields = [f.strip() for f in line.split(",")] if free else _fields_small(line)
        if is_cont and cur is not None:
            cur.extend(fields[1:])
            continue
        if cur is not None:
            yield cur
        cur = fields
    if cur is not None:
        yield cur


def _num(s: str) -> float:
    s = s.strip()
    if not s:
        return 0.0
    # Nastran short exponents: 1.5-3 means 1.5e-3
    for k in range(1, len(s)):
        if s[k] in "+-" and s[k - 1] not in "eEdD":
            s = s[:k] + "e" + s[k:]
            break
    return float(s.replace("D", "e").replace("d", "e"))


def read_bdf(path: str, node_order: str = "tensor", E: float = 70e9, nu: float = 0.3, t: float = 1.0,
             states=None) -> Mesh:
    """A Mesh from a BDF file (one element order per file, as the reference requires).
    Node ids are renumbered 0..N-1 in ascending GRID id order."""
    if node_order not in ("tensor", "gmsh"):
        raise ValueError("node_order must be 'tensor' or 'gmsh'")
    grids, elems, order = {}, [], None
    with open(path) as f:
        for card in _cards(f):
            name = card[0].upper().rstrip("*")
            if name == "GRID":
                gid = int(card[1])
                grids[gid] = (_num(card[3]), _num(card[4]))
            elif name.startswith("CQUAD"):
                nodes = [int(x) for x in card[3:] if x.strip()]
                n = len(nodes)
                p = int(round(np.sqrt(n))) - 1
                if (p + 1) ** 2 != n or not 1 <= p <= 4:
                    raise ValueError(f"element {card[1]}: {n} nodes is not a quad of order 1..4")
                if order is None:
                    order = p
                elif order != p:
                    raise ValueError("mixed element orders in one file")
                elems.append(nodes)
    if order is None:
        raise ValueError("no CQUAD elements")
    ids = np.array(sorted(grids), dtype=np.int64)
    index = {g: i for i, g in enumerate(ids)}
    coords = np.array([grids[g] for g in ids], dtype=np.float64)
    conn = np.array([[index[g] for g in e] for e in elems], dtype=np.int64)
    if node_order == "gmsh" and order > 1:
        conn = conn[:, gmsh_to_tensor(order)]
    nn = (order + 1) ** 2
    conn_ptr = (np.arange(len(elems) + 1, dtype=np.int64) * nn).astype(np.int32)
    st = np.zeros_like(coords) if states is None else np.ascontiguousarray(states, dtype=np.float64)
    return Mesh(order, np.ascontiguousarray(coords), conn_ptr, np.ascontiguousarray(conn.reshape(-1), dtype=np.int32),
                st, E, nu, t, path)


def write_bdf(mesh: Mesh, path: str, node_order: str = "tensor") -> None:
    """Small-field BDF: GRID cards (ids from 1) and CQUADn cards (ids from 1, PID 1)."""
    n = mesh.nodes_per_element
    conn = mesh.conn.reshape(-1, n).astype(np.int64)
    if node_order == "gmsh" and mesh.order > 1:
        inv = np.argsort(gmsh_to_tensor(mesh.order))
        conn = conn[:, inv]
    with open(path, "w") as f:
        f.write("$ written by gpu-fem-project_b200\nBEGIN BULK\n")
        for i, (x, y) in enumerate(mesh.coords):
            # free-field GRID cards keep every digit of the coordinates
            f.write(f"GRID,{i + 1},0,{float(x)!r},{float(y)!r},0.0\n")
        for e, row in enumerate(conn):
            fields = [f"CQUAD{n}", str(e + 1), "1"] + [str(v + 1) for v in row]
            lines, cur = [], ""
            for k, fld in enumerate(fields):
                if k >= 9 and (k - 9) % 8 == 0:  # 8 data fields per line, continuation field blank
                    lines.append(cur)
                    cur = " " * 8
                cur += fld.ljust(8)
            lines.append(cur)
            f.write("\n".join(lines) + "\n")
        f.write("ENDDATA\n")
