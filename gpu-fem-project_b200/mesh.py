"""Seeded structured meshes of Lagrange quads in tensor-product node order.

Node placement follows the reference's cosine knots
x_k = -cos(pi/2 * (xLin + 1)), xLin = -1 + 2k/p (element/LagrangeShapeFuncs.h:7-10),
mapped onto each element; local node a = ay*(p+1) + ax (element/FEKernels.h:136,452).
The reference reads gmsh BDF meshes through TACS (verification/TACSHelpers.h:35-129);
those files and tools are absent, so the workloads are generated here from
their stated shapes and distributions with fixed seeds.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Mesh:
    order: int
    coords: np.ndarray      # float64 [numNodes, 2]
    conn_ptr: np.ndarray    # int32 [numElements + 1]
    conn: np.ndarray        # int32 [numElements * (p+1)^2]
    states: np.ndarray      # float64 [numNodes, 2]
    E: float
    nu: float
    t: float = 1.0
    name: str = ""
    seed: int = 0

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def num_elements(self) -> int:
        return int(self.conn_ptr.shape[0] - 1)

    @property
    def nodes_per_element(self) -> int:
        return (self.order + 1) ** 2

    @property
    def num_dof(self) -> int:
        return 2 * self.num_nodes


def cosine_knots(p: int) -> np.ndarray:
    """Local knot fractions in [0, 1] of the order-p cosine-spaced nodes."""
    xlin = -1.0 + 2.0 * np.arange(p + 1) / p
    x = -np.cos(np.pi / 2 * (xlin + 1.0))
    x[0], x[-1] = -1.0, 1.0
    return (x + 1.0) / 2.0


def _axis(n_el: int, p: int, length: float) -> np.ndarray:
    """Coordinates of the n_el*p + 1 nodes of one axis."""
    f = cosine_knots(p)
    idx = np.arange(n_el * p + 1)
    e = np.minimum(idx // p, n_el - 1)
    loc = idx - e * p
    return (e + f[loc]) * (length / n_el)


def _structured_conn(nx: int, ny: int, p: int, nodes_x: int, wrap_y: int = 0) -> np.ndarray:
    """conn[e, a] for element e = ey*nx + ex, a = ay*(p+1) + ax; node = J*nodes_x + I.
    With wrap_y > 0 the J index is taken modulo wrap_y (periodic direction)."""
    p1 = p + 1
    ex = np.arange(nx)
    ey = np.arange(ny)
    ax = np.arange(p1)
    I = ex[None, :, None, None] * p + ax[None, None, None, :]
    J = ey[:, None, None, None] * p + ax[None, None, :, None]
    if wrap_y:
        J = J % wrap_y
    conn = J * nodes_x + I
    return conn.reshape(nx * ny * p1 * p1).astype(np.int32)


def square_mesh(nx: int, ny: int, p: int, lx: float = 1.0, ly: float = 1.0, perturb: float = 0.0,
                disp: float = 1e-3, E: float = 70e9, nu: float = 0.3, t: float = 1.0, seed: int = 0,
                name: str = "square") -> Mesh:
    """nx x ny order-p quads on [0,lx]x[0,ly]; nodal displacements U(-disp, disp).

    Perturbation: element vertices not on the domain boundary move by
    U(-perturb*h, +perturb*h) per direction (h = element size along it); every
    higher-order node then sits at the cosine knots of its element's bilinear map
    of the perturbed vertices, so elements stay valid (a node-by-node move of
    +-0.2h would push the first interior knot, 0.25h from the edge at p=3 and
    0.146h at p=4, past its neighbour and invert the element)."""
    rng = np.random.default_rng(seed)
    nxn, nyn = nx * p + 1, ny * p + 1
    V = np.empty((ny + 1, nx + 1, 2))
    V[:, :, 0] = np.linspace(0.0, lx, nx + 1)[None, :]
    V[:, :, 1] = np.linspace(0.0, ly, ny + 1)[:, None]
    if perturb and nx > 1 and ny > 1:
        d = rng.uniform(-1.0, 1.0, size=(ny - 1, nx - 1, 2))
        V[1:-1, 1:-1, 0] += perturb * (lx / nx) * d[:, :, 0]
        V[1:-1, 1:-1, 1] += perturb * (ly / ny) * d[:, :, 1]
    f = cosine_knots(p)

    def split(n_el, n_nodes):
        idx = np.arange(n_nodes)
        e = np.minimum(idx // p, n_el - 1)
        return e, f[idx - e * p]

    ex, fx = split(nx, nxn)
    ey, fy = split(ny, nyn)
    fx, fy = fx[None, :, None], fy[:, None, None]
    v00 = V[ey][:, ex]
    v10 = V[ey][:, ex + 1]
    v01 = V[ey + 1][:, ex]
    v11 = V[ey + 1][:, ex + 1]
    X = (1 - fx) * (1 - fy) * v00 + fx * (1 - fy) * v10 + (1 - fx) * fy * v01 + fx * fy * v11
    coords = np.ascontiguousarray(X.reshape(-1, 2))
    conn = _structured_conn(nx, ny, p, nxn)
    nn = (p + 1) ** 2
    conn_ptr = (np.arange(nx * ny + 1, dtype=np.int64) * nn).astype(np.int32)
    states = rng.uniform(-disp, disp, size=coords.shape)
    return Mesh(p, coords, conn_ptr, conn, states, E, nu, t, name, seed)


def annulus_mesh(nr: int, nth: int, p: int, r0: float = 1.0, r1: float = 2.0, k: int | None = None,
                 amp: float = 1e-3, noise: float = 1e-5, E: float = 200e9, nu: float = 0.28, t: float = 1.0,
                 seed: int = 0, name: str = "annulus") -> Mesh:
    """nr (radial) x nth (circumferential, periodic) order-p quads on r in [r0, r1]
    with nodes at exact polar positions.  Both displacement components are
    amp*sin(k*theta)*r + U(-noise, noise); k in 1..8 drawn from the seed unless given."""
    rng = np.random.default_rng(seed)
    if k is None:
        k = int(rng.integers(1, 9))
    nrn, ntn = nr * p + 1, nth * p
    r = r0 + _axis(nr, p, r1 - r0)
    th = 2.0 * np.pi * _axis(nth, p, 1.0)[:ntn]
    R, TH = np.meshgrid(r, th, indexing="xy")          # [ntn, nrn]
    coords = np.stack([R * np.cos(TH), R * np.sin(TH)], axis=-1).reshape(-1, 2)
    conn = _structured_conn(nr, nth, p, nrn, wrap_y=ntn)
    nn = (p + 1) ** 2
    conn_ptr = (np.arange(nr * nth + 1, dtype=np.int64) * nn).astype(np.int32)
    base = (amp * np.sin(k * TH) * R).reshape(-1)
    states = np.stack([base, base], axis=-1) + rng.uniform(-noise, noise, size=(ntn * nrn, 2))
    m = Mesh(p, np.ascontiguousarray(coords), conn_ptr, conn, np.ascontiguousarray(states), E, nu, t, name, seed)
    m.k = k
    return m


# ---- the workloads -------------------------------------------------------------------

SEEDS = {"square64_p1": 0x5EED0001, "square1024_p3": 0x5EED0002, "annulus_p2": 0x5EED0003,
         "batch256": 0x5EED0004, "serve64": 0x5EED0005}


def square64_p1(scale: int = 64) -> Mesh:
    """64x64 order-1 quads on the unit square, interior +-0.1h, u in [-1e-3,1e-3],
    E=70e9, nu=0.3, t=1 (2x2 Gauss points)."""
    return square_mesh(scale, scale, 1, 1.0, 1.0, 0.1, 1e-3, 70e9, 0.3, 1.0, SEEDS["square64_p1"],
                       f"square{scale}_p1")


def square1024_p3(n: int = 1024) -> Mesh:
    """n x n order-3 quads on a 10x10 square, interior +-0.2h, u in [-1e-3,1e-3],
    E=70e9, nu=0.3 (4x4 Gauss points); n=1024 gives 18,886,658 DOF."""
    return square_mesh(n, n, 3, 10.0, 10.0, 0.2, 1e-3, 70e9, 0.3, 1.0, SEEDS["square1024_p3"], f"square{n}_p3")


def annulus512x2048_p2(nr: int = 512, nth: int = 2048) -> Mesh:
    """Annulus r in [1,2], nr x nth order-2 quads (3x3 Gauss points), E=200e9, nu=0.28."""
    return annulus_mesh(nr, nth, 2, seed=SEEDS["annulus_p2"], name=f"annulus{nr}x{nth}_p2")


@dataclasses.dataclass
class MeshSpec:
    nx: int
    ny: int
    order: int
    aspect: float
    perturb: float
    E: float
    nu: float
    seed: int

    @property
    def num_elements(self) -> int:
        return self.nx * self.ny

    def num_nodes(self) -> int:
        return (self.nx * self.order + 1) * (self.ny * self.order + 1)

    def nnzb(self) -> int:
        p = self.order
        return (self.nx * (p * p + 2 * p) + 1) * (self.ny * (p * p + 2 * p) + 1)

    def build(self) -> Mesh:
        hy = 1.0 / self.ny
        hx = self.aspect * hy
        return square_mesh(self.nx, self.ny, self.order, hx * self.nx, 1.0, self.perturb, 1e-3, self.E, self.nu, 1.0,
                           self.seed, f"q{self.order}_{self.nx}x{self.ny}")


def batch_specs(count: int = 256, lo: float = 1e3, hi: float = 1e6, seed: int | None = None,
                perturb: float = 0.15, max_elements: float | None = None, max_dof: float | None = None
                ) -> list[MeshSpec]:
    """Independent meshes: element counts log-uniform in [lo, hi], order uniform in
    {1,2,3,4}, element aspect ratio (hx/hy) uniform in [1,4], perturbation +-0.15h,
    E in U[50e9, 210e9], nu in U[0.25, 0.35], all drawn from one seed.  With
    max_dof, the element count is capped so that 2*(p*nx+1)*(p*ny+1) <= max_dof."""
    rng = np.random.default_rng(SEEDS["batch256"] if seed is None else seed)
    out = []
    for i in range(count):
        ne = float(np.exp(rng.uniform(math.log(lo), math.log(hi))))
        if max_elements is not None:
            ne = min(ne, max_elements)
        order = int(rng.integers(1, 5))
        if max_dof is not None:
            ne = min(ne, 0.98 * (math.sqrt(max_dof / 2.0) - 1.0) ** 2 / (order * order))
        aspect = float(rng.uniform(1.0, 4.0))
        E = float(rng.uniform(50e9, 210e9))
        nu = float(rng.uniform(0.25, 0.35))
        ny = max(1, int(round(math.sqrt(ne))))
        nx = max(1, int(round(ne / ny)))
        out.append(MeshSpec(nx, ny, order, aspect, perturb, E, nu, int(rng.integers(0, 2**31 - 1))))
    return out


def submesh(mesh: Mesh, e0: int, e1: int) -> Mesh:
    """Elements [e0, e1) of `mesh` with their nodes renumbered compactly (ascending
    original id), keeping coordinates, states and material."""
    cp = mesh.conn_ptr.astype(np.int64)
    conn = mesh.conn[cp[e0]:cp[e1]]
    nodes, inv = np.unique(conn, return_inverse=True)
    new_ptr = (cp[e0:e1 + 1] - cp[e0]).astype(np.int32)
    return Mesh(mesh.order, np.ascontiguousarray(mesh.coords[nodes]), new_ptr, inv.astype(np.int32),
                np.ascontiguousarray(mesh.states[nodes]), mesh.E, mesh.nu, mesh.t, f"{mesh.name}[{e0}:{e1}]",
                mesh.seed)


def submesh_elements(mesh: Mesh, elements) -> Mesh:
    """The listed elements of `mesh` (ascending ids) with their nodes renumbered
    compactly in ascending original id, so that sorted node lists keep their order."""
    el = np.unique(np.asarray(elements, dtype=np.int64))
    n = mesh.nodes_per_element
    cp = mesh.conn_ptr.astype(np.int64)
    conn = np.concatenate([mesh.conn[cp[e]:cp[e] + n] for e in el]) if el.size else np.zeros(0, np.int32)
    nodes, inv = np.unique(conn, return_inverse=True)
    ptr = (np.arange(el.size + 1, dtype=np.int64) * n).astype(np.int32)
    sub = Mesh(mesh.order, np.ascontiguousarray(mesh.coords[nodes]), ptr, inv.astype(np.int32),
               np.ascontiguousarray(mesh.states[nodes]), mesh.E, mesh.nu, mesh.t, f"{mesh.name}[patch]", mesh.seed)
    sub.global_nodes = nodes
    return sub


def row_complete_patch(mesh: Mesh, core_elements):
    """Node rows that a small submesh assembles completely: S = every node of the
    core elements, and the patch = every element that touches a node of S.  Each
    node of S has all its elements in the patch, so the patch's assembled residual
    and matrix rows of S equal the full mesh's.  Returns (patch, S as global ids,
    S as patch-local ids); the mesh must list each element's nodes contiguously
    with a fixed count (structured meshes)."""
    n = mesh.nodes_per_element
    conn = mesh.conn.reshape(-1, n)
    S = np.unique(conn[np.asarray(core_elements, dtype=np.int64)])
    touching = np.nonzero(np.isin(conn, S).any(axis=1))[0]
    patch = submesh_elements(mesh, touching)
    local = np.searchsorted(patch.global_nodes, S)
    return patch, S, local
