"""ctypes wrapper of the FP64 CPU oracle (oracle/libfemoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check in
__graft_entry__.py and by the CPU-baseline leg of bench.py, where it is the
checker or the timed CPU reference -- never part of the product path.
See fem_oracle.cpp for what is restated from which reference file:line and for
the pinning status (tables pinned against the reference's own headers; element
physics not pinned by reference outputs).
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libfemoracle.so"


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def _load():
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    p, i, i64, d = C.c_void_p, C.c_int, C.c_int64, C.c_double
    lib.oracle_tables.argtypes = [i, p, p, p]
    lib.oracle_lagrange1d.argtypes = [i, i, p, p, p]
    lib.oracle_element.argtypes = [i, p, p, d, d, d, p, p]
    lib.oracle_element_ex.argtypes = [i, p, p, d, d, d, i, p, p]
    lib.oracle_element_energy.argtypes = [i, p, p, d, d, d, i, p]
    lib.oracle_assemble.argtypes = [i, p, p, i64, p, p, d, d, d, p, p, p]
    lib.oracle_assemble_ex.argtypes = [i, p, p, i64, p, p, d, d, d, i, p, p, p]
    lib.oracle_assemble_parallel.argtypes = [i, p, p, i64, p, p, d, d, d, p, p, p]
    lib.oracle_bsr_pattern.argtypes = [i, p, p, i64, p, p]
    lib.oracle_bsr_pattern.restype = i64
    lib.oracle_element_bsr_map.argtypes = [p, p, i64, i, p, p, p]
    lib.oracle_element_bsr_map.restype = i64
    lib.oracle_check_colouring.argtypes = [i, p, p, i64, p, i]
    lib.oracle_check_colouring.restype = i64
    lib.oracle_bsr_spmv.argtypes = [i, p, p, p, p, p]
    lib.oracle_set_num_threads.argtypes = [i]
    lib.oracle_set_extended_j.argtypes = [i]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def set_threads(n: int) -> None:
    lib().oracle_set_num_threads(int(n))


def set_extended_j(on: bool) -> None:
    """Accumulate the isoparametric Jacobian in long double (True) or with the
    reference's plain FP64 sum (False, the default)."""
    lib().oracle_set_extended_j(1 if on else 0)


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def tables(p: int):
    """(xi[p+1], w[p+1], dN[(p+1)^2, (p+1)^2, 2]) with q = qy*(p+1)+qx, a = ay*(p+1)+ax."""
    n = (p + 1) ** 2
    xi, w, dN = np.zeros(p + 1), np.zeros(p + 1), np.zeros((n, n, 2))
    assert lib().oracle_tables(p, _ptr(xi), _ptr(w), _ptr(dN)) == 0
    return xi, w, dN


def lagrange1d(p: int, x):
    x = _c(x, np.float64)
    N = np.zeros((x.size, p + 1))
    dN = np.zeros((x.size, p + 1))
    assert lib().oracle_lagrange1d(p, x.size, _ptr(x), _ptr(N), _ptr(dN)) == 0
    return N, dN


STRAIN = {"linear": 0, "nonlinear": 1}


def element(p: int, X, U, E: float, nu: float, t: float, strain: str = "linear"):
    """Element residual [2n] and stiffness [2n, 2n] for node coords X [n,2], states U [n,2]."""
    n = (p + 1) ** 2
    X, U = _c(X, np.float64), _c(U, np.float64)
    Re, Ke = np.zeros(2 * n), np.zeros((2 * n, 2 * n))
    assert lib().oracle_element_ex(p, _ptr(X), _ptr(U), E, nu, t, STRAIN[strain], _ptr(Re), _ptr(Ke)) == 0
    return Re, Ke


def element_energy(p: int, X, U, E: float, nu: float, t: float, strain: str = "linear") -> float:
    """Element strain energy sum_q 1/2 w detJ t S:E."""
    X, U = _c(X, np.float64), _c(U, np.float64)
    W = np.zeros(1)
    assert lib().oracle_element_energy(p, _ptr(X), _ptr(U), E, nu, t, STRAIN[strain], _ptr(W)) == 0
    return float(W[0])


def bsr_pattern(num_nodes: int, conn_ptr, conn):
    conn_ptr, conn = _c(conn_ptr, np.int32), _c(conn, np.int32)
    ne = conn_ptr.size - 1
    nnz = lib().oracle_bsr_pattern(num_nodes, _ptr(conn_ptr), _ptr(conn), ne, None, None)
    rowp = np.zeros(num_nodes + 1, np.int32)
    cols = np.zeros(nnz, np.int32)
    lib().oracle_bsr_pattern(num_nodes, _ptr(conn_ptr), _ptr(conn), ne, _ptr(rowp), _ptr(cols))
    return rowp, cols


def element_bsr_map(conn_ptr, conn, nodes_per_element: int, rowp, cols):
    conn_ptr, conn = _c(conn_ptr, np.int32), _c(conn, np.int32)
    rowp, cols = _c(rowp, np.int32), _c(cols, np.int32)
    ne = conn_ptr.size - 1
    m = np.zeros(ne * nodes_per_element ** 2, np.int32)
    missing = lib().oracle_element_bsr_map(_ptr(conn_ptr), _ptr(conn), ne, nodes_per_element, _ptr(rowp), _ptr(cols),
                                           _ptr(m))
    assert missing == 0, f"{missing} blocks missing from pattern"
    return m


def check_colouring(num_nodes: int, conn_ptr, conn, colour, num_colours: int) -> int:
    conn_ptr, conn, colour = _c(conn_ptr, np.int32), _c(conn, np.int32), _c(colour, np.int32)
    return int(lib().oracle_check_colouring(num_nodes, _ptr(conn_ptr), _ptr(conn), conn_ptr.size - 1, _ptr(colour),
                                            num_colours))


def assemble(mesh, bsr_map=None, nnzb: int | None = None, residual: bool = True, jacobian: bool = True,
             parallel: bool = False, num_elements: int | None = None, strain: str = "linear"):
    """Residual [numNodes*2] and BSR values [nnzb*4] (zero-initialised, then
    accumulated as runJacobianKernel does).  parallel=True uses the OpenMP
    atomic-scatter variant (timed CPU baseline; summation order not fixed;
    linear strain only)."""
    ne = mesh.num_elements if num_elements is None else num_elements
    cp, cn = _c(mesh.conn_ptr, np.int32), _c(mesh.conn, np.int32)
    st, xy = _c(mesh.states, np.float64), _c(mesh.coords, np.float64)
    res = np.zeros(mesh.num_nodes * 2) if residual else None
    mat = None
    mp = None
    if jacobian:
        mp = _c(bsr_map, np.int32)
        mat = np.zeros(int(nnzb) * 4)
    if parallel:
        assert strain == "linear"
        rc = lib().oracle_assemble_parallel(mesh.order, _ptr(cp), _ptr(cn), ne, _ptr(st), _ptr(xy), mesh.E, mesh.nu,
                                            mesh.t, _ptr(mp), _ptr(res), _ptr(mat))
    else:
        rc = lib().oracle_assemble_ex(mesh.order, _ptr(cp), _ptr(cn), ne, _ptr(st), _ptr(xy), mesh.E, mesh.nu, mesh.t,
                                      STRAIN[strain], _ptr(mp), _ptr(res), _ptr(mat))
    assert rc == 0
    return res, mat


REF_LIB_PATH = HERE / "_ref" / "libfemref.so"
_ref_lib = None


def ref_available() -> bool:
    """Whether oracle/_ref/libfemref.so (the reference's own CPU assembly compiled
    from its header, oracle/Makefile target `ref`) has been built here."""
    return REF_LIB_PATH.exists()


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        lib = C.CDLL(str(REF_LIB_PATH))
        p, i, d = C.c_void_p, C.c_int, C.c_double
        lib.ref_run_residual.argtypes = [i, p, p, i, p, p, d, d, d, p]
        lib.ref_run_residual.restype = d
        lib.ref_run_jacobian.argtypes = [i, p, p, i, p, p, d, d, d, p, p, p]
        lib.ref_run_jacobian.restype = d
        lib.ref_assemble_nonlinear.argtypes = [i, p, p, i, p, p, d, d, d, p, p, p]
        lib.ref_assemble_nonlinear.restype = i
        _ref_lib = lib
    return _ref_lib


def ref_assemble(mesh, bsr_map=None, nnzb: int | None = None, jacobian: bool = True, strain: str = "linear"):
    """Residual and BSR values from the reference's own CPU assembly
    (runResidualKernel / runJacobianKernel, element/FEKernels.h:1030-1225, host
    build, serial), zero-initialised then accumulated as the reference driver does."""
    cp, cn = _c(mesh.conn_ptr, np.int32), _c(mesh.conn, np.int32)
    st, xy = _c(mesh.states, np.float64), _c(mesh.coords, np.float64)
    res = np.zeros(mesh.num_nodes * 2)
    mat = mp = None
    if jacobian:
        mp = _c(bsr_map, np.int32)
        mat = np.zeros(int(nnzb) * 4)
    ne = mesh.num_elements
    if strain == "nonlinear":
        rc = ref_lib().ref_assemble_nonlinear(mesh.order, _ptr(cp), _ptr(cn), ne, _ptr(st), _ptr(xy), mesh.E, mesh.nu,
                                              mesh.t, _ptr(mp), _ptr(res), _ptr(mat))
        assert rc == 0
    elif jacobian:
        ref_lib().ref_run_jacobian(mesh.order, _ptr(cp), _ptr(cn), ne, _ptr(st), _ptr(xy), mesh.E, mesh.nu, mesh.t,
                                   _ptr(mp), _ptr(res), _ptr(mat))
    else:
        ref_lib().ref_run_residual(mesh.order, _ptr(cp), _ptr(cn), ne, _ptr(st), _ptr(xy), mesh.E, mesh.nu, mesh.t,
                                   _ptr(res))
    return res, mat


def bsr_spmv(rowp, cols, A, x):
    rowp, cols, A, x = _c(rowp, np.int32), _c(cols, np.int32), _c(A, np.float64), _c(x, np.float64)
    y = np.zeros(x.size)
    lib().oracle_bsr_spmv(rowp.size - 1, _ptr(rowp), _ptr(cols), _ptr(A), _ptr(x), _ptr(y))
    return y
