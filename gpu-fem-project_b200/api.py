"""Python host mirror of the reference's element-kernel API over the C ABI.

`run_residual_kernel` / `run_jacobian_kernel` keep the argument order and
meaning of runResidualKernel / runJacobianKernel (element/FEKernels.h:1030,1125):
device arrays in, accumulate into the caller-zeroed outputs, elapsed seconds
out.  Device arrays are torch CUDA tensors (or raw device pointers as ints).
Errors raise FemError instead of exiting the process (GPUMacros.h:23-31).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import FEM_KERNELS, FEM_PRECISION_FP64, FEM_PRECISION_MIXED, FEM_STRAIN_LINEAR, FEM_STRAIN_NONLINEAR, check, lib

_PRECISION = {"fp64": FEM_PRECISION_FP64, "mixed": FEM_PRECISION_MIXED}
# A2D::GreenStrainType of the reference kernels' strainType template argument
_STRAIN = {"linear": FEM_STRAIN_LINEAR, "nonlinear": FEM_STRAIN_NONLINEAR}


def _prec(p) -> int:
    if isinstance(p, int):
        return p
    return _PRECISION[p]


def _strain(s) -> int:
    if isinstance(s, int):
        return s
    return _STRAIN[s]


def _dptr(x, dtype=None, name="array"):
    """Device pointer of a CUDA tensor (or an int pointer); None stays None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    import torch
    if not isinstance(x, torch.Tensor):
        raise TypeError(f"{name}: expected a CUDA tensor or a device pointer, got {type(x).__name__}")
    if not x.is_cuda:
        raise ValueError(f"{name}: tensor is on {x.device}; the assembly path runs on the GPU only")
    if not x.is_contiguous():
        raise ValueError(f"{name}: tensor must be contiguous")
    if dtype is not None and x.dtype != dtype:
        raise TypeError(f"{name}: dtype {x.dtype}, expected {dtype}")
    return x.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _np(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def run_residual_kernel(element_order, conn_ptr, conn, num_elements, states, node_coords, E, nu, t, residual, *,
                        precision="fp64", strain="linear", stream=None, timed=True):
    """runResidualKernel: adds element residuals into `residual`; returns seconds (timed) or None.
    strain="nonlinear" selects GreenStrainType::NONLINEAR (FP64 only)."""
    import torch
    el = C.c_double(0.0)
    args = (int(element_order), _dptr(conn_ptr, torch.int32, "connPtr"), _dptr(conn, torch.int32, "conn"),
            int(num_elements), _dptr(states, torch.float64, "states"), _dptr(node_coords, torch.float64, "nodeCoords"),
            float(E), float(nu), float(t), _dptr(residual, torch.float64, "residual"))
    tail = (_stream(stream), C.byref(el) if timed else None)
    if _strain(strain) != FEM_STRAIN_LINEAR:
        check(lib.fem_run_residual_ex(*args, _prec(precision), _strain(strain), *tail), "fem_run_residual_ex")
    else:
        fn = lib.fem_run_residual if _prec(precision) == FEM_PRECISION_FP64 else lib.fem_run_residual_mixed
        check(fn(*args, *tail), "fem_run_residual")
    return el.value if timed else None


def run_jacobian_kernel(element_order, conn_ptr, conn, num_elements, states, node_coords, E, nu, t,
                        element_bcsr_map, residual, mat_entries, *, precision="fp64", strain="linear", stream=None,
                        timed=True):
    """runJacobianKernel: adds element matrices (and residuals when `residual` is
    not None) into the caller-zeroed outputs; returns seconds (timed) or None.
    strain="nonlinear" selects GreenStrainType::NONLINEAR (FP64 only)."""
    import torch
    el = C.c_double(0.0)
    args = (int(element_order), _dptr(conn_ptr, torch.int32, "connPtr"), _dptr(conn, torch.int32, "conn"),
            int(num_elements), _dptr(states, torch.float64, "states"), _dptr(node_coords, torch.float64, "nodeCoords"),
            float(E), float(nu), float(t), _dptr(element_bcsr_map, torch.int32, "elementBCSRMap"),
            _dptr(residual, torch.float64, "residual"), _dptr(mat_entries, torch.float64, "matEntries"))
    tail = (_stream(stream), C.byref(el) if timed else None)
    if _strain(strain) != FEM_STRAIN_LINEAR:
        check(lib.fem_run_jacobian_ex(*args, _prec(precision), _strain(strain), *tail), "fem_run_jacobian_ex")
    else:
        fn = lib.fem_run_jacobian if _prec(precision) == FEM_PRECISION_FP64 else lib.fem_run_jacobian_mixed
        check(fn(*args, *tail), "fem_run_jacobian")
    return el.value if timed else None


def build_bsr_pattern(num_nodes, conn_ptr, conn):
    """(rowp int32[numNodes+1], cols int32[nnzb]) of the nodal adjacency (host)."""
    cp, cn = _np(conn_ptr, np.int32), _np(conn, np.int32)
    ne = cp.size - 1
    rowp = np.zeros(int(num_nodes) + 1, np.int32)
    nnzb = C.c_int64(0)
    check(lib.fem_build_bsr_pattern(int(num_nodes), cp.ctypes.data, cn.ctypes.data, ne, rowp.ctypes.data, None,
                                    C.byref(nnzb)), "fem_build_bsr_pattern")
    cols = np.zeros(nnzb.value, np.int32)
    check(lib.fem_build_bsr_pattern(int(num_nodes), cp.ctypes.data, cn.ctypes.data, ne, rowp.ctypes.data,
                                    cols.ctypes.data, C.byref(nnzb)), "fem_build_bsr_pattern")
    return rowp, cols


def build_element_bsr_map(conn_ptr, conn, nodes_per_element, rowp, cols):
    """generateElementBCSRMap: int32[numElements * n * n] of block offsets * 4 (host)."""
    cp, cn = _np(conn_ptr, np.int32), _np(conn, np.int32)
    rp, cl = _np(rowp, np.int32), _np(cols, np.int32)
    ne = cp.size - 1
    out = np.zeros(ne * int(nodes_per_element) ** 2, np.int32)
    check(lib.fem_build_element_bsr_map(cp.ctypes.data, cn.ctypes.data, ne, int(nodes_per_element), rp.ctypes.data,
                                        cl.ctypes.data, out.ctypes.data), "fem_build_element_bsr_map")
    return out


def colour_elements(num_nodes, conn_ptr, conn):
    """(colour int32[numElements], numColours): greedy, element order, no shared nodes per colour."""
    cp, cn = _np(conn_ptr, np.int32), _np(conn, np.int32)
    ne = cp.size - 1
    colour = np.zeros(ne, np.int32)
    nc = C.c_int(0)
    check(lib.fem_colour_elements(int(num_nodes), cp.ctypes.data, cn.ctypes.data, ne, colour.ctypes.data,
                                  C.byref(nc)), "fem_colour_elements")
    return colour, nc.value


def pair_layout(order, num_nodes, conn_ptr, conn, codes=False):
    """The pair layout of an order-2..4 plan (host): (elemList, colourPtr, numPairs,
    codes uint8[numElements, codeStride] or None).  colourPtr is empty when the plan
    has no pair layout."""
    cp, cn = _np(conn_ptr, np.int32), _np(conn, np.int32)
    ne = cp.size - 1
    nn = (order + 1) ** 2
    stride = (nn * nn + nn + 15) // 16 * 16
    elist = np.zeros(max(ne, 1), np.int32)
    cptr = np.zeros(65, np.int32)
    nc, npairs, cs = C.c_int(0), C.c_int64(0), C.c_int(0)
    rec = np.zeros((max(ne, 1), stride), np.uint8) if codes else None
    check(lib.fem_pair_layout(int(order), int(num_nodes), cp.ctypes.data, cn.ctypes.data, ne, elist.ctypes.data,
                              cptr.ctypes.data, C.byref(nc), C.byref(npairs),
                              rec.ctypes.data if codes else None, C.byref(cs)), "fem_pair_layout")
    assert not codes or cs.value == stride
    return elist[:ne], cptr[:nc.value + 1] if nc.value else cptr[:0], npairs.value, (rec[:ne] if codes else None)


def bsr_spmv(rowp, cols, values, x, y, stream=None):
    """y = A x on the device for the 2x2-block BSR matrix (rowp, cols, values)."""
    import torch
    n = int(rowp.numel()) - 1
    check(lib.fem_bsr_spmv(n, _dptr(rowp, torch.int32), _dptr(cols, torch.int32), _dptr(values, torch.float64),
                           _dptr(x, torch.float64), _dptr(y, torch.float64), _stream(stream)), "fem_bsr_spmv")


class Plan:
    """Device-resident assembly plan of one mesh (fem_plan_*): BSR pattern,
    colouring and block codes.  `assemble` overwrites the outputs completely."""

    def __init__(self, element_order, num_nodes, conn_ptr, conn):
        cp, cn = _np(conn_ptr, np.int32), _np(conn, np.int32)
        self._h = C.c_void_p()
        check(lib.fem_plan_create(int(element_order), int(num_nodes), cp.ctypes.data, cn.ctypes.data, cp.size - 1,
                                  C.byref(self._h)), "fem_plan_create")
        self.order = int(element_order)
        nn, ne, nc = C.c_int(), C.c_int(), C.c_int()
        nnzb, nbytes = C.c_int64(), C.c_int64()
        check(lib.fem_plan_info(self._h, C.byref(nn), C.byref(ne), C.byref(nnzb), C.byref(nc), C.byref(nbytes)),
              "fem_plan_info")
        self.num_nodes, self.num_elements, self.nnzb = nn.value, ne.value, nnzb.value
        self.num_colours, self.device_bytes = nc.value, nbytes.value
        rc = C.c_int()
        check(lib.fem_plan_row_chunks(self._h, C.byref(rc)), "fem_plan_row_chunks")
        self.row_chunks = rc.value

    def launches(self, strain="linear", precision="fp64") -> int:
        """Kernel launches of one assemble(): 1 for order-1 row assembly and for a
        dependency-ordered plan, else one per colour."""
        if self.row_chunks > 0 and _strain(strain) == FEM_STRAIN_LINEAR:
            return 1
        if self.scheduled(strain, precision):
            return 1
        lay, _, pair_colours = self.layout()
        return pair_colours if lay == "pairs" and self.fragment(strain, precision) else self.num_colours

    def fragment(self, strain="linear", precision="fp64") -> bool:
        """Whether assemble() runs the warp-fragment kernel (orders 2-3, order 4 in
        FP64 LINEAR)."""
        nl, fp64 = _strain(strain) != FEM_STRAIN_LINEAR, _prec(precision) == FEM_PRECISION_FP64
        if nl:
            return fp64 and self.order in (2, 3)
        return self.order in (2, 3) or (self.order == 4 and fp64)

    def scheduled(self, strain="linear", precision="fp64") -> bool:
        """Whether assemble() runs all colours in one dependency-ordered launch: the
        plan has a schedule and the assembly runs the fragment kernel (orders 2-3,
        and order 4 in FP64 LINEAR)."""
        if self.schedule()["groups"] == 0:
            return False
        return self.fragment(strain, precision)

    def schedule(self):
        """The dependency-ordered schedule: band and tile lengths (elements), groups, tiles."""
        b, t, g, n = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib.fem_plan_get_schedule(self._h, C.byref(b), C.byref(t), C.byref(g), C.byref(n)),
              "fem_plan_get_schedule")
        return {"band": b.value, "tile": t.value, "groups": g.value, "tiles": n.value}

    def schedule_tables(self):
        """Host copies of the schedule: tile (begin, count, group) arrays, tiles per
        group and the dependency CSR (dep_ptr, deps)."""
        info = self.schedule()
        T, G = info["tiles"], info["groups"]
        begin, count, group = np.zeros(T, np.int64), np.zeros(T, np.int32), np.zeros(T, np.int32)
        gt, ptr = np.zeros(G, np.int32), np.zeros(G + 1, np.int32)
        check(lib.fem_plan_get_schedule_tables(self._h, begin.ctypes.data, count.ctypes.data, group.ctypes.data,
                                               gt.ctypes.data, ptr.ctypes.data, None), "fem_plan_get_schedule_tables")
        deps = np.zeros(max(int(ptr[-1]), 1), np.int32)
        check(lib.fem_plan_get_schedule_tables(self._h, None, None, None, None, None, deps.ctypes.data),
              "fem_plan_get_schedule_tables")
        return {"tile_begin": begin, "tile_count": count, "tile_group": group, "group_tiles": gt, "dep_ptr": ptr,
                "deps": deps[:int(ptr[-1])]}

    def set_layout(self, layout):
        """'pairs' (default where built) or 'colours': the element order of the
        fragment kernel's single-mesh colour launches."""
        code = {"colours": _lib.FEM_LAYOUT_COLOURS, "pairs": _lib.FEM_LAYOUT_PAIRS}[layout]
        check(lib.fem_plan_set_layout(self._h, code), "fem_plan_set_layout")

    def layout(self):
        """(layout name, pairs formed, pair colours)."""
        lay, npairs, ncol = C.c_int(), C.c_int64(), C.c_int()
        check(lib.fem_plan_get_layout(self._h, C.byref(lay), C.byref(npairs), C.byref(ncol)), "fem_plan_get_layout")
        return ("pairs" if lay.value == _lib.FEM_LAYOUT_PAIRS else "colours"), npairs.value, ncol.value

    def set_schedule(self, band=-1, tile=0):
        """band = -1: the default band (about 8 MB of blocks), 0: colour launches;
        tile = 0: the default tile length."""
        check(lib.fem_plan_set_schedule(self._h, int(band), int(tile)), "fem_plan_set_schedule")

    def wait_status(self, stream=None) -> int:
        """Waits for the stream; in-kernel waits that ran out since the last call."""
        n = C.c_int64()
        check(lib.fem_plan_wait_status(self._h, _stream(stream), C.byref(n)), "fem_plan_wait_status")
        return n.value

    def set_schedule_waits(self, wait_limit_ns=0, stall_group=-1):
        """Failure injection for tests: the wait limit and a group no wait sees finished."""
        check(lib.fem_plan_set_schedule_waits(self._h, int(wait_limit_ns), int(stall_group)),
              "fem_plan_set_schedule_waits")

    @property
    def handle(self) -> int:
        return self._h.value

    def pattern(self):
        rowp = np.zeros(self.num_nodes + 1, np.int32)
        cols = np.zeros(self.nnzb, np.int32)
        check(lib.fem_plan_get_pattern(self._h, rowp.ctypes.data, cols.ctypes.data), "fem_plan_get_pattern")
        return rowp, cols

    def device_pattern(self):
        """(rowp, cols) device pointers owned by the plan."""
        r, c = C.c_void_p(), C.c_void_p()
        check(lib.fem_plan_device_pattern(self._h, C.byref(r), C.byref(c)), "fem_plan_device_pattern")
        return r.value, c.value

    def assemble(self, states, node_coords, E, nu, t, residual=None, mat_entries=None, *, precision="fp64",
                 strain="linear", stream=None, timed=False):
        import torch
        el = C.c_double(0.0)
        check(lib.fem_plan_assemble_ex(self._h, _dptr(states, torch.float64, "states"),
                                       _dptr(node_coords, torch.float64, "nodeCoords"), float(E), float(nu), float(t),
                                       _dptr(residual, torch.float64, "residual"),
                                       _dptr(mat_entries, torch.float64, "matEntries"), _prec(precision),
                                       _strain(strain), _stream(stream), C.byref(el) if timed else None),
              "fem_plan_assemble_ex")
        return el.value if timed else None

    def assemble_host(self, host_states, states, node_coords, E, nu, t, host_residual, residual, mat_entries=None, *,
                      precision="fp64", strain="linear", bands=8, stream=None, timed=False):
        """fem_plan_assemble_host: upload `host_states` (CPU tensor, pinned for overlap)
        into the device `states`, assemble, download `residual` into `host_residual`,
        the copies overlapped with the band-split assembly; results equal assemble()'s."""
        import torch
        for name, x in (("host_states", host_states), ("host_residual", host_residual)):
            if not isinstance(x, torch.Tensor) or x.is_cuda or x.dtype != torch.float64 or not x.is_contiguous():
                raise ValueError(f"{name}: expected a contiguous float64 CPU tensor")
        el = C.c_double(0.0)
        check(lib.fem_plan_assemble_host(self._h, host_states.data_ptr(), _dptr(states, torch.float64, "states"),
                                         _dptr(node_coords, torch.float64, "nodeCoords"), float(E), float(nu),
                                         float(t), host_residual.data_ptr(),
                                         _dptr(residual, torch.float64, "residual"),
                                         _dptr(mat_entries, torch.float64, "matEntries"), _prec(precision),
                                         _strain(strain), int(bands), _stream(stream),
                                         C.byref(el) if timed else None), "fem_plan_assemble_host")
        return el.value if timed else None

    def close(self):
        if self._h and self._h.value:
            lib.fem_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many meshes assembled together (fem_batch_*): one persistent kernel per
    (order, colour) pulls element tiles from a work queue; orders run concurrently.
    The plans must stay alive as long as the batch (the batch keeps references)."""

    def __init__(self, plans):
        self.plans = list(plans)
        arr = (C.c_void_p * len(self.plans))(*[p.handle for p in self.plans])
        self._h = C.c_void_p()
        check(lib.fem_batch_create(len(self.plans), arr, C.byref(self._h)), "fem_batch_create")

    def bind(self, mesh, states, node_coords, E, nu, t, residual, mat_entries):
        import torch
        check(lib.fem_batch_bind(self._h, int(mesh), _dptr(states, torch.float64, "states"),
                                 _dptr(node_coords, torch.float64, "nodeCoords"), float(E), float(nu), float(t),
                                 _dptr(residual, torch.float64, "residual"),
                                 _dptr(mat_entries, torch.float64, "matEntries")), "fem_batch_bind")

    def info(self):
        ne, nt, bytes_ = C.c_int64(), C.c_int64(), C.c_int64()
        nl = C.c_int()
        check(lib.fem_batch_info(self._h, C.byref(ne), C.byref(nt), C.byref(nl), C.byref(bytes_)), "fem_batch_info")
        tiles = (C.c_int * 4)()
        check(lib.fem_batch_get_tiles(self._h, tiles), "fem_batch_get_tiles")
        return {"elements": ne.value, "tiles": nt.value, "launches": nl.value, "device_bytes": bytes_.value,
                "tile_batches": list(tiles), "kernels_fp64": self.kernels("fp64"), "kernels_mixed": self.kernels("mixed"),
                "ordered": self.ordered()}

    def ordered(self):
        """Per order (1..4): 1 where its colours run as one dependency-ordered launch."""
        arr = (C.c_int * 4)()
        check(lib.fem_batch_get_ordered(self._h, arr), "fem_batch_get_ordered")
        return list(arr)

    def set_ordered(self, ordered):
        """Per order (1..4; order 1 must be 0): one dependency-ordered launch for all colours."""
        arr = (C.c_int * 4)(*[int(x) for x in ordered])
        check(lib.fem_batch_set_ordered(self._h, arr), "fem_batch_set_ordered")

    def wait_status(self, *, stream=None):
        """Bounded in-kernel waits of the dependency-ordered launches that ran out (cleared)."""
        n = C.c_int64(0)
        check(lib.fem_batch_wait_status(self._h, _stream(stream), C.byref(n)), "fem_batch_wait_status")
        return n.value

    def set_schedule_waits(self, order, wait_limit_ns=0, stall_group=-1):
        """Failure injection: wait limit and a group whose completion no wait observes."""
        check(lib.fem_batch_set_schedule_waits(self._h, int(wait_limit_ns), int(order), int(stall_group)),
              "fem_batch_set_schedule_waits")

    def kernels(self, precision="fp64"):
        """Kernel variant per order (1..4) for `precision`, by name (FEM_KERNEL_*)."""
        arr = (C.c_int * 4)()
        check(lib.fem_batch_get_kernels(self._h, _prec(precision), arr), "fem_batch_get_kernels")
        return [FEM_KERNELS[int(v)] for v in arr]

    def set_kernels(self, names, precision="fp64"):
        """Kernel variants per order (1..4) by name; "default" = the plan path's kernel."""
        ids = {v: k for k, v in FEM_KERNELS.items()}
        arr = (C.c_int * 4)(*[ids[n] for n in names])
        check(lib.fem_batch_set_kernels(self._h, _prec(precision), arr), "fem_batch_set_kernels")

    def set_tiles(self, tile_batches):
        arr = (C.c_int * 4)(*[int(x) for x in tile_batches])
        check(lib.fem_batch_set_tiles(self._h, arr), "fem_batch_set_tiles")

    def assemble(self, *, precision="fp64", stream=None, timed=False):
        el = C.c_double(0.0)
        check(lib.fem_batch_assemble(self._h, _prec(precision), _stream(stream), C.byref(el) if timed else None),
              "fem_batch_assemble")
        return el.value if timed else None

    def tune(self, *, precision="fp64", stream=None, reps=3):
        best = C.c_double(0.0)
        check(lib.fem_batch_tune(self._h, _prec(precision), _stream(stream), int(reps), C.byref(best)),
              "fem_batch_tune")
        return best.value

    def capture(self, *, precision="fp64", stream=None):
        check(lib.fem_batch_capture(self._h, _prec(precision), _stream(stream)), "fem_batch_capture")

    def replay(self, *, stream=None, timed=False):
        el = C.c_double(0.0)
        check(lib.fem_batch_replay(self._h, _stream(stream), C.byref(el) if timed else None), "fem_batch_replay")
        return el.value if timed else None

    def close(self):
        if self._h and self._h.value:
            lib.fem_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _hptr(x):
    """Host pointer of a numpy array or a (pinned) CPU tensor."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous or x.dtype != np.float64:
            raise ValueError("host arrays must be contiguous float64")
        return x.ctypes.data
    import torch
    if isinstance(x, torch.Tensor):
        if x.is_cuda or x.dtype != torch.float64 or not x.is_contiguous():
            raise ValueError("host tensors must be contiguous float64 CPU tensors")
        return x.data_ptr()
    raise TypeError(type(x).__name__)


class Server:
    """Continuous-batching assembly server over device-resident meshes (fem_server_*)."""

    def __init__(self, budget_bytes, *, precision="fp64", max_batch=64):
        self._h = C.c_void_p()
        check(lib.fem_server_create(int(budget_bytes), _prec(precision), int(max_batch), C.byref(self._h)),
              "fem_server_create")
        self._inflight = {}

    def add_mesh(self, mesh):
        cp, cn = _np(mesh.conn_ptr, np.int32), _np(mesh.conn, np.int32)
        xy = _np(mesh.coords, np.float64)
        mid = C.c_int()
        check(lib.fem_server_add_mesh(self._h, mesh.order, mesh.num_nodes, cp.ctypes.data, cn.ctypes.data, cp.size - 1,
                                      xy.ctypes.data, float(mesh.E), float(mesh.nu), float(mesh.t), C.byref(mid)),
              "fem_server_add_mesh")
        return mid.value

    def remove_mesh(self, mesh_id):
        check(lib.fem_server_remove_mesh(self._h, int(mesh_id)), "fem_server_remove_mesh")

    def outputs(self, mesh_id):
        r, a, rp, cl = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        nnzb = C.c_int64()
        check(lib.fem_server_mesh_outputs(self._h, int(mesh_id), C.byref(r), C.byref(a), C.byref(rp), C.byref(cl),
                                          C.byref(nnzb)), "fem_server_mesh_outputs")
        return {"residual": r.value, "mat": a.value, "rowp": rp.value, "cols": cl.value, "nnzb": nnzb.value}

    def submit(self, mesh_id, host_states, host_residual=None):
        tk = C.c_int64()
        check(lib.fem_server_submit(self._h, int(mesh_id), _hptr(host_states), _hptr(host_residual), C.byref(tk)),
              "fem_server_submit")
        self._inflight[tk.value] = (host_states, host_residual)
        return tk.value

    def wait(self, ticket, timeout_ms=120000):
        lat = C.c_double()
        try:
            check(lib.fem_server_wait(self._h, int(ticket), int(timeout_ms), C.byref(lat)), "fem_server_wait")
        finally:
            self._inflight.pop(ticket, None)
        return lat.value

    def stats(self):
        w, c, e, u, b = (C.c_int64() for _ in range(5))
        check(lib.fem_server_stats(self._h, C.byref(w), C.byref(c), C.byref(e), C.byref(u), C.byref(b)),
              "fem_server_stats")
        return {"waves": w.value, "completed": c.value, "elements": e.value, "used_bytes": u.value,
                "budget_bytes": b.value}

    def close(self):
        if self._h and self._h.value:
            lib.fem_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceMesh:
    """A Mesh uploaded to the GPU as torch tensors (int32 topology, float64 data)."""

    def __init__(self, mesh, device="cuda"):
        import torch
        self.mesh = mesh
        self.order = mesh.order
        self.conn_ptr = torch.from_numpy(_np(mesh.conn_ptr, np.int32)).to(device)
        self.conn = torch.from_numpy(_np(mesh.conn, np.int32)).to(device)
        self.coords = torch.from_numpy(_np(mesh.coords, np.float64)).to(device)
        self.states = torch.from_numpy(_np(mesh.states, np.float64)).to(device)
