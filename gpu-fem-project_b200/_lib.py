"""ctypes binding of libfemb200.so (the C ABI declared in include/fem_b200.h).

The library is required: importing this module without the built .so, or
calling a device entry point on a machine without a CUDA device, raises.  There
is no CPU fallback for the assembly path.
"""
from __future__ import annotations

import ctypes as C
import pathlib

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfemb200.so"

FEM_SUCCESS = 0
FEM_ERR_INVALID_ORDER = 1
FEM_ERR_INVALID_ARGUMENT = 2
FEM_ERR_MISALIGNED = 3
FEM_ERR_CUDA = 4
FEM_ERR_OVERFLOW = 5
FEM_ERR_NOT_FOUND = 6
FEM_ERR_UNSUPPORTED = 7
FEM_ERR_BUDGET = 8
FEM_ERR_TIMEOUT = 9

FEM_PRECISION_FP64 = 0
FEM_PRECISION_MIXED = 1

FEM_STRAIN_LINEAR = 0
FEM_STRAIN_NONLINEAR = 1

# element order of the fragment kernel's single-mesh colour launches (fem_plan_set_layout)
FEM_LAYOUT_COLOURS = 0
FEM_LAYOUT_PAIRS = 1

# batch kernel variants (fem_batch_get_kernels / fem_batch_set_kernels)
FEM_KERNELS = {0: "default", 1: "rows", 2: "fragment_fp64", 3: "fragment_bf16x6", 4: "element_fp64",
               5: "element_fp32", 6: "element_tcgen05"}

_i = C.c_int
_i64 = C.c_int64
_d = C.c_double
_p = C.c_void_p
_pi = C.POINTER(C.c_int)
_pi64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol declared in include/fem_b200.h
SIGNATURES = {
    "fem_status_string": (C.c_char_p, [_i]),
    "fem_last_error": (C.c_char_p, []),
    "fem_version": (_i, []),
    "fem_run_residual": (_i, [_i, _p, _p, _i, _p, _p, _d, _d, _d, _p, _p, _pd]),
    "fem_run_jacobian": (_i, [_i, _p, _p, _i, _p, _p, _d, _d, _d, _p, _p, _p, _p, _pd]),
    "fem_run_residual_mixed": (_i, [_i, _p, _p, _i, _p, _p, _d, _d, _d, _p, _p, _pd]),
    "fem_run_jacobian_mixed": (_i, [_i, _p, _p, _i, _p, _p, _d, _d, _d, _p, _p, _p, _p, _pd]),
    "fem_run_residual_ex": (_i, [_i, _p, _p, _i, _p, _p, _d, _d, _d, _p, _i, _i, _p, _pd]),
    "fem_run_jacobian_ex": (_i, [_i, _p, _p, _i, _p, _p, _d, _d, _d, _p, _p, _p, _i, _i, _p, _pd]),
    "fem_build_bsr_pattern": (_i, [_i, _p, _p, _i, _p, _p, _pi64]),
    "fem_build_element_bsr_map": (_i, [_p, _p, _i, _i, _p, _p, _p]),
    "fem_colour_elements": (_i, [_i, _p, _p, _i, _p, _pi]),
    "fem_pair_layout": (_i, [_i, _i, _p, _p, _i, _p, _p, _pi, _pi64, _p, _pi]),
    "fem_bsr_spmv": (_i, [_i, _p, _p, _p, _p, _p, _p]),
    "fem_plan_create": (_i, [_i, _i, _p, _p, _i, C.POINTER(_p)]),
    "fem_plan_destroy": (_i, [_p]),
    "fem_plan_info": (_i, [_p, _pi, _pi, _pi64, _pi, _pi64]),
    "fem_plan_get_pattern": (_i, [_p, _p, _p]),
    "fem_plan_device_pattern": (_i, [_p, C.POINTER(_p), C.POINTER(_p)]),
    "fem_plan_assemble": (_i, [_p, _p, _p, _d, _d, _d, _p, _p, _i, _p, _pd]),
    "fem_plan_row_chunks": (_i, [_p, _pi]),
    "fem_plan_set_layout": (_i, [_p, _i]),
    "fem_plan_get_layout": (_i, [_p, _pi, _pi64, _pi]),
    "fem_plan_assemble_ex": (_i, [_p, _p, _p, _d, _d, _d, _p, _p, _i, _i, _p, _pd]),
    "fem_plan_assemble_host": (_i, [_p, _p, _p, _p, _d, _d, _d, _p, _p, _p, _i, _i, _i, _p, _pd]),
    "fem_plan_set_schedule": (_i, [_p, _i, _i]),
    "fem_plan_get_schedule": (_i, [_p, _pi, _pi, _pi, _pi]),
    "fem_plan_wait_status": (_i, [_p, _p, _pi64]),
    "fem_plan_get_schedule_tables": (_i, [_p, _p, _p, _p, _p, _p, _p]),
    "fem_plan_set_schedule_waits": (_i, [_p, _i64, _i]),
    "fem_server_create": (_i, [_i64, _i, _i, C.POINTER(_p)]),
    "fem_server_destroy": (_i, [_p]),
    "fem_server_add_mesh": (_i, [_p, _i, _i, _p, _p, _i, _p, _d, _d, _d, _pi]),
    "fem_server_remove_mesh": (_i, [_p, _i]),
    "fem_server_mesh_outputs": (_i, [_p, _i, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p), C.POINTER(_p), _pi64]),
    "fem_server_submit": (_i, [_p, _i, _p, _p, _pi64]),
    "fem_server_wait": (_i, [_p, _i64, _i, _pd]),
    "fem_server_stats": (_i, [_p, _pi64, _pi64, _pi64, _pi64, _pi64]),
    "fem_run_jacobian_batched_static": (_i, [_i, _p, _p]),
    "fem_batch_create": (_i, [_i, _p, C.POINTER(_p)]),
    "fem_batch_destroy": (_i, [_p]),
    "fem_batch_bind": (_i, [_p, _i, _p, _p, _d, _d, _d, _p, _p]),
    "fem_batch_info": (_i, [_p, _pi64, _pi64, _pi, _pi64]),
    "fem_batch_get_tiles": (_i, [_p, _p]),
    "fem_batch_set_tiles": (_i, [_p, _p]),
    "fem_batch_assemble": (_i, [_p, _i, _p, _pd]),
    "fem_batch_tune": (_i, [_p, _i, _p, _i, _pd]),
    "fem_batch_get_kernels": (_i, [_p, _i, _p]),
    "fem_batch_set_kernels": (_i, [_p, _i, _p]),
    "fem_batch_set_ordered": (_i, [_p, _p]),
    "fem_batch_get_ordered": (_i, [_p, _p]),
    "fem_batch_wait_status": (_i, [_p, _p, _pi64]),
    "fem_batch_set_schedule_waits": (_i, [_p, _i64, _i, _i]),
    "fem_batch_capture": (_i, [_p, _i, _p]),
    "fem_batch_replay": (_i, [_p, _p, _pd]),
}


class FemError(RuntimeError):
    """A non-zero status from the C ABI, with the library's message."""

    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: status {status} ({message})")


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python gpu-fem-project_b200/build.py` "
            "(the assembly path has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int, where: str) -> None:
    if status != FEM_SUCCESS:
        msg = lib.fem_last_error().decode() or lib.fem_status_string(status).decode()
        raise FemError(status, where, msg)


def exported_symbols():
    """Names from SIGNATURES that the loaded library exports."""
    return [n for n in SIGNATURES if getattr(lib, n, None) is not None]
