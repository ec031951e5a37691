"""B200-native global residual / 2x2-block BSR Jacobian assembly for 2D
plane-stress Lagrange quadrilaterals of order 1..4.

A drop-in for the element-kernel API of A-CGray/GPU-FEM-Project
(runResidualKernel / runJacobianKernel, element/FEKernels.h:1030,1125).  The
compute lives in libfemb200.so (CUDA sm_100a, C ABI in include/fem_b200.h);
this package is the host-side mirror of the reference interface.
"""
from ._lib import (FEM_ERR_BUDGET, FEM_ERR_CUDA, FEM_ERR_INVALID_ARGUMENT, FEM_ERR_INVALID_ORDER,
                   FEM_ERR_MISALIGNED, FEM_ERR_NOT_FOUND, FEM_ERR_OVERFLOW, FEM_ERR_TIMEOUT, FEM_ERR_UNSUPPORTED,
                   FEM_PRECISION_FP64, FEM_PRECISION_MIXED, FEM_SUCCESS, LIB_PATH, FemError, check, lib)
from .bdf import gmsh_to_tensor, read_bdf, write_bdf
from .api import (Batch, DeviceMesh, Plan, Server, bsr_spmv, build_bsr_pattern, build_element_bsr_map, colour_elements,
                  pair_layout, run_jacobian_kernel, run_residual_kernel)
from .mesh import (Mesh, annulus512x2048_p2, annulus_mesh, batch_specs, square1024_p3, square64_p1, square_mesh,
                   submesh)

__all__ = [
    "FEM_ERR_BUDGET", "FEM_ERR_CUDA", "FEM_ERR_INVALID_ARGUMENT", "FEM_ERR_INVALID_ORDER", "FEM_ERR_MISALIGNED",
    "FEM_ERR_NOT_FOUND", "FEM_ERR_OVERFLOW", "FEM_ERR_TIMEOUT", "FEM_ERR_UNSUPPORTED", "FEM_PRECISION_FP64", "FEM_PRECISION_MIXED",
    "FEM_SUCCESS", "LIB_PATH", "FemError", "check", "lib", "Batch", "DeviceMesh", "Server", "Plan", "bsr_spmv", "build_bsr_pattern",
    "build_element_bsr_map", "colour_elements", "pair_layout", "run_jacobian_kernel", "run_residual_kernel", "Mesh",
    "annulus512x2048_p2", "annulus_mesh", "batch_specs", "square1024_p3", "square64_p1", "square_mesh", "submesh", "read_bdf", "write_bdf", "gmsh_to_tensor",
]
