// The reference's own FP64 CPU assembly (element/FEKernels.h:317-508 and its
// dispatchers runResidualKernel / runJacobianKernel, :1030-1225), compiled from
// the header where it lies in the reference checkout with the A2D interface
// restated in oracle/a2d_shim/ (A2D is not part of the checkout).  Built by
// oracle/Makefile (target `ref`) twice:
//   * oracle/_ref/libfemref.so without OpenMP: the reference's CPU matrix scatter
//     has no atomic (FEKernels.h:95-99), so serial execution is what makes it
//     deterministic; the tests and the golden vectors use this one;
//   * oracle/_ref/libfemref_omp.so with OpenMP, the reference's parallel loops as
//     written (their unsynchronised matrix scatter included), timed as the CPU
//     baseline of bench.py and never used as a checker.
//
// TEST INFRASTRUCTURE ONLY: tests/ compare the oracle restatement (and, through
// the committed fixtures of tests/golden/, the CUDA library) with it.
#include "FEKernels.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
template <int order>
void jac_nl(const int *connPtr, const int *conn, int nE, const double *states, const double *coords, double E,
            double nu, double t, int *map, double *residual, double *mat) {
  assemblePlaneStressJacobian<order, 2, 2, A2D::GreenStrainType::NONLINEAR>(connPtr, conn, nE, states, coords, E, nu,
                                                                            t, map, residual, mat);
}
template <int order>
void res_nl(const int *connPtr, const int *conn, int nE, const double *states, const double *coords, double E,
            double nu, double t, double *residual) {
  assemblePlaneStressResidual<order, 2, 2, A2D::GreenStrainType::NONLINEAR>(connPtr, conn, nE, states, coords, E, nu,
                                                                            t, residual);
}
}  // namespace

extern "C" {

// Threads of the OpenMP build's parallel loops (no effect in the serial build).
void ref_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// runResidualKernel (FEKernels.h:1030-1102), host build.  Accumulates into residual.
double ref_run_residual(int order, const int *connPtr, const int *conn, int nE, const double *states,
                        const double *coords, double E, double nu, double t, double *residual) {
  return runResidualKernel(order, connPtr, conn, nE, states, coords, E, nu, t, residual);
}

// runJacobianKernel (FEKernels.h:1125-1225), host build.  Accumulates into
// matEntries through the element map and, when residual != NULL, into residual.
double ref_run_jacobian(int order, const int *connPtr, const int *conn, int nE, const double *states,
                        const double *coords, double E, double nu, double t, int *map, double *residual,
                        double *mat) {
  return runJacobianKernel(order, connPtr, conn, nE, states, coords, E, nu, t, map, residual, mat);
}

// The same CPU loops with GreenStrainType::NONLINEAR (a template option the
// dispatchers never select, FEKernels.h:317,379).  Returns 0, or -1 for an
// order outside 1..4.
int ref_assemble_nonlinear(int order, const int *connPtr, const int *conn, int nE, const double *states,
                           const double *coords, double E, double nu, double t, int *map, double *residual,
                           double *mat) {
  switch (order) {
    case 1: mat ? jac_nl<1>(connPtr, conn, nE, states, coords, E, nu, t, map, residual, mat)
                : res_nl<1>(connPtr, conn, nE, states, coords, E, nu, t, residual); break;
    case 2: mat ? jac_nl<2>(connPtr, conn, nE, states, coords, E, nu, t, map, residual, mat)
                : res_nl<2>(connPtr, conn, nE, states, coords, E, nu, t, residual); break;
    case 3: mat ? jac_nl<3>(connPtr, conn, nE, states, coords, E, nu, t, map, residual, mat)
                : res_nl<3>(connPtr, conn, nE, states, coords, E, nu, t, residual); break;
    case 4: mat ? jac_nl<4>(connPtr, conn, nE, states, coords, E, nu, t, map, residual, mat)
                : res_nl<4>(connPtr, conn, nE, states, coords, E, nu, t, residual); break;
    default: return -1;
  }
  return 0;
}

}  // extern "C"
