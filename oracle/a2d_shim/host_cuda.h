// Force-included (g++ -include) when element/FEKernels.h is compiled for the
// host as oracle/_ref: the header's GPU kernels are templates that the host
// build never instantiates, but g++ still parses them, so the CUDA keywords and
// built-in names they mention are given host meanings here (keywords empty,
// built-ins declared, never defined or called).
//
// FEKernels.h's host runResidualKernel (FEKernels.h:1067-1076) names
// `elemPerBlock` in the template argument list of assemblePlaneStressResidual,
// where the fourth parameter is the strain type; the reference's CPU build
// stops there.  The constant below gives that name the strain type the
// dispatcher means (the default, LINEAR); the kernel templates' own parameters
// of that name shadow it.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref); nothing in the library uses it.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdio>

#include "a2dcore.h"

#define __global__
#define __device__
#define __host__
#define __shared__
#define __forceinline__ inline

struct HostDim3 {
  unsigned x, y, z;
};
extern const HostDim3 threadIdx, blockIdx, blockDim, gridDim;
double atomicAdd(double *address, double value);
void __syncthreads();

constexpr A2D::GreenStrainType elemPerBlock = A2D::GreenStrainType::LINEAR;

// FEKernels.h:363 and :430 (the CPU residual and Jacobian loops) call
// interpRealGradient without template arguments, and its `order` cannot be
// deduced (it appears only in an array bound, FEKernels.h:260-264), so those
// calls fail with any A2D.  The overload below, in A2D's namespace, is found by
// argument-dependent lookup at those calls (their arguments are A2D::Mat); it
// takes order from the node count of the matrix, (order + 1)^2 rows, and calls
// the reference's own template with it, as the GPU kernel's call does
// (FEKernels.h:920).  The declaration is the reference's (FEKernels.h:260-264).
template <int order, int numVals, int numDim>
void interpRealGradient(const double xi[numDim], const double nodalValues[(order + 1) * (order + 1) * numVals],
                        const A2D::Mat<double, numDim, numDim> JInv, A2D::Mat<double, numVals, numDim> &dudx);
namespace A2D {
constexpr int order_of_nodes(int n) { return n == 4 ? 1 : n == 9 ? 2 : n == 16 ? 3 : n == 25 ? 4 : -1; }
template <int numNodes, int numVals, int numDim>
void interpRealGradient(const double xi[numDim], const Mat<double, numNodes, numVals> &nodalValues,
                        const Mat<double, numDim, numDim> &JInv, Mat<double, numVals, numDim> &dudx) {
  static_assert(order_of_nodes(numNodes) > 0, "interpRealGradient: 4, 9, 16 or 25 nodes");
  ::interpRealGradient<order_of_nodes(numNodes), numVals, numDim>(xi, nodalValues.get_data(), JInv, dudx);
}
}  // namespace A2D
