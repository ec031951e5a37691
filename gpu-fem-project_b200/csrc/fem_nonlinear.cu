// Instantiations of the GreenStrainType::NONLINEAR assembly kernels (FP64 tensor
// cores; drop-in and plan modes), kept in their own translation unit so they
// compile in parallel with the linear ones.
#include "fem_launch.h"

namespace fem {

int launch_nl(int order, int mode, const dev::AsmArgs &a, cudaStream_t s) {
  using namespace dev;
  switch (mode) {
    case kRes: return launch_mode<double, kNL | kRes>(order, a, s);
    case kJac: return launch_mode<double, kNL | kJac>(order, a, s);
    case kRes | kJac: return launch_mode<double, kNL | kRes | kJac>(order, a, s);
    case kPlan | kRes: return launch_mode<double, kNL | kPlan | kRes>(order, a, s);
    case kPlan | kJac: return launch_mode<double, kNL | kPlan | kJac>(order, a, s);
    case kPlan | kRes | kJac: return launch_mode<double, kNL | kPlan | kRes | kJac>(order, a, s);
    default: return fail(FEM_ERR_INVALID_ARGUMENT, "bad kernel mode %d", mode);
  }
}

}  // namespace fem
