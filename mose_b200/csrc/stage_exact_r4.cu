// stage_exact_r4.cu -- 2-D stage kernels, precision exact (MOSE_PRECISION_* = 0),
// the Riemann solvers selected at run time (MOSE_RIEMANN_* >= 4).
#include "stage_inst.cuh"

namespace mose {
bool launch_stage2d_p0_r4(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  return stage2d_dispatch_lim<0, 4>(a, nsm, mode, uni, lim, s);
}
}  // namespace mose
