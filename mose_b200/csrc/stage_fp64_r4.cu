// stage_fp64_r4.cu -- 2-D stage kernels, precision fp64 (MOSE_PRECISION_* = 1),
// the Riemann solvers selected at run time (MOSE_RIEMANN_* >= 4).
#include "stage_inst.cuh"

namespace mose {
bool launch_stage2d_p1_r4(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  return stage2d_dispatch_lim<1, 4>(a, nsm, mode, uni, lim, s);
}
}  // namespace mose
