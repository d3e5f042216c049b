// stage_exact_r1.cu -- 2-D stage kernels, precision exact (MOSE_PRECISION_* = 0),
// Riemann solver 1 (MOSE_RIEMANN_*).
#include "stage_inst.cuh"

namespace mose {
bool launch_stage2d_p0_r1(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  return stage2d_dispatch_lim<0, 1>(a, nsm, mode, uni, lim, s);
}
}  // namespace mose
