// stage3d_mixed_r0.cu -- 3-D stage sweeps, precision mixed (MOSE_PRECISION_* = 2),
// Riemann solver 0 (MOSE_RIEMANN_*).
#include "stage3d_inst.cuh"

namespace mose {
bool launch_stage3d_p2_r0(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  return stage3d_dispatch_lim<2, 0>(a, nsm, mode, uni, lim, s);
}
}  // namespace mose
