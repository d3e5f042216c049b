// stage3d_fp64_r0.cu -- 3-D stage sweeps, precision fp64 (MOSE_PRECISION_* = 1),
// Riemann solver 0 (MOSE_RIEMANN_*).
#include "stage3d_inst.cuh"

namespace mose {
bool launch_stage3d_p1_r0(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  return stage3d_dispatch_lim<1, 0>(a, nsm, mode, uni, lim, s);
}
}  // namespace mose
