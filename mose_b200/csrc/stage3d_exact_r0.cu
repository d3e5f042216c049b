// stage3d_exact_r0.cu -- 3-D stage sweeps, precision exact (MOSE_PRECISION_* = 0),
// Riemann solver 0 (MOSE_RIEMANN_*).
#include "stage3d_inst.cuh"

namespace mose {
bool launch_stage3d_p0_r0(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  return stage3d_dispatch_lim<0, 0>(a, nsm, mode, uni, lim, s);
}
}  // namespace mose
