// stage3d_mixed_r4.cu -- 3-D stage sweeps, precision mixed (MOSE_PRECISION_* = 2),
// the run-time solver unit (every MOSE_RIEMANN_* index from 2).
#include "stage3d_inst.cuh"

namespace mose {
bool launch_stage3d_p2_r4(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  return stage3d_dispatch_lim<2, 4>(a, nsm, mode, uni, lim, s);
}
}  // namespace mose
