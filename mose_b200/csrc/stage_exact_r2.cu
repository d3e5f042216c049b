// stage_exact_r2.cu -- instantiations of the reference-exact 2-D stage kernel
// for Riemann solver 2 (see MOSE_RIEMANN_* in mose_gpu.h).  Built with
// --fmad=false like every reference-exact unit.
#include "stage_exact_inst.cuh"

namespace mose {
bool launch_stage2d_exact_r2(const StageArgs& a, int grid, int mode, bool uni, int lim, cudaStream_t s) {
  return stage2d_dispatch_lim<2>(a, grid, mode, uni, lim, s);
}
}  // namespace mose
