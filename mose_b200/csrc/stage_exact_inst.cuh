// stage_exact_inst.cuh -- launch dispatch of the reference-exact 2-D stage
// kernel over limiter, metric mode and kernel mode.  The residual-only mode
// (phase-by-phase C-ABI path) always reads the metric arrays; the fused mode
// has a constant-metric variant for uniform grids.
#pragma once

#include <cuda_runtime.h>

#include "stage2d.cuh"

namespace mose {

template <int RIE, int LIM>
static void stage2d_dispatch_uni(const StageArgs& a, int grid, int mode, bool uni, cudaStream_t s) {
  if (mode == 1) k_stage2d<RIE, LIM, false, 1><<<grid, STRIP_T, 0, s>>>(a);
  else if (uni) k_stage2d<RIE, LIM, true, 0><<<grid, STRIP_T, 0, s>>>(a);
  else k_stage2d<RIE, LIM, false, 0><<<grid, STRIP_T, 0, s>>>(a);
}

template <int RIE>
static bool stage2d_dispatch_lim(const StageArgs& a, int grid, int mode, bool uni, int lim, cudaStream_t s) {
  switch (lim) {
    case 0: stage2d_dispatch_uni<RIE, 0>(a, grid, mode, uni, s); return true;
    case 1: stage2d_dispatch_uni<RIE, 1>(a, grid, mode, uni, s); return true;
    case 2: stage2d_dispatch_uni<RIE, 2>(a, grid, mode, uni, s); return true;
    case 3: stage2d_dispatch_uni<RIE, 3>(a, grid, mode, uni, s); return true;
    case 4: stage2d_dispatch_uni<RIE, 4>(a, grid, mode, uni, s); return true;
    case 5: stage2d_dispatch_uni<RIE, 5>(a, grid, mode, uni, s); return true;
  }
  return false;
}

}  // namespace mose
