// stage_inst.cuh -- launch dispatch of the 2-D stage kernel over arithmetic
// policy, limiter, metric mode and kernel mode.  Each translation unit
// stage_<precision>_r<solver>.cu instantiates one (precision, Riemann solver)
// pair.  The residual-only mode (the phase-by-phase C-ABI path) exists for the
// reference-exact policy with metric arrays and for the fp64 policy; the
// fused mode has constant-metric variants for uniform grids.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "stage2d.cuh"

namespace mose {

template <int PREC, int RIE, int LIM>
using StagePolicy = typename std::conditional<PREC == 0, PolExact<RIE, LIM>, PolFast<RIE, LIM, PREC == 2>>::type;

// Persistent grid: as many CTAs as the SMs hold at once (registers and the
// shared-memory ring decide), never more than there are work items.
template <int PREC, int RIE, int LIM, bool UNI, int MODE, bool BC>
static void launch_persistent_list(const StageArgs& a, int nitems, int nsm, cudaStream_t s) {
  using PH = StagePolicy<PREC, RIE, LIM>;
  constexpr size_t smem = stage_smem_bytes<UNI, stage_fp32_pipeline<PH, RIE, UNI>(), BC, RIE == 4>();
  static int occ = 0;   // one per kernel instance
  if (occ == 0) {
    cudaFuncSetAttribute(k_stage2d<PH, RIE, LIM, UNI, MODE, BC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage2d<PH, RIE, LIM, UNI, MODE, BC>, SB_T, smem) !=
            cudaSuccess ||
        occ < 1)
      occ = 1;
  }
  const int per_sm = (a.grid_cap > 0 && a.grid_cap < occ) ? a.grid_cap : occ;
  const int grid = nitems < per_sm * nsm ? nitems : per_sm * nsm;
  k_stage2d<PH, RIE, LIM, UNI, MODE, BC><<<grid, SB_T, smem, s>>>(a);
}

// The items without physical boundary faces, then those with.
template <int PREC, int RIE, int LIM, bool UNI, int MODE>
static void launch_persistent(const StageArgs& a, int nsm, cudaStream_t s) {
  if (a.nitems_nb > 0) launch_persistent_list<PREC, RIE, LIM, UNI, MODE, false>(a, a.nitems_nb, nsm, s);
  if (a.nitems > 0) launch_persistent_list<PREC, RIE, LIM, UNI, MODE, true>(a, a.nitems, nsm, s);
}

template <int PREC, int RIE, int LIM>
static bool stage2d_dispatch_uni(const StageArgs& a, int nsm, int mode, bool uni, cudaStream_t s) {
  if (mode == 1) {
    // residual only: the reference-exact policy with metric arrays, and the
    // fp64 policy in both metric modes (its residual is checked against the
    // oracle's per evaluation)
    if constexpr (PREC == 0) {
      launch_persistent<PREC, RIE, LIM, false, 1>(a, nsm, s);
      return true;
    } else if constexpr (PREC == 1) {
      if (uni) launch_persistent<PREC, RIE, LIM, true, 1>(a, nsm, s);
      else launch_persistent<PREC, RIE, LIM, false, 1>(a, nsm, s);
      return true;
    }
    return false;
  }
  if (mode == 2) {
    if (uni) launch_persistent<PREC, RIE, LIM, true, 2>(a, nsm, s);
    else launch_persistent<PREC, RIE, LIM, false, 2>(a, nsm, s);
    return true;
  }
  if (uni) launch_persistent<PREC, RIE, LIM, true, 0>(a, nsm, s);
  else launch_persistent<PREC, RIE, LIM, false, 0>(a, nsm, s);
  return true;
}

template <int PREC, int RIE>
static bool stage2d_dispatch_lim(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  switch (lim) {
    case 0: return stage2d_dispatch_uni<PREC, RIE, 0>(a, nsm, mode, uni, s);
    case 1: return stage2d_dispatch_uni<PREC, RIE, 1>(a, nsm, mode, uni, s);
    case 2: return stage2d_dispatch_uni<PREC, RIE, 2>(a, nsm, mode, uni, s);
    case 3: return stage2d_dispatch_uni<PREC, RIE, 3>(a, nsm, mode, uni, s);
    case 4: return stage2d_dispatch_uni<PREC, RIE, 4>(a, nsm, mode, uni, s);
    case 5: return stage2d_dispatch_uni<PREC, RIE, 5>(a, nsm, mode, uni, s);
  }
  return false;
}

}  // namespace mose
