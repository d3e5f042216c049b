// stage3d_inst.cuh -- launch dispatch of the 3-D sweeps over arithmetic
// policy, limiter and metric mode.  Each translation unit
// stage3d_<precision>_r<solver>.cu instantiates one (precision, Riemann
// solver) pair for the six limiters (first order, minmod, van Leer, van
// Albada, MC, superbee).
#pragma once

#include <cuda_runtime.h>

#include "stage3d.cuh"
#include "stage_inst.cuh"

namespace mose {

template <class K>
static int occupancy_grid(K kernel, int nitems, int nsm, int& occ) {
  if (occ == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, SB_T, 0) != cudaSuccess || occ < 1) occ = 1;
  }
  const int g = occ * nsm;
  return nitems < g ? nitems : g;
}

// One RK stage (or one residual evaluation, MODE 1): the i-sweep, the
// j-march, then the k-march that finishes the residual.
template <int PREC, int RIE, int LIM, bool UNI, int MODE>
static void launch3d(const StageArgs& a, int nsm, cudaStream_t s) {
  using PH = StagePolicy<PREC, RIE, LIM>;
  static int occ[3] = {0, 0, 0};
  if (a.nitems3[0] > 0) {
    auto k0 = k_sweep3d_i<PH, RIE, LIM, UNI>;
    k0<<<occupancy_grid(k0, a.nitems3[0], nsm, occ[0]), SB_T, 0, s>>>(a, a.items3[0], a.nitems3[0]);
  }
  auto k1 = k_march3d<PH, RIE, LIM, UNI, 1, 3>;
  k1<<<occupancy_grid(k1, a.nitems3[1], nsm, occ[1]), SB_T, 0, s>>>(a, a.items3[1], a.nitems3[1]);
  auto k2 = k_march3d<PH, RIE, LIM, UNI, 2, MODE>;
  k2<<<occupancy_grid(k2, a.nitems3[2], nsm, occ[2]), SB_T, 0, s>>>(a, a.items3[2], a.nitems3[2]);
}

template <int PREC, int RIE, int LIM>
static bool stage3d_dispatch_uni(const StageArgs& a, int nsm, int mode, bool uni, cudaStream_t s) {
  if (mode == 1) {
    // residual only: the reference-exact policy with metric arrays, and the
    // fp64 policy in both metric modes (its residual is checked against the
    // oracle's per evaluation)
    if constexpr (PREC == 0) {
      launch3d<PREC, RIE, LIM, false, 1>(a, nsm, s);
      return true;
    } else if constexpr (PREC == 1) {
      if (uni) launch3d<PREC, RIE, LIM, true, 1>(a, nsm, s);
      else launch3d<PREC, RIE, LIM, false, 1>(a, nsm, s);
      return true;
    }
    return false;
  }
  if (mode == 2) {
    if (uni) launch3d<PREC, RIE, LIM, true, 2>(a, nsm, s);
    else launch3d<PREC, RIE, LIM, false, 2>(a, nsm, s);
    return true;
  }
  if (uni) launch3d<PREC, RIE, LIM, true, 0>(a, nsm, s);
  else launch3d<PREC, RIE, LIM, false, 0>(a, nsm, s);
  return true;
}

template <int PREC, int RIE>
static bool stage3d_dispatch_lim(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s) {
  switch (lim) {
    case 0: return stage3d_dispatch_uni<PREC, RIE, 0>(a, nsm, mode, uni, s);
    case 1: return stage3d_dispatch_uni<PREC, RIE, 1>(a, nsm, mode, uni, s);
    case 2: return stage3d_dispatch_uni<PREC, RIE, 2>(a, nsm, mode, uni, s);
    case 3: return stage3d_dispatch_uni<PREC, RIE, 3>(a, nsm, mode, uni, s);
    case 4: return stage3d_dispatch_uni<PREC, RIE, 4>(a, nsm, mode, uni, s);
    case 5: return stage3d_dispatch_uni<PREC, RIE, 5>(a, nsm, mode, uni, s);
  }
  return false;
}

}  // namespace mose
