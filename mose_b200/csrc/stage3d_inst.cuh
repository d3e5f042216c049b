// stage3d_inst.cuh -- launch dispatch of the 3-D stage kernels over
// arithmetic policy, limiter and metric mode.  Each translation unit
// stage3d_<precision>_r<solver>.cu instantiates one (precision, Riemann
// solver) pair for the six limiters (first order, minmod, van Leer, van
// Albada, MC, superbee).
#pragma once

#include <cuda_runtime.h>

#include "stage3d.cuh"
#include "stage_inst.cuh"

namespace mose {

// The persistent grid of a kernel instance: one CTA per resident slot, at
// most one per item.
template <class K>
static int persistent_grid(K kernel, int threads, size_t smem, int nsm, int n, int& occ) {
  if (occ == 0) {
    if (smem > 0) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem) != cudaSuccess || occ < 1)
      occ = 1;
  }
  return n < occ * nsm ? n : occ * nsm;
}

// One RK stage (or one residual evaluation, MODE 1): the k-face march over
// every tile (items3[2]), then the plane stage over the connection-only tiles
// (items3[0]) and over the tiles with a physical boundary face (items3[1]).
// A list with no items launches nothing, so a caller may pass each part on
// its own stream.
template <int PREC, int RIE, int LIM, bool UNI, int MODE>
static void launch3d(const StageArgs& a, int nsm, cudaStream_t s) {
  using PH = StagePolicy<PREC, RIE, LIM>;
  constexpr size_t smem = stage3d_smem_bytes<UNI, stage3d_f32<PH, UNI>()>();
  static int occ_k = 0, occ_n = 0, occ_b = 0;   // one set per kernel instance
  if (a.nitems3[2] > 0) {
    const int n = a.nitems3[2];
    const int g = persistent_grid(k_kface3d<PH, RIE, LIM, UNI>, SB_T, 0, nsm, n, occ_k);
    k_kface3d<PH, RIE, LIM, UNI><<<g, SB_T, 0, s>>>(a, a.items3[2], n);
  }
  if (a.nitems3[0] > 0) {
    const int n = a.nitems3[0];
    const int g = persistent_grid(k_stage3d<PH, RIE, LIM, UNI, MODE, false>, s3_threads<PH>(), smem, nsm, n, occ_n);
    k_stage3d<PH, RIE, LIM, UNI, MODE, false><<<g, s3_threads<PH>(), smem, s>>>(a, a.items3[0], n);
  }
  if (a.nitems3[1] > 0) {
    const int n = a.nitems3[1];
    const int g = persistent_grid(k_stage3d<PH, RIE, LIM, UNI, MODE, true>, s3_threads<PH>(), smem, nsm, n, occ_b);
    k_stage3d<PH, RIE, LIM, UNI, MODE, true><<<g, s3_threads<PH>(), smem, s>>>(a, a.items3[1], n);
  }
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
