// kernels_exact.cu -- the reference-exact FP64 kernels.  Built with
// --fmad=false: no multiply-add contraction, every operation rounds once in
// the order of the reference's Fortran expressions.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "metrics.cuh"
#include "stage2d.cuh"

namespace mose {

// ---------------------------------------------------------------------------
// Metrics (Mod_Metrics.f90:8-107)
// ---------------------------------------------------------------------------
// Interior cells: Compute_Metric_Tensor -> dl, vol, CFL versors.
__global__ void k_cell_metrics(const BlockDesc* blk, int b, NodeView nv, double* dl, double* vol,
                               double* vers, double* Mt, int nd, int ndir, DevError* err) {
  const BlockDesc& d = blk[b];
  long long n = (long long)d.ni * d.nj * d.nk;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    int I = i + 1, J = j + 1, K = k + 1;   // reference indices
    double M[9], l[3], v;
    bool ok = metric_tensor(nv.at(I - 1, J - 1, K - 1), nv.at(I - 1, J - 1, K), nv.at(I - 1, J, K - 1),
                            nv.at(I - 1, J, K), nv.at(I, J - 1, K - 1), nv.at(I, J - 1, K), nv.at(I, J, K - 1),
                            nv.at(I, J, K), M, l, &v);
    if (!ok) report(err, 6, b, i, j, k);
    long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    long long vs = d.vstride, mb = d.mbase;
    for (int h = 0; h < 3; ++h) dl[3 * mb + h * vs + o] = l[h];
    vol[mb + o] = v;
    // the 2-D metric tensor of the viscous fluxes: M(r,s) at plane (r-1) + 2(s-1)
    if (Mt)
      for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) Mt[4 * mb + (r + 2 * c) * vs + o] = M[r + 3 * c];
    // versor = M(d,:)/norm2(M(d,:))  (Mod_dt.f90:78-80)
    for (int dd = 0; dd < ndir; ++dd) {
      double m0 = M[dd + 0], m1 = M[dd + 3], m2 = M[dd + 6];
      double nrm = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
      vers[9 * mb + (3 * dd + 0) * vs + o] = m0 / nrm;
      vers[9 * mb + (3 * dd + 1) * vs + o] = m1 / nrm;
      vers[9 * mb + (3 * dd + 2) * vs + o] = m2 / nrm;
    }
  }
}

// Compute_Norm_Area (Lib_Metrics.f90:69-247).  One thread per face of the
// direction; stored with the cell on the high side of the face.
__global__ void k_face_metrics(const BlockDesc* blk, int b, NodeView nv, double* face, int nd, int dir) {
  const BlockDesc& d = blk[b];
  int ei = d.ni + (dir == 0), ej = d.nj + (dir == 1), ek = d.nk + (dir == 2);
  long long n = (long long)ei * ej * ek;
  double s[3];
  face_signs(nv, s);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % ei), j = (int)((q / ei) % ej), k = (int)(q / ((long long)ei * ej));
    // reference face indices: dir(1)%f(0:ni,1:nj,1:nk) etc.
    int I = (dir == 0) ? i : i + 1, J = (dir == 1) ? j : j + 1, K = (dir == 2) ? k : k + 1;
    double nrm[3], A;
    face_metric(nv, dir, I, J, K, s[dir], nrm, &A);
    // the face with reference index I (dir 0) is the low face of 0-based cell I
    int ci = (dir == 0) ? I : I - 1, cj = (dir == 1) ? J : J - 1, ck = (dir == 2) ? K : K - 1;
    if (nd == 2 && dir == 2) continue;
    long long o = (nd == 3) ? cell_off3(d, ci, cj, ck) : cell_off2(d, ci, cj);
    long long vs = d.vstride, mb = d.mbase;
    double* f = face + 12 * mb + (4 * dir) * vs + o;
    f[0] = nrm[0]; f[vs] = nrm[1]; f[2 * vs] = nrm[2]; f[3 * vs] = A;
  }
}

// Precomputed metrics of block b handed to mose_gpu_add_block: the
// reference's Setup_Metrics arrays in their Fortran memory order (vol, dl%c(3),
// M%c(3,3) over 1-gc:n+gc in every direction, then dir(1..3)%f as (N(3), A)),
// laid over the planes the node kernels above formed.  Interior cells take
// vol, dl and the CFL versors M(d,:)/norm2(M(d,:)) (and M(1:2,1:2) for the
// viscous terms); the ghost layers take dl along their boundary's normal (and
// M in the first layer), as the ghost-metric kernel stores them.
__global__ void k_metrics_from_ref(const BlockDesc* blk, int b, const double* src, double* dl, double* vol,
                                   double* vers, double* Mt, int nd, int ndir) {
  const BlockDesc& d = blk[b];
  const int ni = d.ni, nj = d.nj, nk = d.nk;
  const long long gi = ni + 4, gj = nj + 4, gk = nk + 4, NG = gi * gj * gk;
  const double* rvol = src;
  const double* rdl = src + NG;
  const double* rM = src + 4 * NG;
  const long long n = gi * gj * (nd == 3 ? gk : 1);
  const long long vs = d.vstride, mb = d.mbase;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % gi) - 2, j = (int)((q / gi) % gj) - 2, k = nd == 3 ? (int)(q / (gi * gj)) - 2 : 0;
    const bool oi = i < 0 || i >= ni, oj = j < 0 || j >= nj, ok = nd == 3 && (k < 0 || k >= nk);
    if ((int)oi + (int)oj + (int)ok > 1) continue;   // corners: not metric cells
    const long long r = (i + 2) + gi * ((j + 2) + gj * (long long)(k + 2));   // reference linear index
    const long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    const double* M = rM + 9 * r;   // M(a, c) at (a - 1) + 3 (c - 1)
    if (!oi && !oj && !ok) {
      vol[mb + o] = rvol[r];
      for (int h = 0; h < 3; ++h) dl[3 * mb + h * vs + o] = rdl[3 * r + h];
      if (Mt)
        for (int a = 0; a < 2; ++a)
          for (int c = 0; c < 2; ++c) Mt[4 * mb + (a + 2 * c) * vs + o] = M[a + 3 * c];
      for (int dd = 0; dd < ndir; ++dd) {
        double m0 = M[dd + 0], m1 = M[dd + 3], m2 = M[dd + 6];
        double nrm = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
        vers[9 * mb + (3 * dd + 0) * vs + o] = m0 / nrm;
        vers[9 * mb + (3 * dd + 1) * vs + o] = m1 / nrm;
        vers[9 * mb + (3 * dd + 2) * vs + o] = m2 / nrm;
      }
    } else {
      const int dir = oi ? 0 : oj ? 1 : 2;
      dl[3 * mb + dir * vs + o] = rdl[3 * r + dir];
      const bool first = (oi && (i == -1 || i == ni)) || (oj && (j == -1 || j == nj));
      if (Mt && nd == 2 && first)
        for (int a = 0; a < 2; ++a)
          for (int c = 0; c < 2; ++c) Mt[4 * mb + (a + 2 * c) * vs + o] = M[a + 3 * c];
    }
  }
}

// The face part of the same input: dir(dir+1)%f, (N(3), A) per face, onto the
// low-face planes (the face of reference index I along i is the low face of
// 0-based cell I).
__global__ void k_faces_from_ref(const BlockDesc* blk, int b, const double* src, double* face, int nd, int dir) {
  const BlockDesc& d = blk[b];
  const int ei = d.ni + (dir == 0), ej = d.nj + (dir == 1), ek = d.nk + (dir == 2);
  const long long n = (long long)ei * ej * ek;
  const long long vs = d.vstride, mb = d.mbase;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % ei), j = (int)((q / ei) % ej), k = (int)(q / ((long long)ei * ej));
    const long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    const double* f = src + 4 * q;
    double* g = face + 12 * mb + (4 * dir) * vs + o;
    g[0] = f[0]; g[vs] = f[1]; g[2 * vs] = f[2]; g[3 * vs] = f[3];
  }
}

// Ghost dl along the face direction for each boundary record:
// BC_Connect_Metrics (101), BC_Symmetry_Metrics (300), BC_Extrapolate_Metrics
// (everything else), Lib_Metrics.f90:535-1092.
__device__ void store_ghost_dl(const BlockDesc* blk, double* dl, int b, int nd, int I, int J, int K, int dir,
                               double val, DevError* err) {
  const BlockDesc& d = blk[b];
  // bounds self-check: the cell must lie inside the ghosted extents
  const bool in = I - 1 >= -GW && I - 1 < d.ni + GW && J - 1 >= -GW && J - 1 < d.nj + GW &&
                  (nd == 2 || (K - 1 >= -GW && K - 1 < d.nk + GW));
  if (!in) {
    if (atomicCAS(&err->code, 0, 1) == 0) { err->b = b + 1; err->i = I; err->j = J; err->k = K; }
    return;
  }
  long long o = (nd == 3) ? cell_off3(d, I - 1, J - 1, K - 1) : cell_off2(d, I - 1, J - 1);
  dl[3 * d.mbase + dir * d.vstride + o] = val;
}

// The metric tensor of the first ghost layer (viscous fluxes; Mt null otherwise).
__device__ void store_ghost_M(const BlockDesc* blk, double* Mt, int b, int nd, int I, int J, int K, const double* M,
                              DevError* err) {
  if (!Mt || nd != 2) return;
  const BlockDesc& d = blk[b];
  const bool in = I - 1 >= -GW && I - 1 < d.ni + GW && J - 1 >= -GW && J - 1 < d.nj + GW;
  if (!in) {
    if (atomicCAS(&err->code, 0, 1) == 0) { err->b = b + 1; err->i = I; err->j = J; err->k = K; }
    return;
  }
  const long long o = cell_off2(d, I - 1, J - 1);
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 2; ++c) Mt[4 * d.mbase + (r + 2 * c) * d.vstride + o] = M[r + 3 * c];
}

__global__ void k_ghost_metrics(const BlockDesc* blk, const GhostMetricRec* recs, int nrec,
                                const NodeView* nodes, double* dl, double* Mt, int nd, int ndir, DevError* err) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nrec) return;
  const GhostMetricRec e = recs[q];
  const int dir = (e.F - 1) / 2;
  if (dir >= nd) return;
  const BlockDesc& bm = blk[e.b];
  const NodeView& nv = nodes[e.b];
  const int Im = e.I, Jm = e.J, Km = e.K;
  // self-check: the node view must describe this record's block (and source)
  if (nv.p == nullptr || nv.ni != bm.ni || nv.nj != bm.nj || nv.nk != bm.nk ||
      (e.type == 101 && (nodes[e.bs].p == nullptr || nodes[e.bs].ni != blk[e.bs].ni))) {
    if (atomicCAS(&err->code, 0, 1) == 0) { err->b = -2; err->i = q; err->j = e.b; err->k = e.bs; }
    return;
  }
  double M[9], l[3], v;
  bool ok = true;
  if (e.type == 300) {
    // BC_Symmetry_Metrics: ghost g takes the metrics of the g-th interior cell
    for (int g = 1; g <= GW; ++g) {
      int gi = Im, gj = Jm, gk = Km, si = Im, sj = Jm, sk = Km;
      switch (e.F) {
        case 1: gi = Im - g; si = Im + g - 1; break;
        case 2: gi = Im + g; si = Im - g + 1; break;
        case 3: gj = Jm - g; sj = Jm + g - 1; break;
        case 4: gj = Jm + g; sj = Jm - g + 1; break;
        case 5: gk = Km - g; sk = Km + g - 1; break;
        case 6: gk = Km + g; sk = Km - g + 1; break;
      }
      long long so = (nd == 3) ? cell_off3(bm, si - 1, sj - 1, sk - 1) : cell_off2(bm, si - 1, sj - 1);
      double val = dl[3 * bm.mbase + dir * bm.vstride + so];
      store_ghost_dl(blk, dl, e.b, nd, gi, gj, gk, dir, val, err);
      if (g == 1 && Mt && nd == 2) {
        double Ms[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int r = 0; r < 2; ++r)
          for (int c = 0; c < 2; ++c) Ms[r + 3 * c] = Mt[4 * bm.mbase + (r + 2 * c) * bm.vstride + so];
        store_ghost_M(blk, Mt, e.b, nd, gi, gj, gk, Ms, err);
      }
    }
    return;
  }
  V3 N[8][2 * GW + 1];
  if (e.type == 101) {
    const NodeView& ns = nodes[e.bs];
    const int guides[6][3] = {{0, 0, 0}, {-1, 0, 0}, {0, 0, 0}, {0, -1, 0}, {0, 0, 0}, {0, 0, -1}};
    const int guides2[6][3] = {{1, 0, 0}, {-2, 0, 0}, {0, 1, 0}, {0, -2, 0}, {0, 0, 1}, {0, 0, -2}};
    switch (e.F) {
      case 1: N[0][0] = nv.at(Im - 1, Jm - 1, Km - 1); N[1][0] = nv.at(Im - 1, Jm - 1, Km);
              N[2][0] = nv.at(Im - 1, Jm, Km - 1); N[3][0] = nv.at(Im - 1, Jm, Km); break;
      case 2: N[4][0] = nv.at(Im, Jm - 1, Km - 1); N[5][0] = nv.at(Im, Jm - 1, Km);
              N[6][0] = nv.at(Im, Jm, Km - 1); N[7][0] = nv.at(Im, Jm, Km); break;
      case 3: N[0][0] = nv.at(Im - 1, Jm - 1, Km - 1); N[1][0] = nv.at(Im - 1, Jm - 1, Km);
              N[4][0] = nv.at(Im, Jm - 1, Km - 1); N[5][0] = nv.at(Im, Jm - 1, Km); break;
      case 4: N[2][0] = nv.at(Im - 1, Jm, Km - 1); N[3][0] = nv.at(Im - 1, Jm, Km);
              N[6][0] = nv.at(Im, Jm, Km - 1); N[7][0] = nv.at(Im, Jm, Km); break;
      case 5: N[0][0] = nv.at(Im - 1, Jm - 1, Km - 1); N[2][0] = nv.at(Im - 1, Jm, Km - 1);
              N[4][0] = nv.at(Im, Jm - 1, Km - 1); N[6][0] = nv.at(Im, Jm, Km - 1); break;
      case 6: N[1][0] = nv.at(Im - 1, Jm - 1, Km); N[3][0] = nv.at(Im - 1, Jm, Km);
              N[5][0] = nv.at(Im, Jm - 1, Km); N[7][0] = nv.at(Im, Jm, Km); break;
    }
    const int slotA[6] = {3, 7, 5, 7, 6, 7}, slotB[6] = {1, 5, 1, 3, 2, 3};
    const int slotC[6] = {2, 6, 4, 6, 4, 5}, slotD[6] = {0, 4, 0, 2, 0, 1};
    const int Fs = e.Fs;
    for (int g = 1; g <= GW; ++g) {
      int Is1 = e.Is + (GW - g) * guides[Fs - 1][0] + (g - 1) * guides2[Fs - 1][0];
      int Js1 = e.Js + (GW - g) * guides[Fs - 1][1] + (g - 1) * guides2[Fs - 1][1];
      int Ks1 = e.Ks + (GW - g) * guides[Fs - 1][2] + (g - 1) * guides2[Fs - 1][2];
      int II, JJ, KK;
      if (Fs <= 2) { II = Is1; JJ = (2 * Js1 + e.d11 + e.d21) / 2; KK = (2 * Ks1 + e.d12 + e.d22) / 2; }
      else if (Fs <= 4) { II = (2 * Is1 + e.d11 + e.d21) / 2; JJ = Js1; KK = (2 * Ks1 + e.d12 + e.d22) / 2; }
      else { II = (2 * Is1 + e.d11 + e.d21) / 2; JJ = (2 * Js1 + e.d12 + e.d22) / 2; KK = Ks1; }
      N[slotA[e.F - 1]][g] = ns.at(II, JJ, KK);
      int a1, a2, a3;
      if (Fs <= 2) { a1 = II; a2 = JJ - e.d11; a3 = KK - e.d12; }
      else if (Fs <= 4) { a1 = II - e.d11; a2 = JJ; a3 = KK - e.d12; }
      else { a1 = II - e.d11; a2 = JJ - e.d12; a3 = KK; }
      N[slotB[e.F - 1]][g] = ns.at(a1, a2, a3);
      if (Fs <= 2) { a1 = II; a2 = JJ - e.d21; a3 = KK - e.d22; }
      else if (Fs <= 4) { a1 = II - e.d21; a2 = JJ; a3 = KK - e.d22; }
      else { a1 = II - e.d21; a2 = JJ - e.d22; a3 = KK; }
      N[slotC[e.F - 1]][g] = ns.at(a1, a2, a3);
      if (Fs <= 2) { a1 = II; a2 = JJ - e.d11 - e.d21; a3 = KK - e.d12 - e.d22; }
      else if (Fs <= 4) { a1 = II - e.d11 - e.d21; a2 = JJ; a3 = KK - e.d12 - e.d22; }
      else { a1 = II - e.d11 - e.d21; a2 = JJ - e.d12 - e.d22; a3 = KK; }
      N[slotD[e.F - 1]][g] = ns.at(a1, a2, a3);
      int gi = Im, gj = Jm, gk = Km;
      switch (e.F) {
        case 1: ok &= metric_tensor(N[0][g], N[1][g], N[2][g], N[3][g], N[0][g - 1], N[1][g - 1], N[2][g - 1], N[3][g - 1], M, l, &v); gi = Im - g; break;
        case 2: ok &= metric_tensor(N[4][g - 1], N[5][g - 1], N[6][g - 1], N[7][g - 1], N[4][g], N[5][g], N[6][g], N[7][g], M, l, &v); gi = Im + g; break;
        case 3: ok &= metric_tensor(N[0][g], N[1][g], N[0][g - 1], N[1][g - 1], N[4][g], N[5][g], N[4][g - 1], N[5][g - 1], M, l, &v); gj = Jm - g; break;
        case 4: ok &= metric_tensor(N[2][g - 1], N[3][g - 1], N[2][g], N[3][g], N[6][g - 1], N[7][g - 1], N[6][g], N[7][g], M, l, &v); gj = Jm + g; break;
        case 5: ok &= metric_tensor(N[0][g], N[0][g - 1], N[2][g], N[2][g - 1], N[4][g], N[4][g - 1], N[6][g], N[6][g - 1], M, l, &v); gk = Km - g; break;
        case 6: ok &= metric_tensor(N[1][g - 1], N[1][g], N[3][g - 1], N[3][g], N[5][g - 1], N[5][g], N[7][g - 1], N[7][g], M, l, &v); gk = Km + g; break;
      }
      store_ghost_dl(blk, dl, e.b, nd, gi, gj, gk, dir, l[dir], err);
      if (g == 1) store_ghost_M(blk, Mt, e.b, nd, gi, gj, gk, M, err);
    }
  } else {
    // BC_Extrapolate_Metrics (delthe = 0 branches)
    auto at = [&](int slot, int g) -> V3& { return N[slot][g + GW]; };
    switch (e.F) {
      case 1:
        for (int g = 0; g <= GW; ++g) {
          at(0, g) = nv.at(Im + g - 1, Jm - 1, Km - 1); at(1, g) = nv.at(Im + g - 1, Jm - 1, Km);
          at(2, g) = nv.at(Im + g - 1, Jm, Km - 1); at(3, g) = nv.at(Im + g - 1, Jm, Km);
        }
        for (int g = -1; g >= -GW; --g) {
          for (int s = 0; s < 4; ++s) at(s, g) = v3lin3(at(s, g + 1), at(s, g + 2), at(s, g + 3));
          ok &= metric_tensor(at(0, g), at(1, g), at(2, g), at(3, g), at(0, g + 1), at(1, g + 1), at(2, g + 1), at(3, g + 1), M, l, &v);
          store_ghost_dl(blk, dl, e.b, nd, Im + g, Jm, Km, dir, l[dir], err);
          if (g == -1 || g == 1) store_ghost_M(blk, Mt, e.b, nd, Im + g, Jm, Km, M, err);
        }
        break;
      case 2:
        for (int g = 0; g >= -GW; --g) {
          at(4, g) = nv.at(Im + g, Jm - 1, Km - 1); at(5, g) = nv.at(Im + g, Jm - 1, Km);
          at(6, g) = nv.at(Im + g, Jm, Km - 1); at(7, g) = nv.at(Im + g, Jm, Km);
        }
        for (int g = 1; g <= GW; ++g) {
          for (int s = 4; s < 8; ++s) at(s, g) = v3lin3(at(s, g - 1), at(s, g - 2), at(s, g - 3));
          ok &= metric_tensor(at(4, g - 1), at(5, g - 1), at(6, g - 1), at(7, g - 1), at(4, g), at(5, g), at(6, g), at(7, g), M, l, &v);
          store_ghost_dl(blk, dl, e.b, nd, Im + g, Jm, Km, dir, l[dir], err);
          if (g == -1 || g == 1) store_ghost_M(blk, Mt, e.b, nd, Im + g, Jm, Km, M, err);
        }
        break;
      case 3: {
        bool cubic = bm.nj > 2;
        int gtop = cubic ? GW : 1;
        for (int g = 0; g <= gtop; ++g) {
          at(0, g) = nv.at(Im - 1, Jm + g - 1, Km - 1); at(1, g) = nv.at(Im - 1, Jm + g - 1, Km);
          at(4, g) = nv.at(Im, Jm + g - 1, Km - 1); at(5, g) = nv.at(Im, Jm + g - 1, Km);
        }
        for (int g = -1; g >= -GW; --g) {
          const int sl[4] = {0, 1, 4, 5};
          for (int s : sl) at(s, g) = cubic ? v3lin3(at(s, g + 1), at(s, g + 2), at(s, g + 3)) : v3lin2(at(s, g + 1), at(s, g + 2));
          ok &= metric_tensor(at(0, g), at(1, g), at(0, g + 1), at(1, g + 1), at(4, g), at(5, g), at(4, g + 1), at(5, g + 1), M, l, &v);
          store_ghost_dl(blk, dl, e.b, nd, Im, Jm + g, Km, dir, l[dir], err);
          if (g == -1 || g == 1) store_ghost_M(blk, Mt, e.b, nd, Im, Jm + g, Km, M, err);
        }
        break;
      }
      case 4: {
        bool cubic = bm.nj > 2;
        int gbot = cubic ? -GW : -1;
        for (int g = 0; g >= gbot; --g) {
          at(2, g) = nv.at(Im - 1, Jm + g, Km - 1); at(3, g) = nv.at(Im - 1, Jm + g, Km);
          at(6, g) = nv.at(Im, Jm + g, Km - 1); at(7, g) = nv.at(Im, Jm + g, Km);
        }
        for (int g = 1; g <= GW; ++g) {
          const int sl[4] = {2, 3, 6, 7};
          for (int s : sl) at(s, g) = cubic ? v3lin3(at(s, g - 1), at(s, g - 2), at(s, g - 3)) : v3lin2(at(s, g - 1), at(s, g - 2));
          ok &= metric_tensor(at(2, g - 1), at(3, g - 1), at(2, g), at(3, g), at(6, g - 1), at(7, g - 1), at(6, g), at(7, g), M, l, &v);
          store_ghost_dl(blk, dl, e.b, nd, Im, Jm + g, Km, dir, l[dir], err);
          if (g == -1 || g == 1) store_ghost_M(blk, Mt, e.b, nd, Im, Jm + g, Km, M, err);
        }
        break;
      }
      case 5: {
        bool cubic = (ndir == 3);
        int gtop = cubic ? GW : 1;
        for (int g = 0; g <= gtop; ++g) {
          at(0, g) = nv.at(Im - 1, Jm - 1, Km + g - 1); at(2, g) = nv.at(Im - 1, Jm, Km + g - 1);
          at(4, g) = nv.at(Im, Jm - 1, Km + g - 1); at(6, g) = nv.at(Im, Jm, Km + g - 1);
        }
        for (int g = -1; g >= -GW; --g) {
          const int sl[4] = {0, 2, 4, 6};
          for (int s : sl) at(s, g) = cubic ? v3lin3(at(s, g + 1), at(s, g + 2), at(s, g + 3)) : v3lin2(at(s, g + 1), at(s, g + 2));
          ok &= metric_tensor(at(0, g), at(0, g + 1), at(2, g), at(2, g + 1), at(4, g), at(4, g + 1), at(6, g), at(6, g + 1), M, l, &v);
          store_ghost_dl(blk, dl, e.b, nd, Im, Jm, Km + g, dir, l[dir], err);
          if (g == -1 || g == 1) store_ghost_M(blk, Mt, e.b, nd, Im, Jm, Km + g, M, err);
        }
        break;
      }
      case 6: {
        bool cubic = (ndir == 3);
        int gbot = cubic ? -GW : -1;
        for (int g = 0; g >= gbot; --g) {
          at(1, g) = nv.at(Im - 1, Jm - 1, Km + g); at(3, g) = nv.at(Im - 1, Jm, Km + g);
          at(5, g) = nv.at(Im, Jm - 1, Km + g); at(7, g) = nv.at(Im, Jm, Km + g);
        }
        for (int g = 1; g <= GW; ++g) {
          const int sl[4] = {1, 3, 5, 7};
          for (int s : sl) at(s, g) = cubic ? v3lin3(at(s, g - 1), at(s, g - 2), at(s, g - 3)) : v3lin2(at(s, g - 1), at(s, g - 2));
          ok &= metric_tensor(at(1, g - 1), at(1, g), at(3, g - 1), at(3, g), at(5, g - 1), at(5, g), at(7, g - 1), at(7, g), M, l, &v);
          store_ghost_dl(blk, dl, e.b, nd, Im, Jm, Km + g, dir, l[dir], err);
          if (g == -1 || g == 1) store_ghost_M(blk, Mt, e.b, nd, Im, Jm, Km + g, M, err);
        }
        break;
      }
    }
  }
  if (!ok) report(err, 6, e.b, Im - 1, Jm - 1, Km - 1);
}

// Uniformity check: flags[b] bit p set when plane p differs from its first
// valid value somewhere in its valid region.  tol = 0 asks for bitwise
// equality; tol > 0 accepts values within tol relative to the first one
// (last-bit differences of nodes placed by floating-point arithmetic).
__global__ void k_uniform_check(const BlockDesc* blk, int b, MetricArgs m, int nd, int ndir, int* flags,
                                double* firsts, double tol) {
  const BlockDesc& d = blk[b];
  auto ne = [tol](double a, double a0) -> bool {
    return tol == 0.0 ? (a != a0) : !(fabs(a - a0) <= tol * fabs(a0));
  };
  const long long vs = d.vstride, mb = d.mbase;
  // reference values: cell (0,0,0) metrics; faces of cell (0,0,0)
  long long o0 = (nd == 3) ? cell_off3(d, 0, 0, 0) : cell_off2(d, 0, 0);
  long long n = (long long)(d.ni + 4) * (d.nj + 4) * (nd == 3 ? d.nk + 4 : 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % (d.ni + 4)) - GW, j = (int)((q / (d.ni + 4)) % (d.nj + 4)) - GW;
    int k = (nd == 3) ? (int)(q / ((long long)(d.ni + 4) * (d.nj + 4))) - GW : 0;
    bool in_i = i >= 0 && i < d.ni, in_j = j >= 0 && j < d.nj, in_k = (nd == 2) || (k >= 0 && k < d.nk);
    long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    int f = 0;
    // dl along each active direction on that direction's ghosted line
    if (in_j && in_k && ne(m.dl[3 * mb + 0 * vs + o], m.dl[3 * mb + 0 * vs + o0])) f |= 1;
    if (in_i && in_k && ne(m.dl[3 * mb + 1 * vs + o], m.dl[3 * mb + 1 * vs + o0])) f |= 2;
    if (nd == 3 && in_i && in_j && ne(m.dl[3 * mb + 2 * vs + o], m.dl[3 * mb + 2 * vs + o0])) f |= 4;
    if (in_i && in_j && in_k) {
      if (ne(m.vol[mb + o], m.vol[mb + o0])) f |= 8;
      for (int p = 0; p < 3 * ndir; ++p)
        if (ne(m.vers[9 * mb + p * vs + o], m.vers[9 * mb + p * vs + o0])) f |= 16;
    }
    for (int dir = 0; dir < nd; ++dir) {
      bool in = (dir == 0 ? (i >= 0 && i <= d.ni) : in_i) && (dir == 1 ? (j >= 0 && j <= d.nj) : in_j) &&
                (nd == 2 || (dir == 2 ? (k >= 0 && k <= d.nk) : in_k));
      if (!in) continue;
      for (int p = 0; p < 4; ++p)
        if (ne(m.face[12 * mb + (4 * dir + p) * vs + o], m.face[12 * mb + (4 * dir + p) * vs + o0])) f |= 32 << dir;
    }
    if (f) atomicOr(&flags[b], f);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int h = 0; h < 3; ++h) firsts[h] = m.dl[3 * mb + h * vs + o0];
    for (int dir = 0; dir < 3; ++dir)
      for (int p = 0; p < 4; ++p) firsts[3 + 4 * dir + p] = (dir < nd) ? m.face[12 * mb + (4 * dir + p) * vs + o0] : 0.0;
    firsts[15] = m.vol[mb + o0];
    for (int p = 0; p < 9; ++p) firsts[16 + p] = (p < 3 * ndir) ? m.vers[9 * mb + p * vs + o0] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Fill_Ghost_Cell (Lib_Ghost.f90:11-137), one thread per boundary record.
// ---------------------------------------------------------------------------
template <int NV>
__global__ void k_fill_ghosts(const BlockDesc* blk, const GhostRec* recs, int nrec, double* P, MetricArgs m,
                              int nd, DevError* err) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nrec) return;
  const GhostRec e = recs[q];
  const BlockDesc& d = blk[e.b];
  const int dir = (e.f - 1) / 2;
  if (dir >= nd) return;
  const int gi = (e.f == 1) ? 1 : (e.f == 2) ? -1 : 0;   // guide(Fm,:) inward step
  const int gj = (e.f == 3) ? 1 : (e.f == 4) ? -1 : 0;
  const int gk = (e.f == 5) ? 1 : (e.f == 6) ? -1 : 0;
  double* Pb = P + d.sbase;
  const long long vs = d.vstride;
  // offset of a cell; self-check: -1 (and the access is skipped) for a cell
  // outside the ghosted extents of its block
  auto off = [&](const BlockDesc& bb, int i, int j, int k) -> long long {
    const bool in = i >= -GW && i < bb.ni + GW && j >= -GW && j < bb.nj + GW &&
                    (nd == 2 || (k >= -GW && k < bb.nk + GW));
    if (!in) {
      if (atomicCAS(&err->code, 0, 1) == 0) { err->b = -3; err->i = i; err->j = j; err->k = k; }
      return -1;
    }
    return (nd == 3) ? cell_off3(bb, i, j, k) : cell_off2(bb, i, j);
  };
  if (e.type == BC_CONN) {     // Ghost_Connection :140-160
    const BlockDesc& s = blk[e.bs];
    const int si = (e.fs == 1) ? 1 : (e.fs == 2) ? -1 : 0;
    const int sj = (e.fs == 3) ? 1 : (e.fs == 4) ? -1 : 0;
    const int sk = (e.fs == 5) ? 1 : (e.fs == 6) ? -1 : 0;
    const double* Ps = P + s.sbase;
    for (int g = 1; g <= GW; ++g) {
      long long od = off(d, e.i - gi * g, e.j - gj * g, e.k - gk * g);
      long long os = off(s, e.is + si * (g - 1), e.js + sj * (g - 1), e.ks + sk * (g - 1));
      if (od < 0 || os < 0) continue;
      for (int v = 0; v < NV; ++v) Pb[v * vs + od] = Ps[v * s.vstride + os];
    }
  } else if (e.type == BC_SYM) {  // Ghost_Symmetry :193-225 (first ghost only)
    long long ob = off(d, e.i, e.j, e.k);
    long long og = off(d, e.i - gi, e.j - gj, e.k - gk);
    // normal of the boundary face: low face of the boundary cell (odd faces)
    // or of the next cell (even faces)
    int fi = e.i + (e.f == 2), fj = e.j + (e.f == 4), fk = e.k + (e.f == 6);
    long long of = off(d, fi, fj, fk);
    if (ob < 0 || og < 0 || of < 0) return;
    const double* fp = m.face + 12 * d.mbase + (4 * dir) * vs + of;
    double n[3] = {fp[0], fp[vs], fp[2 * vs]};
    double q[NV];
    for (int v = 0; v < NV; ++v) q[v] = Pb[v * vs + ob];
    double udotn = ex::dot_vel<NV>(q, n);
    for (int c = 0; c < NV - 2; ++c) q[1 + c] = q[1 + c] - 2.0 * udotn * n[c];
    for (int v = 0; v < NV; ++v) Pb[v * vs + og] = q[v];
  } else if (e.type == BC_EXTRAP) {   // Ghost_Extrapolate :363-402
    for (int g = 1; g <= GW; ++g) {
      long long od = off(d, e.i - gi * g, e.j - gj * g, e.k - gk * g);
      long long oa = off(d, e.i - gi * (g - 1), e.j - gj * (g - 1), e.k - gk * (g - 1));
      long long oc = off(d, e.i - gi * (g - 2), e.j - gj * (g - 2), e.k - gk * (g - 2));
      long long oe = off(d, e.i - gi * (g - 3), e.j - gj * (g - 3), e.k - gk * (g - 3));
      if (od < 0 || oa < 0 || oc < 0 || oe < 0) continue;
      for (int v = 0; v < NV; ++v)
        Pb[v * vs + od] = 3.0 * Pb[v * vs + oa] - 3.0 * Pb[v * vs + oc] + Pb[v * vs + oe];
    }
  } else {                        // Ghost_ZG_Extrapolate :279-304 (0, 401-407, 420)
    long long ob = off(d, e.i, e.j, e.k);
    if (ob < 0) return;
    for (int g = 1; g <= GW; ++g) {
      long long od = off(d, e.i - gi * g, e.j - gj * g, e.k - gk * g);
      if (od < 0) continue;
      for (int v = 0; v < NV; ++v) Pb[v * vs + od] = Pb[v * vs + ob];
    }
  }
}

// ---------------------------------------------------------------------------
// Compute_dt (Mod_dt.f90:10-106): local dt and a global minimum.
// dtmin_bits holds the running minimum as the bit pattern of a positive double.
// ---------------------------------------------------------------------------
template <int NV, bool UNI>
__global__ void k_compute_dt(const BlockDesc* blk, int nblk, const double* P, MetricArgs m, double* dtl,
                             unsigned long long* dtmin_bits, Gas g, double cfl, int ndir, int nd, int iter,
                             int ramp_iter, int store_local, const int* iterp) {
  if (iterp) iter = *iterp + 1;   // the fused steps' device counter: completed steps + 1
  // blockIdx.y = block; CTAs stride over the block's cell rows (j, k), threads
  // over the cells of a row, so no per-cell index division
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  const int rows = d.nj * d.nk;
  const long long vs = d.vstride, mb = d.mbase;
  const double* Pb = P + d.sbase;
  double local_min = __longlong_as_double(0x7ff0000000000000LL);
  for (int row = blockIdx.x; row < rows; row += gridDim.x)
  for (int i = threadIdx.x; i < d.ni; i += blockDim.x) {
    const int j = row % d.nj, k = row / d.nj;
    long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    double Q[NV];
    for (int v = 0; v < NV; ++v) Q[v] = Pb[v * vs + o];
    double dtcell = cfl_dt<NV, UNI, false>(g, Q, d, m, o, ndir, cfl);
    if (g.model > 0) {
      // VNN condition (Mod_dt.f90:87-103), laminar: mi = 0 + mil
      const double mi = 0.0 + g.mu;
      for (int dd = 0; dd < ndir; ++dd) {
        double dlv;
        if constexpr (UNI) dlv = d.u_dl[dd]; else dlv = m.dl[3 * mb + dd * vs + o];
        const double dtv = (Q[0] * (dlv * dlv) * g.vnn) / mi;
        dtcell = fmin(dtv, dtcell);
      }
    }
    if (ramp_iter > 0 && iter < ramp_iter) dtcell = dtcell * (double)iter / (double)ramp_iter;
    if (store_local) dtl[mb + o] = dtcell;
    local_min = fmin(local_min, dtcell);
  }
  // warp + CTA min, one atomic per CTA
  for (int s = 16; s > 0; s >>= 1) local_min = fmin(local_min, __shfl_xor_sync(0xffffffffu, local_min, s));
  __shared__ double wmin[32];
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = local_min;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? wmin[threadIdx.x] : __longlong_as_double(0x7ff0000000000000LL);
    for (int s = 16; s > 0; s >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, s));
    if (threadIdx.x == 0) atomicMin(dtmin_bits, (unsigned long long)__double_as_longlong(v));
  }
}

// Set_Global_dt: every interior dtlocal = dtglobal (device scalar).
__global__ void k_set_global_dt(const BlockDesc* blk, double* dtl, const double* dtg, int nd) {
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  long long ncell = (long long)d.ni * d.nj * d.nk;
  double v = *dtg;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    dtl[d.mbase + o] = v;
  }
}

// Device-side step bookkeeping (no host round trip between steps).
//   begin: dtmin = dt_start ; finish: dtglobal = dtmin, time += dtglobal
__global__ void k_step_begin(unsigned long long* dtmin_bits, double dt_start, int* iter) {
  *dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
  if (iter) *iter = *iter + 1;
}
__global__ void k_step_dt_final(const unsigned long long* dtmin_bits, double* dtg, double* time, int advance_time) {
  double v = __longlong_as_double((long long)*dtmin_bits);
  *dtg = v;
  if (advance_time) *time = *time + v;
}
// The cell attaining a step's global dt (smallest flat index on ties), for
// the discrete adjoint.  Built here, with the reference arithmetic of the dt
// pass, so that the cell's dt equals the recorded dtglobal bit for bit.
template <bool UNI>
__global__ void k_dt_argmin(const BlockDesc* blk, int b, MetricArgs m, Gas g, const double* P, const double* dtg,
                            double cfl, int ndir, unsigned long long* arg) {
  const BlockDesc& d = blk[b];
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= d.ni || j >= d.nj) return;
  const long long o = cell_off2(d, i, j);
  double Q[4];
  for (int v = 0; v < 4; ++v) Q[v] = P[d.sbase + o + v * d.vstride];
  const double dt = cfl_dt<4, UNI, false>(g, Q, d, m, o, ndir, cfl);
  if (dt == *dtg) atomicMin(arg, ((unsigned long long)b << 40) | (unsigned long long)o);
}

// Fused-step bookkeeping: dtglobal = the running minimum (from the standalone
// pass, or from the previous step's last RK stage), time += dtglobal, then
// the minimum restarts from dt_start for this step's last stage.
__global__ void k_step_dt_take(unsigned long long* dtmin_bits, double* dtg, double* time, int advance_time,
                               double dt_start, int* iter) {
  const double v = __longlong_as_double((long long)*dtmin_bits);
  *dtg = v;
  if (advance_time) *time = *time + v;
  *dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
  if (iter) *iter = *iter + 1;
}

// ---------------------------------------------------------------------------
// RK_Newstate pointwise (phase path): P <- update(P, PO, R)
// ---------------------------------------------------------------------------
// Pout = RK stage of Pin (in place when Pout == Pin); dt from *dtg when
// given (time accurate), else the local dt plane.
template <int NV, bool UNI>
__global__ void k_rk_stage(const BlockDesc* blk, const double* P, const double* PO, const double* R, MetricArgs m,
                           const double* dtl, const double* dtg, double* Pout, Gas g, double c, int nd,
                           DevError* err) {
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  long long ncell = (long long)d.ni * d.nj * d.nk;
  const long long vs = d.vstride, mb = d.mbase;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    double Q[NV], QO[NV], Rv[NV];
    for (int v = 0; v < NV; ++v) {
      Q[v] = P[d.sbase + v * vs + o];
      QO[v] = PO[d.sbase + v * vs + o];
      Rv[v] = R[d.sbase + v * vs + o];
    }
    double vol;
    if constexpr (UNI) vol = d.u_vol; else vol = m.vol[mb + o];
    double dt = dtg ? *dtg : dtl[mb + o];
    bool ok = rk_update<NV>(g, Q, QO, Rv, vol, dt, c, false);
    if (!ok) report(err, 5, b, i, j, k);
    for (int v = 0; v < NV; ++v) Pout[d.sbase + v * vs + o] = Q[v];
  }
}

// ---------------------------------------------------------------------------
// Implicit residual smoothing (Newstate_Conservative with IRS,
// Lib_Newstate.f90:40-72, and Lib_IRS.f90), in the reference's arithmetic:
// scale R to the conservative increment, then per direction the first ghost
// layer of R and two Jacobi sweeps, then the RK stage on the smoothed
// increment.  NV = 4: 2-D blocks (ni x nj); NV = 5: 3-D (ni x nj x nk).
// ---------------------------------------------------------------------------
// Scale_Residual_Cons :98-103 (strangcoeff = 1): R = -(R / vol * dt); with
// integration-variables = prim, Compute_Prim_Residual (:255-302) of the
// stage's primitives P (Newstate_Primitive's IRS branch, :195-231)
template <int NV>
__global__ void k_irs_scale(const BlockDesc* blk, const double* P, double* R, MetricArgs m, const double* dtl,
                            const double* dtg, int use_dtg, Gas g) {
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  const long long ncell = (long long)d.ni * d.nj * (NV == 5 ? d.nk : 1), vs = d.vstride;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    const long long o = NV == 5 ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    const double vol = m.vol[d.mbase + o];
    const double dt = use_dtg ? *dtg : dtl[d.mbase + o];
    if (g.prim) {
      double Q[NV], Rv[NV];
      for (int v = 0; v < NV; ++v) { Q[v] = P[d.sbase + v * vs + o]; Rv[v] = R[d.sbase + v * vs + o]; }
      prim_residual<NV>(g, Q, Rv, vol, dt);
      for (int v = 0; v < NV; ++v) R[d.sbase + v * vs + o] = Rv[v];
      continue;
    }
    for (int v = 0; v < NV; ++v) {
      double* r = R + d.sbase + v * vs + o;
      *r = -(*r / vol * dt);
    }
  }
}
// Ghost_Residual_Extrapolation :130-187: 101 copies the source cell, every
// other record its own boundary cell (ghost and source cells are disjoint)
template <int NV>
__global__ void k_irs_ghost(const IrsCopy* list, int n, double* R) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const IrsCopy e = list[q];
  for (int v = 0; v < NV; ++v) R[e.dst + v * e.vsd] = R[e.src + v * e.vss];
}
// One Jacobi sweep along dir (Residual_Smoothing_Blk :64-80, the i, j and k
// loops alike): out = (R + beta (Rs(-1) + Rs(+1))) / (1 + 2 beta).  out may
// be R itself: each cell reads its own R before writing it, neighbours come
// from Rs.
template <int NV>
__global__ void k_irs_jacobi(const BlockDesc* blk, const double* R, const double* Rs, double* out, int dir,
                             double beta) {
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  const long long ncell = (long long)d.ni * d.nj * (NV == 5 ? d.nk : 1), vs = d.vstride;
  const long long step = dir == 0 ? 1 : dir == 1 ? d.px : d.plane;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    const long long o = d.sbase + (NV == 5 ? cell_off3(d, i, j, k) : cell_off2(d, i, j));
    for (int v = 0; v < NV; ++v) {
      const long long ov = o + v * vs;
      const double r = R[ov];
      out[ov] = (r + beta * (Rs[ov - step] + Rs[ov + step])) / (1.0 + 2.0 * beta);
    }
  }
}
// Update_State_Cons_IRS :106-131: RK_stage on the smoothed increment, then
// cons2prim and Check_And_Fix_State.  Pout may be Pin (the phase path).
template <int NV>
__global__ void k_irs_update(const BlockDesc* blk, const double* Pin, const double* PO, const double* R, double* Pout,
                             Gas g, double c, DevError* err) {
  constexpr int P = NV - 1;
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  const long long ncell = (long long)d.ni * d.nj * (NV == 5 ? d.nk : 1), vs = d.vstride;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    const long long o = d.sbase + (NV == 5 ? cell_off3(d, i, j, k) : cell_off2(d, i, j));
    double Q[NV], QO[NV], U[NV], U0[NV];
    for (int v = 0; v < NV; ++v) { Q[v] = Pin[o + v * vs]; QO[v] = PO[o + v * vs]; }
    if (g.prim) {   // Newstate_Primitive :218-226: RK_stage on the smoothed primitive increment
      double Rp[NV];
      for (int v = 0; v < NV; ++v) Rp[v] = R[o + v * vs];
      if (!rk_prim_stage<NV>(Q, QO, Rp, c)) report(err, 5, b, i, j, k);
      for (int v = 0; v < NV; ++v) Pout[o + v * vs] = Q[v];
      continue;
    }
    ex::prim2cons<NV>(g, QO, U0);
    ex::prim2cons<NV>(g, Q, U);
    for (int v = 0; v < NV; ++v) {
      const double r_ = (U[v] - U0[v] + R[o + v * vs]) * c;
      U[v] = U0[v] + r_;
    }
    ex::cons2prim<NV>(g, U, Q);
    bool bad = false;
    for (int v = 0; v < NV; ++v) bad |= isnan(Q[v]);
    bad |= (Q[P] < 0.0);
    if (bad) report(err, 5, b, i, j, k);
    if (Q[0] < 1e-20) Q[0] = 1e-20;
    for (int v = 0; v < NV; ++v) Pout[o + v * vs] = Q[v];
  }
}

// The shock detector of every cell of the 3-D blocks (Fluxes_blk's SD_Tramel
// pass, Mod_Fluxes.f90:78-85) into the beta plane arena, from the pressures
// of the cell and its six face neighbours (ghosts at the block edges).
__global__ void k_sd_beta3d(const BlockDesc* blk, const double* P, double* beta) {
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  const long long ncell = (long long)d.ni * d.nj * d.nk, vs = d.vstride;
  const double* p = P + d.sbase + 4 * vs;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    const long long o = cell_off3(d, i, j, k);
    beta[d.mbase + o] = ex::sd_tramel3(p[o], p[cell_off3(d, i - 1, j, k)], p[cell_off3(d, i + 1, j, k)],
                                       p[cell_off3(d, i, j - 1, k)], p[cell_off3(d, i, j + 1, k)],
                                       p[cell_off3(d, i, j, k - 1)], p[cell_off3(d, i, j, k + 1)]);
  }
}

// ---------------------------------------------------------------------------
// Compute_Residual (Mod_Diagnostic.f90:13-50): per-CTA partial sums of
// (|d rho|, |du|, |dv|, |dw|, |dp|)^2, reduced in a fixed order afterwards.
// ---------------------------------------------------------------------------
template <int NV>
__global__ void k_residual_norms(const BlockDesc* blk, const double* P, const double* PO, int nd,
                                 double* partial) {
  const int b = blockIdx.y;
  const BlockDesc& d = blk[b];
  long long ncell = (long long)d.ni * d.nj * d.nk;
  const long long vs = d.vstride;
  double acc[5] = {0, 0, 0, 0, 0};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    for (int v = 0; v < NV; ++v) {
      double r = fabs(P[d.sbase + v * vs + o] - PO[d.sbase + v * vs + o]);
      int slot = (NV == 4 && v == 3) ? 4 : v;     // 2-D: (rho,u,v,p) -> slots 0,1,2,4
      acc[slot] = acc[slot] + r * r;
    }
  }
  __shared__ double red[5][256];
  for (int s = 0; s < 5; ++s) red[s][threadIdx.x] = acc[s];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int s = 0; s < 5; ++s) red[s][threadIdx.x] = red[s][threadIdx.x] + red[s][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    long long slot = (long long)blockIdx.y * gridDim.x + blockIdx.x;
    for (int s = 0; s < 5; ++s) partial[5 * slot + s] = red[s][0];
  }
}

__global__ void k_sum_partials(const double* partial, int n, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t[5] = {0, 0, 0, 0, 0};
  for (int q = 0; q < n; ++q)
    for (int s = 0; s < 5; ++s) t[s] = t[s] + partial[5 * q + s];
  for (int s = 0; s < 5; ++s) out[s] = t[s];
}

// ---------------------------------------------------------------------------
// Layout conversion between the reference's AoS P(5, 1-gc:ni+gc, ...) and the
// device SoA planes.  ref: the transferred slab of one block's reference
// array -- the whole array in 3-D, the k = 1 plane in 2-D (the only plane the
// 2-D path reads or writes).
// ---------------------------------------------------------------------------
__global__ void k_ref_to_soa(const BlockDesc* blk, int b, const double* ref, double* dst, int nv, int nd) {
  const BlockDesc& d = blk[b];
  const int ex = d.ni + 4, ey = d.nj + 4, ez = (nd == 3) ? d.nk + 4 : 1;
  const long long n = (long long)ex * ey * ez;
  const long long vs = d.vstride;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int x = (int)(q % ex), y = (int)((q / ex) % ey), z = (int)(q / ((long long)ex * ey));
    const double* src = ref + 5 * q;
    long long o = (nd == 3) ? cell_off3(d, x - GW, y - GW, z - GW) : cell_off2(d, x - GW, y - GW);
    if (nv == 5) {
      for (int v = 0; v < 5; ++v) dst[d.sbase + v * vs + o] = src[v];
    } else {
      dst[d.sbase + 0 * vs + o] = src[0];
      dst[d.sbase + 1 * vs + o] = src[1];
      dst[d.sbase + 2 * vs + o] = src[2];
      dst[d.sbase + 3 * vs + o] = src[4];
    }
  }
}

// Writes the slab of the reference layout (see k_ref_to_soa); in 2-D the w
// slot is 0.
__global__ void k_soa_to_ref(const BlockDesc* blk, int b, const double* src, double* ref, int nv, int nd) {
  const BlockDesc& d = blk[b];
  const int ex = d.ni + 4, ey = d.nj + 4, ez = (nd == 3) ? d.nk + 4 : 1;
  const long long n = (long long)ex * ey * ez;
  const long long vs = d.vstride;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int x = (int)(q % ex), y = (int)((q / ex) % ey), z = (int)(q / ((long long)ex * ey));
    double* out = ref + 5 * q;
    if (nd == 3) {
      long long o = cell_off3(d, x - GW, y - GW, z - GW);
      for (int v = 0; v < 5; ++v) out[v] = src[d.sbase + v * vs + o];
    } else {
      long long o = cell_off2(d, x - GW, y - GW);
      out[0] = src[d.sbase + 0 * vs + o];
      out[1] = src[d.sbase + 1 * vs + o];
      out[2] = src[d.sbase + 2 * vs + o];
      out[3] = 0.0;
      out[4] = src[d.sbase + 3 * vs + o];
    }
  }
}

// one-plane quantity (dtlocal, interior only) <-> reference (1:ni,1:nj,1:nk)
__global__ void k_plane_io(const BlockDesc* blk, int b, double* plane_arena, double* ref, int nd, int to_ref) {
  const BlockDesc& d = blk[b];
  long long n = (long long)d.ni * d.nj * d.nk;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % d.ni), j = (int)((q / d.ni) % d.nj), k = (int)(q / ((long long)d.ni * d.nj));
    long long o = (nd == 3) ? cell_off3(d, i, j, k) : cell_off2(d, i, j);
    if (to_ref) ref[q] = plane_arena[d.mbase + o];
    else plane_arena[d.mbase + o] = ref[q];
  }
}

// metrics of one block -> reference-shaped vol(ghosted) and dl(3, ghosted)
__global__ void k_metrics_to_ref(const BlockDesc* blk, int b, MetricArgs m, double* vol, double* dl, int nd) {
  const BlockDesc& d = blk[b];
  const int ex = d.ni + 4, ey = d.nj + 4, ez = d.nk + 4;
  long long n = (long long)ex * ey * ez;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int x = (int)(q % ex), y = (int)((q / ex) % ey), z = (int)(q / ((long long)ex * ey));
    if (nd == 2 && z != GW) continue;
    long long o = (nd == 3) ? cell_off3(d, x - GW, y - GW, z - GW) : cell_off2(d, x - GW, y - GW);
    if (vol) vol[q] = m.vol[d.mbase + o];
    if (dl)
      for (int h = 0; h < 3; ++h) dl[3 * q + h] = m.dl[3 * d.mbase + h * d.vstride + o];
  }
}

__global__ void k_faces_to_ref(const BlockDesc* blk, int b, MetricArgs m, int dir, double* N, double* A, int nd) {
  const BlockDesc& d = blk[b];
  int ei = d.ni + (dir == 0), ej = d.nj + (dir == 1), ek = d.nk + (dir == 2);
  long long n = (long long)ei * ej * ek;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % ei), j = (int)((q / ei) % ej), k = (int)(q / ((long long)ei * ej));
    int ci = (dir == 0) ? i : i, cj = (dir == 1) ? j : j, ck = (dir == 2) ? k : k;
    if (nd == 2 && dir == 2) continue;
    long long o = (nd == 3) ? cell_off3(d, ci, cj, ck) : cell_off2(d, ci, cj);
    const double* f = m.face + 12 * d.mbase + (4 * dir) * d.vstride + o;
    if (N) { N[3 * q] = f[0]; N[3 * q + 1] = f[d.vstride]; N[3 * q + 2] = f[2 * d.vstride]; }
    if (A) A[q] = f[3 * d.vstride];
  }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static inline int grid_for(long long n, int threads, int cap = 148 * 16) {
  long long g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

void launch_cell_metrics(const BlockDesc* dblk, int b, long long ncell, NodeView nv, MetricArgs m, int nd,
                         int ndir, DevError* err, cudaStream_t s) {
  k_cell_metrics<<<grid_for(ncell, 256), 256, 0, s>>>(dblk, b, nv, const_cast<double*>(m.dl),
                                                       const_cast<double*>(m.vol), const_cast<double*>(m.vers),
                                                       const_cast<double*>(m.Mt), nd, ndir, err);
}
void launch_face_metrics(const BlockDesc* dblk, int b, long long nface, NodeView nv, MetricArgs m, int nd,
                         int dir, cudaStream_t s) {
  k_face_metrics<<<grid_for(nface, 256), 256, 0, s>>>(dblk, b, nv, const_cast<double*>(m.face), nd, dir);
}
void launch_ghost_metrics(const BlockDesc* dblk, const void* recs, int nrec, const NodeView* nodes, MetricArgs m,
                          int nd, int ndir, DevError* err, cudaStream_t s) {
  if (nrec == 0) return;
  k_ghost_metrics<<<(nrec + 127) / 128, 128, 0, s>>>(dblk, (const GhostMetricRec*)recs, nrec, nodes,
                                                     const_cast<double*>(m.dl), const_cast<double*>(m.Mt), nd, ndir,
                                                     err);
}
void launch_metrics_from_ref(const BlockDesc* dblk, int b, const int* dims, const double* src, MetricArgs m, int nd,
                             int ndir, cudaStream_t s) {
  const int ni = dims[0], nj = dims[1], nk = dims[2];
  const long long ncell = (long long)(ni + 4) * (nj + 4) * (nd == 3 ? nk + 4 : 1);
  k_metrics_from_ref<<<grid_for(ncell, 256), 256, 0, s>>>(dblk, b, src, const_cast<double*>(m.dl),
                                                           const_cast<double*>(m.vol), const_cast<double*>(m.vers),
                                                           const_cast<double*>(m.Mt), nd, ndir);
  const long long NG = (long long)(ni + 4) * (nj + 4) * (nk + 4);
  const double* f = src + 13 * NG;
  for (int dir = 0; dir < 3; ++dir) {
    const long long nf = (long long)(ni + (dir == 0)) * (nj + (dir == 1)) * (nk + (dir == 2));
    if (dir < nd)
      k_faces_from_ref<<<grid_for(nf, 256), 256, 0, s>>>(dblk, b, f, const_cast<double*>(m.face), nd, dir);
    f += 4 * nf;
  }
}
void launch_uniform_check(const BlockDesc* dblk, int b, long long ncell, MetricArgs m, int nd, int ndir,
                          int* flags, double* firsts, double tol, cudaStream_t s) {
  k_uniform_check<<<grid_for(ncell, 256), 256, 0, s>>>(dblk, b, m, nd, ndir, flags, firsts, tol);
}
void launch_fill_ghosts(const BlockDesc* dblk, const GhostRec* recs, int nrec, double* P, MetricArgs m, int nd,
                        DevError* err, cudaStream_t s) {
  if (nrec == 0) return;
  if (nd == 3) k_fill_ghosts<5><<<(nrec + 127) / 128, 128, 0, s>>>(dblk, recs, nrec, P, m, nd, err);
  else k_fill_ghosts<4><<<(nrec + 127) / 128, 128, 0, s>>>(dblk, recs, nrec, P, m, nd, err);
}
void launch_compute_dt(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, MetricArgs m,
                       double* dtl, unsigned long long* dtmin_bits, Gas g, double cfl, int ndir, int nd, int iter,
                       int ramp_iter, int store_local, bool uniform, cudaStream_t s, const int* iterp) {
  // one CTA per cell row (rows <= cells), at most 16 per SM
  dim3 grid((unsigned)std::min<long long>(maxcell, 148 * 16), nblk);
  if (nd == 3) {
    if (uniform) k_compute_dt<5, true><<<grid, 256, 0, s>>>(dblk, nblk, P, m, dtl, dtmin_bits, g, cfl, ndir, nd, iter, ramp_iter, store_local, iterp);
    else k_compute_dt<5, false><<<grid, 256, 0, s>>>(dblk, nblk, P, m, dtl, dtmin_bits, g, cfl, ndir, nd, iter, ramp_iter, store_local, iterp);
  } else {
    if (uniform) k_compute_dt<4, true><<<grid, 256, 0, s>>>(dblk, nblk, P, m, dtl, dtmin_bits, g, cfl, ndir, nd, iter, ramp_iter, store_local, iterp);
    else k_compute_dt<4, false><<<grid, 256, 0, s>>>(dblk, nblk, P, m, dtl, dtmin_bits, g, cfl, ndir, nd, iter, ramp_iter, store_local, iterp);
  }
}
void launch_set_global_dt(const BlockDesc* dblk, int nblk, long long maxcell, double* dtl, const double* dtg, int nd,
                          cudaStream_t s) {
  dim3 grid(grid_for(maxcell, 256, 148 * 8), nblk);
  k_set_global_dt<<<grid, 256, 0, s>>>(dblk, dtl, dtg, nd);
}
void launch_step_begin(unsigned long long* dtmin_bits, double dt_start, int* iter, cudaStream_t s) {
  k_step_begin<<<1, 1, 0, s>>>(dtmin_bits, dt_start, iter);
}
void launch_step_dt_final(const unsigned long long* dtmin_bits, double* dtg, double* time, int advance_time,
                          cudaStream_t s) {
  k_step_dt_final<<<1, 1, 0, s>>>(dtmin_bits, dtg, time, advance_time);
}
void launch_dt_argmin(const BlockDesc* dblk, int b, int ni, int nj, MetricArgs m, Gas g, const double* P,
                      const double* dtg, double cfl, int ndir, bool uniform, unsigned long long* arg, cudaStream_t s) {
  const dim3 grid((ni + 127) / 128, nj);
  if (uniform) k_dt_argmin<true><<<grid, 128, 0, s>>>(dblk, b, m, g, P, dtg, cfl, ndir, arg);
  else k_dt_argmin<false><<<grid, 128, 0, s>>>(dblk, b, m, g, P, dtg, cfl, ndir, arg);
}
void launch_step_dt_take(unsigned long long* dtmin_bits, double* dtg, double* time, int advance_time, double dt_start,
                         int* iter, cudaStream_t s) {
  k_step_dt_take<<<1, 1, 0, s>>>(dtmin_bits, dtg, time, advance_time, dt_start, iter);
}
void launch_rk_stage(const BlockDesc* dblk, int nblk, long long maxcell, double* P, const double* PO, const double* R,
                     MetricArgs m, const double* dtl, Gas g, double c, int nd, bool uniform, DevError* err,
                     cudaStream_t s) {
  launch_rk_stage_to(dblk, nblk, maxcell, P, PO, R, m, dtl, nullptr, P, g, c, nd, uniform, err, s);
}
void launch_rk_stage_to(const BlockDesc* dblk, int nblk, long long maxcell, const double* Pin, const double* PO,
                        const double* R, MetricArgs m, const double* dtl, const double* dtg, double* Pout, Gas g,
                        double c, int nd, bool uniform, DevError* err, cudaStream_t s) {
  dim3 grid(grid_for(maxcell, 256, 148 * 8), nblk);
  if (nd == 3) {
    if (uniform) k_rk_stage<5, true><<<grid, 256, 0, s>>>(dblk, Pin, PO, R, m, dtl, dtg, Pout, g, c, nd, err);
    else k_rk_stage<5, false><<<grid, 256, 0, s>>>(dblk, Pin, PO, R, m, dtl, dtg, Pout, g, c, nd, err);
  } else {
    if (uniform) k_rk_stage<4, true><<<grid, 256, 0, s>>>(dblk, Pin, PO, R, m, dtl, dtg, Pout, g, c, nd, err);
    else k_rk_stage<4, false><<<grid, 256, 0, s>>>(dblk, Pin, PO, R, m, dtl, dtg, Pout, g, c, nd, err);
  }
}
void launch_irs_scale(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, double* R, MetricArgs m,
                      const double* dtl, const double* dtg, int use_dtg, Gas g, int nd, cudaStream_t s) {
  dim3 grid(grid_for(maxcell, 256, 148 * 4), nblk);
  if (nd == 3) k_irs_scale<5><<<grid, 256, 0, s>>>(dblk, P, R, m, dtl, dtg, use_dtg, g);
  else k_irs_scale<4><<<grid, 256, 0, s>>>(dblk, P, R, m, dtl, dtg, use_dtg, g);
}
void launch_irs_ghost(const IrsCopy* list, int n, double* R, int nd, cudaStream_t s) {
  if (n <= 0) return;
  if (nd == 3) k_irs_ghost<5><<<(n + 255) / 256, 256, 0, s>>>(list, n, R);
  else k_irs_ghost<4><<<(n + 255) / 256, 256, 0, s>>>(list, n, R);
}
void launch_irs_jacobi(const BlockDesc* dblk, int nblk, long long maxcell, const double* R, const double* Rs,
                       double* out, int dir, double beta, int nd, cudaStream_t s) {
  dim3 grid(grid_for(maxcell, 256, 148 * 4), nblk);
  if (nd == 3) k_irs_jacobi<5><<<grid, 256, 0, s>>>(dblk, R, Rs, out, dir, beta);
  else k_irs_jacobi<4><<<grid, 256, 0, s>>>(dblk, R, Rs, out, dir, beta);
}
void launch_irs_update(const BlockDesc* dblk, int nblk, long long maxcell, const double* Pin, const double* PO,
                       const double* R, double* Pout, Gas g, double c, DevError* err, int nd, cudaStream_t s) {
  dim3 grid(grid_for(maxcell, 256, 148 * 4), nblk);
  if (nd == 3) k_irs_update<5><<<grid, 256, 0, s>>>(dblk, Pin, PO, R, Pout, g, c, err);
  else k_irs_update<4><<<grid, 256, 0, s>>>(dblk, Pin, PO, R, Pout, g, c, err);
}
void launch_sd_beta3d(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, double* beta,
                      cudaStream_t s) {
  dim3 grid(grid_for(maxcell, 256, 148 * 4), nblk);
  k_sd_beta3d<<<grid, 256, 0, s>>>(dblk, P, beta);
}
int norms_partial_count(int nblk, long long maxcell) { return grid_for(maxcell, 256, 148 * 4) * nblk; }
void launch_residual_norms(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, const double* PO,
                           int nd, double* partial, double* out, cudaStream_t s) {
  dim3 grid(grid_for(maxcell, 256, 148 * 4), nblk);
  if (nd == 3) k_residual_norms<5><<<grid, 256, 0, s>>>(dblk, P, PO, nd, partial);
  else k_residual_norms<4><<<grid, 256, 0, s>>>(dblk, P, PO, nd, partial);
  k_sum_partials<<<1, 1, 0, s>>>(partial, grid.x * grid.y, out);
}
void launch_ref_to_soa(const BlockDesc* dblk, int b, long long n, const double* ref, double* dst, int nv, int nd,
                       cudaStream_t s) {
  k_ref_to_soa<<<grid_for(n, 256), 256, 0, s>>>(dblk, b, ref, dst, nv, nd);
}
void launch_soa_to_ref(const BlockDesc* dblk, int b, long long n, const double* src, double* ref, int nv, int nd,
                       cudaStream_t s) {
  k_soa_to_ref<<<grid_for(n, 256), 256, 0, s>>>(dblk, b, src, ref, nv, nd);
}
void launch_plane_io(const BlockDesc* dblk, int b, long long n, double* arena, double* ref, int nd, int to_ref,
                     cudaStream_t s) {
  k_plane_io<<<grid_for(n, 256), 256, 0, s>>>(dblk, b, arena, ref, nd, to_ref);
}
void launch_metrics_to_ref(const BlockDesc* dblk, int b, long long n, MetricArgs m, double* vol, double* dl, int nd,
                           cudaStream_t s) {
  k_metrics_to_ref<<<grid_for(n, 256), 256, 0, s>>>(dblk, b, m, vol, dl, nd);
}
void launch_faces_to_ref(const BlockDesc* dblk, int b, long long n, MetricArgs m, int dir, double* N, double* A,
                         int nd, cudaStream_t s) {
  k_faces_to_ref<<<grid_for(n, 256), 256, 0, s>>>(dblk, b, m, dir, N, A, nd);
}

}  // namespace mose

namespace mose {

// ---- 402 inlets: p0 from the time table (Series_Data_m.f90:55-86) -----------------
// Linear interpolation at the device time; a periodic table first wraps the
// time into [t_1, t_n) (Fortran MODULO of reals: fmod, plus the period where
// the signs differ).  Before t_1 the reference's value is undefined; here it
// is v_1.  Runs in this --fmad=false unit: the same roundings as the host.
__global__ void k_series_p0(const SeriesRec* recs, int n, const double* tv, const double* time, BcParam* bcp) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const SeriesRec r = recs[q];
  const double* T = tv + 2 * (long long)r.off;   // (t, v) pairs
  double t_ = *time;
  if (r.periodic) {
    const double period = T[2 * (r.n - 1)] - T[0];
    if (period > 0.0) {
      double m = fmod(t_ - T[0], period);
      if (m != 0.0 && ((m < 0.0) != (period < 0.0))) m = m + period;
      t_ = T[0] + m;
    }
  }
  double out = T[1];
  if (t_ == T[0]) {
    out = T[1];
  } else {
    bool found = false;
    for (int i = 1; i < r.n && !found; ++i) {
      const double t0 = T[2 * (i - 1)], t1 = T[2 * i];
      if (t_ > t0 && t_ <= t1) {
        const double v0 = T[2 * (i - 1) + 1], v1 = T[2 * i + 1];
        out = (v1 - v0) / (t1 - t0) * (t_ - t0) + v0;
        found = true;
      }
    }
    if (!found && t_ > T[2 * (r.n - 1)]) out = T[2 * (r.n - 1) + 1];
  }
  bcp[r.pidx].p = out;
}

void launch_series_p0(const SeriesRec* recs, int n, const double* tv, const double* time, BcParam* bcp,
                      cudaStream_t s) {
  if (n <= 0) return;
  k_series_p0<<<(n + 127) / 128, 128, 0, s>>>(recs, n, tv, time, bcp);
}
}  // namespace mose
