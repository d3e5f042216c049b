// metrics.cuh -- setup-time geometry on the device (Lib_Metrics.f90).
// Compiled into the --fmad=false translation unit so the metrics are
// bit-identical to the reference's FP64 algorithm.
#pragma once

#include "common.cuh"

namespace mose {

struct V3 { double c[3]; };

__device__ __forceinline__ V3 v3sub(const V3& a, const V3& b) {
  return V3{{a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]}};
}
__device__ __forceinline__ V3 v3lin3(const V3& a, const V3& b, const V3& c) {   // 3a - 3b + c
  V3 r;
  for (int q = 0; q < 3; ++q) r.c[q] = 3.0 * a.c[q] - 3.0 * b.c[q] + c.c[q];
  return r;
}
__device__ __forceinline__ V3 v3lin2(const V3& a, const V3& b) {                 // 2a - b
  V3 r;
  for (int q = 0; q < 3; ++q) r.c[q] = 2.0 * a.c[q] - b.c[q];
  return r;
}

// Node array of one block: Fortran node(3, 0:ni, 0:nj, 0:nk).
struct NodeView {
  const double* p;
  int ni, nj, nk;
  DevError* err;   // bounds self-check: an index outside 0..n is recorded here and clamped
  __device__ __forceinline__ V3 at(int i, int j, int k) const {
    if (i < 0 || i > ni || j < 0 || j > nj || k < 0 || k > nk) {
      if (err && atomicCAS(&err->code, 0, 1) == 0) { err->b = -1; err->i = i; err->j = j; err->k = k; }
      i = i < 0 ? 0 : (i > ni ? ni : i);
      j = j < 0 ? 0 : (j > nj ? nj : j);
      k = k < 0 ? 0 : (k > nk ? nk : k);
    }
    const double* q = p + 3 * ((long long)i + (long long)(ni + 1) * ((long long)j + (long long)(nj + 1) * k));
    return V3{{q[0], q[1], q[2]}};
  }
};

__device__ __forceinline__ double tvol(const double* vx, const double* vy, const double* vz, int i1, int i2,
                                       int i3, int i4) {
  --i1; --i2; --i3; --i4;
  return fabs(((vx[i2] - vx[i1]) * ((vy[i3] - vy[i1]) * (vz[i4] - vz[i1]) - (vy[i4] - vy[i1]) * (vz[i3] - vz[i1])) +
               (vy[i2] - vy[i1]) * ((vx[i4] - vx[i1]) * (vz[i3] - vz[i1]) - (vx[i3] - vx[i1]) * (vz[i4] - vz[i1])) +
               (vz[i2] - vz[i1]) * ((vx[i3] - vx[i1]) * (vy[i4] - vy[i1]) - (vx[i4] - vx[i1]) * (vy[i3] - vy[i1]))) /
              6.0);
}

// Compute_Metric_Tensor, Lib_Metrics.f90:250-376.  M is c(3,3) column-major.
__device__ __forceinline__ bool metric_tensor(const V3& N1, const V3& N2, const V3& N3, const V3& N4,
                                              const V3& N5, const V3& N6, const V3& N7, const V3& N8,
                                              double* M, double* dl, double* vol) {
  double A[3][3];
  for (int c = 0; c < 3; ++c) {
    A[0][c] = N5.c[c] - N1.c[c] + N6.c[c] - N2.c[c] + N7.c[c] - N3.c[c] + N8.c[c] - N4.c[c];
    A[1][c] = N3.c[c] - N1.c[c] + N4.c[c] - N2.c[c] + N7.c[c] - N5.c[c] + N8.c[c] - N6.c[c];
    A[2][c] = N2.c[c] - N1.c[c] + N4.c[c] - N3.c[c] + N6.c[c] - N5.c[c] + N8.c[c] - N7.c[c];
  }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[r][c] = 0.25 * A[r][c];
  double det = A[0][0] * A[1][1] * A[2][2] - A[0][0] * A[1][2] * A[2][1] - A[0][1] * A[1][0] * A[2][2] +
               A[0][1] * A[1][2] * A[2][0] + A[0][2] * A[1][0] * A[2][1] - A[0][2] * A[1][1] * A[2][0];
  bool ok = true;
  if (fabs(det) == 0.0) {
    ok = false;
    for (int q = 0; q < 9; ++q) M[q] = 0.0;
    M[0] = M[4] = M[8] = 1.0;
  } else {
    double cof[3][3];
    cof[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]);
    cof[0][1] = -(A[1][0] * A[2][2] - A[1][2] * A[2][0]);
    cof[0][2] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    cof[1][0] = -(A[0][1] * A[2][2] - A[0][2] * A[2][1]);
    cof[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]);
    cof[1][2] = -(A[0][0] * A[2][1] - A[0][1] * A[2][0]);
    cof[2][0] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]);
    cof[2][1] = -(A[0][0] * A[1][2] - A[0][2] * A[1][0]);
    cof[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) M[r + 3 * c] = cof[r][c] / det;
  }
  for (int h = 0; h < 3; ++h) dl[h] = sqrt(A[h][0] * A[h][0] + A[h][1] * A[h][1] + A[h][2] * A[h][2]);
  double vx[8], vy[8], vz[8];
  const V3* ord[8] = {&N1, &N5, &N3, &N7, &N2, &N6, &N4, &N8};
  for (int q = 0; q < 8; ++q) { vx[q] = ord[q]->c[0]; vy[q] = ord[q]->c[1]; vz[q] = ord[q]->c[2]; }
  double v = tvol(vx, vy, vz, 1, 2, 3, 5) + tvol(vx, vy, vz, 2, 4, 3, 8) + tvol(vx, vy, vz, 5, 8, 6, 2) +
             tvol(vx, vy, vz, 5, 7, 8, 3) + tvol(vx, vy, vz, 5, 8, 2, 3);
  *vol = v;
  if (v <= 0.0) ok = false;
  return ok;
}

__device__ __forceinline__ void cross3(const V3& d1, const V3& d2, double* d3) {
  d3[0] = (d1.c[1] * d2.c[2] - d1.c[2] * d2.c[1]);
  d3[1] = (d1.c[2] * d2.c[0] - d1.c[0] * d2.c[2]);
  d3[2] = (d1.c[0] * d2.c[1] - d1.c[1] * d2.c[0]);
}
__device__ __forceinline__ V3 avg4(const V3& a, const V3& b, const V3& c, const V3& d) {
  V3 r;
  for (int q = 0; q < 3; ++q) r.c[q] = 0.25 * (a.c[q] + b.c[q] + c.c[q] + d.c[q]);
  return r;
}

// Orientation signs of Compute_Norm_Area, Lib_Metrics.f90:84-153.
__device__ __forceinline__ void face_signs(const NodeView& nv, double* s) {
  double sn[3];
  cross3(v3sub(nv.at(1, 1, 1), nv.at(1, 0, 0)), v3sub(nv.at(1, 0, 1), nv.at(1, 1, 0)), sn);
  V3 d = v3sub(avg4(nv.at(1, 1, 1), nv.at(1, 0, 1), nv.at(1, 0, 0), nv.at(1, 1, 0)),
               avg4(nv.at(0, 1, 1), nv.at(0, 0, 1), nv.at(0, 0, 0), nv.at(0, 1, 0)));
  s[0] = copysign(1.0, d.c[0] * sn[0] + d.c[1] * sn[1] + d.c[2] * sn[2]);
  cross3(v3sub(nv.at(0, 1, 1), nv.at(1, 1, 0)), v3sub(nv.at(1, 1, 1), nv.at(0, 1, 0)), sn);
  d = v3sub(avg4(nv.at(1, 1, 1), nv.at(0, 1, 1), nv.at(0, 1, 0), nv.at(1, 1, 0)),
            avg4(nv.at(1, 0, 1), nv.at(0, 0, 1), nv.at(0, 0, 0), nv.at(1, 0, 0)));
  s[1] = copysign(1.0, d.c[0] * sn[0] + d.c[1] * sn[1] + d.c[2] * sn[2]);
  cross3(v3sub(nv.at(0, 1, 1), nv.at(1, 0, 1)), v3sub(nv.at(0, 0, 1), nv.at(1, 1, 1)), sn);
  d = v3sub(avg4(nv.at(1, 1, 1), nv.at(0, 1, 1), nv.at(0, 0, 1), nv.at(1, 0, 1)),
            avg4(nv.at(1, 1, 0), nv.at(0, 1, 0), nv.at(0, 0, 0), nv.at(1, 0, 0)));
  s[2] = copysign(1.0, d.c[0] * sn[0] + d.c[1] * sn[1] + d.c[2] * sn[2]);
}

// Normal and area of one face (Compute_Norm_Area loops :159-244).  dir 0/1/2;
// (i, j, k) are the reference's face indices of dir(d)%f.
__device__ __forceinline__ void face_metric(const NodeView& nv, int dir, int i, int j, int k, double sgn,
                                            double* n, double* A) {
  double d3[3];
  if (dir == 0) cross3(v3sub(nv.at(i, j, k), nv.at(i, j - 1, k - 1)), v3sub(nv.at(i, j - 1, k), nv.at(i, j, k - 1)), d3);
  else if (dir == 1) cross3(v3sub(nv.at(i - 1, j, k), nv.at(i, j, k - 1)), v3sub(nv.at(i, j, k), nv.at(i - 1, j, k - 1)), d3);
  else cross3(v3sub(nv.at(i - 1, j, k), nv.at(i, j - 1, k)), v3sub(nv.at(i - 1, j - 1, k), nv.at(i, j, k)), d3);
  for (int q = 0; q < 3; ++q) d3[q] = d3[q] * 0.5;
  double a = sqrt(d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2]);
  if (a == 0.0) { n[0] = n[1] = n[2] = 0.0; }
  else for (int q = 0; q < 3; ++q) n[q] = d3[q] / a * sgn;
  *A = a;
}

}  // namespace mose
