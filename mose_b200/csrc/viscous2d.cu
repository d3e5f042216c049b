// viscous2d.cu -- the Navier-Stokes residual of 2-D blocks (model = 1,
// laminar, one species, constant transport properties) in the reference's
// operation order, compiled with --fmad=false like every reference-exact
// unit, so it matches the oracle bit for bit.
//
// Two launches per residual.  k_visc_faces2d forms every interior face's
// convective (4 values) and diffusive (3 values) flux once, one thread per
// cell for its i+1/2 and j+1/2 faces, into the viscous face arena.  Then one
// thread per cell forms the cell's whole residual, in the order the reference
// accumulates it (Mod_Fluxes.f90:86-206, then BC_Fluxes by block and face,
// Mod_BC_Fluxes.f90:52-216):
//   convective i-faces (i-1/2, i+1/2), diffusive i-faces, convective j-faces,
//   diffusive j-faces (from the arena), then the block-edge faces in face
//   order 1..4, each with its Euler flux followed by its viscous one (101/201:
//   BC_Connection_Eul + BC_Connection_Visc; 300: symmetry + BC_Symmetry_Visc;
//   301: symmetry + BC_Wall_Heat; 302: symmetry + BC_Wall_Temperature; the
//   others inviscid).
//
// 2-D specialisation of Lib_Diffusive.f90: the out-of-plane gradients are
// exact zeros in the reference (its k ghost planes are zero-gradient copies,
// w = 0, n_z = 0 and M(1:2,3) = M(3,1:2) = 0 on planar meshes), so every
// term they contribute is an exact zero and is left out; so are the species
// diffusion and its enthalpy flux, which multiply the exactly zero gradient
// of rho_1 / rho = 1.
#include <cuda_runtime.h>

#include "kernels.h"
#include "stage2d.cuh"

namespace mose {
namespace {

constexpr int NV = 4;   // rho, u, v, p

struct Cell2 {
  const BlockDesc& d;
  const StageArgs& a;
  const double* P;
  __device__ long long off(int i, int j) const { return cell_off2(d, i, j); }
  __device__ void q(int i, int j, double* out) const {
    const long long o = off(i, j);
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = P[v * d.vstride + o];
  }
  __device__ double dl(int dir, int i, int j) const { return a.m.dl[3 * d.mbase + dir * d.vstride + off(i, j)]; }
  // normal and area of the low face of cell (i, j) along dir
  __device__ double face(int dir, int i, int j, double* n) const {
    const double* f = a.m.face + 12 * d.mbase + (4 * dir) * d.vstride + off(i, j);
    n[0] = f[0]; n[1] = f[d.vstride]; n[2] = f[2 * d.vstride];
    return f[3 * d.vstride];
  }
  // metric tensor entries M(1,1), M(2,1), M(1,2), M(2,2)
  __device__ void M(int i, int j, double* m) const {
    const long long o = off(i, j);
#pragma unroll
    for (int q = 0; q < 4; ++q) m[q] = a.m.Mt[4 * d.mbase + q * d.vstride + o];
  }
};

// visc variables (u, v, T) of a state (Visc_Variables; T = p / (rho R), with
// co_rotot_Rtot's R = (rho_1 / rho) R_1)
__device__ __forceinline__ void visc3(const Gas& g, const double* q, double* V) {
  const double rho = q[0];
  const double Rg = (q[0] / rho) * g.R;
  V[0] = q[1];
  V[1] = q[2];
  V[2] = q[3] / (rho * Rg);
}

// matmul(Gradient, M) for the (u, v, T) rows: Gx = G1 M(1,1) + G2 M(2,1),
// Gy = G1 M(1,2) + G2 M(2,2) (the third index direction adds exact zeros);
// G1 / G2 are the index-direction gradients along i / j
__device__ __forceinline__ void grad_phys(const double* G1, const double* G2, const double* m, double* Gx,
                                          double* Gy) {
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    Gx[v] = G1[v] * m[0] + G2[v] * m[1];
    Gy[v] = G1[v] * m[2] + G2[v] * m[3];
  }
}

// Stress_Vector_Std (Lib_Fluid.f90:23-46), planar: (S1, S2)
__device__ __forceinline__ void stress2(const double* Gx, const double* Gy, const double* n, double mu, double* S) {
  const double mi = mu + 0.0;
  const double lam = (-2.0 / 3.0) * mi;
  const double Divervel = Gx[0] + Gy[1];
  const double lamDivervel = lam * Divervel;
  const double Txx = lamDivervel + 2.0 * mi * Gx[0];
  const double Tyy = lamDivervel + 2.0 * mi * Gy[1];
  const double Txy = mi * (Gy[0] + Gx[1]);
  S[0] = Txx * n[0] + Txy * n[1];
  S[1] = Txy * n[0] + Tyy * n[1];
}

// Compute_Diffusive_Flux (Lib_Diffusive.f90:90-172) for (rho u, rho v, E) at
// a face with mean state (ubar, vbar): F[0] momentum x, F[1] momentum y,
// F[2] energy; the mass flux is an exact zero
__device__ __forceinline__ void diff_flux(const Gas& g, const double* Gx, const double* Gy, double ubar, double vbar,
                                          const double* n, double area, double* F) {
  double S[2];
  stress2(Gx, Gy, n, g.mu, S);
  const double kappa = g.kappa + 0.0;
  F[0] = area * S[0];
  F[1] = area * S[1];
  F[2] = area * ((S[0] * ubar + S[1] * vbar) + kappa * (Gx[2] * n[0] + Gy[2] * n[1]));
}

// Convective face flux between cells A and B = A + 1 along dir: the
// reference's reconstruction on the 4-cell stencil (A-1, A, B, B+1) and the
// face solve (Convective_Flux, Lib_Convective.f90:10-85), as the exact stage
// kernels form it.  (i, j) = cell A.
template <int LIM>
__device__ bool conv_face(const Cell2& c, int dir, int i, int j, double* F) {
  const int di = dir == 0, dj = dir == 1;
  double qm[NV], q0[NV], q1[NV], q2[NV];
  c.q(i - di, j - dj, qm);
  c.q(i, j, q0);
  c.q(i + di, j + dj, q1);
  c.q(i + 2 * di, j + 2 * dj, q2);
  const double dm = c.dl(dir, i - di, j - dj), d0 = c.dl(dir, i, j), d1 = c.dl(dir, i + di, j + dj),
               d2 = c.dl(dir, i + 2 * di, j + 2 * dj);
  const double la = 0.5 * (dm + d0), lb = 0.5 * (d0 + d1), lc = 0.5 * (d1 + d2);
  const double lm = 0.5 * d0, lp = 0.5 * d1;
  double QL[NV], QR[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double sA = ex::limiter<LIM>((q1[v] - q0[v]) / lb, (q0[v] - qm[v]) / la);
    const double sB = ex::limiter<LIM>((q2[v] - q1[v]) / lc, (q1[v] - q0[v]) / lb);
    QL[v] = q0[v] + sA * lm;
    QR[v] = q1[v] - sB * lp;
  }
  double n[3];
  const double A = c.face(dir, i + di, j + dj, n);
  return ex::face_flux<4, NV>(c.a.g, QL, QR, n, A, F, 1.0);
}

// Diffusive_Flux (Lib_Diffusive.f90:10-52) between cells A = (i, j) and
// B = A + 1 along dir; F = (momentum x, momentum y, energy)
__device__ void diff_face(const Cell2& c, int dir, int i, int j, double* F) {
  const Gas& g = c.a.g;
  const int di = dir == 0, dj = dir == 1;
  const int ti = dj, tj = di;   // tangential step
  double qA[NV], qB[NV], V1[3], V2[3];
  c.q(i, j, qA);
  c.q(i + di, j + dj, qB);
  visc3(g, qA, V1);
  visc3(g, qB, V2);
  double Ga[3], Gt[3];
#pragma unroll
  for (int v = 0; v < 3; ++v) Ga[v] = V2[v] - V1[v];
  // Tangential_Gradient(P(A - t), P(A + t), P(B - t), P(B + t))
  double q3[NV], q4[NV], q5[NV], q6[NV], W1[3], W2[3], W3[3], W4[3];
  c.q(i - ti, j - tj, q3);
  c.q(i + ti, j + tj, q4);
  c.q(i + di - ti, j + dj - tj, q5);
  c.q(i + di + ti, j + dj + tj, q6);
  visc3(g, q3, W1);
  visc3(g, q4, W2);
  visc3(g, q5, W3);
  visc3(g, q6, W4);
#pragma unroll
  for (int v = 0; v < 3; ++v) Gt[v] = (W2[v] - W1[v] + W4[v] - W3[v]) * 0.25;
  double mA[4], mB[4], m[4];
  c.M(i, j, mA);
  c.M(i + di, j + dj, mB);
#pragma unroll
  for (int q = 0; q < 4; ++q) m[q] = 0.5 * (mA[q] + mB[q]);
  double Gx[3], Gy[3];
  if (dir == 0) grad_phys(Ga, Gt, m, Gx, Gy);
  else grad_phys(Gt, Ga, m, Gx, Gy);
  const double ubar = 0.5 * (qA[1] + qB[1]), vbar = 0.5 * (qA[2] + qB[2]);
  double n[3];
  const double A = c.face(dir, i + di, j + dj, n);
  diff_flux(g, Gx, Gy, ubar, vbar, n, A, F);
}

// BC_Connection_Visc (Lib_BC_Fluxes_Connection.f90:117-224), 2-D: R of the
// boundary cell (i, j) on face f minus 0.5 modfm2 (Flux_loc + Flux_ghost)
__device__ void conn_visc(const Cell2& c, const VConn& vc, int f, int i, int j, double* R) {
  const Gas& g = c.a.g;
  const int dir = (f - 1) / 2;
  const int modfm2 = 1 - 2 * (f % 2);
  const int gi = (f == 1) ? 1 : (f == 2) ? -1 : 0, gj = (f == 3) ? 1 : (f == 4) ? -1 : 0;   // guide(f,:)
  const int ig = i - gi, jg = j - gj;   // first ghost
  double n[3];
  const double area = c.face(dir, i + (f == 2), j + (f == 4), n);
  double mA[4], mG[4], m[4];
  c.M(i, j, mA);
  c.M(ig, jg, mG);
#pragma unroll
  for (int q = 0; q < 4; ++q) m[q] = 0.5 * (mA[q] + mG[q]);
  double ql[NV], qg[NV], Vl[3], Vg[3];
  c.q(i, j, ql);
  c.q(ig, jg, qg);
  visc3(g, ql, Vl);
  visc3(g, qg, Vg);
  // the boundary cell's own tangential neighbours
  const int ti = dir == 1, tj = dir == 0;
  double qp[NV], qm[NV], Vp[3], Vm[3];
  c.q(i + ti, j + tj, qp);
  c.q(i - ti, j - tj, qm);
  visc3(g, qp, Vp);
  visc3(g, qm, Vm);
  // Pg(:,3:4): the source cell's tangential neighbours (Fill_BC_Ghost_Connection)
  const BlockDesc& s = c.a.blk[vc.bs];
  const Cell2 cs{s, c.a, c.P - c.d.sbase + s.sbase};
  const int sti = (vc.fs <= 2) ? 0 : vc.d11, stj = (vc.fs <= 2) ? vc.d11 : 0;
  double q3[NV], q4[NV], V3[3], V4[3];
  cs.q(vc.is - sti, vc.js - stj, q3);
  cs.q(vc.is + sti, vc.js + stj, q4);
  visc3(g, q3, V3);
  visc3(g, q4, V4);
  double Gl_a[3], Gl_t[3], Gg_a[3], Gg_t[3];
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    Gl_a[v] = (Vg[v] - Vl[v]) * (double)modfm2;
    Gl_t[v] = (Vp[v] - Vm[v]) * 0.5;
    Gg_a[v] = (Vl[v] - Vg[v]) * (double)(-modfm2);
    Gg_t[v] = (V4[v] - V3[v]) * 0.5;
  }
  double Gx_l[3], Gy_l[3], Gx_g[3], Gy_g[3];
  if (dir == 0) {
    grad_phys(Gl_a, Gl_t, m, Gx_l, Gy_l);
    grad_phys(Gg_a, Gg_t, m, Gx_g, Gy_g);
  } else {
    grad_phys(Gl_t, Gl_a, m, Gx_l, Gy_l);
    grad_phys(Gg_t, Gg_a, m, Gx_g, Gy_g);
  }
  const double ubar = (ql[1] + qg[1]) * 0.5, vbar = (ql[2] + qg[2]) * 0.5;
  double Fl[3], Fg[3];
  diff_flux(g, Gx_l, Gy_l, ubar, vbar, n, area, Fl);
  diff_flux(g, Gx_g, Gy_g, ubar, vbar, n, area, Fg);
#pragma unroll
  for (int v = 0; v < 3; ++v) R[1 + v] = R[1 + v] - 0.5 * (double)modfm2 * (Fl[v] + Fg[v]);
}

// BC_Symmetry_Visc (Lib_BC_Fluxes_Symmetry.f90:128-247), 2-D
__device__ void sym_visc(const Cell2& c, int f, int i, int j, double* R) {
  const Gas& g = c.a.g;
  const int dir = (f - 1) / 2;
  const int modfm2 = 1 - 2 * (f % 2);
  double n[3];
  const double area = c.face(dir, i + (f == 2), j + (f == 4), n);
  double m[4];
  c.M(i, j, m);
  const int ti = dir == 1, tj = dir == 0;
  double q1[NV], q3[NV], q4[NV];
  c.q(i, j, q1);
  c.q(i - ti, j - tj, q3);
  c.q(i + ti, j + tj, q4);
  auto mirror = [&](const double* q, double* W) {
    const double dn = q[1] * n[0] + q[2] * n[1];
    W[0] = q[1] - 2.0 * dn * n[0];
    W[1] = q[2] - 2.0 * dn * n[1];
  };
  const double V1[2] = {q1[1], q1[2]}, V3[2] = {q3[1], q3[2]}, V4[2] = {q4[1], q4[2]};
  double V2[2], V5[2], V6[2];
  mirror(q1, V2);
  mirror(q3, V5);
  mirror(q4, V6);
  double Ga[3], Gt[3];
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    Ga[v] = (V2[v] - V1[v]) * (double)modfm2;
    Gt[v] = (V4[v] - V3[v] + V6[v] - V5[v]) * 0.25;
  }
  Ga[2] = Gt[2] = 0.0;
  double Gx[3], Gy[3];
  if (dir == 0) grad_phys(Ga, Gt, m, Gx, Gy);
  else grad_phys(Gt, Ga, m, Gx, Gy);
  double S[2];
  stress2(Gx, Gy, n, g.mu, S);
  const double Vx = 0.5 * (V1[0] + V2[0]), Vy = 0.5 * (V1[1] + V2[1]);
  const double F[3] = {area * S[0], area * S[1], area * (Vx * S[0] + Vy * S[1])};
#pragma unroll
  for (int v = 0; v < 3; ++v) R[1 + v] = R[1 + v] - (double)modfm2 * F[v];
}

// BC_Wall_Heat (301) / BC_Wall_Temperature (302), 2-D: no-slip velocity
// gradient across the face (Prim(nu:nw) * modfm3), the wall's temperature
// gradient (302) or heat flux (301)
__device__ void wall_visc(const Cell2& c, int code, const BcParam& bp, int f, int i, int j, double* R) {
  const Gas& g = c.a.g;
  const int dir = (f - 1) / 2;
  const int modfm = f % 2, modfm2 = 1 - 2 * modfm, modfm3 = 2 * (2 * modfm - 1);
  double n[3];
  const double area = c.face(dir, i + (f == 2), j + (f == 4), n);
  double m[4];
  c.M(i, j, m);
  double q[NV];
  c.q(i, j, q);
  double Ga[3], Gz[3] = {0.0, 0.0, 0.0};
  Ga[0] = q[1] * (double)modfm3;
  Ga[1] = q[2] * (double)modfm3;
  if (code == BC_WALL_T) {
    const double rho = q[0];
    const double Rg = (q[0] / rho) * g.R;
    const double T = q[3] / (rho * Rg);
    Ga[2] = (T - bp.T) * (double)modfm3;
  } else {
    Ga[2] = 0.0;   // the heat-flux wall's temperature gradient enters no flux
  }
  double Gx[3], Gy[3];
  if (dir == 0) grad_phys(Ga, Gz, m, Gx, Gy);
  else grad_phys(Gz, Ga, m, Gx, Gy);
  double S[2];
  stress2(Gx, Gy, n, g.mu, S);
  double F[3];
  F[0] = S[0] * area;
  F[1] = S[1] * area;
  if (code == BC_WALL_T) F[2] = area * g.kappa * (Gx[2] * n[0] + Gy[2] * n[1]);
  else F[2] = area * bp.p;
#pragma unroll
  for (int v = 0; v < 3; ++v) R[1 + v] = R[1 + v] - (double)modfm2 * F[v];
}

// a boundary-face contribution sgn * F, masked as BC_Fluxes adds it
__device__ __forceinline__ void add_masked(double* R, const double* F, double sgn, int mask) {
  if (mask == ADD_ALL) {
    for (int v = 0; v < NV; ++v) R[v] = R[v] + sgn * F[v];
  } else if (mask == ADD_MOMENTUM) {
    for (int v = 1; v < NV - 1; ++v) R[v] = R[v] + sgn * F[v];
  }
}

// The viscous face arena: 14 planes per block (offset 14 mbase), at the low
// cell of each interior face: the convective i-face flux (planes 0-3), the
// diffusive one (4-6), then the same for the j-face (7-10, 11-13).
constexpr int kVisc_CX = 0, kVisc_DX = 4, kVisc_CY = 7, kVisc_DY = 11;

template <int LIM>
__global__ void __launch_bounds__(128) k_visc_faces2d(StageArgs a) {
  const int b = blockIdx.y;
  const BlockDesc& d = a.blk[b];
  const Cell2 c{d, a, a.Pc + d.sbase};
  const long long ncell = (long long)d.ni * d.nj, vs = d.vstride;
  double* Fv = a.Fv + 14 * d.mbase;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % d.ni), j = (int)(q / d.ni);
    const long long o = c.off(i, j);
    double F[NV];
    bool ok = true;
    if (i < d.ni - 1) {
      ok &= conv_face<LIM>(c, 0, i, j, F);
      for (int v = 0; v < NV; ++v) Fv[(kVisc_CX + v) * vs + o] = F[v];
      diff_face(c, 0, i, j, F);
      for (int v = 0; v < 3; ++v) Fv[(kVisc_DX + v) * vs + o] = F[v];
    }
    if (d.nj > 1 && j < d.nj - 1) {
      ok &= conv_face<LIM>(c, 1, i, j, F);
      for (int v = 0; v < NV; ++v) Fv[(kVisc_CY + v) * vs + o] = F[v];
      diff_face(c, 1, i, j, F);
      for (int v = 0; v < 3; ++v) Fv[(kVisc_DY + v) * vs + o] = F[v];
    }
    if (!ok) report(a.err, 4, b, i, j, 0);
  }
}

template <int LIM>
__global__ void __launch_bounds__(128) k_visc_residual2d(StageArgs a) {
  const int b = blockIdx.y;
  const BlockDesc& d = a.blk[b];
  const Cell2 c{d, a, a.Pc + d.sbase};
  const long long ncell = (long long)d.ni * d.nj, vs = d.vstride;
  const double* Fv = a.Fv + 14 * d.mbase;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % d.ni), j = (int)(q / d.ni);
    double R[NV] = {0.0, 0.0, 0.0, 0.0};
    double F[NV];
    // plane p of the face whose low cell is (ii, jj)
    auto fv = [&](int p, int ii, int jj) { return Fv[p * vs + c.off(ii, jj)]; };
    // convective i faces, diffusive i faces (Mod_Fluxes.f90:89-126)
    if (i > 0)
      for (int v = 0; v < NV; ++v) R[v] = R[v] - fv(kVisc_CX + v, i - 1, j);
    if (i < d.ni - 1)
      for (int v = 0; v < NV; ++v) R[v] = R[v] + fv(kVisc_CX + v, i, j);
    if (i > 0)
      for (int v = 0; v < 3; ++v) R[1 + v] = R[1 + v] + fv(kVisc_DX + v, i - 1, j);
    if (i < d.ni - 1)
      for (int v = 0; v < 3; ++v) R[1 + v] = R[1 + v] - fv(kVisc_DX + v, i, j);
    // convective j faces, diffusive j faces (:129-166)
    if (d.nj > 1) {
      if (j > 0)
        for (int v = 0; v < NV; ++v) R[v] = R[v] - fv(kVisc_CY + v, i, j - 1);
      if (j < d.nj - 1)
        for (int v = 0; v < NV; ++v) R[v] = R[v] + fv(kVisc_CY + v, i, j);
      if (j > 0)
        for (int v = 0; v < 3; ++v) R[1 + v] = R[1 + v] + fv(kVisc_DY + v, i, j - 1);
      if (j < d.nj - 1)
        for (int v = 0; v < 3; ++v) R[1 + v] = R[1 + v] - fv(kVisc_DY + v, i, j);
    }
    // block-edge faces in face order, Euler part then viscous part
    for (int f = 1; f <= 4; ++f) {
      const bool on = (f == 1 && i == 0) || (f == 2 && i == d.ni - 1) || (f == 3 && j == 0) ||
                      (f == 4 && j == d.nj - 1);
      if (!on) continue;
      const int w = a.bcw[d.bcoff[f - 1] + ((f <= 2) ? j : i)];
      const int code = bc_code(w);
      if (code == BC_NONE) continue;
      const int dir = (f - 1) / 2;
      const double sgn = (f % 2) ? -1.0 : 1.0;
      if (code == BC_CONN) {
        // the interior formula on the ghost stencil (BC_Connection_Eul)
        conv_face<LIM>(c, dir, (f == 1) ? i - 1 : i, (f == 3) ? j - 1 : j, F);
        add_masked(R, F, sgn, ADD_ALL);
        conn_visc(c, reinterpret_cast<const VConn*>(a.vconn)[bc_param(w)], f, i, j, R);
        continue;
      }
      double Q[NV], Qi[NV], n[3];
      const int ii = i + ((f == 1) ? 1 : (f == 2) ? -1 : 0), ji = j + ((f == 3) ? 1 : (f == 4) ? -1 : 0);
      c.q(i, j, Q);
      c.q(ii, ji, Qi);
      const double A = c.face(dir, i + (f == 2), j + (f == 4), n);
      const int mask = boundary_flux<4, LIM, NV>(a, w, Q, Qi, c.dl(dir, i, j), c.dl(dir, ii, ji), n, A, f, F);
      add_masked(R, F, sgn, mask);
      if (code == BC_SYM) sym_visc(c, f, i, j, R);
      else if (code == BC_WALL_Q || code == BC_WALL_T) wall_visc(c, code, a.bcp[bc_param(w)], f, i, j, R);
    }
    double* Rb = a.R + d.sbase;
    const long long o = c.off(i, j);
    for (int v = 0; v < NV; ++v) Rb[v * d.vstride + o] = R[v];
  }
}

}  // namespace

bool launch_visc_residual2d(const StageArgs& a, int nblk, long long maxcell, int lim, cudaStream_t s) {
  const dim3 grid((unsigned)std::min<long long>((maxcell + 127) / 128, 148 * 8), (unsigned)nblk);
  switch (lim) {
#define MOSE_VISC_LIM(L)                                      \
  case L:                                                      \
    k_visc_faces2d<L><<<grid, 128, 0, s>>>(a);                 \
    k_visc_residual2d<L><<<grid, 128, 0, s>>>(a);              \
    return true;
    MOSE_VISC_LIM(0)
    MOSE_VISC_LIM(1)
    MOSE_VISC_LIM(2)
    MOSE_VISC_LIM(3)
    MOSE_VISC_LIM(4)
    MOSE_VISC_LIM(5)
#undef MOSE_VISC_LIM
  }
  return false;
}

}  // namespace mose
