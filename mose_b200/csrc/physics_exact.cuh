// physics_exact.cuh -- FP64 face physics in the reference's operation order.
//
// Every expression below keeps MOSE's Fortran evaluation order (left to right
// for equal precedence, x**2 as x*x) and this header is only compiled into a
// translation unit built with --fmad=false, so each operation rounds once
// exactly as the Fortran source reads.  The results are bit-identical to the
// reference algorithm's FP64 arithmetic.
//
// NV = 4 (2-D: rho, u, v, p) or 5 (3-D: rho, u, v, w, p).  In 2-D the w terms
// of the reference are identically zero (w = 0, n_z = 0) and are omitted; the
// omitted terms only ever add an exact zero.
//
// Thermodynamics: the reference calls FLINT (absent from its tree) for
// rho, R, a, h, e.  This file uses FLINT's documented model for one
// calorically perfect species: T = p/(rho R), a = sqrt(gamma R T),
// h = cp T, e = cv T.
#pragma once

#include "common.cuh"

namespace mose {
namespace ex {

template <int NV> struct V { double q[NV]; };

// ---- limiters: Lib_Limiters.f90:24-105 ------------------------------------
template <int LIM>
__device__ __forceinline__ double limiter(double x, double y) {
  if constexpr (LIM == 1) {            // minmod :35-45
    double r = 0.0;
    if (x * y < 0.0) return r;
    r = x;
    if (fabs(x) > fabs(y)) r = y;
    return r;
  } else if constexpr (LIM == 2) {     // van Leer :49-60
    double ru = y / (x + 1e-30);
    double phi = (ru + fabs(ru)) / (1.0 + fabs(ru));
    return phi * x;
  } else if constexpr (LIM == 3) {     // van Albada :64-75
    double ru = y / (x + 1e-30);
    double phi = (ru * ru + ru) / (1.0 + ru * ru);
    return phi * x;
  } else if constexpr (LIM == 4) {     // MC :79-90
    double ru = y / (x + 1e-30);
    double m = fmin(fmin(2.0 * ru, 0.5 * (1.0 + ru)), 2.0);
    double phi = fmax(0.0, m);
    return phi * x;
  } else if constexpr (LIM == 5) {     // superbee :94-104
    double ru = y / (x + 1e-30);
    double phi = fmax(fmax(0.0, fmin(2.0 * ru, 1.0)), fmin(ru, 2.0));
    return phi * x;
  } else {                             // first order :24-31
    return 0.0;
  }
}

// ---- thermodynamic closure --------------------------------------------------
// co_rotot_Rtot + f_ss for one species: R = (rho/rho) R_1 = R_1 exactly.
__device__ __forceinline__ double sound(const Gas& g, double rho, double p) {
  double T = p / (rho * g.R);
  return sqrt(g.gamma * g.R * T);
}
// H0(p, rho_s, |u|) with |u|^2 passed squared-of-norm as the reference does.
__device__ __forceinline__ double H0(const Gas& g, double p, double rho, double umag) {
  double T = p / (rho * g.R);
  double h = g.cp * T;
  return h + 0.5 * (umag * umag);
}

template <int NV>
__device__ __forceinline__ double dot_vel(const double* q, const double* n) {
  if constexpr (NV == 5) return q[1] * n[0] + q[2] * n[1] + q[3] * n[2];
  else return q[1] * n[0] + q[2] * n[1];
}
template <int NV>
__device__ __forceinline__ double vel_sq(const double* q) {
  if constexpr (NV == 5) return q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  else return q[1] * q[1] + q[2] * q[2];
}

// ---- Riemann solvers (interface of Mod_Riemann.f90:13-28) -------------------
// Input states q = (rho, u, v, [w,] p) with sound speed a; output per unit area
// (F_r, F_u, F_v, [F_w,] F_E).
template <int NV>
__device__ __forceinline__ void hllc(const Gas& g, const double* L, double aL, const double* R,
                                     double aR, const double* n, double* F) {
  // riemann_HLLC, Lib_Riemann_HLL.f90:147-258, with roe_averages :550-647
  constexpr int P = NV - 1;
  const double rl = L[0], rr = R[0];
  double unl = dot_vel<NV>(L, n);
  double unr = dot_vel<NV>(R, n);
  double inv_dltot = 1.0 / rl;
  double inv_drtot = 1.0 / rr;
  double Tl = L[P] * inv_dltot / g.R;
  double Tr = R[P] * inv_drtot / g.R;
  double srL = sqrt(rl);
  double srR = sqrt(rr);
  double inv_sr = 1.0 / (srL + srR);
  double u_roe = (srR * R[1] + srL * L[1]) * inv_sr;
  double v_roe = (srR * R[2] + srL * L[2]) * inv_sr;
  double w_roe = 0.0;
  if constexpr (NV == 5) w_roe = (srR * R[3] + srL * L[3]) * inv_sr;
  double R_roe = (srR * g.R + srL * g.R) * inv_sr;
  double T_roe = (srR * Tr + srL * Tl) * inv_sr;
  double hl = g.cp * Tl;
  double hr = g.cp * Tr;
  double el = hl - g.R * Tl;
  double er = hr - g.R * Tr;
  double h0l = hl * rl * inv_dltot;
  double h0r = hr * rr * inv_drtot;
  double d_roe = (srR * rr * inv_drtot + srL * rl * inv_dltot) * inv_sr;
  double cv_roe = d_roe * g.cpmR;
  double sum_ei = d_roe * (srR * er + srL * el) * inv_sr;
  h0l = h0l + 0.5 * vel_sq<NV>(L);
  h0r = h0r + 0.5 * vel_sq<NV>(R);
  double h0_roe = (srR * h0r + srL * h0l) * inv_sr;
  double gam_roe = 1.0 + R_roe / cv_roe;
  double vel2;
  if constexpr (NV == 5) vel2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  else vel2 = u_roe * u_roe + v_roe * v_roe;
  double a_roe = sqrt((gam_roe - 1.0) * (h0_roe - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
  double un_roe;
  if constexpr (NV == 5) un_roe = u_roe * n[0] + v_roe * n[1] + w_roe * n[2];
  else un_roe = u_roe * n[0] + v_roe * n[1];
  double e0l = h0l - L[P] / rl;
  double e0r = h0r - R[P] / rr;
  double S1 = fmin(fmin(0.0, unl - aL), un_roe - a_roe);
  double S4 = fmax(fmax(0.0, unr + aR), un_roe + a_roe);
  double inv_denom = 1.0 / (rl * (S1 - unl) - rr * (S4 - unr));
  double Sstar = (R[P] - L[P] + rl * unl * (S1 - unl) - rr * unr * (S4 - unr)) * inv_denom;
  double pstar = rl * (unl - S1) * (unl - Sstar) + L[P];
  if (S1 >= 0.0) {
    F[0] = rl * unl;
    for (int d = 0; d < NV - 2; ++d) F[1 + d] = F[0] * L[1 + d] + L[P] * n[d];
    F[P] = F[0] * h0l;
  } else if (Sstar >= 0.0) {
    F[0] = rl * unl;
    for (int d = 0; d < NV - 2; ++d) F[1 + d] = F[0] * L[1 + d] + L[P] * n[d];
    F[P] = F[0] * h0l;
    double inv = 1.0 / (S1 - Sstar);
    double U1S = rl * (S1 - unl) * inv;
    F[0] = F[0] + S1 * (U1S - rl);
    for (int d = 0; d < NV - 2; ++d) {
      double UdS = ((S1 - unl) * rl * L[1 + d] + (pstar - L[P]) * n[d]) * inv;
      F[1 + d] = F[1 + d] + S1 * (UdS - rl * L[1 + d]);
    }
    double U5S = ((S1 - unl) * rl * e0l - L[P] * unl + pstar * Sstar) * inv;
    F[P] = F[P] + S1 * (U5S - rl * e0l);
  } else if (S4 > 0.0) {
    F[0] = rr * unr;
    for (int d = 0; d < NV - 2; ++d) F[1 + d] = F[0] * R[1 + d] + R[P] * n[d];
    F[P] = F[0] * h0r;
    double inv = 1.0 / (S4 - Sstar);
    double U1S = rr * (S4 - unr) * inv;
    F[0] = F[0] + S4 * (U1S - rr);
    for (int d = 0; d < NV - 2; ++d) {
      double UdS = ((S4 - unr) * rr * R[1 + d] + (pstar - R[P]) * n[d]) * inv;
      F[1 + d] = F[1 + d] + S4 * (UdS - rr * R[1 + d]);
    }
    double U5S = ((S4 - unr) * rr * e0r - R[P] * unr + pstar * Sstar) * inv;
    F[P] = F[P] + S4 * (U5S - rr * e0r);
  } else {
    F[0] = rr * unr;
    for (int d = 0; d < NV - 2; ++d) F[1 + d] = F[0] * R[1 + d] + R[P] * n[d];
    F[P] = F[0] * h0r;
  }
}

template <int NV>
__device__ __forceinline__ void ausmp(const Gas& g, const double* L, double aL, const double* R,
                                      double aR, const double* n, double* F) {
  // riemann_AUSMp, Lib_Riemann_AUSM.f90:150-238
  constexpr int P = NV - 1;
  const double beta = 0.125, alpha = 0.1875;
  double unl = dot_vel<NV>(L, n);
  double unr = dot_vel<NV>(R, n);
  double H_L = H0(g, L[P], L[0], sqrt(vel_sq<NV>(L)));
  double H_R = H0(g, R[P], R[0], sqrt(vel_sq<NV>(R)));
  double a_half = sqrt(aL * aR);
  double ML = unl / a_half;
  double MR = unr / a_half;
  double MplusL, pplusL, MminusR, pminusR;
  if (fabs(ML) < 1.0) {
    MplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) + beta * ((ML * ML - 1.0) * (ML * ML - 1.0));
    pplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) * (2.0 - ML) + alpha * ML * ((ML * ML - 1.0) * (ML * ML - 1.0));
  } else {
    MplusL = 0.5 * (ML + fabs(ML));
    pplusL = 0.5 * (1.0 + copysign(1.0, ML));
  }
  if (fabs(MR) < 1.0) {
    MminusR = -(0.25 * ((MR - 1.0) * (MR - 1.0))) - beta * ((MR * MR - 1.0) * (MR * MR - 1.0));
    pminusR = 0.25 * ((MR - 1.0) * (MR - 1.0)) * (2.0 + MR) - alpha * MR * ((MR * MR - 1.0) * (MR * MR - 1.0));
  } else {
    MminusR = 0.5 * (MR - fabs(MR));
    pminusR = 0.5 * (1.0 - copysign(1.0, MR));
  }
  double Mhalf = MplusL + MminusR;
  double phalf = pplusL * L[P] + pminusR * R[P];
  double mdotp = L[0] * a_half * 0.5 * (Mhalf + fabs(Mhalf));
  double mdotm = R[0] * a_half * 0.5 * (Mhalf - fabs(Mhalf));
  F[0] = mdotp + mdotm;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = mdotp * L[1 + d] + mdotm * R[1 + d] + n[d] * phalf;
  F[P] = mdotp * H_L + mdotm * H_R;
}

template <int NV>
__device__ __forceinline__ void slau(const Gas& g, const double* L, double aL, const double* R,
                                     double aR, const double* n, double* F, bool slau2) {
  // riemann_SLAU / riemann_SLAU2, Lib_Riemann_SLAU.f90:19-141
  constexpr int P = NV - 1;
  const double rl = L[0], rr = R[0];
  double unl = dot_vel<NV>(L, n);
  double unr = dot_vel<NV>(R, n);
  double sq_veli = vel_sq<NV>(L);
  double sq_velj = vel_sq<NV>(R);
  double aF = 0.5 * (aL + aR);
  double mL = unl / aF;
  double mR = unr / aF;
  double Mach_tilde = fmin(1.0, sqrt(0.5 * (sq_veli + sq_velj)) / aF);
  double Chi = (1.0 - Mach_tilde) * (1.0 - Mach_tilde);
  double Vn_mag = (rl * fabs(unl) + rr * fabs(unr)) / (rl + rr);
  double f_rho = -fmax(fmin(mL, 0.0), -1.0) * fmin(fmax(mR, 0.0), 1.0);
  double Vn_magL = (1.0 - f_rho) * Vn_mag + f_rho * fabs(unl);
  double Vn_magR = (1.0 - f_rho) * Vn_mag + f_rho * fabs(unr);
  F[0] = 0.5 * (rl * (unl + Vn_magL) + rr * (unr - Vn_magR) - (Chi / aF) * (R[P] - L[P]));
  double BetaL, BetaR;
  if (fabs(mL) < 1.0) BetaL = 0.25 * (2.0 - mL) * ((mL + 1.0) * (mL + 1.0));
  else if (mL >= 0.0) BetaL = 1.0;
  else BetaL = 0.0;
  if (fabs(mR) < 1.0) BetaR = 0.25 * (2.0 + mR) * ((mR - 1.0) * (mR - 1.0));
  else if (mR >= 0.0) BetaR = 0.0;
  else BetaR = 1.0;
  double p_half;
  if (!slau2)
    p_half = 0.5 * (L[P] + R[P]) + 0.5 * (BetaL - BetaR) * (L[P] - R[P]) +
             (1.0 - Chi) * (BetaL + BetaR - 1.0) * 0.5 * (L[P] + R[P]);
  else
    p_half = 0.5 * (L[P] + R[P]) + 0.5 * (BetaL - BetaR) * (L[P] - R[P]) +
             sqrt(0.5 * (sq_veli + sq_velj)) * (BetaL + BetaR - 1.0) * aF * 0.5 * (rl + rr);
  double H_L = H0(g, L[P], rl, sqrt(sq_veli));
  double H_R = H0(g, R[P], rr, sqrt(sq_velj));
  const double* S = (F[0] >= 0.0) ? L : R;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = F[0] * S[1 + d] + n[d] * p_half;
  F[P] = F[0] * ((F[0] >= 0.0) ? H_L : H_R);
}

// ---- the solvers selected at run time (Gas::rie >= 4) -------------------------
// They work on three-component velocities and normals, w = 0 and n_z = 0 in
// 2-D, with every term the reference forms (an exact zero where it vanishes).
struct St3 { double r, u, v, w, p, a; };
template <int NV>
__device__ __forceinline__ St3 st3(const double* q, double a) {
  constexpr int P = NV - 1;
  St3 s;
  s.r = q[0]; s.u = q[1]; s.v = q[2]; s.w = (NV == 5) ? q[3] : 0.0; s.p = q[P]; s.a = a;
  return s;
}
struct Fl5 { double r, u, v, w, E; };
__device__ __forceinline__ double E0(const Gas& g, double p, double rho, double umag) {
  double T = p / (rho * g.R);
  double e = g.cv * T;
  return e + 0.5 * (umag * umag);
}
__device__ __forceinline__ double umag3(const St3& s) { return sqrt(s.u * s.u + s.v * s.v + s.w * s.w); }
// fluxes(p, r, u, v, w, n), Lib_Riemann_LF.f90:105-126
__device__ __forceinline__ Fl5 phys3(const Gas& g, const St3& q, double nx, double ny, double nz) {
  Fl5 F;
  F.r = q.r * (q.u * nx + q.v * ny + q.w * nz);
  F.u = F.r * q.u + q.p * nx;
  F.v = F.r * q.v + q.p * ny;
  F.w = F.r * q.w + q.p * nz;
  F.E = F.r * H0(g, q.p, q.r, umag3(q));
  return F;
}
// roe_averages, Lib_Riemann_HLL.f90:550-647 (one calorically perfect species)
struct Roe { double h0l, h0r, rho, u, v, w, a, h0; };
__device__ __forceinline__ Roe roe3(const Gas& g, const St3& L, const St3& R) {
  Roe o;
  double inv_dltot = 1.0 / L.r, inv_drtot = 1.0 / R.r;
  double Tl = L.p * inv_dltot / g.R, Tr = R.p * inv_drtot / g.R;
  double srL = sqrt(L.r), srR = sqrt(R.r);
  o.rho = srL * srR;
  double inv_sr = 1.0 / (srL + srR);
  o.u = (srR * R.u + srL * L.u) * inv_sr;
  o.v = (srR * R.v + srL * L.v) * inv_sr;
  o.w = (srR * R.w + srL * L.w) * inv_sr;
  double R_roe = (srR * g.R + srL * g.R) * inv_sr;
  double T_roe = (srR * Tr + srL * Tl) * inv_sr;
  double hl = g.cp * Tl, hr = g.cp * Tr;
  double el = hl - g.R * Tl, er = hr - g.R * Tr;
  o.h0l = hl * L.r * inv_dltot;
  o.h0r = hr * R.r * inv_drtot;
  double d_roe = (srR * R.r * inv_drtot + srL * L.r * inv_dltot) * inv_sr;
  double cv_roe = d_roe * g.cpmR;
  double sum_ei = d_roe * (srR * er + srL * el) * inv_sr;
  o.h0l = o.h0l + 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w);
  o.h0r = o.h0r + 0.5 * (R.u * R.u + R.v * R.v + R.w * R.w);
  o.h0 = (srR * o.h0r + srL * o.h0l) * inv_sr;
  double gam_roe = 1.0 + R_roe / cv_roe;
  double vel2 = o.u * o.u + o.v * o.v + o.w * o.w;
  o.a = sqrt((gam_roe - 1.0) * (o.h0 - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
  return o;
}

// riemann_HLLE, Lib_Riemann_HLL.f90:259-317
__device__ __forceinline__ Fl5 hlle3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz) {
  Fl5 F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  Roe o = roe3(g, L, R);
  double un_roe = o.u * nx + o.v * ny + o.w * nz;
  double S1 = fmin(fmin(0.0, unl - L.a), un_roe - o.a);
  double S4 = fmax(fmax(0.0, unr + R.a), un_roe + o.a);
  double inv_denom = 1.0 / (S4 - S1);
  double FrL = L.r * unl, FrR = R.r * unr;
  F.r = (S4 * FrL - S1 * FrR + S1 * S4 * (R.r - L.r)) * inv_denom;
  F.u = (S4 * (FrL * L.u + L.p * nx) - S1 * (FrR * R.u + R.p * nx) + S1 * S4 * (R.r * R.u - L.r * L.u)) * inv_denom;
  F.v = (S4 * (FrL * L.v + L.p * ny) - S1 * (FrR * R.v + R.p * ny) + S1 * S4 * (R.r * R.v - L.r * L.v)) * inv_denom;
  F.w = (S4 * (FrL * L.w + L.p * nz) - S1 * (FrR * R.w + R.p * nz) + S1 * S4 * (R.r * R.w - L.r * L.w)) * inv_denom;
  F.E = (S4 * (FrL * o.h0l) - S1 * (FrR * o.h0r) +
         S1 * S4 * (R.r * (o.h0r - R.p / R.r) - L.r * (o.h0l - L.p / L.r))) * inv_denom;
  return F;
}

// riemann_HLLEM, Lib_Riemann_HLL.f90:23-146
__device__ __forceinline__ Fl5 hllem3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz) {
  Fl5 F;
  Roe o = roe3(g, L, R);
  double un_roe = o.u * nx + o.v * ny + o.w * nz;
  double S1 = fmin(fmin(0.0, (L.u * nx + L.v * ny + L.w * nz) - L.a), un_roe - o.a);
  double S4 = fmax(fmax(0.0, (R.u * nx + R.v * ny + R.w * nz) + R.a), un_roe + o.a);
  Fl5 Fl = phys3(g, L, nx, ny, nz), Fr = phys3(g, R, nx, ny, nz);
  F.r = (S4 * Fl.r - S1 * Fr.r + S1 * S4 * (R.r - L.r)) / (S4 - S1);
  F.u = (S4 * Fl.u - S1 * Fr.u + S1 * S4 * (R.r * R.u - L.r * L.u)) / (S4 - S1);
  F.v = (S4 * Fl.v - S1 * Fr.v + S1 * S4 * (R.r * R.v - L.r * L.v)) / (S4 - S1);
  F.w = (S4 * Fl.w - S1 * Fr.w + S1 * S4 * (R.r * R.w - L.r * L.w)) / (S4 - S1);
  F.E = (S4 * Fl.E - S1 * Fr.E + S1 * S4 * (R.r * E0(g, R.p, R.r, umag3(R)) - L.r * E0(g, L.p, L.r, umag3(L)))) /
        (S4 - S1);
  if (S1 < 0.0 && S4 > 0.0) {
    double drho = R.r - L.r, dp = R.p - L.p;
    double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w;
    double t1x, t1y, t1z;
    if (fabs(nx) < 0.9) { t1x = 0.0; t1y = -nz; t1z = ny; }
    else { t1x = -nz; t1y = 0.0; t1z = nx; }
    double normt = sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
    t1x = t1x / normt; t1y = t1y / normt; t1z = t1z / normt;
    double t2x = ny * t1z - nz * t1y, t2y = nz * t1x - nx * t1z, t2z = nx * t1y - ny * t1x;
    double alpha_c = drho - dp / (o.a * o.a);
    double alpha_s1 = o.rho * (du * t1x + dv * t1y + dw * t1z);
    double alpha_s2 = o.rho * (du * t2x + dv * t2y + dw * t2z);
    double delta = o.a / (o.a + fabs(0.5 * (S1 + S4)));
    double C = (S1 * S4) / (S4 - S1);
    F.r = F.r - C * delta * alpha_c;
    F.u = F.u - C * delta * (alpha_c * o.u);
    F.v = F.v - C * delta * (alpha_c * o.v);
    F.w = F.w - C * delta * (alpha_c * o.w);
    F.u = F.u - C * delta * (alpha_s1 * t1x + alpha_s2 * t2x);
    F.v = F.v - C * delta * (alpha_s1 * t1y + alpha_s2 * t2y);
    F.w = F.w - C * delta * (alpha_s1 * t1z + alpha_s2 * t2z);
    F.E = F.E - C * delta * (alpha_c * 0.5 * (o.u * o.u + o.v * o.v + o.w * o.w));
    F.E = F.E - C * delta * (alpha_s1 * (o.u * t1x + o.v * t1y + o.w * t1z) + alpha_s2 * (o.u * t2x + o.v * t2y + o.w * t2z));
  }
  return F;
}

// 0.5 (F_L + F_R - A (U_R - U_L)), Lib_Riemann_LF.f90:39-44 / :96-101
__device__ __forceinline__ Fl5 lf3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz,
                                   double A) {
  Fl5 Fr = phys3(g, R, nx, ny, nz), Fl = phys3(g, L, nx, ny, nz), F;
  F.r = 0.5 * (Fl.r + Fr.r - A * (R.r - L.r));
  F.u = 0.5 * (Fr.u + Fl.u - A * (R.r * R.u - L.r * L.u));
  F.v = 0.5 * (Fr.v + Fl.v - A * (R.r * R.v - L.r * L.v));
  F.w = 0.5 * (Fr.w + Fl.w - A * (R.r * R.w - L.r * L.w));
  F.E = 0.5 * (Fl.E + Fr.E - A * (R.r * E0(g, R.p, R.r, umag3(R)) - L.r * E0(g, L.p, L.r, umag3(L))));
  return F;
}
// riemann_LLF (Rusanov), Lib_Riemann_LF.f90:10-45
__device__ __forceinline__ Fl5 llf3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz) {
  double uln = L.u * nx + L.v * ny + L.w * nz;
  double urn = R.u * nx + R.v * ny + R.w * nz;
  double A = fmax(fmax(fmax(fabs(uln - L.a), fabs(urn - R.a)), fabs(uln + L.a)), fabs(urn + R.a));
  return lf3(g, L, R, nx, ny, nz, A);
}
// Riemann_PLLF, Lib_Riemann_LF.f90:48-102 (theta_L/R are formed there but unused)
__device__ __forceinline__ Fl5 pllf3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz) {
  double uln = L.u * nx + L.v * ny + L.w * nz;
  double urn = R.u * nx + R.v * ny + R.w * nz;
  double U_rl = fmax(1e-5 * L.a, fmin(fabs(uln), L.a));
  double U_rr = fmax(1e-5 * R.a, fmin(fabs(urn), R.a));
  double betal = 1.0 / (L.a * L.a), betar = 1.0 / (R.a * R.a);
  double alphal = 0.5 * (1.0 - betal * (U_rl * U_rl));
  double alphar = 0.5 * (1.0 - betar * (U_rr * U_rr));
  double ul_mod = fabs(uln * (1.0 - alphal));
  double ur_mod = fabs(urn * (1.0 - alphar));
  double al_mod = sqrt((alphal * alphal) * (uln * uln) + U_rl * U_rl);
  double ar_mod = sqrt((alphar * alphar) * (urn * urn) + U_rr * U_rr);
  double A = fmax(ul_mod + al_mod, ur_mod + ar_mod);
  return lf3(g, L, R, nx, ny, nz, A);
}
// riemann_Hanel, Lib_Riemann_AUSM.f90:48-117
__device__ __forceinline__ Fl5 hanel3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz) {
  Fl5 F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double H_L = H0(g, L.p, L.r, umag3(L));
  double H_R = H0(g, R.p, R.r, umag3(R));
  double uLp, uRm, pLp, pRm;
  if (fabs(unl) <= L.a) uLp = ((unl + L.a) * (unl + L.a)) / (4.0 * L.a);
  else uLp = 0.5 * (unl + fabs(unl));
  if (fabs(unr) <= R.a) uRm = (-((unr - R.a) * (unr - R.a))) / (4.0 * R.a);
  else uRm = 0.5 * (unr - fabs(unr));
  if (fabs(unl) <= L.a) pLp = L.p * uLp * (2.0 - unl / L.a) / L.a;
  else pLp = L.p * uLp / unl;
  if (fabs(unr) <= R.a) pRm = R.p * uRm * (-2.0 - unr / R.a) / R.a;
  else pRm = R.p * uRm / unr;
  double phalf = pLp + pRm;
  F.r = uLp * L.r + uRm * R.r;
  F.u = uLp * (L.r * L.u) + uRm * (R.r * R.u) + phalf * nx;
  F.v = uLp * (L.r * L.v) + uRm * (R.r * R.v) + phalf * ny;
  F.w = uLp * (L.r * L.w) + uRm * (R.r * R.w) + phalf * nz;
  F.E = uLp * (L.r * H_L) + uRm * (R.r * H_R);
  return F;
}
// riemann_AUSMp_up, Lib_Riemann_AUSM.f90:273-418; riemann_AUSMp_up2, :455-570
__device__ __forceinline__ Fl5 ausmpup3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz,
                                        bool up2) {
  const double Kp = 0.25, Ku = 0.75, sigma = 1.0, beta = 0.125;
  Fl5 F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double sq_vel = 0.5 * ((L.u * L.u + L.v * L.v + L.w * L.w) + (R.u * R.u + R.v * R.v + R.w * R.w));
  double H_L = H0(g, L.p, L.r, umag3(L));
  double H_R = H0(g, R.p, R.r, umag3(R));
  double astarL2 = 2.0 * (g.gamma - 1.0) / (g.gamma + 1.0) * H_L;
  double astarR2 = 2.0 * (g.gamma - 1.0) / (g.gamma + 1.0) * H_R;
  double astarL = sqrt(astarL2), astarR = sqrt(astarR2);
  double atildeL = astarL2 / fmax(astarL, unl);
  double atildeR = astarR2 / fmax(astarR, -unr);
  double aF = fmin(atildeL, atildeR);
  double mL = unl / aF, mR = unr / aF;
  double MFsq = 0.5 * (mL * mL + mR * mR);
  double Mrefsq = fmin(1.0, fmax(MFsq, g.minf * g.minf));
  double fa = 2.0 * sqrt(Mrefsq) - Mrefsq;
  double alpha = up2 ? 3.0 / 16.0 * (-4.0 + 5.0 * fa * fa) : 0.1875 * (-4.0 + 5.0 * fa * fa);
  double mLP, mRM, bLP, bRM;
  if (fabs(mL) <= 1.0) {
    double p1 = 0.25 * ((mL + 1.0) * (mL + 1.0));
    double p2 = (mL * mL - 1.0) * (mL * mL - 1.0);
    mLP = p1 + beta * p2;
    bLP = p1 * (2.0 - mL) + alpha * mL * p2;
  } else {
    mLP = 0.5 * (mL + fabs(mL));
    bLP = mLP / mL;
  }
  if (fabs(mR) <= 1.0) {
    double p1 = 0.25 * ((mR - 1.0) * (mR - 1.0));
    double p2 = (mR * mR - 1.0) * (mR * mR - 1.0);
    mRM = -p1 - beta * p2;
    bRM = p1 * (2.0 + mR) - alpha * mR * p2;
  } else {
    mRM = 0.5 * (mR - fabs(mR));
    bRM = mRM / mR;
  }
  double rhoF = 0.5 * (L.r + R.r);
  double Mp = -(Kp / fa) * fmax(0.0, 1.0 - sigma * MFsq) * (R.p - L.p) / (rhoF * aF * aF);
  double mF = mLP + mRM + Mp;
  double mdot = aF * (fmax(mF, 0.0) * L.r + fmin(mF, 0.0) * R.r);
  double phalf;
  if (!up2) {
    double Pu = -Ku * fa * bLP * bRM * 2.0 * rhoF * aF * (unr - unl);
    phalf = bLP * L.p + bRM * R.p + Pu;
  } else {
    phalf = 0.5 * (R.p + L.p) + 0.5 * (bLP - bRM) * (L.p - R.p) + sqrt(sq_vel) * (bLP + bRM - 1.0) * rhoF * aF;
  }
  const bool up = mF >= 0.0;
  F.r = mdot;
  F.u = mdot * (up ? L.u : R.u) + nx * phalf;
  F.v = mdot * (up ? L.v : R.v) + ny * phalf;
  F.w = mdot * (up ? L.w : R.w) + nz * phalf;
  F.E = mdot * (up ? H_L : H_R);
  return F;
}

// hartenHyman, Lib_Riemann_HLL.f90:537-547
__device__ __forceinline__ double harten_hyman(double v, double e) {
  double al = fabs(v);
  double l = al;
  if (al <= e) l = (v * v + e * e) / (2.0 * e);
  return l;
}
// riemann_HLLEpp ('HLLE++'), Lib_Riemann_HLL.f90:320-464
__device__ __forceinline__ Fl5 hllepp3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz,
                                       double beta) {
  Fl5 F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  Roe o = roe3(g, L, R);
  double un_roe = o.u * nx + o.v * ny + o.w * nz;
  double Sm = fmin(fmin(0.0, unl - L.a), un_roe - o.a);
  double Sp = fmax(fmax(0.0, unr + R.a), un_roe + o.a);
  double inv_denom = 1.0 / (Sp - Sm);
  double lam1_hlle = fabs((Sp + Sm) * un_roe * inv_denom - 2.0 * Sp * Sm * inv_denom);
  double lam2_hlle = fabs((Sp + Sm) * (un_roe - o.a) * inv_denom - 2.0 * Sp * Sm * inv_denom);
  double lam3_hlle = fabs((Sp + Sm) * (un_roe + o.a) * inv_denom - 2.0 * Sp * Sm * inv_denom);
  double eps = 0.3 * (fabs(un_roe) + o.a);
  double lam1_roe = fabs(un_roe);
  double lam2_roe = harten_hyman(un_roe - o.a, eps);
  double lam3_roe = harten_hyman(un_roe + o.a, eps);
  double lam1_pp = beta * lam1_roe + (1.0 - beta) * lam1_hlle;
  double lam2_pp = beta * lam2_roe + (1.0 - beta) * lam2_hlle;
  double lam3_pp = beta * lam3_roe + (1.0 - beta) * lam3_hlle;
  Fl5 Fl = phys3(g, L, nx, ny, nz), Fr = phys3(g, R, nx, ny, nz);
  F.r = 0.5 * (Fl.r + Fr.r);
  F.u = 0.5 * (Fl.u + Fr.u);
  F.v = 0.5 * (Fl.v + Fr.v);
  F.w = 0.5 * (Fl.w + Fr.w);
  F.E = 0.5 * (Fl.E + Fr.E);
  double drho = R.r - L.r, dp = R.p - L.p;
  double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w, dun = unr - unl;
  double t1x, t1y, t1z;
  if (fabs(nx) < 0.9) { t1x = 0.0; t1y = -nz; t1z = ny; }
  else { t1x = -nz; t1y = 0.0; t1z = nx; }
  double normt = sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
  t1x = t1x / normt; t1y = t1y / normt; t1z = t1z / normt;
  double t2x = ny * t1z - nz * t1y, t2y = nz * t1x - nx * t1z, t2z = nx * t1y - ny * t1x;
  double alpha_m = (dp - o.rho * o.a * dun) / (2.0 * o.a * o.a);
  double alpha_c = drho - dp / (o.a * o.a);
  double alpha_s1 = o.rho * (du * t1x + dv * t1y + dw * t1z);
  double alpha_s2 = o.rho * (du * t2x + dv * t2y + dw * t2z);
  double alpha_p = (dp + o.rho * o.a * dun) / (2.0 * o.a * o.a);
  F.r = F.r - 0.5 * (alpha_c * lam1_pp + alpha_m * lam2_pp + alpha_p * lam3_pp);
  F.u = F.u - 0.5 * (alpha_c * lam1_pp * o.u);
  F.v = F.v - 0.5 * (alpha_c * lam1_pp * o.v);
  F.w = F.w - 0.5 * (alpha_c * lam1_pp * o.w);
  F.u = F.u - 0.5 * lam1_pp * (alpha_s1 * t1x + alpha_s2 * t2x);
  F.v = F.v - 0.5 * lam1_pp * (alpha_s1 * t1y + alpha_s2 * t2y);
  F.w = F.w - 0.5 * lam1_pp * (alpha_s1 * t1z + alpha_s2 * t2z);
  F.u = F.u - 0.5 * (alpha_m * lam2_pp * (o.u - o.a * nx) + alpha_p * lam3_pp * (o.u + o.a * nx));
  F.v = F.v - 0.5 * (alpha_m * lam2_pp * (o.v - o.a * ny) + alpha_p * lam3_pp * (o.v + o.a * ny));
  F.w = F.w - 0.5 * (alpha_m * lam2_pp * (o.w - o.a * nz) + alpha_p * lam3_pp * (o.w + o.a * nz));
  F.E = F.E - 0.5 * lam1_pp * (alpha_c * 0.5 * (o.u * o.u + o.v * o.v + o.w * o.w));
  F.E = F.E - 0.5 * lam1_pp * (alpha_s1 * (o.u * t1x + o.v * t1y + o.w * t1z) + alpha_s2 * (o.u * t2x + o.v * t2y + o.w * t2z));
  F.E = F.E - 0.5 * (alpha_m * lam2_pp * (o.h0 - o.a * un_roe) + alpha_p * lam3_pp * (o.h0 + o.a * un_roe));
  return F;
}

// SD_Tramel, Lib_Shock_Detector.f90:9-38 (DELTA = 20) over the face
// neighbours of a 2-D cell; the k pair of the reference is zero-gradient
// there (2-D k faces are null) and contributes an exact 0 to the maximum.
__device__ __forceinline__ double sd_tramel2(double p, double p1, double p2, double p3, double p4) {
  const double DELTA = 20.0;
  double kp1 = fabs((p2 - 2.0 * p + p1) / (p2 + 2.0 * p + p1));
  double kp2 = fabs((p4 - 2.0 * p + p3) / (p4 + 2.0 * p + p3));
  double sw = fmax(kp1, kp2);
  if (sw < 1.0 / DELTA) {
    double phi = fmax(sw / DELTA, 0.0);
    return 1.0 - tanh(10.0 * phi * phi * phi);
  }
  return 0.0;
}

// SD_Tramel over the six face neighbours of a 3-D cell (p1/p2 along i, p3/p4
// along j, p5/p6 along k).
__device__ __forceinline__ double sd_tramel3(double p, double p1, double p2, double p3, double p4, double p5,
                                             double p6) {
  const double DELTA = 20.0;
  double kp1 = fabs((p2 - 2.0 * p + p1) / (p2 + 2.0 * p + p1));
  double kp2 = fabs((p4 - 2.0 * p + p3) / (p4 + 2.0 * p + p3));
  double kp3 = fabs((p6 - 2.0 * p + p5) / (p6 + 2.0 * p + p5));
  double sw = fmax(fmax(kp1, kp2), kp3);
  if (sw < 1.0 / DELTA) {
    double phi = fmax(sw / DELTA, 0.0);
    return 1.0 - tanh(10.0 * phi * phi * phi);
  }
  return 0.0;
}

// riemann_HLLCHLLE ('HLLC Rotated'), Lib_Riemann_HLL.f90:672-755: HLLE along
// n1, the direction of the velocity jump, and HLLC along n2 = (-n1y, n1x,
// n1z), weighted by the (non-negative) projections of the face normal on
// them; HLLC along the normal where the jump is negligible.
template <int NV>
__device__ __forceinline__ void hllc_rot(const Gas& g, const double* Lq, double aL, const double* Rq, double aR,
                                         const double* n, double* F) {
  const St3 L = st3<NV>(Lq, aL), R = st3<NV>(Rq, aR);
  const double nx = n[0], ny = n[1], nz = (NV == 5) ? n[2] : 0.0;
  const double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w;
  const double abs_dv = sqrt(du * du + dv * dv + dw * dw);
  const double dum = 0.5 * (umag3(L) + umag3(R));
  if (!(abs_dv / (dum + 1.0e-10) > 1.0e-12)) {
    hllc<NV>(g, Lq, aL, Rq, aR, n, F);
    return;
  }
  double nx1 = du / abs_dv, ny1 = dv / abs_dv, nz1 = dw / abs_dv;
  double alfa1 = nx * nx1 + ny * ny1 + nz * nz1;
  const double s1 = copysign(1.0, alfa1);
  nx1 = s1 * nx1; ny1 = s1 * ny1; nz1 = s1 * nz1; alfa1 = s1 * alfa1;
  double n2[3] = {-ny1, nx1, nz1};
  double alfa2 = nx * n2[0] + ny * n2[1] + nz * n2[2];
  const double s2 = copysign(1.0, alfa2);
  n2[0] = s2 * n2[0]; n2[1] = s2 * n2[1]; n2[2] = s2 * n2[2]; alfa2 = s2 * alfa2;
  if (nz > 0.1) {
    alfa1 = 0.0;
    n2[0] = nx; n2[1] = ny; n2[2] = nz;
    alfa2 = 1.0;
  }
  const Fl5 E = hlle3(g, L, R, nx1, ny1, nz1);
  double C[NV];
  hllc<NV>(g, Lq, aL, Rq, aR, n2, C);
  F[0] = E.r * alfa1 + C[0] * alfa2;
  F[1] = E.u * alfa1 + C[1] * alfa2;
  F[2] = E.v * alfa1 + C[2] * alfa2;
  if constexpr (NV == 5) {
    double fw = E.w * alfa1 + C[3] * alfa2;
    if (fw != 0.0 && fabs(nz) <= 1.0e-10) fw = 0.0;
    F[3] = fw;
    F[4] = E.E * alfa1 + C[4] * alfa2;
  } else {
    F[3] = E.E * alfa1 + C[3] * alfa2;
  }
}

// riemann_exact ('exact'), Lib_Riemann_Godunov.f90:10-224: Newton iteration
// on the contact velocity (relative pressure tolerance 1e-5, at most 1001
// iterations) with the shock or rarefaction relation of each side
// (shockleft / rareleft / shockright / rareright, :153-224), then the
// Godunov state sampled at the face.  The sampling reads the wave speeds of
// the last iteration that set them (0 before).  Its energy flux carries the
// normal kinetic energy only, H0(p, rho, |u_n|), as the reference's does.
__device__ __forceinline__ Fl5 exact3(const Gas& g, const St3& L, const St3& R, double nx, double ny, double nz) {
  const double gam = g.gamma;
  const double p1 = L.p, a1 = L.a, p4 = R.p, a4 = R.a;
  const double gm1 = gam - 1.0;
  const double delta = 0.5 * gm1;
  const double eta = gam / delta;
  const double un1 = L.u * nx + L.v * ny + L.w * nz;
  const double ut1 = L.u - un1 * nx, vt1 = L.v - un1 * ny, wt1 = L.w - un1 * nz;
  const double un4 = R.u * nx + R.v * ny + R.w * nz;
  const double ut4 = R.u - un4 * nx, vt4 = R.v - un4 * ny, wt4 = R.w - un4 * nz;
  const double R2I = un1 + (2.0 / gm1) * a1;
  const double R1IV = un4 - (2.0 / gm1) * a4;
  const double dum = gm1 / (2.0 * gam);
  const double z = (gm1 / gm1) * (a4 / a1) * pow(p1 / p4, dum);
  double vel = (z * R2I + R1IV) / (1.0 + z);
  // rareleft / rareright: delta = .5 (gamma - 1), exponent 2 gamma / (gamma - 1)
  const double rdelta = 0.5 * (gam - 1.0);
  const double dum1 = 2.0 * gam / (gam - 1.0);
  double p3 = 1.0, p2 = 2.0 * p3, a2 = 0.0, a3 = 0.0;
  double swl = 0.0, swr = 0.0, vw1 = 0.0, vw2 = 0.0, vw3 = 0.0, vw4 = 0.0;
  int iter = 0;
  while (fabs(1.0 - (p2 / p3)) >= 1e-5 && iter <= 1000) {
    double dpr, dpl;
    if (vel < un1) {                 // shockleft(un1, a1, p1, vel, a2, p2, dpr, swl)
      const double x1 = (gam + 1.0) * (vel - un1) / (4.0 * a1);
      const double M = x1 - sqrt(1.0 + x1 * x1);
      const double C1 = gam * p1 / a1;
      p2 = p1 + C1 * (vel - un1) * M;
      dpr = 2.0 * C1 * pow(M, 3.0) / (1.0 + M * M);
      const double rpd = p2 / p1;
      swl = un1 + a1 * M;
      a2 = a1 * sqrt((gam + 1.0 + (gam - 1.0) * rpd) / (gam + 1.0 + (gam - 1.0) / rpd));
    } else {                         // rareleft(p1, a1, un1, vel, p2, a2, dpr, vw1, vw2)
      a2 = a1 - rdelta * (vel - un1);
      p2 = p1 * pow(a2 / a1, dum1);
      dpr = -(gam * p2 / a2);
      vw1 = un1 - a1;
      vw2 = vel - a2;
    }
    if (vel > un4) {                 // shockright(un4, a4, p4, vel, a3, p3, dpl, swr)
      const double x4 = (gam + 1.0) * (vel - un4) / (4.0 * a4);
      const double M = x4 + sqrt(1.0 + x4 * x4);
      const double C4 = gam * p4 / a4;
      p3 = p4 + C4 * (vel - un4) * M;
      dpl = 2.0 * C4 * pow(M, 3.0) / (1.0 + M * M);
      const double rps = p3 / p4;
      swr = un4 + a4 * M;
      a3 = a4 * sqrt((gam + 1.0 + (gam - 1.0) * rps) / (gam + 1.0 + (gam - 1.0) / rps));
    } else {                         // rareright(p4, a4, un4, vel, p3, a3, dpl, vw3, vw4)
      a3 = a4 + rdelta * (vel - un4);
      p3 = p4 * pow(a3 / a4, dum1);
      dpl = gam * p3 / a3;
      vw3 = vel + a3;
      vw4 = un4 + a4;
    }
    vel = vel - ((p2 - p3) / (dpr - dpl));
    iter = iter + 1;
  }
  double af, pf, rhof, uf, vf, wf;
  if (vel > 0.0) {
    af = a2; pf = p2;
    if (vel <= un1) {
      if (swl > 0.0) { af = a1; vel = un1; pf = p1; }
    } else if (vw1 > 0.0) {
      vel = un1; af = a1; pf = p1;
    } else if (vw2 > 0.0) {
      af = (un1 + a1 / delta) / (1.0 + 1.0 / delta);
      vel = af;
      pf = p1 * pow(af / a1, eta);
    }
    rhof = gam * pf / (af * af);
    uf = vel * nx + ut1; vf = vel * ny + vt1; wf = vel * nz + wt1;
  } else {
    af = a3; pf = p3;
    if (vel >= un4) {
      if (swr < 0.0) { af = a4; vel = un4; pf = p4; }
    } else if (vw4 < 0.0) {
      af = a4; vel = un4; pf = p4;
    } else if (vw3 < 0.0) {
      af = -(un4 - a4 / delta) / (1.0 + 1.0 / delta);
      vel = -af;
      pf = p4 * pow(af / a4, eta);
    }
    rhof = gam * pf / (af * af);
    uf = vel * nx + ut4; vf = vel * ny + vt4; wf = vel * nz + wt4;
  }
  Fl5 F;
  F.r = rhof * vel;
  F.u = F.r * uf + pf * nx;
  F.v = F.r * vf + pf * ny;
  F.w = F.r * wf + pf * nz;
  F.E = F.r * H0(g, pf, 1.0 * rhof, sqrt(vel * vel));
  return F;
}

// Every solver selected at run time by Gas::rie (MOSE_RIEMANN_*); beta is
// the face's shock detector (1 without one).
template <int NV>
__device__ __noinline__ void riemann_rt(const Gas& g, const double* Lq, double aL, const double* Rq, double aR,
                                        const double* n, double* F, double beta) {
  switch (g.rie) {
    case 0: hllc<NV>(g, Lq, aL, Rq, aR, n, F); return;
    case 1: ausmp<NV>(g, Lq, aL, Rq, aR, n, F); return;
    case 2: slau<NV>(g, Lq, aL, Rq, aR, n, F, false); return;
    case 3: slau<NV>(g, Lq, aL, Rq, aR, n, F, true); return;
    case 11: {   // riemann_HLLCSD ('HLLC+'), Lib_Riemann_HLL.f90:500-534
      if (beta >= 1.0) { hllc<NV>(g, Lq, aL, Rq, aR, n, F); return; }
      const St3 L = st3<NV>(Lq, aL), R = st3<NV>(Rq, aR);
      const Fl5 E = hlle3(g, L, R, n[0], n[1], n[2]);
      if (beta == 0.0) {
        F[0] = E.r; F[1] = E.u; F[2] = E.v;
        if constexpr (NV == 5) { F[3] = E.w; F[4] = E.E; } else F[3] = E.E;
        return;
      }
      double C[NV];
      hllc<NV>(g, Lq, aL, Rq, aR, n, C);
      F[0] = beta * C[0] + (1.0 - beta) * E.r;
      F[1] = beta * C[1] + (1.0 - beta) * E.u;
      F[2] = beta * C[2] + (1.0 - beta) * E.v;
      if constexpr (NV == 5) {
        F[3] = beta * C[3] + (1.0 - beta) * E.w;
        F[4] = beta * C[4] + (1.0 - beta) * E.E;
      } else {
        F[3] = beta * C[3] + (1.0 - beta) * E.E;
      }
      return;
    }
    case 13: hllc_rot<NV>(g, Lq, aL, Rq, aR, n, F); return;
    default: break;
  }
  const St3 L = st3<NV>(Lq, aL), R = st3<NV>(Rq, aR);
  Fl5 f;
  switch (g.rie) {
    case 12: f = hllepp3(g, L, R, n[0], n[1], n[2], beta); break;
    case 14: f = exact3(g, L, R, n[0], n[1], (NV == 5) ? n[2] : 0.0); break;
    case 4: f = hlle3(g, L, R, n[0], n[1], n[2]); break;
    case 5: f = hllem3(g, L, R, n[0], n[1], n[2]); break;
    case 6: f = llf3(g, L, R, n[0], n[1], n[2]); break;
    case 7: f = pllf3(g, L, R, n[0], n[1], n[2]); break;
    case 8: f = hanel3(g, L, R, n[0], n[1], n[2]); break;
    case 9: f = ausmpup3(g, L, R, n[0], n[1], n[2], false); break;
    default: f = ausmpup3(g, L, R, n[0], n[1], n[2], true); break;
  }
  F[0] = f.r; F[1] = f.u; F[2] = f.v;
  if constexpr (NV == 5) { F[3] = f.w; F[4] = f.E; }
  else F[3] = f.E;
}

template <int RIE, int NV>
__device__ __forceinline__ void riemann(const Gas& g, const double* L, double aL, const double* R,
                                        double aR, const double* n, double* F, double beta = 1.0) {
  if constexpr (RIE == 1) ausmp<NV>(g, L, aL, R, aR, n, F);
  else if constexpr (RIE == 2) slau<NV>(g, L, aL, R, aR, n, F, false);
  else if constexpr (RIE == 3) slau<NV>(g, L, aL, R, aR, n, F, true);
  else if constexpr (RIE == 4) riemann_rt<NV>(g, L, aL, R, aR, n, F, beta);
  else hllc<NV>(g, L, aL, R, aR, n, F);
}

// Interface flux times area, including the species upwinding of
// Lib_Convective.f90:66-75.  For one species the species flux
// F_r*A*(sp*(rho1/rho1) - sm*(rho4/rho4)) equals F_r*A exactly.
// Returns false when check_gas_state rejects either state.
template <int RIE, int NV>
__device__ __forceinline__ bool face_flux(const Gas& g, const double* QL, const double* QR,
                                          const double* n, double area, double* F, double beta = 1.0) {
  constexpr int P = NV - 1;
  bool ok = (QL[0] > 0.0 && QL[P] > 0.0 && QR[0] > 0.0 && QR[P] > 0.0);
  double aL = sound(g, QL[0], QL[P]);
  double aR = sound(g, QR[0], QR[P]);
  riemann<RIE, NV>(g, QL, aL, QR, aR, n, F, beta);
  for (int v = 0; v < NV; ++v) F[v] = F[v] * area;
  return ok;
}

// ---- boundary-face fluxes ---------------------------------------------------
// All return the flux oriented along the face normal (the low-to-high index
// direction); the caller adds modfm2 * flux.

// BC_Extrapolation, Lib_BC_Fluxes_Extrapolation.f90:13-47
template <int NV>
__device__ __forceinline__ void bc_extrapolation(const Gas& g, const double* Q, const double* n,
                                                 double area, double* F) {
  constexpr int P = NV - 1;
  double Un = dot_vel<NV>(Q, n);
  F[0] = Q[0] * Un * area;
  double Fmass = F[0];
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = Fmass * Q[1 + d] + Q[P] * area * n[d];
  F[P] = Fmass * H0(g, Q[P], Q[0], sqrt(vel_sq<NV>(Q)));
}

// BC_Symmetry_Eul, Lib_BC_Fluxes_Symmetry.f90:14-125 (no rotating frame).
// Bound = boundary cell, Int = first interior cell, s = modfm2 (-1 odd faces).
// Only the momentum components are meaningful (the caller adds only those).
template <int RIE, int LIM, int NV>
__device__ __forceinline__ void bc_symmetry(const Gas& g, const double* Bound, const double* Int,
                                            double dlB, double dlI, const double* n, double area,
                                            int face, double* F) {
  constexpr int P = NV - 1;
  const double fm = (double)(face % 2), fm1 = (double)(1 - face % 2), s = (double)(1 - 2 * (face % 2));
  double Bound_Dl = 0.5 * dlB;
  double Int_Dl = 0.5 * dlI;
  double Un = dot_vel<NV>(Bound, n);
  double Ghost[NV];
  for (int v = 0; v < NV; ++v) Ghost[v] = Bound[v];
  for (int d = 0; d < NV - 2; ++d) Ghost[1 + d] = Ghost[1 + d] - 2.0 * Un * n[d];
  double Dist12 = 2.0 * Bound_Dl * fm + (Bound_Dl + Int_Dl) * fm1;
  double Dist23 = (Bound_Dl + Int_Dl) * fm + 2.0 * Bound_Dl * fm1;
  double Face[NV];
  double Dist = Bound_Dl * s;
  for (int v = 0; v < NV; ++v) {
    double p1 = fm * Ghost[v] + fm1 * Int[v];
    double p3 = fm * Int[v] + fm1 * Ghost[v];
    double s32 = (p3 - Bound[v]) / Dist23;
    double s21 = (Bound[v] - p1) / Dist12;
    double sl = limiter<LIM>(s32, s21);
    Face[v] = Bound[v] + sl * Dist;
  }
  double Sound = sound(g, Face[0], Face[P]);
  double Unf = dot_vel<NV>(Face, n);
  double Un1 = Unf * s;
  double U1[NV], U4[NV];
  U1[0] = U4[0] = Face[0];
  U1[P] = U4[P] = Face[P];
  for (int d = 0; d < NV - 2; ++d) {
    double velt = Face[1 + d] - Unf * n[d];
    U1[1 + d] = Un1 * n[d] + velt;
    U4[1 + d] = -Un1 * n[d] + velt;
  }
  riemann<RIE, NV>(g, U1, Sound, U4, Sound, n, F);
  for (int v = 0; v < NV; ++v) F[v] = F[v] * area;
}

// Supersonic_Inflow, Lib_BC_Fluxes_Inflow.f90:289-382 (called from
// BC_Inlet_Supersonic_Static :244-281 once BC_Sign*Un < 0 has been checked).
template <int RIE, int LIM, int NV>
__device__ __forceinline__ bool bc_supersonic_inflow(const Gas& g, const double* Prim2, const double* Int,
                                                     const BcParam& bp, const double* n, double area,
                                                     int face, double* F) {
  constexpr int P = NV - 1;
  const double fm = (double)(face % 2), fm1 = (double)(1 - face % 2), s = (double)(1 - 2 * (face % 2));
  double flow_Sound = sound(g, Prim2[0], Prim2[P]);
  double flow_Mach = sqrt(vel_sq<NV>(Prim2)) / flow_Sound;
  double BC_Mach_local = bp.rel_fac * bp.mach + (1.0 - bp.rel_fac) * flow_Mach;
  double BC_p0_local = bp.rel_fac * bp.p + (1.0 - bp.rel_fac) * Prim2[P];
  double Sup[NV];
  Sup[P] = BC_p0_local;
  double Sup_Rgas = 1.0 * g.R;
  double Sup_rho = Sup[P] / (Sup_Rgas * bp.T);
  Sup[0] = Sup_rho * 1.0;
  double Sup_Sound = sound(g, Sup[0], Sup[P]);
  Sup[1] = BC_Mach_local * Sup_Sound * bp.ca * bp.cb;
  Sup[2] = BC_Mach_local * Sup_Sound * bp.sa * bp.cb;
  if constexpr (NV == 5) Sup[3] = BC_Mach_local * Sup_Sound * bp.sb;
  double PL[NV], PR[NV];
  for (int v = 0; v < NV; ++v) {
    double p1 = fm * Sup[v] + fm1 * Int[v];
    double p3 = fm * Int[v] + fm1 * Sup[v];
    double d32 = p3 - Prim2[v];
    double d21 = Prim2[v] - p1;
    double sl = limiter<LIM>(d32, d21);
    double face_v = Prim2[v] + 0.5 * sl * s;
    PL[v] = fm * Sup[v] + fm1 * face_v;
    PR[v] = fm * face_v + fm1 * Sup[v];
  }
  double aL = sound(g, PL[0], PL[P]);
  double aR = sound(g, PR[0], PR[P]);
  riemann<RIE, NV>(g, PL, aL, PR, aR, n, F);
  for (int v = 0; v < NV; ++v) F[v] = F[v] * area;
  return true;
}

// Outflow, Lib_BC_Fluxes_Outflow.f90:59-129 (after BC_Sign*Un >= 0 was checked).
template <int NV>
__device__ __forceinline__ void bc_outflow(const Gas& g, const double* Bound, double Un,
                                           const double* n, double area, double pexit_in,
                                           int face, double* F) {
  constexpr int P = NV - 1;
  const double BC_Sign = (double)(1 - 2 * (face % 2));
  double Bound_rho = Bound[0];
  double Bound_Sound = sound(g, Bound[0], Bound[P]);
  double Bound_Gamma = g.gamma;
  double Riem = Bound_Sound + BC_Sign * 0.5 * (Bound_Gamma - 1.0) * Un;
  double Mach_N = fabs(Un / Bound_Sound);
  double Face[NV], Face_Un, Face_rho;
  if (Mach_N < 1.0 && pexit_in > 0.0) {
    double p_exit = pexit_in;
    double delta = 0.5 * (Bound_Gamma - 1.0);
    double den = 1.0 / pow(1.0 + delta, Bound_Gamma / (Bound_Gamma - 1.0));
    double pstar = Bound[P] * den * pow(1.0 + delta * (Mach_N * Mach_N), Bound_Gamma / (Bound_Gamma - 1.0));
    if (pstar >= p_exit) p_exit = pstar;
    double Isentropic = (Bound_Gamma - 1.0) / (2.0 * Bound_Gamma);
    double Face_Sound = Bound_Sound * pow(p_exit / Bound[P], Isentropic);
    Face_Un = (Riem - Face_Sound) / (BC_Sign * 0.5 * (Bound_Gamma - 1.0));
    Face[P] = p_exit;
    Face_rho = Bound_Gamma * Face[P] / (Face_Sound * Face_Sound);
    Face[0] = Bound[0] / Bound_rho * Face_rho;
    for (int d = 0; d < NV - 2; ++d) {
      double velt = Bound[1 + d] - Un * n[d];
      Face[1 + d] = velt + Face_Un * n[d];
    }
  } else {
    for (int v = 0; v < NV; ++v) Face[v] = Bound[v];
    Face_Un = Un;
    Face_rho = Bound_rho;
  }
  double Face_T = Face[P] / (g.R * Face_rho);
  double Face_Enthalpy = Face[0] / Face_rho * (g.cp * Face_T);
  F[0] = Face[0] * area * Face_Un;
  double BC_mdot = Face_rho * area * Face_Un;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = Face[1 + d] * BC_mdot + Face[P] * area * n[d];
  F[P] = BC_mdot * (0.5 * vel_sq<NV>(Face) + Face_Enthalpy);
}

// ---- inlets 401 / 403 / 404 and the ambient far field 407 --------------------
// The part of Setup_Inflow_Geometry (Lib_BC_Fluxes_Inflow.f90:502-559) that
// depends on the state: the boundary cell's normal velocity, sound speed and
// the Riemann invariant toward the face (the tangent and the direction
// coefficients come precomputed in BcParam).
struct InGeo {
  double Un, sign, sound, riem;
};
template <int NV>
__device__ __forceinline__ InGeo inflow_geo(const Gas& g, const double* Q, const double* n, int face) {
  InGeo G;
  G.Un = dot_vel<NV>(Q, n);
  G.sign = (double)(1 - 2 * (face % 2));
  G.sound = sound(g, Q[0], Q[NV - 1]);
  G.riem = G.sound + G.sign * 0.5 * (g.gamma - 1.0) * G.Un;
  return G;
}

// Compute_Flux_from_Face (Lib_BC_Fluxes_Inflow.f90:565-587) for a face state
// of density rho and velocity Un3 (n + E1 t + E2 b).
template <int NV>
__device__ __forceinline__ void face_state_flux(const Gas& g, double rho, double p, double Un3, const BcParam& bp,
                                                const double* n, double area, bool known_un, double* F) {
  constexpr int P = NV - 1;
  double Face[NV];
  Face[0] = rho * 1.0;
  Face[P] = p;
  const double Ut3 = Un3 * bp.E1, Ub3 = Un3 * bp.E2;
  for (int d = 0; d < NV - 2; ++d) Face[1 + d] = Un3 * n[d] + Ut3 * bp.tv[d] + Ub3 * bp.bv[d];
  // Stagn_Inflow takes Un3 as the face's normal velocity; the mass-flux
  // inlets dot the face velocity with the normal
  const double Face_Un = known_un ? Un3 : dot_vel<NV>(Face, n);
  const double Face_T = Face[P] / (g.R * rho);
  const double Fmass = rho * Face_Un * area;
  const double Face_Enthalpy = Face[0] / rho * (g.cp * Face_T);
  F[0] = Face[0] * Face_Un * area;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = Fmass * Face[1 + d] + Face[P] * area * n[d];
  F[P] = Fmass * (0.5 * vel_sq<NV>(Face) + Face_Enthalpy);
}

// Stagn_Inflow, Lib_BC_Fluxes_Inflow.f90:388-473: total conditions (bp.T =
// T0, bp.p = p0); p0 relaxes toward the boundary pressure while the
// quadratic for the face's normal velocity has no real root, at most 1000
// times.
template <int NV>
__device__ __forceinline__ void stagn_inflow(const Gas& g, const double* Prim, const InGeo& G, const BcParam& bp,
                                             const double* n, double area, double* F) {
  constexpr int P = NV - 1;
  const double Gamma = g.gamma;
  double Discr = -1.0, p0_try = bp.p, Sound0 = 0.0, Coef_D = 0.0, YA = 0.0, YB = 0.0;
  int iter = 0;
  while (Discr < 0.0) {
    iter = iter + 1;
    const double Face_Rgas = 1.0 * g.R;
    Sound0 = sqrt(Gamma * Face_Rgas * bp.T);
    Coef_D = (1.0 + bp.E1 * bp.E1 + bp.E2 * bp.E2) * (Gamma - 1.0) / 2.0;
    double Coef_C = pow(p0_try / Prim[P], (Gamma - 1.0) / Gamma);
    const double ratio = G.sound / Sound0;
    Coef_C = Coef_C * (ratio * ratio);
    const double hg = (Gamma - 1.0) / 2.0;
    YA = hg * hg + Coef_C * Coef_D;
    YB = G.sign * G.riem * hg;
    const double YC = G.riem * G.riem - Coef_C * (Sound0 * Sound0);
    Discr = YB * YB - YA * YC;
    if (Discr < 0.0 && fabs(Discr) < 1e-2) Discr = 0.0;
    if (Discr < 0.0 && fabs(Discr) > 1e-2) p0_try = bp.rel_fac * p0_try + (1.0 - bp.rel_fac) * Prim[P];
    if (iter > 1000) {
      Discr = 0.0;
      break;
    }
  }
  const double Un_Sign = copysign(1.0, G.Un);
  const double Un3 = (YB + Un_Sign * sqrt(Discr)) / YA;
  const double Sound3 = sqrt(Sound0 * Sound0 - Coef_D * (Un3 * Un3));
  const double p3 = p0_try * pow(Sound3 / Sound0, 2.0 * Gamma / (Gamma - 1.0));
  const double rho = Gamma * p3 / (Sound3 * Sound3);
  face_state_flux<NV>(g, rho, p3, Un3, bp, n, area, true, F);
}

// BC_Inlet_MassFlux_T0 (403, Lib_BC_Fluxes_Inflow.f90:81-159) and
// BC_Inlet_MassFlux_T (404, :165-236): mass flux bp.p through the face at the
// boundary cell's pressure, with the total (403) or static (404)
// temperature bp.T.
template <int NV>
__device__ __forceinline__ void mass_flux_inflow(const Gas& g, const double* Prim, const BcParam& bp, const double* n,
                                                 double area, bool total, double* F) {
  const double Rgas3 = 0.0 + 1.0 * g.R;
  const double p3 = Prim[NV - 1];
  const double BC_g = bp.p;
  double T3 = bp.T;
  if (total) {
    const double cp3 = 0.0 + 1.0 * g.cp;
    const double X = BC_g * Rgas3 / p3, Y = p3 / (BC_g * Rgas3);
    T3 = (-cp3 + sqrt(cp3 * cp3 + 2.0 * cp3 * bp.T * (X * X))) * (Y * Y);
  }
  const double rho3 = p3 / (Rgas3 * T3);
  const double Un3 = BC_g / rho3;
  face_state_flux<NV>(g, rho3, p3, Un3, bp, n, area, false, F);
}

// ---- state update: Newstate_Conservative (Lib_Newstate.f90:134-160) --------
template <int NV>
__device__ __forceinline__ void prim2cons(const Gas& g, const double* Q, double* U) {
  constexpr int P = NV - 1;
  double rho = Q[0];
  double T = Q[P] / (rho * g.R);
  double e = g.cv * T;
  U[0] = rho;
  for (int d = 0; d < NV - 2; ++d) U[1 + d] = rho * Q[1 + d];
  U[P] = rho * (e + 0.5 * vel_sq<NV>(Q));
}
template <int NV>
__device__ __forceinline__ void cons2prim(const Gas& g, const double* U, double* Q) {
  constexpr int P = NV - 1;
  double rho = U[0];
  Q[0] = rho;
  for (int d = 0; d < NV - 2; ++d) Q[1 + d] = U[1 + d] / rho;
  double e = U[P] / rho - 0.5 * vel_sq<NV>(Q);
  double T = e / g.cv;
  Q[P] = rho * g.R * T;
}

}  // namespace ex
}  // namespace mose
