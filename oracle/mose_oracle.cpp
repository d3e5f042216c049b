// mose_oracle.cpp -- CPU oracle for MOSE's explicit inviscid residual-and-update
// path on multi-block structured grids.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
// baseline.  Nothing in the product links or calls this file.
//
// This is a restatement, routine by routine, of the reference Fortran.  The
// data model is the reference's own: P, PO, R are Fortran-ordered
// (nprim, 1-gc:ni+gc, 1-gc:nj+gc, 1-gc:nk+gc) arrays, metrics carry ghost
// layers in every direction, the boundary list is walked in bc.txt order.
// Each arithmetic expression keeps the Fortran evaluation order (left to
// right for equal precedence, `x**2` as x*x) and the file is compiled with
// -ffp-contract=off, so every operation rounds once.
//
// Thermodynamic closure.  MOSE calls the FLINT library (submodule lib/FLINT,
// https://github.com/MarcoGrossi92/FLINT, pinned commit not recoverable: the
// submodule is empty in the reference tree) for every thermodynamic quantity.
// Its source is absent, so this oracle restates FLINT's documented model
// (docs/theory/thermo.md) for ONE calorically perfect species, consistent
// with the constant-cp tables the reference ships (test/common/*/thermo.dat):
//   rho = sum(rho_s) = rho_1,  R = sum(rho_s/rho * R_s) = R_1
//   T = p / (rho R),  a = sqrt(gamma R T),  h(T) = cp T  (table h_tab)
//   cp = gamma R / (gamma - 1),  cv = R / (gamma - 1)
//   H0(p, rho_s, |u|) = h(T) + 0.5 |u|^2
//   E0(p, rho_s, |u|) = e(T) + 0.5 |u|^2,  e(T) = cv T
//   f_gamma = gamma,  f_cp = cp
//   prim2cons: (rho, rho u, rho v, rho w, rho (cv T + 0.5 |u|^2))
//   cons2prim: u = (rho u)/rho ..., T = (E/rho - 0.5|u|^2)/cv, p = rho R T
//   check_gas_state: error unless rho_s > 0 and p > 0
// norm2(v) is restated as sqrt(v1*v1 + v2*v2 + v3*v3).
// Parity at this boundary is therefore against the restated closure; the
// FLINT table path (1 K tables, int(T) index) cannot be reproduced without
// its source.
//
// Transport closure (Navier-Stokes, model = 1).  FLINT's laminar transport
// (co_k_mi_lam_Wilke_expr, f_laminarViscosity) interpolates mu(T) and k(T)
// in 1 K tables and mixes species by Wilke's rule.  For one species Wilke's
// weight is 1, and the reference's viscous tables are constant
// (test/common/Air-viscous/transport.dat), so both interpolations return the
// table's constant exactly: mu and kappa are configuration constants here.

#include "mose_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int GC = 2;                 // Global_m.f90:17
constexpr int NPRIM = 5;              // rho, u, v, w, p (one species)
constexpr int NU = 1, NV = 2, NW = 3, NP = 4;   // 0-based nu, nv, nw, np
constexpr int NRES = NPRIM;           // nres = nprim - nsc + 1

// Parameters_m.f90:29-34: guide(face, dir) is the inward unit step of a face.
const int guide[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
                         {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
inline int G(int f, int d) { return guide[f - 1][d - 1]; }

struct Vec3 { double c[3]; };

struct Thermo {
  double gamma, R, cp, cv;
};

struct Block {
  int ni = 0, nj = 0, nk = 0;
  int sx = 0, sy = 0, sz = 0;           // ghosted extents
  std::vector<double> node;             // (3, 0:ni, 0:nj, 0:nk)
  std::vector<double> P, PO, R;         // (5, ghosted cells)
  std::vector<double> M;                // (3,3, ghosted cells), c(r,s) at r + 3 s
  std::vector<double> dl;               // (3, ghosted cells)
  std::vector<double> vol;              // (ghosted cells)
  std::vector<double> fN[3], fA[3];     // dir(d)%f : N(3), A
  std::vector<double> dtlocal, beta;    // (1:ni, 1:nj, 1:nk)

  size_t cell(int i, int j, int k) const {
    return (size_t)(i + GC - 1) + (size_t)sx * ((size_t)(j + GC - 1) + (size_t)sy * (size_t)(k + GC - 1));
  }
  size_t inner(int i, int j, int k) const {
    return (size_t)(i - 1) + (size_t)ni * ((size_t)(j - 1) + (size_t)nj * (size_t)(k - 1));
  }
  const double* nodep(int i, int j, int k) const {
    return &node[3 * ((size_t)i + (size_t)(ni + 1) * ((size_t)j + (size_t)(nj + 1) * (size_t)k))];
  }
  Vec3 nd(int i, int j, int k) const {
    const double* p = nodep(i, j, k);
    return Vec3{{p[0], p[1], p[2]}};
  }
  // dir(1)%f(0:ni, 1:nj, 1:nk), dir(2)%f(1:ni, 0:nj, 1:nk), dir(3)%f(1:ni, 1:nj, 0:nk)
  size_t face(int d, int i, int j, int k) const {
    if (d == 1) return (size_t)i + (size_t)(ni + 1) * ((size_t)(j - 1) + (size_t)nj * (size_t)(k - 1));
    if (d == 2) return (size_t)(i - 1) + (size_t)ni * ((size_t)j + (size_t)(nj + 1) * (size_t)(k - 1));
    return (size_t)(i - 1) + (size_t)ni * ((size_t)(j - 1) + (size_t)nj * (size_t)k);
  }
  double* Pc(int i, int j, int k) { return &P[NPRIM * cell(i, j, k)]; }
  double* POc(int i, int j, int k) { return &PO[NPRIM * cell(i, j, k)]; }
  double* Rc(int i, int j, int k) { return &R[NPRIM * cell(i, j, k)]; }
  double& M_(int r, int s, int i, int j, int k) { return M[9 * cell(i, j, k) + (r - 1) + 3 * (s - 1)]; }
  double& dl_(int h, int i, int j, int k) { return dl[3 * cell(i, j, k) + (h - 1)]; }
  double& vol_(int i, int j, int k) { return vol[cell(i, j, k)]; }
};

struct BCrec {
  int b, i, j, k, f, type, bs, is, js, ks, fs, d11, d12, d21, d22;
  double data[6];
};

}  // namespace

struct orc_domain {
  orc_config cfg;
  Thermo th;
  int ndir = 0;
  double delthe = 0.0;
  int nthreads = 1;
  std::vector<Block> blk;
  std::vector<BCrec> bc;
  std::vector<int> n_bf;                // (nb, 6)
  struct Series { std::vector<double> t, v; bool periodic = false; };
  std::vector<Series> series;           // 402 time tables
  double time = 0.0, dtglobal = 0.0;
  int iter = 0, iter_from_call = 0;
  int err = 0, eb = 0, ei = 0, ej = 0, ek = 0;

  void fail(int code, int b, int i, int j, int k) {
#ifdef _OPENMP
#pragma omp critical(orc_err)
#endif
    {
      if (err == 0) { err = code; eb = b; ei = i; ej = j; ek = k; }
    }
  }
};

namespace {

// ---------------------------------------------------------------------------
// Thermodynamic closure (restated FLINT, see header comment)
// ---------------------------------------------------------------------------
inline void co_rotot_Rtot(const Thermo& t, double rhos, double& rho, double& R) {
  rho = rhos;
  R = (rhos / rho) * t.R;
}
inline double f_ss(const Thermo& t, double /*rhos*/, double p, double rho, double R) {
  double T = p / (rho * R);
  return std::sqrt(t.gamma * R * T);
}
inline double H0(const Thermo& t, double p, double rhos, double umag) {
  double rho = rhos, R = t.R;
  double T = p / (rho * R);
  double h = (rhos / rho) * (t.cp * T);
  return h + 0.5 * (umag * umag);
}
inline double E0(const Thermo& t, double p, double rhos, double umag) {
  double rho = rhos, R = t.R;
  double T = p / (rho * R);
  double e = (rhos / rho) * (t.cv * T);
  return e + 0.5 * (umag * umag);
}
inline double norm2(double a, double b, double c) { return std::sqrt(a * a + b * b + c * c); }
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline int check_gas_state(double rhos, double p) { return (rhos > 0.0 && p > 0.0) ? 0 : 1; }

inline void prim2cons(const Thermo& t, const double* P, double* U) {
  double rho = P[0];
  double T = P[NP] / (rho * t.R);
  double e = t.cv * T;
  U[0] = rho;
  U[NU] = rho * P[NU];
  U[NV] = rho * P[NV];
  U[NW] = rho * P[NW];
  U[NP] = rho * (e + 0.5 * (P[NU] * P[NU] + P[NV] * P[NV] + P[NW] * P[NW]));
}
inline void cons2prim(const Thermo& t, const double* U, double* P) {
  double rho = U[0];
  double u = U[NU] / rho, v = U[NV] / rho, w = U[NW] / rho;
  double e = U[NP] / rho - 0.5 * (u * u + v * v + w * w);
  double T = e / t.cv;
  P[0] = rho;
  P[NU] = u;
  P[NV] = v;
  P[NW] = w;
  P[NP] = rho * t.R * T;
}

// ---------------------------------------------------------------------------
// Limiters: Lib_Limiters.f90:24-105
// ---------------------------------------------------------------------------
inline double lim_minmod(double x, double y) {        // :35-45
  double r = 0.0;
  if (x * y < 0.0) return r;
  r = x;
  if (std::fabs(x) > std::fabs(y)) r = y;
  return r;
}
inline double lim_vanleer(double x, double y) {       // :49-60
  double ru = y / (x + 1e-30);
  double phi = (ru + std::fabs(ru)) / (1.0 + std::fabs(ru));
  return phi * x;
}
inline double lim_vanalbada(double x, double y) {     // :64-75
  double ru = y / (x + 1e-30);
  double phi = (ru * ru + ru) / (1.0 + ru * ru);
  return phi * x;
}
inline double lim_mc(double x, double y) {            // :79-90
  double ru = y / (x + 1e-30);
  double m = std::min(std::min(2.0 * ru, 0.5 * (1.0 + ru)), 2.0);
  double phi = std::max(0.0, m);
  return phi * x;
}
inline double lim_superbee(double x, double y) {      // :94-104
  double ru = y / (x + 1e-30);
  double phi = std::max(std::max(0.0, std::min(2.0 * ru, 1.0)), std::min(ru, 2.0));
  return phi * x;
}
inline double rlimiter(int lim, double x, double y) {
  switch (lim) {
    case ORC_LIM_MINMOD: return lim_minmod(x, y);
    case ORC_LIM_VANLEER: return lim_vanleer(x, y);
    case ORC_LIM_VANALBADA: return lim_vanalbada(x, y);
    case ORC_LIM_MC: return lim_mc(x, y);
    case ORC_LIM_SUPERBEE: return lim_superbee(x, y);
    default: return 0.0;                            // rlimiter_IORD :24-31
  }
}

// ---------------------------------------------------------------------------
// Riemann solvers: interface of Mod_Riemann.f90:13-28
// ---------------------------------------------------------------------------
struct RState { double d, u, v, w, p, a, rho; };
struct RFlux { double r, u, v, w, E; };

// roe_averages, Lib_Riemann_HLL.f90:550-647, with the table thermo restated
// for constant cp (h_tab(T) = cp T, cp_tab = cp, Runiv/Wm = R).
inline void roe_averages(const Thermo& t, const RState& L, const RState& Rr, double& h0l,
                         double& h0r, double& u_roe, double& v_roe, double& w_roe,
                         double& a_roe, double& h0_roe) {
  double Rl = t.R, Rrr = t.R;                               // f_Rtot
  double inv_dltot = 1.0 / L.rho;
  double inv_drtot = 1.0 / Rr.rho;
  double Tl = L.p * inv_dltot / Rl;
  double Tr = Rr.p * inv_drtot / Rrr;
  double srL = std::sqrt(L.rho);
  double srR = std::sqrt(Rr.rho);
  double inv_sr = 1.0 / (srL + srR);
  u_roe = (srR * Rr.u + srL * L.u) * inv_sr;
  v_roe = (srR * Rr.v + srL * L.v) * inv_sr;
  w_roe = (srR * Rr.w + srL * L.w) * inv_sr;
  double R_roe = (srR * Rrr + srL * Rl) * inv_sr;
  double T_roe = (srR * Tr + srL * Tl) * inv_sr;
  // species loop (one species); the leading 0 + of each accumulation is exact
  double invW = t.R;
  double hl = t.cp * Tl;
  double hr = t.cp * Tr;
  double el = hl - invW * Tl;
  double er = hr - invW * Tr;
  h0l = hl * L.d * inv_dltot;
  h0r = hr * Rr.d * inv_drtot;
  double d_roe = (srR * Rr.d * inv_drtot + srL * L.d * inv_dltot) * inv_sr;
  double cv_roe = d_roe * (0.5 * (t.cp + t.cp) - invW);
  double sum_ei = d_roe * (srR * er + srL * el) * inv_sr;
  h0l = h0l + 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w);
  h0r = h0r + 0.5 * (Rr.u * Rr.u + Rr.v * Rr.v + Rr.w * Rr.w);
  h0_roe = (srR * h0r + srL * h0l) * inv_sr;
  double gam_roe = 1.0 + R_roe / cv_roe;
  double vel2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  a_roe = std::sqrt((gam_roe - 1.0) * (h0_roe - 0.5 * vel2 + cv_roe * T_roe - sum_ei));
}
// rho_roe of roe_averages (Lib_Riemann_HLL.f90, roe_averages: rho_roe = srL srR)
inline double rho_roe_of(const RState& L, const RState& R) { return std::sqrt(L.rho) * std::sqrt(R.rho); }

// fluxes(p, r, u, v, w, n), Lib_Riemann_LF.f90 (and its twin in
// Lib_Riemann_HLL.f90): the physical flux of one state
inline RFlux phys_flux(const Thermo& t, const RState& Q, double nx, double ny, double nz) {
  RFlux F;
  F.r = Q.d * (Q.u * nx + Q.v * ny + Q.w * nz);
  F.u = F.r * Q.u + Q.p * nx;
  F.v = F.r * Q.v + Q.p * ny;
  F.w = F.r * Q.w + Q.p * nz;
  F.E = F.r * H0(t, Q.p, Q.d, std::sqrt(Q.u * Q.u + Q.v * Q.v + Q.w * Q.w));
  return F;
}

// riemann_HLLC (Batten), Lib_Riemann_HLL.f90:147-258
inline RFlux riemann_HLLC(const Thermo& t, const RState& L, const RState& R, double nx,
                          double ny, double nz) {
  RFlux F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe;
  roe_averages(t, L, R, h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe);
  double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  double e0l = h0l - L.p / L.rho;
  double e0r = h0r - R.p / R.rho;
  double S1 = std::min(std::min(0.0, unl - L.a), un_roe - a_roe);
  double S4 = std::max(std::max(0.0, unr + R.a), un_roe + a_roe);
  double inv_denom = 1.0 / (L.rho * (S1 - unl) - R.rho * (S4 - unr));
  double Sstar = (R.p - L.p + L.rho * unl * (S1 - unl) - R.rho * unr * (S4 - unr)) * inv_denom;
  double pstar = L.rho * (unl - S1) * (unl - Sstar) + L.p;
  if (S1 >= 0.0) {
    F.r = L.rho * unl;
    F.u = F.r * L.u + L.p * nx;
    F.v = F.r * L.v + L.p * ny;
    F.w = F.r * L.w + L.p * nz;
    F.E = F.r * h0l;
  } else if (Sstar >= 0.0) {
    F.r = L.rho * unl;
    F.u = F.r * L.u + L.p * nx;
    F.v = F.r * L.v + L.p * ny;
    F.w = F.r * L.w + L.p * nz;
    F.E = F.r * h0l;
    inv_denom = 1.0 / (S1 - Sstar);
    double U1S = L.rho * (S1 - unl) * inv_denom;
    double U2S = ((S1 - unl) * L.rho * L.u + (pstar - L.p) * nx) * inv_denom;
    double U3S = ((S1 - unl) * L.rho * L.v + (pstar - L.p) * ny) * inv_denom;
    double U4S = ((S1 - unl) * L.rho * L.w + (pstar - L.p) * nz) * inv_denom;
    double U5S = ((S1 - unl) * L.rho * e0l - L.p * unl + pstar * Sstar) * inv_denom;
    F.r = F.r + S1 * (U1S - L.rho);
    F.u = F.u + S1 * (U2S - L.rho * L.u);
    F.v = F.v + S1 * (U3S - L.rho * L.v);
    F.w = F.w + S1 * (U4S - L.rho * L.w);
    F.E = F.E + S1 * (U5S - L.rho * e0l);
  } else if (S4 > 0.0) {
    F.r = R.rho * unr;
    F.u = F.r * R.u + R.p * nx;
    F.v = F.r * R.v + R.p * ny;
    F.w = F.r * R.w + R.p * nz;
    F.E = F.r * h0r;
    inv_denom = 1.0 / (S4 - Sstar);
    double U1S = R.rho * (S4 - unr) * inv_denom;
    double U2S = ((S4 - unr) * R.rho * R.u + (pstar - R.p) * nx) * inv_denom;
    double U3S = ((S4 - unr) * R.rho * R.v + (pstar - R.p) * ny) * inv_denom;
    double U4S = ((S4 - unr) * R.rho * R.w + (pstar - R.p) * nz) * inv_denom;
    double U5S = ((S4 - unr) * R.rho * e0r - R.p * unr + pstar * Sstar) * inv_denom;
    F.r = F.r + S4 * (U1S - R.rho);
    F.u = F.u + S4 * (U2S - R.rho * R.u);
    F.v = F.v + S4 * (U3S - R.rho * R.v);
    F.w = F.w + S4 * (U4S - R.rho * R.w);
    F.E = F.E + S4 * (U5S - R.rho * e0r);
  } else {
    F.r = R.rho * unr;
    F.u = F.r * R.u + R.p * nx;
    F.v = F.r * R.v + R.p * ny;
    F.w = F.r * R.w + R.p * nz;
    F.E = F.r * h0r;
  }
  return F;
}

// riemann_AUSMp, Lib_Riemann_AUSM.f90:150-238
inline RFlux riemann_AUSMp(const Thermo& t, const RState& L, const RState& R, double nx,
                           double ny, double nz) {
  const double beta = 0.125, alpha = 0.1875;
  RFlux F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double H_L = H0(t, L.p, L.d, std::sqrt(L.u * L.u + L.v * L.v + L.w * L.w));
  double H_R = H0(t, R.p, R.d, std::sqrt(R.u * R.u + R.v * R.v + R.w * R.w));
  double a_half = std::sqrt(L.a * R.a);
  double ML = unl / a_half;
  double MR = unr / a_half;
  double MplusL, pplusL, MminusR, pminusR;
  if (std::fabs(ML) < 1.0) {
    MplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) + beta * ((ML * ML - 1.0) * (ML * ML - 1.0));
    pplusL = 0.25 * ((ML + 1.0) * (ML + 1.0)) * (2.0 - ML) + alpha * ML * ((ML * ML - 1.0) * (ML * ML - 1.0));
  } else {
    MplusL = 0.5 * (ML + std::fabs(ML));
    pplusL = 0.5 * (1.0 + std::copysign(1.0, ML));
  }
  if (std::fabs(MR) < 1.0) {
    MminusR = -(0.25 * ((MR - 1.0) * (MR - 1.0))) - beta * ((MR * MR - 1.0) * (MR * MR - 1.0));
    pminusR = 0.25 * ((MR - 1.0) * (MR - 1.0)) * (2.0 + MR) - alpha * MR * ((MR * MR - 1.0) * (MR * MR - 1.0));
  } else {
    MminusR = 0.5 * (MR - std::fabs(MR));
    pminusR = 0.5 * (1.0 - std::copysign(1.0, MR));
  }
  double Mhalf = MplusL + MminusR;
  double phalf = pplusL * L.p + pminusR * R.p;
  double mdotp = L.rho * a_half * 0.5 * (Mhalf + std::fabs(Mhalf));
  double mdotm = R.rho * a_half * 0.5 * (Mhalf - std::fabs(Mhalf));
  F.r = mdotp + mdotm;
  F.u = mdotp * L.u + mdotm * R.u + nx * phalf;
  F.v = mdotp * L.v + mdotm * R.v + ny * phalf;
  F.w = mdotp * L.w + mdotm * R.w + nz * phalf;
  F.E = mdotp * H_L + mdotm * H_R;
  return F;
}

// riemann_SLAU / SLAU2, Lib_Riemann_SLAU.f90:19-141
inline RFlux riemann_SLAU(const Thermo& t, const RState& L, const RState& R, double nx,
                          double ny, double nz, bool slau2) {
  RFlux F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double sq_veli = L.u * L.u + L.v * L.v + L.w * L.w;
  double sq_velj = R.u * R.u + R.v * R.v + R.w * R.w;
  double aF = 0.5 * (L.a + R.a);
  double mL = unl / aF;
  double mR = unr / aF;
  double Mach_tilde = std::min(1.0, std::sqrt(0.5 * (sq_veli + sq_velj)) / aF);
  double Chi = (1.0 - Mach_tilde) * (1.0 - Mach_tilde);
  double Vn_mag = (L.rho * std::fabs(unl) + R.rho * std::fabs(unr)) / (L.rho + R.rho);
  double f_rho = -std::max(std::min(mL, 0.0), -1.0) * std::min(std::max(mR, 0.0), 1.0);
  double Vn_magL = (1.0 - f_rho) * Vn_mag + f_rho * std::fabs(unl);
  double Vn_magR = (1.0 - f_rho) * Vn_mag + f_rho * std::fabs(unr);
  F.r = 0.5 * (L.rho * (unl + Vn_magL) + R.rho * (unr - Vn_magR) - (Chi / aF) * (R.p - L.p));
  double BetaL, BetaR;
  if (std::fabs(mL) < 1.0) BetaL = 0.25 * (2.0 - mL) * ((mL + 1.0) * (mL + 1.0));
  else if (mL >= 0.0) BetaL = 1.0;
  else BetaL = 0.0;
  if (std::fabs(mR) < 1.0) BetaR = 0.25 * (2.0 + mR) * ((mR - 1.0) * (mR - 1.0));
  else if (mR >= 0.0) BetaR = 0.0;
  else BetaR = 1.0;
  double p_half;
  if (!slau2) {
    p_half = 0.5 * (L.p + R.p) + 0.5 * (BetaL - BetaR) * (L.p - R.p) +
             (1.0 - Chi) * (BetaL + BetaR - 1.0) * 0.5 * (L.p + R.p);
  } else {
    p_half = 0.5 * (L.p + R.p) + 0.5 * (BetaL - BetaR) * (L.p - R.p) +
             std::sqrt(0.5 * (sq_veli + sq_velj)) * (BetaL + BetaR - 1.0) * aF * 0.5 * (L.rho + R.rho);
  }
  double H_L = H0(t, L.p, L.d, std::sqrt(sq_veli));
  double H_R = H0(t, R.p, R.d, std::sqrt(sq_velj));
  if (F.r >= 0.0) {
    F.u = F.r * L.u + nx * p_half;
    F.v = F.r * L.v + ny * p_half;
    F.w = F.r * L.w + nz * p_half;
    F.E = F.r * H_L;
  } else {
    F.u = F.r * R.u + nx * p_half;
    F.v = F.r * R.v + ny * p_half;
    F.w = F.r * R.w + nz * p_half;
    F.E = F.r * H_R;
  }
  return F;
}

// riemann_HLLE, Lib_Riemann_HLL.f90:259-317 (Batten signal speeds)
inline RFlux riemann_HLLE(const Thermo& t, const RState& L, const RState& R, double nx, double ny,
                          double nz) {
  RFlux F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe;
  roe_averages(t, L, R, h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe);
  double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  double S1 = std::min(std::min(0.0, unl - L.a), un_roe - a_roe);
  double S4 = std::max(std::max(0.0, unr + R.a), un_roe + a_roe);
  double inv_denom = 1.0 / (S4 - S1);
  double FrL = L.rho * unl, FrR = R.rho * unr;
  F.r = (S4 * FrL - S1 * FrR + S1 * S4 * (R.rho - L.rho)) * inv_denom;
  F.u = (S4 * (FrL * L.u + L.p * nx) - S1 * (FrR * R.u + R.p * nx) + S1 * S4 * (R.rho * R.u - L.rho * L.u)) * inv_denom;
  F.v = (S4 * (FrL * L.v + L.p * ny) - S1 * (FrR * R.v + R.p * ny) + S1 * S4 * (R.rho * R.v - L.rho * L.v)) * inv_denom;
  F.w = (S4 * (FrL * L.w + L.p * nz) - S1 * (FrR * R.w + R.p * nz) + S1 * S4 * (R.rho * R.w - L.rho * L.w)) * inv_denom;
  F.E = (S4 * (FrL * h0l) - S1 * (FrR * h0r) +
         S1 * S4 * (R.rho * (h0r - R.p / R.rho) - L.rho * (h0l - L.p / L.rho))) * inv_denom;
  return F;
}

// riemann_HLLEM (Einfeldt et al. 1991), Lib_Riemann_HLL.f90:23-146: HLL flux of
// the physical fluxes plus the anti-diffusion of the contact and shear waves
// when S1 < 0 < S4
inline RFlux riemann_HLLEM(const Thermo& t, const RState& L, const RState& R, double nx, double ny,
                           double nz) {
  RFlux F;
  double h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe;
  roe_averages(t, L, R, h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe);
  double rho_roe = rho_roe_of(L, R);
  double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  double S1 = std::min(std::min(0.0, (L.u * nx + L.v * ny + L.w * nz) - L.a), un_roe - a_roe);
  double S4 = std::max(std::max(0.0, (R.u * nx + R.v * ny + R.w * nz) + R.a), un_roe + a_roe);
  RFlux Fl = phys_flux(t, L, nx, ny, nz), Fr = phys_flux(t, R, nx, ny, nz);
  F.r = (S4 * Fl.r - S1 * Fr.r + S1 * S4 * (R.rho - L.rho)) / (S4 - S1);
  F.u = (S4 * Fl.u - S1 * Fr.u + S1 * S4 * (R.rho * R.u - L.rho * L.u)) / (S4 - S1);
  F.v = (S4 * Fl.v - S1 * Fr.v + S1 * S4 * (R.rho * R.v - L.rho * L.v)) / (S4 - S1);
  F.w = (S4 * Fl.w - S1 * Fr.w + S1 * S4 * (R.rho * R.w - L.rho * L.w)) / (S4 - S1);
  F.E = (S4 * Fl.E - S1 * Fr.E +
         S1 * S4 * (R.rho * E0(t, R.p, R.d, std::sqrt(R.u * R.u + R.v * R.v + R.w * R.w)) -
                    L.rho * E0(t, L.p, L.d, std::sqrt(L.u * L.u + L.v * L.v + L.w * L.w)))) / (S4 - S1);
  if (S1 < 0.0 && S4 > 0.0) {
    double drho = R.rho - L.rho, dp = R.p - L.p;
    double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w;
    double t1x, t1y, t1z;
    if (std::fabs(nx) < 0.9) { t1x = 0.0; t1y = -nz; t1z = ny; }
    else { t1x = -nz; t1y = 0.0; t1z = nx; }
    double normt = std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
    t1x = t1x / normt; t1y = t1y / normt; t1z = t1z / normt;
    double t2x = ny * t1z - nz * t1y, t2y = nz * t1x - nx * t1z, t2z = nx * t1y - ny * t1x;
    double alpha_c = drho - dp / (a_roe * a_roe);
    double alpha_s1 = rho_roe * (du * t1x + dv * t1y + dw * t1z);
    double alpha_s2 = rho_roe * (du * t2x + dv * t2y + dw * t2z);
    double delta = a_roe / (a_roe + std::fabs(0.5 * (S1 + S4)));
    double C = (S1 * S4) / (S4 - S1);
    F.r = F.r - C * delta * alpha_c;
    F.u = F.u - C * delta * (alpha_c * u_roe);
    F.v = F.v - C * delta * (alpha_c * v_roe);
    F.w = F.w - C * delta * (alpha_c * w_roe);
    F.u = F.u - C * delta * (alpha_s1 * t1x + alpha_s2 * t2x);
    F.v = F.v - C * delta * (alpha_s1 * t1y + alpha_s2 * t2y);
    F.w = F.w - C * delta * (alpha_s1 * t1z + alpha_s2 * t2z);
    F.E = F.E - C * delta * (alpha_c * 0.5 * (u_roe * u_roe + v_roe * v_roe + w_roe * w_roe));
    F.E = F.E - C * delta * (alpha_s1 * (u_roe * t1x + v_roe * t1y + w_roe * t1z) +
                             alpha_s2 * (u_roe * t2x + v_roe * t2y + w_roe * t2z));
  }
  return F;
}

// Shared by the Lax-Friedrichs pair: 0.5 (F_L + F_R - A (U_R - U_L)),
// Lib_Riemann_LF.f90:39-44 / :96-101
inline RFlux lf_flux(const Thermo& t, const RState& L, const RState& R, double nx, double ny, double nz,
                     double A) {
  RFlux Fr = phys_flux(t, R, nx, ny, nz), Fl = phys_flux(t, L, nx, ny, nz), F;
  F.r = 0.5 * (Fl.r + Fr.r - A * (R.rho - L.rho));
  F.u = 0.5 * (Fr.u + Fl.u - A * (R.rho * R.u - L.rho * L.u));
  F.v = 0.5 * (Fr.v + Fl.v - A * (R.rho * R.v - L.rho * L.v));
  F.w = 0.5 * (Fr.w + Fl.w - A * (R.rho * R.w - L.rho * L.w));
  F.E = 0.5 * (Fl.E + Fr.E - A * (R.rho * E0(t, R.p, R.d, std::sqrt(R.u * R.u + R.v * R.v + R.w * R.w)) -
                                  L.rho * E0(t, L.p, L.d, std::sqrt(L.u * L.u + L.v * L.v + L.w * L.w))));
  return F;
}

// riemann_LLF (Rusanov), Lib_Riemann_LF.f90:10-45
inline RFlux riemann_LLF(const Thermo& t, const RState& L, const RState& R, double nx, double ny,
                         double nz) {
  double uln = L.u * nx + L.v * ny + L.w * nz;
  double urn = R.u * nx + R.v * ny + R.w * nz;
  double A = std::max(std::max(std::max(std::fabs(uln - L.a), std::fabs(urn - R.a)), std::fabs(uln + L.a)),
                      std::fabs(urn + R.a));
  return lf_flux(t, L, R, nx, ny, nz, A);
}

// Riemann_PLLF (preconditioned Rusanov), Lib_Riemann_LF.f90:48-102
inline RFlux riemann_PLLF(const Thermo& t, const RState& L, const RState& R, double nx, double ny,
                          double nz) {
  double uln = L.u * nx + L.v * ny + L.w * nz;
  double urn = R.u * nx + R.v * ny + R.w * nz;
  double Tl = L.p / (L.rho * t.R), Tr = R.p / (R.rho * t.R);
  double rho_Tl = -L.rho / Tl, rho_Tr = -R.rho / Tr;
  double cpl = t.cp, cpr = t.cp;
  double U_rl = std::max(1e-5 * L.a, std::min(std::fabs(uln), L.a));
  double U_rr = std::max(1e-5 * R.a, std::min(std::fabs(urn), R.a));
  double thetal = 1.0 / (U_rl * U_rl) - rho_Tl / (L.rho * cpl);
  double thetar = 1.0 / (U_rr * U_rr) - rho_Tr / (R.rho * cpr);
  (void)thetal;
  (void)thetar;
  double betal = 1.0 / (L.a * L.a), betar = 1.0 / (R.a * R.a);
  double alphal = 0.5 * (1.0 - betal * (U_rl * U_rl));
  double alphar = 0.5 * (1.0 - betar * (U_rr * U_rr));
  double ul_mod = std::fabs(uln * (1.0 - alphal));
  double ur_mod = std::fabs(urn * (1.0 - alphar));
  double al_mod = std::sqrt((alphal * alphal) * (uln * uln) + U_rl * U_rl);
  double ar_mod = std::sqrt((alphar * alphar) * (urn * urn) + U_rr * U_rr);
  double A = std::max(ul_mod + al_mod, ur_mod + ar_mod);
  return lf_flux(t, L, R, nx, ny, nz, A);
}

// riemann_Hanel, Lib_Riemann_AUSM.f90:48-117
inline RFlux riemann_Hanel(const Thermo& t, const RState& L, const RState& R, double nx, double ny,
                           double nz) {
  RFlux F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double H_L = H0(t, L.p, L.d, std::sqrt(L.u * L.u + L.v * L.v + L.w * L.w));
  double H_R = H0(t, R.p, R.d, std::sqrt(R.u * R.u + R.v * R.v + R.w * R.w));
  double uLp, uRm, pLp, pRm;
  if (std::fabs(unl) <= L.a) uLp = ((unl + L.a) * (unl + L.a)) / (4.0 * L.a);
  else uLp = 0.5 * (unl + std::fabs(unl));
  if (std::fabs(unr) <= R.a) uRm = (-((unr - R.a) * (unr - R.a))) / (4.0 * R.a);
  else uRm = 0.5 * (unr - std::fabs(unr));
  if (std::fabs(unl) <= L.a) pLp = L.p * uLp * (2.0 - unl / L.a) / L.a;
  else pLp = L.p * uLp / unl;
  if (std::fabs(unr) <= R.a) pRm = R.p * uRm * (-2.0 - unr / R.a) / R.a;
  else pRm = R.p * uRm / unr;
  double phalf = pLp + pRm;
  F.r = uLp * L.rho + uRm * R.rho;
  F.u = uLp * (L.rho * L.u) + uRm * (R.rho * R.u) + phalf * nx;
  F.v = uLp * (L.rho * L.v) + uRm * (R.rho * R.v) + phalf * ny;
  F.w = uLp * (L.rho * L.w) + uRm * (R.rho * R.w) + phalf * nz;
  F.E = uLp * (L.rho * H_L) + uRm * (R.rho * H_R);
  return F;
}

// riemann_AUSMp_up (SU2 form), Lib_Riemann_AUSM.f90:273-418, and
// riemann_AUSMp_up2 (Kitamura-Shima pressure flux), :455-570
inline RFlux riemann_AUSMp_up(const Thermo& t, const RState& L, const RState& R, double nx, double ny,
                              double nz, double minf, bool up2) {
  const double Kp = 0.25, Ku = 0.75, sigma = 1.0, beta = 0.125;
  RFlux F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double sq_vel = 0.5 * ((L.u * L.u + L.v * L.v + L.w * L.w) + (R.u * R.u + R.v * R.v + R.w * R.w));
  double H_L = H0(t, L.p, L.d, std::sqrt(L.u * L.u + L.v * L.v + L.w * L.w));
  double H_R = H0(t, R.p, R.d, std::sqrt(R.u * R.u + R.v * R.v + R.w * R.w));
  double gamma_L = t.gamma, gamma_R = t.gamma;
  double astarL2 = 2.0 * (gamma_L - 1.0) / (gamma_L + 1.0) * H_L;
  double astarR2 = 2.0 * (gamma_R - 1.0) / (gamma_R + 1.0) * H_R;
  double astarL = std::sqrt(astarL2), astarR = std::sqrt(astarR2);
  double atildeL = astarL2 / std::max(astarL, unl);
  double atildeR = astarR2 / std::max(astarR, -unr);
  double aF = std::min(atildeL, atildeR);
  double mL = unl / aF, mR = unr / aF;
  double MFsq = 0.5 * (mL * mL + mR * mR);
  double Mrefsq = std::min(1.0, std::max(MFsq, minf * minf));
  double fa = 2.0 * std::sqrt(Mrefsq) - Mrefsq;
  double alpha = up2 ? 3.0 / 16.0 * (-4.0 + 5.0 * fa * fa) : 0.1875 * (-4.0 + 5.0 * fa * fa);
  double mLP, mRM, bLP, bRM;
  if (std::fabs(mL) <= 1.0) {
    double p1 = 0.25 * ((mL + 1.0) * (mL + 1.0));
    double p2 = (mL * mL - 1.0) * (mL * mL - 1.0);
    mLP = p1 + beta * p2;
    bLP = p1 * (2.0 - mL) + alpha * mL * p2;
  } else {
    mLP = 0.5 * (mL + std::fabs(mL));
    bLP = mLP / mL;
  }
  if (std::fabs(mR) <= 1.0) {
    double p1 = 0.25 * ((mR - 1.0) * (mR - 1.0));
    double p2 = (mR * mR - 1.0) * (mR * mR - 1.0);
    mRM = -p1 - beta * p2;
    bRM = p1 * (2.0 + mR) - alpha * mR * p2;
  } else {
    mRM = 0.5 * (mR - std::fabs(mR));
    bRM = mRM / mR;
  }
  double rhoF = 0.5 * (L.rho + R.rho);
  double Mp = -(Kp / fa) * std::max(0.0, 1.0 - sigma * MFsq) * (R.p - L.p) / (rhoF * aF * aF);
  double mF = mLP + mRM + Mp;
  double mdot = aF * (std::max(mF, 0.0) * L.rho + std::min(mF, 0.0) * R.rho);
  double phalf;
  if (!up2) {
    double Pu = -Ku * fa * bLP * bRM * 2.0 * rhoF * aF * (unr - unl);
    phalf = bLP * L.p + bRM * R.p + Pu;
  } else {
    phalf = 0.5 * (R.p + L.p) + 0.5 * (bLP - bRM) * (L.p - R.p) + std::sqrt(sq_vel) * (bLP + bRM - 1.0) * rhoF * aF;
  }
  const RState& K = (mF >= 0.0) ? L : R;
  double upwind_H = (mF >= 0.0) ? H_L : H_R;
  F.r = mdot;
  F.u = mdot * K.u + nx * phalf;
  F.v = mdot * K.v + ny * phalf;
  F.w = mdot * K.w + nz * phalf;
  F.E = mdot * upwind_H;
  return F;
}

// riemann_HLLCSD ('HLLC+', Tramel), Lib_Riemann_HLL.f90:500-534: HLLE where
// the shock detector is 0, HLLC where it is >= 1, their blend in between
inline RFlux riemann_HLLCSD(const Thermo& t, const RState& L, const RState& R, double nx, double ny, double nz,
                            double beta) {
  if (beta == 0.0) return riemann_HLLE(t, L, R, nx, ny, nz);
  if (beta >= 1.0) return riemann_HLLC(t, L, R, nx, ny, nz);
  RFlux E = riemann_HLLE(t, L, R, nx, ny, nz), C = riemann_HLLC(t, L, R, nx, ny, nz), F;
  F.r = beta * C.r + (1.0 - beta) * E.r;
  F.u = beta * C.u + (1.0 - beta) * E.u;
  F.v = beta * C.v + (1.0 - beta) * E.v;
  F.w = beta * C.w + (1.0 - beta) * E.w;
  F.E = beta * C.E + (1.0 - beta) * E.E;
  return F;
}

// hartenHyman, Lib_Riemann_HLL.f90:537-547
inline double hartenHyman(double v, double e) {
  double al = std::fabs(v);
  double l = al;
  if (al <= e) l = (v * v + e * e) / (2.0 * e);
  return l;
}

// riemann_HLLEpp ('HLLE++', Tramel), Lib_Riemann_HLL.f90:320-464: central
// flux with the wave-by-wave dissipation whose eigenvalues blend Roe's
// (Harten-Hyman fixed) and HLLE's by the shock detector
inline RFlux riemann_HLLEpp(const Thermo& t, const RState& L, const RState& R, double nx, double ny, double nz,
                            double beta) {
  RFlux F;
  double unl = L.u * nx + L.v * ny + L.w * nz;
  double unr = R.u * nx + R.v * ny + R.w * nz;
  double h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe;
  roe_averages(t, L, R, h0l, h0r, u_roe, v_roe, w_roe, a_roe, h0_roe);
  double rho_roe = rho_roe_of(L, R);
  double un_roe = u_roe * nx + v_roe * ny + w_roe * nz;
  double Sm = std::min(std::min(0.0, unl - L.a), un_roe - a_roe);
  double Sp = std::max(std::max(0.0, unr + R.a), un_roe + a_roe);
  double inv_denom = 1.0 / (Sp - Sm);
  double lam1_hlle = std::fabs((Sp + Sm) * un_roe * inv_denom - 2.0 * Sp * Sm * inv_denom);
  double lam2_hlle = std::fabs((Sp + Sm) * (un_roe - a_roe) * inv_denom - 2.0 * Sp * Sm * inv_denom);
  double lam3_hlle = std::fabs((Sp + Sm) * (un_roe + a_roe) * inv_denom - 2.0 * Sp * Sm * inv_denom);
  double eps = 0.3 * (std::fabs(un_roe) + a_roe);
  double lam1_roe = std::fabs(un_roe);
  double lam2_roe = hartenHyman(un_roe - a_roe, eps);
  double lam3_roe = hartenHyman(un_roe + a_roe, eps);
  double lam1_pp = beta * lam1_roe + (1.0 - beta) * lam1_hlle;
  double lam2_pp = beta * lam2_roe + (1.0 - beta) * lam2_hlle;
  double lam3_pp = beta * lam3_roe + (1.0 - beta) * lam3_hlle;
  RFlux Fl = phys_flux(t, L, nx, ny, nz), Fr = phys_flux(t, R, nx, ny, nz);
  F.r = 0.5 * (Fl.r + Fr.r);
  F.u = 0.5 * (Fl.u + Fr.u);
  F.v = 0.5 * (Fl.v + Fr.v);
  F.w = 0.5 * (Fl.w + Fr.w);
  F.E = 0.5 * (Fl.E + Fr.E);
  double drho = R.rho - L.rho, dp = R.p - L.p;
  double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w, dun = unr - unl;
  double t1x, t1y, t1z;
  if (std::fabs(nx) < 0.9) { t1x = 0.0; t1y = -nz; t1z = ny; }
  else { t1x = -nz; t1y = 0.0; t1z = nx; }
  double normt = std::sqrt(t1x * t1x + t1y * t1y + t1z * t1z);
  t1x = t1x / normt; t1y = t1y / normt; t1z = t1z / normt;
  double t2x = ny * t1z - nz * t1y, t2y = nz * t1x - nx * t1z, t2z = nx * t1y - ny * t1x;
  double alpha_m = (dp - rho_roe * a_roe * dun) / (2.0 * a_roe * a_roe);
  double alpha_c = drho - dp / (a_roe * a_roe);
  double alpha_s1 = rho_roe * (du * t1x + dv * t1y + dw * t1z);
  double alpha_s2 = rho_roe * (du * t2x + dv * t2y + dw * t2z);
  double alpha_p = (dp + rho_roe * a_roe * dun) / (2.0 * a_roe * a_roe);
  F.r = F.r - 0.5 * (alpha_c * lam1_pp + alpha_m * lam2_pp + alpha_p * lam3_pp);
  F.u = F.u - 0.5 * (alpha_c * lam1_pp * u_roe);
  F.v = F.v - 0.5 * (alpha_c * lam1_pp * v_roe);
  F.w = F.w - 0.5 * (alpha_c * lam1_pp * w_roe);
  F.u = F.u - 0.5 * lam1_pp * (alpha_s1 * t1x + alpha_s2 * t2x);
  F.v = F.v - 0.5 * lam1_pp * (alpha_s1 * t1y + alpha_s2 * t2y);
  F.w = F.w - 0.5 * lam1_pp * (alpha_s1 * t1z + alpha_s2 * t2z);
  F.u = F.u - 0.5 * (alpha_m * lam2_pp * (u_roe - a_roe * nx) + alpha_p * lam3_pp * (u_roe + a_roe * nx));
  F.v = F.v - 0.5 * (alpha_m * lam2_pp * (v_roe - a_roe * ny) + alpha_p * lam3_pp * (v_roe + a_roe * ny));
  F.w = F.w - 0.5 * (alpha_m * lam2_pp * (w_roe - a_roe * nz) + alpha_p * lam3_pp * (w_roe + a_roe * nz));
  F.E = F.E - 0.5 * lam1_pp * (alpha_c * 0.5 * (u_roe * u_roe + v_roe * v_roe + w_roe * w_roe));
  F.E = F.E - 0.5 * lam1_pp * (alpha_s1 * (u_roe * t1x + v_roe * t1y + w_roe * t1z) +
                               alpha_s2 * (u_roe * t2x + v_roe * t2y + w_roe * t2z));
  F.E = F.E - 0.5 * (alpha_m * lam2_pp * (h0_roe - a_roe * un_roe) + alpha_p * lam3_pp * (h0_roe + a_roe * un_roe));
  return F;
}

// SD_Tramel, Lib_Shock_Detector.f90:9-38 (DELTA = 20): a Jameson-type
// pressure sensor over the six face neighbours
inline double SD_Tramel(double p, double p1, double p2, double p3, double p4, double p5, double p6) {
  const double DELTA = 20.0;
  double kp1 = std::fabs((p2 - 2.0 * p + p1) / (p2 + 2.0 * p + p1));
  double kp2 = std::fabs((p4 - 2.0 * p + p3) / (p4 + 2.0 * p + p3));
  double kp3 = std::fabs((p6 - 2.0 * p + p5) / (p6 + 2.0 * p + p5));
  double sw = std::max(std::max(kp1, kp2), kp3);
  if (sw < 1.0 / DELTA) {
    double phi = std::max(sw / DELTA, 0.0);
    return 1.0 - std::tanh(10.0 * phi * phi * phi);
  }
  return 0.0;
}
// the shock-detector solvers (Mod_Riemann.f90:79-87 set obj_riemann%SD)
inline bool sd_riemann(const orc_domain* d) {
  return d->cfg.riemann == ORC_RIE_HLLC_SD || d->cfg.riemann == ORC_RIE_HLLE_PP;
}
// any shock detector in use (Assign_Setup.f90:43-47)
inline bool sd_any(const orc_domain* d) { return d->cfg.sd_limiter != 0 || sd_riemann(d); }

// riemann_HLLCHLLE ('HLLC Rotated'), Lib_Riemann_HLL.f90:672-755: HLLE along
// n1, the direction of the velocity jump, and HLLC along n2 = (-n1y, n1x,
// n1z), weighted by the projections of the face normal on them (both made
// non-negative); HLLC along the normal where the jump is negligible.
inline RFlux riemann_HLLCrot(const Thermo& t, const RState& L, const RState& R, double nx, double ny, double nz) {
  double abs_dv = std::sqrt((R.u - L.u) * (R.u - L.u) + (R.v - L.v) * (R.v - L.v) + (R.w - L.w) * (R.w - L.w));
  double dum = 0.5 * (std::sqrt(L.u * L.u + L.v * L.v + L.w * L.w) + std::sqrt(R.u * R.u + R.v * R.v + R.w * R.w));
  if (abs_dv / (dum + 1.0e-10) > 1.0e-12) {
    double nx1 = (R.u - L.u) / abs_dv, ny1 = (R.v - L.v) / abs_dv, nz1 = (R.w - L.w) / abs_dv;
    double alfa1 = nx * nx1 + ny * ny1 + nz * nz1;
    double s1 = std::copysign(1.0, alfa1);
    nx1 = s1 * nx1; ny1 = s1 * ny1; nz1 = s1 * nz1; alfa1 = s1 * alfa1;
    double nx2 = -ny1, ny2 = nx1, nz2 = nz1;
    double alfa2 = nx * nx2 + ny * ny2 + nz * nz2;
    double s2 = std::copysign(1.0, alfa2);
    nx2 = s2 * nx2; ny2 = s2 * ny2; nz2 = s2 * nz2; alfa2 = s2 * alfa2;
    if (nz > 0.1) {
      alfa1 = 0.0;
      nx2 = nx; ny2 = ny; nz2 = nz;
      alfa2 = 1.0;
    }
    RFlux E = riemann_HLLE(t, L, R, nx1, ny1, nz1);
    RFlux C = riemann_HLLC(t, L, R, nx2, ny2, nz2);
    RFlux F;
    F.r = E.r * alfa1 + C.r * alfa2;
    F.u = E.u * alfa1 + C.u * alfa2;
    F.v = E.v * alfa1 + C.v * alfa2;
    F.w = E.w * alfa1 + C.w * alfa2;
    if (F.w != 0.0 && std::fabs(nz) <= 1.0e-10) F.w = 0.0;
    F.E = E.E * alfa1 + C.E * alfa2;
    return F;
  }
  return riemann_HLLC(t, L, R, nx, ny, nz);
}

// riemann_exact ('exact'), Lib_Riemann_Godunov.f90:10-224: Newton iteration
// on the contact velocity (relative pressure tolerance 1e-5, at most 1001
// iterations) with shock or rarefaction relations per side, then the
// Godunov state sampled at the face.  The wave speeds that the sampling reads
// (swl, swr, vw1..vw4) keep the value of the last iteration that set them;
// the reference leaves them undefined before that, here they start at 0.
struct ExactWaves { double swl = 0.0, swr = 0.0, vw1 = 0.0, vw2 = 0.0, vw3 = 0.0, vw4 = 0.0; };
inline void exact_rareleft(double ps, double as, double us, double ud, double& pd, double& ad, double& dpr,
                           double& v1, double& v2, double gamma) {             // :153-169
  double delta = 0.5 * (gamma - 1.0);
  double dum1 = 2.0 * gamma / (gamma - 1.0);
  ad = as - delta * (ud - us);
  pd = ps * std::pow(ad / as, dum1);
  dpr = -(gamma * pd / ad);
  v1 = us - as;
  v2 = ud - ad;
}
inline void exact_rareright(double pd, double ad, double ud, double us, double& ps, double& as, double& dpl,
                            double& v3, double& v4, double gamma) {            // :172-188
  double delta = 0.5 * (gamma - 1.0);
  double dum1 = 2.0 * gamma / (gamma - 1.0);
  as = ad + delta * (us - ud);
  ps = pd * std::pow(as / ad, dum1);
  dpl = gamma * ps / as;
  v3 = us + as;
  v4 = ud + ad;
}
inline void exact_shockleft(double us, double as, double ps, double ud, double& ad, double& pd, double& dpr,
                            double& wl, double gamma) {                          // :191-206
  double x1 = (gamma + 1.0) * (ud - us) / (4.0 * as);
  double Mlrel = x1 - std::sqrt(1.0 + x1 * x1);
  double C1 = gamma * ps / as;
  pd = ps + C1 * (ud - us) * Mlrel;
  dpr = 2.0 * C1 * std::pow(Mlrel, 3.0) / (1.0 + Mlrel * Mlrel);
  double rpd = pd / ps;
  wl = us + as * Mlrel;
  ad = as * std::sqrt((gamma + 1.0 + (gamma - 1.0) * rpd) / (gamma + 1.0 + (gamma - 1.0) / rpd));
}
inline void exact_shockright(double ud, double ad, double pd, double us, double& as, double& ps, double& dpl,
                             double& wr, double gamma) {                         // :209-224
  double x4 = (gamma + 1.0) * (us - ud) / (4.0 * ad);
  double Mrrel = x4 + std::sqrt(1.0 + x4 * x4);
  double C4 = gamma * pd / ad;
  ps = pd + C4 * (us - ud) * Mrrel;
  dpl = 2.0 * C4 * std::pow(Mrrel, 3.0) / (1.0 + Mrrel * Mrrel);
  double rps = ps / pd;
  wr = ud + ad * Mrrel;
  as = ad * std::sqrt((gamma + 1.0 + (gamma - 1.0) * rps) / (gamma + 1.0 + (gamma - 1.0) / rps));
}
inline RFlux riemann_exact(const Thermo& t, const RState& L, const RState& R, double nx, double ny, double nz) {
  const double gam1 = t.gamma, gam4 = t.gamma;                                  // f_gamma
  const double p1 = L.p, a1 = L.a, p4 = R.p, a4 = R.a;
  double gm1_1 = gam1 - 1.0, gm1_4 = gam4 - 1.0;
  double delta1 = 0.5 * gm1_1, delta4 = 0.5 * gm1_4;
  double eta1 = gam1 / delta1, eta4 = gam4 / delta4;
  double un1 = L.u * nx + L.v * ny + L.w * nz;
  double ut1 = L.u - un1 * nx, vt1 = L.v - un1 * ny, wt1 = L.w - un1 * nz;
  double un4 = R.u * nx + R.v * ny + R.w * nz;
  double ut4 = R.u - un4 * nx, vt4 = R.v - un4 * ny, wt4 = R.w - un4 * nz;
  double R2I = un1 + (2.0 / gm1_1) * a1;
  double R1IV = un4 - (2.0 / gm1_4) * a4;
  double dum = (p1 < p4) ? gm1_4 / (2.0 * gam4) : gm1_1 / (2.0 * gam1);
  double z = (gm1_1 / gm1_4) * (a4 / a1) * std::pow(p1 / p4, dum);
  double u0 = (z * R2I + R1IV) / (1.0 + z);
  double vel = u0;
  double p3 = 1.0, p2 = 2.0 * p3, a2 = 0.0, a3 = 0.0, dpr = 0.0, dpl = 0.0;
  ExactWaves w;
  int iter = 0;
  while (std::fabs(1.0 - (p2 / p3)) >= 1e-5 && iter <= 1000) {
    if (vel < un1) exact_shockleft(un1, a1, p1, vel, a2, p2, dpr, w.swl, gam1);
    else exact_rareleft(p1, a1, un1, vel, p2, a2, dpr, w.vw1, w.vw2, gam1);
    if (vel > un4) exact_shockright(un4, a4, p4, vel, a3, p3, dpl, w.swr, gam4);
    else exact_rareright(p4, a4, un4, vel, p3, a3, dpl, w.vw3, w.vw4, gam4);
    vel = vel - ((p2 - p3) / (dpr - dpl));
    iter = iter + 1;
  }
  double af, pf, rhof, uf, vf, wf;
  if (vel > 0.0) {
    af = a2; pf = p2;
    if (vel <= un1) {
      if (w.swl > 0.0) { af = a1; vel = un1; pf = p1; }
    } else {
      if (w.vw1 > 0.0) {
        vel = un1; af = a1; pf = p1;
      } else if (w.vw2 > 0.0) {
        af = (un1 + a1 / delta1) / (1.0 + 1.0 / delta1);
        vel = af;
        pf = p1 * std::pow(af / a1, eta1);
      }
    }
    rhof = gam1 * pf / (af * af);
    uf = vel * nx + ut1; vf = vel * ny + vt1; wf = vel * nz + wt1;
  } else {
    af = a3; pf = p3;
    if (vel >= un4) {
      if (w.swr < 0.0) { af = a4; vel = un4; pf = p4; }
    } else {
      if (w.vw4 < 0.0) {
        af = a4; vel = un4; pf = p4;
      } else if (w.vw3 < 0.0) {
        af = -(un4 - a4 / delta4) / (1.0 + 1.0 / delta4);
        vel = -af;
        pf = p4 * std::pow(af / a4, eta4);
      }
    }
    rhof = gam4 * pf / (af * af);
    uf = vel * nx + ut4; vf = vel * ny + vt4; wf = vel * nz + wt4;
  }
  double df = 1.0 * rhof;                                   // dl/dltot*rhof, one species
  RFlux F;
  F.r = rhof * vel;
  F.u = F.r * uf + pf * nx;
  F.v = F.r * vf + pf * ny;
  F.w = F.r * wf + pf * nz;
  F.E = F.r * H0(t, pf, df, std::sqrt(vel * vel));
  return F;
}

// beta: the shock detector of the face (1 at the physical boundary faces,
// which call Riemann with 1d0)
inline RFlux Riemann(const orc_domain* d, const RState& L, const RState& R, double nx,
                     double ny, double nz, double beta = 1.0) {
  switch (d->cfg.riemann) {
    case ORC_RIE_HLLC_SD: return riemann_HLLCSD(d->th, L, R, nx, ny, nz, beta);
    case ORC_RIE_HLLE_PP: return riemann_HLLEpp(d->th, L, R, nx, ny, nz, beta);
    case ORC_RIE_AUSMP: return riemann_AUSMp(d->th, L, R, nx, ny, nz);
    case ORC_RIE_SLAU: return riemann_SLAU(d->th, L, R, nx, ny, nz, false);
    case ORC_RIE_SLAU2: return riemann_SLAU(d->th, L, R, nx, ny, nz, true);
    case ORC_RIE_HLLE: return riemann_HLLE(d->th, L, R, nx, ny, nz);
    case ORC_RIE_HLLEM: return riemann_HLLEM(d->th, L, R, nx, ny, nz);
    case ORC_RIE_LLF: return riemann_LLF(d->th, L, R, nx, ny, nz);
    case ORC_RIE_PLLF: return riemann_PLLF(d->th, L, R, nx, ny, nz);
    case ORC_RIE_HANEL: return riemann_Hanel(d->th, L, R, nx, ny, nz);
    case ORC_RIE_AUSMP_UP: return riemann_AUSMp_up(d->th, L, R, nx, ny, nz, d->cfg.minf, false);
    case ORC_RIE_AUSMP_UP2: return riemann_AUSMp_up(d->th, L, R, nx, ny, nz, d->cfg.minf, true);
    case ORC_RIE_HLLC_ROT: return riemann_HLLCrot(d->th, L, R, nx, ny, nz);
    case ORC_RIE_EXACT: return riemann_exact(d->th, L, R, nx, ny, nz);
    default: return riemann_HLLC(d->th, L, R, nx, ny, nz);
  }
}

inline RState make_state(const Thermo& t, const double* P, bool& bad) {
  // check_gas_state, co_rotot_Rtot and f_ss as in Lib_Convective.f90:45-58
  RState s;
  if (check_gas_state(P[0], P[NP]) != 0) bad = true;
  double rho, R;
  co_rotot_Rtot(t, P[0], rho, R);
  s.d = P[0]; s.u = P[NU]; s.v = P[NV]; s.w = P[NW]; s.p = P[NP];
  s.rho = rho;
  s.a = f_ss(t, P[0], P[NP], rho, R);
  return s;
}

// Reconstruction (elemental), Lib_Reconstruction.f90:10-29, beta = 1
inline void Reconstruction(int lim, const double* prev, const double* local, const double* next,
                           const double* next2, double dl0, double dl1, double dl2, double dll,
                           double dlr, double beta, double* priml, double* primr) {
  for (int v = 0; v < NPRIM; ++v) {
    double slope0 = (local[v] - prev[v]) / dl0;
    double slope1 = (next[v] - local[v]) / dl1;
    double slope2 = (next2[v] - next[v]) / dl2;
    double slopel = rlimiter(lim, slope1, slope0);
    double sloper = rlimiter(lim, slope2, slope1);
    priml[v] = local[v] + beta * slopel * dll;
    primr[v] = next[v] - beta * sloper * dlr;
  }
}

// Species-upwinded flux times area (Lib_Convective.f90:66-75 and the
// identical block of Lib_BC_Fluxes_Connection.f90:95-105).
inline void face_flux(const RFlux& F, double area, const double* p1, double rho1, const double* p4,
                      double rho4, double* Flux) {
  double su = std::copysign(0.5, F.r);
  double sp = 0.5 + su;
  double sm = su - 0.5;
  Flux[0] = F.r * area * (sp * (p1[0] / rho1) - sm * (p4[0] / rho4));
  Flux[NU] = F.u * area;
  Flux[NV] = F.v * area;
  Flux[NW] = F.w * area;
  Flux[NP] = F.E * area;
}

// Convective_Flux, Lib_Convective.f90:10-85
inline bool Convective_Flux(const orc_domain* d, const double* dl /*-1..2*/, const double* N,
                            double area, const double* Pm1, const double* P0, const double* P1,
                            const double* P2, double* R0, double* R1, double beta) {
  double l0 = 0.5 * (dl[0] + dl[1]);
  double l1 = 0.5 * (dl[1] + dl[2]);
  double l2 = 0.5 * (dl[2] + dl[3]);
  double lm = 0.5 * dl[1];
  double lp = 0.5 * dl[2];
  double Prim1[NPRIM], Prim4[NPRIM];
  // :37-42: the limiter scaled by beta under MUSCL-SD, else by 1
  Reconstruction(d->cfg.limiter, Pm1, P0, P1, P2, l0, l1, l2, lm, lp, d->cfg.sd_limiter ? beta : 1.0, Prim1, Prim4);
  bool bad = false;
  RState L = make_state(d->th, Prim1, bad);
  RState R = make_state(d->th, Prim4, bad);
  RFlux F = Riemann(d, L, R, N[0], N[1], N[2], beta);
  double Flux[NPRIM];
  face_flux(F, area, Prim1, L.rho, Prim4, R.rho, Flux);
  for (int v = 0; v < NPRIM; ++v) R0[v] = R0[v] + Flux[v];
  for (int v = 0; v < NPRIM; ++v) R1[v] = R1[v] - Flux[v];
  return !bad;
}

// ---------------------------------------------------------------------------
// Metrics: Lib_Metrics.f90
// ---------------------------------------------------------------------------
inline double tvol(const double* vx, const double* vy, const double* vz, int i1, int i2, int i3,
                   int i4) {
  --i1; --i2; --i3; --i4;
  return std::fabs(((vx[i2] - vx[i1]) * ((vy[i3] - vy[i1]) * (vz[i4] - vz[i1]) - (vy[i4] - vy[i1]) * (vz[i3] - vz[i1])) +
                    (vy[i2] - vy[i1]) * ((vx[i4] - vx[i1]) * (vz[i3] - vz[i1]) - (vx[i3] - vx[i1]) * (vz[i4] - vz[i1])) +
                    (vz[i2] - vz[i1]) * ((vx[i3] - vx[i1]) * (vy[i4] - vy[i1]) - (vx[i4] - vx[i1]) * (vy[i3] - vy[i1]))) /
                   6.0);
}

// Compute_Metric_Tensor, Lib_Metrics.f90:250-376.  Mout: c(3,3) column-major.
inline bool Compute_Metric_Tensor(const Vec3& N1, const Vec3& N2, const Vec3& N3, const Vec3& N4,
                                  const Vec3& N5, const Vec3& N6, const Vec3& N7, const Vec3& N8,
                                  double* Mout, double* dlout, double* volout) {
  double A[3][3];
  for (int c = 0; c < 3; ++c) {
    A[0][c] = N5.c[c] - N1.c[c] + N6.c[c] - N2.c[c] + N7.c[c] - N3.c[c] + N8.c[c] - N4.c[c];
    A[1][c] = N3.c[c] - N1.c[c] + N4.c[c] - N2.c[c] + N7.c[c] - N5.c[c] + N8.c[c] - N6.c[c];
    A[2][c] = N2.c[c] - N1.c[c] + N4.c[c] - N3.c[c] + N6.c[c] - N5.c[c] + N8.c[c] - N7.c[c];
  }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[r][c] = 0.25 * A[r][c];
  double det = A[0][0] * A[1][1] * A[2][2] - A[0][0] * A[1][2] * A[2][1] -
               A[0][1] * A[1][0] * A[2][2] + A[0][1] * A[1][2] * A[2][0] +
               A[0][2] * A[1][0] * A[2][1] - A[0][2] * A[1][1] * A[2][0];
  bool ok = true;
  if (std::fabs(det) == 0.0) {
    ok = false;
    for (int q = 0; q < 9; ++q) Mout[q] = 0.0;
    Mout[0] = Mout[4] = Mout[8] = 1.0;
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
      for (int c = 0; c < 3; ++c) Mout[r + 3 * c] = cof[r][c] / det;
  }
  for (int h = 0; h < 3; ++h) dlout[h] = std::sqrt(A[h][0] * A[h][0] + A[h][1] * A[h][1] + A[h][2] * A[h][2]);
  double vx[8], vy[8], vz[8];
  const Vec3* order[8] = {&N1, &N5, &N3, &N7, &N2, &N6, &N4, &N8};
  for (int q = 0; q < 8; ++q) { vx[q] = order[q]->c[0]; vy[q] = order[q]->c[1]; vz[q] = order[q]->c[2]; }
  double v = tvol(vx, vy, vz, 1, 2, 3, 5) + tvol(vx, vy, vz, 2, 4, 3, 8) + tvol(vx, vy, vz, 5, 8, 6, 2) +
             tvol(vx, vy, vz, 5, 7, 8, 3) + tvol(vx, vy, vz, 5, 8, 2, 3);
  *volout = v;
  if (v <= 0.0) ok = false;
  return ok;
}

inline Vec3 sub(const Vec3& a, const Vec3& b) { return Vec3{{a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]}}; }
inline Vec3 lin3(const Vec3& a, const Vec3& b, const Vec3& c) {   // 3a - 3b + c
  Vec3 r;
  for (int q = 0; q < 3; ++q) r.c[q] = 3.0 * a.c[q] - 3.0 * b.c[q] + c.c[q];
  return r;
}
inline Vec3 lin2(const Vec3& a, const Vec3& b) {                  // 2a - b
  Vec3 r;
  for (int q = 0; q < 3; ++q) r.c[q] = 2.0 * a.c[q] - b.c[q];
  return r;
}

bool cmt_store(Block& B, int i, int j, int k, const Vec3& N1, const Vec3& N2, const Vec3& N3,
               const Vec3& N4, const Vec3& N5, const Vec3& N6, const Vec3& N7, const Vec3& N8) {
  return Compute_Metric_Tensor(N1, N2, N3, N4, N5, N6, N7, N8, &B.M[9 * B.cell(i, j, k)],
                               &B.dl[3 * B.cell(i, j, k)], &B.vol[B.cell(i, j, k)]);
}

// Compute_Norm_Area, Lib_Metrics.f90:69-247
void Compute_Norm_Area(Block& b) {
  int im = b.ni, jm = b.nj, km = b.nk;
  auto cross = [](const Vec3& d1, const Vec3& d2, double* d3) {
    d3[0] = (d1.c[1] * d2.c[2] - d1.c[2] * d2.c[1]);
    d3[1] = (d1.c[2] * d2.c[0] - d1.c[0] * d2.c[2]);
    d3[2] = (d1.c[0] * d2.c[1] - d1.c[1] * d2.c[0]);
  };
  auto avg4 = [](const Vec3& a, const Vec3& bb, const Vec3& c, const Vec3& d) {
    Vec3 r;
    for (int q = 0; q < 3; ++q) r.c[q] = 0.25 * (a.c[q] + bb.c[q] + c.c[q] + d.c[q]);
    return r;
  };
  double d3[3], sn[3];
  // i direction sign
  cross(sub(b.nd(1, 1, 1), b.nd(1, 0, 0)), sub(b.nd(1, 0, 1), b.nd(1, 1, 0)), sn);
  Vec3 c1 = avg4(b.nd(1, 1, 1), b.nd(1, 0, 1), b.nd(1, 0, 0), b.nd(1, 1, 0));
  Vec3 c2 = avg4(b.nd(0, 1, 1), b.nd(0, 0, 1), b.nd(0, 0, 0), b.nd(0, 1, 0));
  Vec3 dd = sub(c1, c2);
  double signi = std::copysign(1.0, dd.c[0] * sn[0] + dd.c[1] * sn[1] + dd.c[2] * sn[2]);
  // j direction sign
  cross(sub(b.nd(0, 1, 1), b.nd(1, 1, 0)), sub(b.nd(1, 1, 1), b.nd(0, 1, 0)), sn);
  c1 = avg4(b.nd(1, 1, 1), b.nd(0, 1, 1), b.nd(0, 1, 0), b.nd(1, 1, 0));
  c2 = avg4(b.nd(1, 0, 1), b.nd(0, 0, 1), b.nd(0, 0, 0), b.nd(1, 0, 0));
  dd = sub(c1, c2);
  double signj = std::copysign(1.0, dd.c[0] * sn[0] + dd.c[1] * sn[1] + dd.c[2] * sn[2]);
  // k direction sign
  cross(sub(b.nd(0, 1, 1), b.nd(1, 0, 1)), sub(b.nd(0, 0, 1), b.nd(1, 1, 1)), sn);
  c1 = avg4(b.nd(1, 1, 1), b.nd(0, 1, 1), b.nd(0, 0, 1), b.nd(1, 0, 1));
  c2 = avg4(b.nd(1, 1, 0), b.nd(0, 1, 0), b.nd(0, 0, 0), b.nd(1, 0, 0));
  dd = sub(c1, c2);
  double signk = std::copysign(1.0, dd.c[0] * sn[0] + dd.c[1] * sn[1] + dd.c[2] * sn[2]);

  auto store = [&](int dir, size_t f, double sgn) {
    for (int q = 0; q < 3; ++q) d3[q] = d3[q] * 0.5;
    double A = std::sqrt(d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2]);
    double n[3];
    if (A == 0.0) { n[0] = n[1] = n[2] = 0.0; }
    else for (int q = 0; q < 3; ++q) n[q] = d3[q] / A * sgn;
    b.fA[dir][f] = A;
    for (int q = 0; q < 3; ++q) b.fN[dir][3 * f + q] = n[q];
  };
  for (int k = 1; k <= km; ++k)
    for (int j = 1; j <= jm; ++j)
      for (int i = 0; i <= im; ++i) {
        cross(sub(b.nd(i, j, k), b.nd(i, j - 1, k - 1)), sub(b.nd(i, j - 1, k), b.nd(i, j, k - 1)), d3);
        store(0, b.face(1, i, j, k), signi);
      }
  for (int k = 1; k <= km; ++k)
    for (int j = 0; j <= jm; ++j)
      for (int i = 1; i <= im; ++i) {
        cross(sub(b.nd(i - 1, j, k), b.nd(i, j, k - 1)), sub(b.nd(i, j, k), b.nd(i - 1, j, k - 1)), d3);
        store(1, b.face(2, i, j, k), signj);
      }
  for (int k = 0; k <= km; ++k)
    for (int j = 1; j <= jm; ++j)
      for (int i = 1; i <= im; ++i) {
        cross(sub(b.nd(i - 1, j, k), b.nd(i, j - 1, k)), sub(b.nd(i - 1, j - 1, k), b.nd(i, j, k)), d3);
        store(2, b.face(3, i, j, k), signk);
      }
}

// BC_Extrapolate_Metrics, Lib_Metrics.f90:535-797 (delthe == 0 branches)
bool BC_Extrapolate_Metrics(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& b) {
  const int gc = GC;
  Vec3 N[8][2 * GC + 1];   // N[q][g + gc], q = 0..7 for N1..N8
  auto at = [&](int q, int g) -> Vec3& { return N[q][g + gc]; };
  bool ok = true;
  switch (Fm) {
    case 1:
      for (int g = 0; g <= gc; ++g) {
        at(0, g) = b.nd(Im + g - 1, Jm - 1, Km - 1);
        at(1, g) = b.nd(Im + g - 1, Jm - 1, Km);
        at(2, g) = b.nd(Im + g - 1, Jm, Km - 1);
        at(3, g) = b.nd(Im + g - 1, Jm, Km);
      }
      for (int g = -1; g >= -gc; --g) {
        for (int q = 0; q < 4; ++q) at(q, g) = lin3(at(q, g + 1), at(q, g + 2), at(q, g + 3));
        ok &= cmt_store(b, Im + g, Jm, Km, at(0, g), at(1, g), at(2, g), at(3, g), at(0, g + 1), at(1, g + 1),
                        at(2, g + 1), at(3, g + 1));
      }
      break;
    case 2:
      for (int g = 0; g >= -gc; --g) {
        at(4, g) = b.nd(Im + g, Jm - 1, Km - 1);
        at(5, g) = b.nd(Im + g, Jm - 1, Km);
        at(6, g) = b.nd(Im + g, Jm, Km - 1);
        at(7, g) = b.nd(Im + g, Jm, Km);
      }
      for (int g = 1; g <= gc; ++g) {
        for (int q = 4; q < 8; ++q) at(q, g) = lin3(at(q, g - 1), at(q, g - 2), at(q, g - 3));
        ok &= cmt_store(b, Im + g, Jm, Km, at(4, g - 1), at(5, g - 1), at(6, g - 1), at(7, g - 1), at(4, g), at(5, g),
                        at(6, g), at(7, g));
      }
      break;
    case 3: {
      bool cubic = b.nj > 2;
      int gtop = cubic ? gc : 1;
      for (int g = 0; g <= gtop; ++g) {
        at(0, g) = b.nd(Im - 1, Jm + g - 1, Km - 1);
        at(1, g) = b.nd(Im - 1, Jm + g - 1, Km);
        at(4, g) = b.nd(Im, Jm + g - 1, Km - 1);
        at(5, g) = b.nd(Im, Jm + g - 1, Km);
      }
      for (int g = -1; g >= -gc; --g) {
        for (int q : {0, 1, 4, 5})
          at(q, g) = cubic ? lin3(at(q, g + 1), at(q, g + 2), at(q, g + 3)) : lin2(at(q, g + 1), at(q, g + 2));
        ok &= cmt_store(b, Im, Jm + g, Km, at(0, g), at(1, g), at(0, g + 1), at(1, g + 1), at(4, g), at(5, g),
                        at(4, g + 1), at(5, g + 1));
      }
      break;
    }
    case 4: {
      bool cubic = b.nj > 2;
      int gbot = cubic ? -gc : -1;
      for (int g = 0; g >= gbot; --g) {
        at(2, g) = b.nd(Im - 1, Jm + g, Km - 1);
        at(3, g) = b.nd(Im - 1, Jm + g, Km);
        at(6, g) = b.nd(Im, Jm + g, Km - 1);
        at(7, g) = b.nd(Im, Jm + g, Km);
      }
      for (int g = 1; g <= gc; ++g) {
        for (int q : {2, 3, 6, 7})
          at(q, g) = cubic ? lin3(at(q, g - 1), at(q, g - 2), at(q, g - 3)) : lin2(at(q, g - 1), at(q, g - 2));
        ok &= cmt_store(b, Im, Jm + g, Km, at(2, g - 1), at(3, g - 1), at(2, g), at(3, g), at(6, g - 1), at(7, g - 1),
                        at(6, g), at(7, g));
      }
      break;
    }
    case 5: {
      bool cubic = (D->ndir == 3);
      int gtop = cubic ? gc : 1;
      for (int g = 0; g <= gtop; ++g) {
        at(0, g) = b.nd(Im - 1, Jm - 1, Km + g - 1);
        at(2, g) = b.nd(Im - 1, Jm, Km + g - 1);
        at(4, g) = b.nd(Im, Jm - 1, Km + g - 1);
        at(6, g) = b.nd(Im, Jm, Km + g - 1);
      }
      for (int g = -1; g >= -gc; --g) {
        for (int q : {0, 2, 4, 6})
          at(q, g) = cubic ? lin3(at(q, g + 1), at(q, g + 2), at(q, g + 3)) : lin2(at(q, g + 1), at(q, g + 2));
        ok &= cmt_store(b, Im, Jm, Km + g, at(0, g), at(0, g + 1), at(2, g), at(2, g + 1), at(4, g), at(4, g + 1),
                        at(6, g), at(6, g + 1));
      }
      break;
    }
    case 6: {
      bool cubic = (D->ndir == 3);
      int gbot = cubic ? -gc : -1;
      for (int g = 0; g >= gbot; --g) {
        at(1, g) = b.nd(Im - 1, Jm - 1, Km + g);
        at(3, g) = b.nd(Im - 1, Jm, Km + g);
        at(5, g) = b.nd(Im, Jm - 1, Km + g);
        at(7, g) = b.nd(Im, Jm, Km + g);
      }
      for (int g = 1; g <= gc; ++g) {
        for (int q : {1, 3, 5, 7})
          at(q, g) = cubic ? lin3(at(q, g - 1), at(q, g - 2), at(q, g - 3)) : lin2(at(q, g - 1), at(q, g - 2));
        ok &= cmt_store(b, Im, Jm, Km + g, at(1, g - 1), at(1, g), at(3, g - 1), at(3, g), at(5, g - 1), at(5, g),
                        at(7, g - 1), at(7, g));
      }
      break;
    }
  }
  return ok;
}

// BC_Symmetry_Metrics, Lib_Metrics.f90:800-857
void BC_Symmetry_Metrics(int Im, int Jm, int Km, int Fm, Block& b) {
  for (int g = 1; g <= GC; ++g) {
    int gi = Im, gj = Jm, gk = Km, si = Im, sj = Jm, sk = Km;
    switch (Fm) {
      case 1: gi = Im - g; si = Im + g - 1; break;
      case 2: gi = Im + g; si = Im - g + 1; break;
      case 3: gj = Jm - g; sj = Jm + g - 1; break;
      case 4: gj = Jm + g; sj = Jm - g + 1; break;
      case 5: gk = Km - g; sk = Km + g - 1; break;
      case 6: gk = Km + g; sk = Km - g + 1; break;
    }
    size_t dst = b.cell(gi, gj, gk), src = b.cell(si, sj, sk);
    for (int q = 0; q < 9; ++q) b.M[9 * dst + q] = b.M[9 * src + q];
    for (int q = 0; q < 3; ++q) b.dl[3 * dst + q] = b.dl[3 * src + q];
    b.vol[dst] = b.vol[src];
  }
}

// BC_Connect_Metrics, Lib_Metrics.f90:860-1092
bool BC_Connect_Metrics(int Im, int Jm, int Km, int Fm, Block& bm, int Is, int Js, int Ks, int Fs,
                        const Block& bs, int d11s, int d12s, int d21s, int d22s) {
  const int guides[6][3] = {{0, 0, 0}, {-1, 0, 0}, {0, 0, 0}, {0, -1, 0}, {0, 0, 0}, {0, 0, -1}};
  const int guides2[6][3] = {{1, 0, 0}, {-2, 0, 0}, {0, 1, 0}, {0, -2, 0}, {0, 0, 1}, {0, 0, -2}};
  Vec3 N[8][GC + 1];
  switch (Fm) {
    case 1: N[0][0] = bm.nd(Im - 1, Jm - 1, Km - 1); N[1][0] = bm.nd(Im - 1, Jm - 1, Km);
            N[2][0] = bm.nd(Im - 1, Jm, Km - 1); N[3][0] = bm.nd(Im - 1, Jm, Km); break;
    case 2: N[4][0] = bm.nd(Im, Jm - 1, Km - 1); N[5][0] = bm.nd(Im, Jm - 1, Km);
            N[6][0] = bm.nd(Im, Jm, Km - 1); N[7][0] = bm.nd(Im, Jm, Km); break;
    case 3: N[0][0] = bm.nd(Im - 1, Jm - 1, Km - 1); N[1][0] = bm.nd(Im - 1, Jm - 1, Km);
            N[4][0] = bm.nd(Im, Jm - 1, Km - 1); N[5][0] = bm.nd(Im, Jm - 1, Km); break;
    case 4: N[2][0] = bm.nd(Im - 1, Jm, Km - 1); N[3][0] = bm.nd(Im - 1, Jm, Km);
            N[6][0] = bm.nd(Im, Jm, Km - 1); N[7][0] = bm.nd(Im, Jm, Km); break;
    case 5: N[0][0] = bm.nd(Im - 1, Jm - 1, Km - 1); N[2][0] = bm.nd(Im - 1, Jm, Km - 1);
            N[4][0] = bm.nd(Im, Jm - 1, Km - 1); N[6][0] = bm.nd(Im, Jm, Km - 1); break;
    case 6: N[1][0] = bm.nd(Im - 1, Jm - 1, Km); N[3][0] = bm.nd(Im - 1, Jm, Km);
            N[5][0] = bm.nd(Im, Jm - 1, Km); N[7][0] = bm.nd(Im, Jm, Km); break;
  }
  bool ok = true;
  for (int g = 1; g <= GC; ++g) {
    int Is1 = Is + (GC - g) * guides[Fs - 1][0] + (g - 1) * guides2[Fs - 1][0];
    int Js1 = Js + (GC - g) * guides[Fs - 1][1] + (g - 1) * guides2[Fs - 1][1];
    int Ks1 = Ks + (GC - g) * guides[Fs - 1][2] + (g - 1) * guides2[Fs - 1][2];
    int II, JJ, KK;
    if (Fs <= 2) { II = Is1; JJ = (2 * Js1 + d11s + d21s) / 2; KK = (2 * Ks1 + d12s + d22s) / 2; }
    else if (Fs <= 4) { II = (2 * Is1 + d11s + d21s) / 2; JJ = Js1; KK = (2 * Ks1 + d12s + d22s) / 2; }
    else { II = (2 * Is1 + d11s + d21s) / 2; JJ = (2 * Js1 + d12s + d22s) / 2; KK = Ks1; }
    const int slotA[6] = {3, 7, 5, 7, 6, 7};   // N4, N8, N6, N8, N7, N8
    N[slotA[Fm - 1]][g] = bs.nd(II, JJ, KK);
    int III, JJJ, KKK;
    if (Fs <= 2) { III = II; JJJ = JJ - d11s; KKK = KK - d12s; }
    else if (Fs <= 4) { III = II - d11s; JJJ = JJ; KKK = KK - d12s; }
    else { III = II - d11s; JJJ = JJ - d12s; KKK = KK; }
    const int slotB[6] = {1, 5, 1, 3, 2, 3};   // N2, N6, N2, N4, N3, N4
    N[slotB[Fm - 1]][g] = bs.nd(III, JJJ, KKK);
    if (Fs <= 2) { III = II; JJJ = JJ - d21s; KKK = KK - d22s; }
    else if (Fs <= 4) { III = II - d21s; JJJ = JJ; KKK = KK - d22s; }
    else { III = II - d21s; JJJ = JJ - d22s; KKK = KK; }
    const int slotC[6] = {2, 6, 4, 6, 4, 5};   // N3, N7, N5, N7, N5, N6
    N[slotC[Fm - 1]][g] = bs.nd(III, JJJ, KKK);
    if (Fs <= 2) { III = II; JJJ = JJ - d11s - d21s; KKK = KK - d12s - d22s; }
    else if (Fs <= 4) { III = II - d11s - d21s; JJJ = JJ; KKK = KK - d12s - d22s; }
    else { III = II - d11s - d21s; JJJ = JJ - d12s - d22s; KKK = KK; }
    const int slotD[6] = {0, 4, 0, 2, 0, 1};   // N1, N5, N1, N3, N1, N2
    N[slotD[Fm - 1]][g] = bs.nd(III, JJJ, KKK);
    switch (Fm) {
      case 1: ok &= cmt_store(bm, Im - g, Jm, Km, N[0][g], N[1][g], N[2][g], N[3][g], N[0][g - 1], N[1][g - 1], N[2][g - 1], N[3][g - 1]); break;
      case 2: ok &= cmt_store(bm, Im + g, Jm, Km, N[4][g - 1], N[5][g - 1], N[6][g - 1], N[7][g - 1], N[4][g], N[5][g], N[6][g], N[7][g]); break;
      case 3: ok &= cmt_store(bm, Im, Jm - g, Km, N[0][g], N[1][g], N[0][g - 1], N[1][g - 1], N[4][g], N[5][g], N[4][g - 1], N[5][g - 1]); break;
      case 4: ok &= cmt_store(bm, Im, Jm + g, Km, N[2][g - 1], N[3][g - 1], N[2][g], N[3][g], N[6][g - 1], N[7][g - 1], N[6][g], N[7][g]); break;
      case 5: ok &= cmt_store(bm, Im, Jm, Km - g, N[0][g], N[0][g - 1], N[2][g], N[2][g - 1], N[4][g], N[4][g - 1], N[6][g], N[6][g - 1]); break;
      case 6: ok &= cmt_store(bm, Im, Jm, Km + g, N[1][g - 1], N[1][g], N[3][g - 1], N[3][g], N[5][g - 1], N[5][g], N[7][g - 1], N[7][g]); break;
    }
  }
  return ok;
}

// Face_Index, Lib_BC_Fluxes.f90:22-45
inline void Face_Index(int face, int ci, int cj, int ck, int& dir, int& fi, int& fj, int& fk) {
  fi = ci; fj = cj; fk = ck;
  if (face <= 2) { dir = 1; fi = ci - face % 2; }
  else if (face <= 4) { dir = 2; fj = cj - face % 2; }
  else { dir = 3; fk = ck - face % 2; }
}

// ---------------------------------------------------------------------------
// Ghost cells: Lib_Ghost.f90
// ---------------------------------------------------------------------------
void Ghost_Connection(int Im, int Jm, int Km, int Fm, Block& bm, int Is, int Js, int Ks, int Fs,
                      const Block& bs) {                     // :140-160
  for (int g = 1; g <= GC; ++g) {
    int Ig = Im - G(Fm, 1) * g, Jg = Jm - G(Fm, 2) * g, Kg = Km - G(Fm, 3) * g;
    const double* src = &bs.P[NPRIM * bs.cell(Is + G(Fs, 1) * (g - 1), Js + G(Fs, 2) * (g - 1),
                                              Ks + G(Fs, 3) * (g - 1))];
    double* dst = bm.Pc(Ig, Jg, Kg);
    for (int v = 0; v < NPRIM; ++v) dst[v] = src[v];
  }
}

void Ghost_Symmetry(int Im, int Jm, int Km, int Fm, Block& b) {   // :193-225
  int Ig = Im - G(Fm, 1), Jg = Jm - G(Fm, 2), Kg = Km - G(Fm, 3);
  const double* normal;
  if (Fm <= 2) normal = &b.fN[0][3 * b.face(1, Im - Fm % 2, Jm, Km)];
  else if (Fm <= 4) normal = &b.fN[1][3 * b.face(2, Im, Jm - Fm % 2, Km)];
  else normal = &b.fN[2][3 * b.face(3, Im, Jm, Km - Fm % 2)];
  double* pm = b.Pc(Im, Jm, Km);
  double* pg = b.Pc(Ig, Jg, Kg);
  double vel[3] = {pm[NU], pm[NV], pm[NW]};
  double udotn = dot3(vel, normal);
  for (int q = 0; q < 3; ++q) vel[q] = vel[q] - 2.0 * udotn * normal[q];
  pg[NU] = vel[0]; pg[NV] = vel[1]; pg[NW] = vel[2];
  pg[0] = pm[0];
  pg[NP] = pm[NP];
}

void Ghost_ZG_Extrapolate(int Im, int Jm, int Km, int Fm, Block& b) {   // :279-304
  for (int g = 1; g <= GC; ++g) {
    double* dst = nullptr;
    switch (Fm) {
      case 1: dst = b.Pc(Im - g, Jm, Km); break;
      case 2: dst = b.Pc(Im + g, Jm, Km); break;
      case 3: dst = b.Pc(Im, Jm - g, Km); break;
      case 4: dst = b.Pc(Im, Jm + g, Km); break;
      case 5: dst = b.Pc(Im, Jm, Km - g); break;
      case 6: dst = b.Pc(Im, Jm, Km + g); break;
    }
    const double* src = b.Pc(Im, Jm, Km);
    for (int v = 0; v < NPRIM; ++v) dst[v] = src[v];
  }
}

void Ghost_Extrapolate(int Im, int Jm, int Km, int Fm, Block& b) {   // :363-402
  for (int g = 1; g <= GC; ++g) {
    int di = -G(Fm, 1), dj = -G(Fm, 2), dk = -G(Fm, 3);   // outward step
    double* dst = b.Pc(Im + di * g, Jm + dj * g, Km + dk * g);
    const double* a = b.Pc(Im + di * (g - 1), Jm + dj * (g - 1), Km + dk * (g - 1));
    const double* c = b.Pc(Im + di * (g - 2), Jm + dj * (g - 2), Km + dk * (g - 2));
    const double* e = b.Pc(Im + di * (g - 3), Jm + dj * (g - 3), Km + dk * (g - 3));
    for (int v = 0; v < NPRIM; ++v) dst[v] = 3.0 * a[v] - 3.0 * c[v] + e[v];
  }
}

// ---------------------------------------------------------------------------
// Boundary fluxes
// ---------------------------------------------------------------------------
inline void compute_modfm(int fm, int& modfm, int& modfm1, int& modfm2) {   // Lib_BC_Fluxes.f90:9-19
  modfm = fm % 2;
  modfm1 = 1 - modfm;
  modfm2 = 1 - 2 * modfm;
}

bool BC_Connection_Eul(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk) {
  // Lib_BC_Fluxes_Connection.f90:13-114
  int modfm, modfm1, modfm2, dir, fi, fj, fk;
  compute_modfm(Fm, modfm, modfm1, modfm2);
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  int I1 = modfm * (Im - G(Fm, 1) * GC) + modfm1 * (Im + G(Fm, 1));
  int J1 = modfm * (Jm - G(Fm, 2) * GC) + modfm1 * (Jm + G(Fm, 2));
  int K1 = modfm * (Km - G(Fm, 3) * GC) + modfm1 * (Km + G(Fm, 3));
  int I2 = modfm1 * Im + modfm * (Im - G(Fm, 1));
  int J2 = modfm1 * Jm + modfm * (Jm - G(Fm, 2));
  int K2 = modfm1 * Km + modfm * (Km - G(Fm, 3));
  int I3 = modfm1 * (Im - G(Fm, 1)) + modfm * Im;
  int J3 = modfm1 * (Jm - G(Fm, 2)) + modfm * Jm;
  int K3 = modfm1 * (Km - G(Fm, 3)) + modfm * Km;
  int I4 = modfm1 * (Im - G(Fm, 1) * GC) + modfm * (Im + G(Fm, 1));
  int J4 = modfm1 * (Jm - G(Fm, 2) * GC) + modfm * (Jm + G(Fm, 2));
  int K4 = modfm1 * (Km - G(Fm, 3) * GC) + modfm * (Km + G(Fm, 3));
  const double* Prim1 = blk.Pc(I1, J1, K1);
  const double* Prim2 = blk.Pc(I2, J2, K2);
  const double* Prim3 = blk.Pc(I3, J3, K3);
  const double* Prim4 = blk.Pc(I4, J4, K4);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  double Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  double Dl1 = blk.dl_(dir, I1, J1, K1) * 0.5;
  double Dl2 = blk.dl_(dir, I2, J2, K2) * 0.5;
  double Dl3 = blk.dl_(dir, I3, J3, K3) * 0.5;
  double Dl4 = blk.dl_(dir, I4, J4, K4) * 0.5;
  double Dist23 = Dl2 + Dl3;
  double Dist12 = Dl1 + Dl2;
  double Dist34 = Dl3 + Dl4;
  double PL[NPRIM], PR[NPRIM];
  // :58-62 / :85-89: the boundary cell's shock detector under MUSCL-SD / an
  // SD Riemann solver, else 1
  const double beta_cell = blk.beta[blk.inner(Im, Jm, Km)];
  Reconstruction(D->cfg.limiter, Prim1, Prim2, Prim3, Prim4, Dist12, Dist23, Dist34, Dl2, Dl3,
                 D->cfg.sd_limiter ? beta_cell : 1.0, PL, PR);
  bool bad = false;   // the connection flux does not call check_gas_state
  RState L = make_state(D->th, PL, bad);
  RState R = make_state(D->th, PR, bad);
  RFlux F = Riemann(D, L, R, Normal[0], Normal[1], Normal[2], sd_riemann(D) ? beta_cell : 1.0);
  double su = std::copysign(0.5, F.r);
  double sel_L = 0.5 + su, sel_R = su - 0.5;
  double Fmass = F.r * Area;
  double Flux[NPRIM];
  Flux[0] = Fmass * (sel_L * PL[0] / L.rho - sel_R * PR[0] / R.rho);
  Flux[NU] = F.u * Area;
  Flux[NV] = F.v * Area;
  Flux[NW] = F.w * Area;
  Flux[NP] = F.E * Area;
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] + Flux[v] * (double)modfm2;
  return true;
}

void BC_Extrapolation(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk) {
  // Lib_BC_Fluxes_Extrapolation.f90:13-47
  int dir, fi, fj, fk;
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  double Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  const double* Prim = blk.Pc(Im, Jm, Km);
  double vel[3] = {Prim[NU], Prim[NV], Prim[NW]};
  double Un = dot3(vel, Normal);
  double Flux[NPRIM];
  Flux[0] = Prim[0] * Un * Area;
  double Fmass = Flux[0];
  for (int q = 0; q < 3; ++q) Flux[NU + q] = Fmass * vel[q] + Prim[NP] * Area * Normal[q];
  Flux[NP] = Fmass * H0(D->th, Prim[NP], Prim[0], norm2(vel[0], vel[1], vel[2]));
  int FluxSign = 1 - 2 * (Fm % 2);
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] + (double)FluxSign * Flux[v];
}

void BC_Symmetry_Eul(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk) {
  // Lib_BC_Fluxes_Symmetry.f90:14-125 (Un_wall = 0: no rotating frame)
  int modfm, modfm1, modfm2, dir, fi, fj, fk;
  compute_modfm(Fm, modfm, modfm1, modfm2);
  int Ii = Im + G(Fm, 1), Ij = Jm + G(Fm, 2), Ik = Km + G(Fm, 3);
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const double* normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  double area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  double Bound_Dl = 0.5 * blk.dl_(dir, Im, Jm, Km);
  double Int_Dl = 0.5 * blk.dl_(dir, Ii, Ij, Ik);
  const double* Bound = blk.Pc(Im, Jm, Km);
  const double* Int = blk.Pc(Ii, Ij, Ik);
  double bvel[3] = {Bound[NU], Bound[NV], Bound[NW]};
  double Un = dot3(bvel, normal);
  double Ghost[NPRIM];
  for (int v = 0; v < NPRIM; ++v) Ghost[v] = Bound[v];
  for (int q = 0; q < 3; ++q) Ghost[NU + q] = Ghost[NU + q] - 2.0 * Un * normal[q];
  double fm = (double)modfm, fm1 = (double)modfm1;
  double Prim1[NPRIM], Prim3[NPRIM];
  for (int v = 0; v < NPRIM; ++v) Prim1[v] = fm * Ghost[v] + fm1 * Int[v];
  double Dist12 = 2.0 * Bound_Dl * fm + (Bound_Dl + Int_Dl) * fm1;
  for (int v = 0; v < NPRIM; ++v) Prim3[v] = fm * Int[v] + fm1 * Ghost[v];
  double Dist23 = (Bound_Dl + Int_Dl) * fm + 2.0 * Bound_Dl * fm1;
  double Slope[NPRIM];
  for (int v = 0; v < NPRIM; ++v) {
    double s32 = (Prim3[v] - Bound[v]) / Dist23;
    double s21 = (Bound[v] - Prim1[v]) / Dist12;
    Slope[v] = rlimiter(D->cfg.limiter, s32, s21);
  }
  double Dist = Bound_Dl * (double)modfm2;
  double Face[NPRIM];
  for (int v = 0; v < NPRIM; ++v) Face[v] = Bound[v] + Slope[v] * Dist;
  double rotot, Rtot;
  co_rotot_Rtot(D->th, Face[0], rotot, Rtot);
  double Sound = f_ss(D->th, Face[0], Face[NP], rotot, Rtot);
  double fvel[3] = {Face[NU], Face[NV], Face[NW]};
  Un = dot3(fvel, normal);
  double Velt[3];
  for (int q = 0; q < 3; ++q) Velt[q] = fvel[q] - Un * normal[q];
  double Un1 = Un * (double)modfm2;
  double U1[3], U4[3];
  for (int q = 0; q < 3; ++q) { U1[q] = Un1 * normal[q] + Velt[q]; U4[q] = -Un1 * normal[q] + Velt[q]; }
  RState L{Face[0], U1[0], U1[1], U1[2], Face[NP], Sound, rotot};
  RState R{Face[0], U4[0], U4[1], U4[2], Face[NP], Sound, rotot};
  RFlux F = Riemann(D, L, R, normal[0], normal[1], normal[2]);
  double Flux[3] = {F.u * area, F.v * area, F.w * area};
  double* r = blk.Rc(Im, Jm, Km);
  for (int q = 0; q < 3; ++q) r[NU + q] = r[NU + q] + (double)modfm2 * Flux[q];
}

// BC_Inlet_Supersonic_Static + Supersonic_Inflow, Lib_BC_Fluxes_Inflow.f90:244-382.
// Returns false when BC_Sign*Un >= 0 (the caller falls back to symmetry).
bool BC_Inlet_Supersonic(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk,
                         const double* data) {
  const Thermo& t = D->th;
  double BC_Mach = data[0], BC_T0 = data[1], BC_p0 = data[2], BC_alpha = data[3],
         BC_beta = data[4], BC_rel_fac = data[5];
  int modfm, modfm1, modfm2, dir, fi, fj, fk;
  compute_modfm(Fm, modfm, modfm1, modfm2);
  int Ii = Im + G(Fm, 1), Ij = Jm + G(Fm, 2), Ik = Km + G(Fm, 3);
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const double* Prim2 = blk.Pc(Im, Jm, Km);
  const double* Int = blk.Pc(Ii, Ij, Ik);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  double Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  double BC_Sign = (double)modfm2;
  double vel2[3] = {Prim2[NU], Prim2[NV], Prim2[NW]};
  double Un = dot3(vel2, Normal);
  if (BC_Sign * Un >= 0.0) return false;
  // Supersonic_Inflow
  double flow_Rgas = t.R;
  double flow_Sound = f_ss(t, Prim2[0], Prim2[NP], Prim2[0], flow_Rgas);
  double flow_Mach = norm2(vel2[0], vel2[1], vel2[2]) / flow_Sound;
  double BC_Mach_local = BC_rel_fac * BC_Mach + (1.0 - BC_rel_fac) * flow_Mach;
  double BC_p0_local = BC_rel_fac * BC_p0 + (1.0 - BC_rel_fac) * Prim2[NP];
  double alpha_eff = BC_alpha, beta_eff = BC_beta;   // Compute_Inflow_Direction :477-495
  if (BC_alpha >= 0.5 * 1.7976931348623157e308) alpha_eff = std::atan(Normal[1] / (Normal[0] + 1e-20));
  if (BC_beta >= 0.5 * 1.7976931348623157e308) beta_eff = std::atan(Normal[2] / (Normal[0] + 1e-20));
  double Sup[NPRIM];
  Sup[NP] = BC_p0_local;
  double Sup_T = BC_T0;
  double Sup_Rgas = 1.0 * t.R;                       // sum(BC_ci*Ri_Tab), ci = 1
  double Sup_rho = Sup[NP] / (Sup_Rgas * Sup_T);
  Sup[0] = Sup_rho * 1.0;
  double Sup_Sound = f_ss(t, Sup[0], Sup[NP], Sup_rho, Sup_Rgas);
  Sup[NU] = BC_Mach_local * Sup_Sound * std::cos(alpha_eff) * std::cos(beta_eff);
  Sup[NV] = BC_Mach_local * Sup_Sound * std::sin(alpha_eff) * std::cos(beta_eff);
  Sup[NW] = BC_Mach_local * Sup_Sound * std::sin(beta_eff);
  double fm = (double)modfm, fm1 = (double)modfm1;
  double Prim1[NPRIM], Prim3[NPRIM], Slope[NPRIM], Face[NPRIM], PL[NPRIM], PR[NPRIM];
  for (int v = 0; v < NPRIM; ++v) {
    Prim1[v] = fm * Sup[v] + fm1 * Int[v];
    Prim3[v] = fm * Int[v] + fm1 * Sup[v];
  }
  for (int v = 0; v < NPRIM; ++v) {
    double d32 = Prim3[v] - Prim2[v];
    double d21 = Prim2[v] - Prim1[v];
    Slope[v] = rlimiter(D->cfg.limiter, d32, d21);
  }
  for (int v = 0; v < NPRIM; ++v) Face[v] = Prim2[v] + 0.5 * Slope[v] * (double)modfm2;
  for (int v = 0; v < NPRIM; ++v) {
    PL[v] = fm * Sup[v] + fm1 * Face[v];
    PR[v] = fm * Face[v] + fm1 * Sup[v];
  }
  bool bad = false;
  RState L = make_state(t, PL, bad);
  RState R = make_state(t, PR, bad);
  RFlux F = Riemann(D, L, R, Normal[0], Normal[1], Normal[2]);
  double su = std::copysign(1.0, F.r);
  double Sel_L = (1.0 + su) / 2.0, Sel_R = (su - 1.0) / 2.0;
  double Fmass = F.r * Area;
  double Flux[NPRIM];
  Flux[0] = Fmass * (Sel_L * PL[0] / L.rho - Sel_R * PR[0] / R.rho);
  Flux[NU] = F.u * Area;
  Flux[NV] = F.v * Area;
  Flux[NW] = F.w * Area;
  Flux[NP] = F.E * Area;
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] + (double)modfm2 * Flux[v];
  return true;
}

// Outflow, Lib_BC_Fluxes_Outflow.f90:59-129: the face flux of an outflow
// face with back pressure BC_pexit (0: extrapolation of every variable).
void Outflow(const Thermo& t, const double* Bound, double BC_Sign, double Un, const double* Normal, double Area,
             double BC_pexit, double* Flux) {
  double bvel[3] = {Bound[NU], Bound[NV], Bound[NW]};
  double Bound_rho, Bound_Rgas;
  co_rotot_Rtot(t, Bound[0], Bound_rho, Bound_Rgas);
  double Bound_Sound = f_ss(t, Bound[0], Bound[NP], Bound_rho, Bound_Rgas);
  double Bound_Gamma = t.gamma;
  double Riem = Bound_Sound + BC_Sign * 0.5 * (Bound_Gamma - 1.0) * Un;
  double Vel_N[3], Vel_T[3];
  for (int q = 0; q < 3; ++q) { Vel_N[q] = Un * Normal[q]; Vel_T[q] = bvel[q] - Vel_N[q]; }
  double Mach_N = std::fabs(Un / Bound_Sound);
  double Face[NPRIM], Face_Un, Face_Sound, Face_rho, Face_Rgas;
  if (Mach_N < 1.0 && BC_pexit > 0.0) {
    double p_exit = BC_pexit;
    double delta = 0.5 * (Bound_Gamma - 1.0);
    double den = 1.0 / std::pow(1.0 + delta, Bound_Gamma / (Bound_Gamma - 1.0));
    double pstar = Bound[NP] * den * std::pow(1.0 + delta * (Mach_N * Mach_N), Bound_Gamma / (Bound_Gamma - 1.0));
    if (pstar >= p_exit) p_exit = pstar;
    double Isentropic = (Bound_Gamma - 1.0) / (2.0 * Bound_Gamma);
    Face_Sound = Bound_Sound * std::pow(p_exit / Bound[NP], Isentropic);
    Face_Un = (Riem - Face_Sound) / (BC_Sign * 0.5 * (Bound_Gamma - 1.0));
    Face[NP] = p_exit;
    Face_rho = Bound_Gamma * Face[NP] / (Face_Sound * Face_Sound);
    Face[0] = Bound[0] / Bound_rho * Face_rho;
    for (int q = 0; q < 3; ++q) Face[NU + q] = Vel_T[q] + Face_Un * Normal[q];
    Face_Rgas = Bound_Rgas;
  } else {
    for (int v = 0; v < NPRIM; ++v) Face[v] = Bound[v];
    Face_Un = Un;
    Face_Sound = Bound_Sound;
    Face_rho = Bound_rho;
    Face_Rgas = Bound_Rgas;
  }
  (void)Face_Sound;
  double Face_T = Face[NP] / (Face_Rgas * Face_rho);
  double Face_Enthalpy = Face[0] / Face_rho * (t.cp * Face_T);
  Flux[0] = Face[0] * Area * Face_Un;
  double BC_mdot = Face_rho * Area * Face_Un;
  for (int q = 0; q < 3; ++q) Flux[NU + q] = Face[NU + q] * BC_mdot + Face[NP] * Area * Normal[q];
  Flux[NP] = BC_mdot * (0.5 * (Face[NU] * Face[NU] + Face[NV] * Face[NV] + Face[NW] * Face[NW]) + Face_Enthalpy);
}

// BC_Outflow, Lib_BC_Fluxes_Outflow.f90:12-56.  Returns false when
// BC_Sign*Un < 0 (the caller falls back to symmetry).
bool BC_Outflow(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk, const double* data) {
  int modfm, modfm1, modfm2, dir, fi, fj, fk;
  compute_modfm(Fm, modfm, modfm1, modfm2);
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const double* Bound = blk.Pc(Im, Jm, Km);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  double Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  double BC_Sign = (double)modfm2;
  double bvel[3] = {Bound[NU], Bound[NV], Bound[NW]};
  double Un = dot3(bvel, Normal);
  if (BC_Sign * Un < 0.0) return false;
  double Flux[NPRIM];
  Outflow(D->th, Bound, BC_Sign, Un, Normal, Area, data[0], Flux);
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] + (double)modfm2 * Flux[v];
  return true;
}

// ---- inlets 401 / 403 / 404 and the ambient far field 407 --------------------
// Setup_Inflow_Geometry, Lib_BC_Fluxes_Inflow.f90:502-559: the boundary face's
// normal and area, the unit tangent t (the face diagonal between two of its
// nodes), the boundary cell's state, Un and the Riemann invariant toward the
// face.
struct InflowGeo {
  const double* Normal;
  double Area, t_Vec[3], BC_Sign, Un, Sound, Gamma, Riem;
  const double* Bound;
  int modfm2;
};

InflowGeo Setup_Inflow_Geometry(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk) {
  const Thermo& t = D->th;
  InflowGeo g;
  int modfm, modfm1, dir, fi, fj, fk;
  compute_modfm(Fm, modfm, modfm1, g.modfm2);
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  g.Bound = blk.Pc(Im, Jm, Km);
  g.Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  g.Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  const double* a = blk.nodep(fi, fj, fk);
  const double* b = (Fm <= 2) ? blk.nodep(fi, fj - 1, fk - 1)
                  : (Fm <= 4) ? blk.nodep(fi - 1, fj, fk - 1)
                              : blk.nodep(fi - 1, fj - 1, fk);
  for (int q = 0; q < 3; ++q) g.t_Vec[q] = a[q] - b[q];
  double t_Mod = norm2(g.t_Vec[0], g.t_Vec[1], g.t_Vec[2]);
  for (int q = 0; q < 3; ++q) g.t_Vec[q] = g.t_Vec[q] / t_Mod;
  g.BC_Sign = (double)g.modfm2;
  double bvel[3] = {g.Bound[NU], g.Bound[NV], g.Bound[NW]};
  g.Un = dot3(bvel, g.Normal);
  double rho, Rgas;
  co_rotot_Rtot(t, g.Bound[0], rho, Rgas);
  g.Sound = f_ss(t, g.Bound[0], g.Bound[NP], rho, Rgas);
  g.Gamma = t.gamma;
  g.Riem = g.Sound + g.BC_Sign * 0.5 * (g.Gamma - 1.0) * g.Un;
  return g;
}

// Compute_Inflow_Direction, Lib_BC_Fluxes_Inflow.f90:479-496: the token
// 'normal' (read as the largest double) takes the angle of the face normal.
void inflow_direction(const double* Normal, double alpha_in, double beta_in, double& alpha, double& beta) {
  alpha = (alpha_in >= 0.5 * 1.7976931348623157e308) ? std::atan(Normal[1] / (Normal[0] + 1e-20)) : alpha_in;
  beta = (beta_in >= 0.5 * 1.7976931348623157e308) ? std::atan(Normal[2] / (Normal[0] + 1e-20)) : beta_in;
}

// The binormal b = n x t / |n x t| and the tangential-to-normal velocity
// ratios E1, E2 that make the face velocity Un (n + E1 t + E2 b) point along
// (alpha, beta) (Lib_BC_Fluxes_Inflow.f90:113-129, 197-213, 404-420).
void inflow_E(const double* Normal, const double* t_Vec, double alpha, double beta, double* b_Vec, double& E1,
              double& E2) {
  b_Vec[0] = Normal[1] * t_Vec[2] - Normal[2] * t_Vec[1];
  b_Vec[1] = Normal[2] * t_Vec[0] - Normal[0] * t_Vec[2];
  b_Vec[2] = Normal[0] * t_Vec[1] - Normal[1] * t_Vec[0];
  double b_Mod = norm2(b_Vec[0], b_Vec[1], b_Vec[2]);
  for (int q = 0; q < 3; ++q) b_Vec[q] = b_Vec[q] / b_Mod;
  double ta = std::tan(alpha), tb = std::tan(beta);
  double XA = Normal[1] - Normal[0] * ta;
  double XB = t_Vec[1] - t_Vec[0] * ta;
  double XC = b_Vec[1] - b_Vec[0] * ta;
  double XD = Normal[2] - Normal[0] * tb;
  double XE = t_Vec[2] - t_Vec[0] * tb;
  double XF = b_Vec[2] - b_Vec[0] * tb;
  double check = (XC * XE - XF * XB);
  E1 = (XF * XA - XC * XD) / check;
  E2 = (XD * XB - XE * XA) / check;
}

// Compute_Flux_from_Face, Lib_BC_Fluxes_Inflow.f90:565-587 (one species).
void Flux_from_Face(const Thermo& t, const double* Face, double Face_rho, double Face_Rgas, double Area,
                    const double* Normal, double* Flux) {
  double fvel[3] = {Face[NU], Face[NV], Face[NW]};
  double Face_Un = dot3(fvel, Normal);
  double Face_T = Face[NP] / (Face_Rgas * Face_rho);
  double Fmass = Face_rho * Face_Un * Area;
  double Face_Enthalpy = 0.0 + Face[0] / Face_rho * (t.cp * Face_T);
  Flux[0] = Face[0] * Face_Un * Area;
  for (int q = 0; q < 3; ++q) Flux[NU + q] = Fmass * Face[NU + q] + Face[NP] * Area * Normal[q];
  Flux[NP] = Fmass * (0.5 * (Face[NU] * Face[NU] + Face[NV] * Face[NV] + Face[NW] * Face[NW]) + Face_Enthalpy);
}

// Stagn_Inflow, Lib_BC_Fluxes_Inflow.f90:388-473: the face state compatible
// with the interior Riemann invariant and the total conditions (T0, p0); p0
// relaxes toward the boundary pressure while the quadratic for Un has no
// real root (at most 1000 tries).
void Stagn_Inflow(const Thermo& t, const InflowGeo& g, double alpha, double beta, double BC_T0, double BC_p0,
                  double BC_rel_fac, double* Flux) {
  const double* Prim = g.Bound;
  const double Gamma = g.Gamma, Riem = g.Riem, Sound = g.Sound;
  double b_Vec[3], E1, E2;
  inflow_E(g.Normal, g.t_Vec, alpha, beta, b_Vec, E1, E2);
  double Discr = -1.0, BC_p0_try = BC_p0, Face_Rgas = 0.0, Sound0 = 0.0, Coef_D = 0.0, Coef_C, YA = 0.0, YB = 0.0, YC;
  int iter_discr = 0;
  while (Discr < 0.0) {
    iter_discr = iter_discr + 1;
    Face_Rgas = 1.0 * t.R;                           // sum(BC_ci*Ri_tab), ci = 1
    Sound0 = std::sqrt(Gamma * Face_Rgas * BC_T0);
    Coef_D = (1.0 + E1 * E1 + E2 * E2) * (Gamma - 1.0) / 2.0;
    Coef_C = std::pow(BC_p0_try / Prim[NP], (Gamma - 1.0) / Gamma);
    Coef_C = Coef_C * ((Sound / Sound0) * (Sound / Sound0));
    YA = ((Gamma - 1.0) / 2.0) * ((Gamma - 1.0) / 2.0) + Coef_C * Coef_D;
    YB = g.BC_Sign * Riem * ((Gamma - 1.0) / 2.0);
    YC = Riem * Riem - Coef_C * (Sound0 * Sound0);
    Discr = YB * YB - YA * YC;
    if (Discr < 0.0 && std::fabs(Discr) < 1e-2) Discr = 0.0;
    if (Discr < 0.0 && std::fabs(Discr) > 1e-2) BC_p0_try = BC_rel_fac * BC_p0_try + (1.0 - BC_rel_fac) * Prim[NP];
    if (iter_discr > 1000) {
      Discr = 0.0;
      break;
    }
  }
  double Un_Sign = std::copysign(1.0, g.Un);
  double Un3 = (YB + Un_Sign * std::sqrt(Discr)) / YA;
  double Sound3 = std::sqrt(Sound0 * Sound0 - Coef_D * (Un3 * Un3));
  double p3 = BC_p0_try * std::pow(Sound3 / Sound0, 2.0 * Gamma / (Gamma - 1.0));
  double Ut3 = Un3 * E1, Ub3 = Un3 * E2;
  double Face[NPRIM];
  Face[NP] = p3;
  double Face_rho = Gamma * Face[NP] / (Sound3 * Sound3);
  Face[0] = 1.0 * Face_rho;
  for (int q = 0; q < 3; ++q) Face[NU + q] = Un3 * g.Normal[q] + Ut3 * g.t_Vec[q] + Ub3 * b_Vec[q];
  double Face_T = Face[NP] / (Face_Rgas * Face_rho);
  double Face_Enthalpy = 0.0 + Face[0] / Face_rho * (t.cp * Face_T);
  Flux[0] = Face[0] * Un3 * g.Area;
  double Fmass = Face_rho * Un3 * g.Area;
  for (int q = 0; q < 3; ++q) Flux[NU + q] = Fmass * Face[NU + q] + Face[NP] * g.Area * g.Normal[q];
  Flux[NP] = Fmass * (0.5 * (Face[NU] * Face[NU] + Face[NV] * Face[NV] + Face[NW] * Face[NW]) + Face_Enthalpy);
}

// ---------------------------------------------------------------------------
// Navier-Stokes diffusive fluxes (model = 1, laminar): Lib_Diffusive.f90,
// Lib_BC_Fluxes_Connection.f90:117-224, Lib_BC_Fluxes_Symmetry.f90:128-247,
// Lib_BC_Fluxes_Wall_Heat.f90, Lib_BC_Fluxes_Wall_Temperature.f90 and the
// standard stress vector Stress_Vector_Std (Lib_Fluid.f90:23-46).  One
// species: the concentration gradient is an exact zero, so the species
// diffusion and its enthalpy flux vanish exactly; the eddy viscosity is 0.
// Gradients are G[v][c], v over the nprim visc variables (Y, u, v, w, T),
// c over the three directions; matmul(G, M) sums over the index direction
// in order 1, 2, 3.
// ---------------------------------------------------------------------------

// matmul(Gradient(nprim,3), M(3,3)) with M stored c(r,s) at r + 3 s
inline void grad_matmul(double G[NPRIM][3], const double* M) {
  double out[NPRIM][3];
  for (int v = 0; v < NPRIM; ++v)
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (int d = 0; d < 3; ++d) s = s + G[v][d] * M[d + 3 * c];
      out[v][c] = s;
    }
  for (int v = 0; v < NPRIM; ++v)
    for (int c = 0; c < 3; ++c) G[v][c] = out[v][c];
}

// Stress_Vector_Std(Gradvel, Normal, mi_l, mi_t): Gradvel(r, c) = d u_r / d x_c
inline void stress_vector(const double Gv[3][3], const double* n, double mi_l, double mi_t, double* S) {
  const double negativetwothird = -2.0 / 3.0;
  double mi = mi_l + mi_t;
  double lam = negativetwothird * mi;
  double Divervel = Gv[0][0] + Gv[1][1] + Gv[2][2];
  double lamDivervel = lam * Divervel;
  double Txx = lamDivervel + 2.0 * mi * Gv[0][0];
  double Tyy = lamDivervel + 2.0 * mi * Gv[1][1];
  double Tzz = lamDivervel + 2.0 * mi * Gv[2][2];
  double Txy = mi * (Gv[0][1] + Gv[1][0]);
  double Txz = mi * (Gv[0][2] + Gv[2][0]);
  double Tyz = mi * (Gv[1][2] + Gv[2][1]);
  S[0] = Txx * n[0] + Txy * n[1] + Txz * n[2];
  S[1] = Txy * n[0] + Tyy * n[1] + Tyz * n[2];
  S[2] = Txz * n[0] + Tyz * n[1] + Tzz * n[2];
}

inline void vel_grad(const double G[NPRIM][3], double Gv[3][3]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) Gv[r][c] = G[NU + r][c];
}

// Compute_Diffusive_Flux (Lib_Diffusive.f90:90-172), laminar, one species
inline void Compute_Diffusive_Flux(const orc_domain* D, const double* Prim, double G[NPRIM][3], double area,
                                   const double* normal, double* Flux) {
  const Thermo& t = D->th;
  double rho, Rgas;
  co_rotot_Rtot(t, Prim[0], rho, Rgas);
  const double mil = D->cfg.mu, kl = D->cfg.kappa, mie = 0.0;
  const double Sc = 1.0;   // obj_rans%Sc; multiplies an exact zero gradient
  double Dm = (mil / Sc + 0.0) / rho;
  double kappa = kl + mie * t.cp / 0.85;
  double Gv[3][3];
  vel_grad(G, Gv);
  double Stress[3];
  stress_vector(Gv, normal, mil, mie, Stress);
  double DiffHFlux = 0.0;
  for (int v = 0; v < NPRIM; ++v) Flux[v] = 0.0;
  double DmGradYi = Dm * (G[0][0] * normal[0] + G[0][1] * normal[1] + G[0][2] * normal[2]);
  Flux[0] = rho * area * DmGradYi;
  double T = Prim[NP] / (rho * Rgas);
  DiffHFlux = DiffHFlux + DmGradYi * (t.cp * T);
  Flux[0] = Flux[0] - Flux[0] * Prim[0] / rho;
  Flux[NU] = area * Stress[0];
  Flux[NV] = area * Stress[1];
  Flux[NW] = area * Stress[2];
  Flux[NP] = area * ((Stress[0] * Prim[NU] + Stress[1] * Prim[NV] + Stress[2] * Prim[NW]) +
                     kappa * (G[NP][0] * normal[0] + G[NP][1] * normal[1] + G[NP][2] * normal[2]) + DiffHFlux * rho);
}

// Visc_Variables: (rho_s / rho, u, v, w, T)
inline void visc_vars(const Thermo& t, const double* P, double* V) {
  double rho, Rgas;
  co_rotot_Rtot(t, P[0], rho, Rgas);
  V[0] = P[0] / rho;
  V[NU] = P[NU];
  V[NV] = P[NV];
  V[NW] = P[NW];
  V[NP] = P[NP] / (rho * Rgas);
}

// Tangential_Gradient (Lib_Diffusive.f90:55-87)
inline void Tangential_Gradient(const Thermo& t, const double* P1, const double* P2, const double* P3, const double* P4,
                                double G[NPRIM][3], int c) {
  double V1[NPRIM], V2[NPRIM], V3[NPRIM], V4[NPRIM];
  visc_vars(t, P1, V1);
  visc_vars(t, P2, V2);
  visc_vars(t, P3, V3);
  visc_vars(t, P4, V4);
  for (int v = 0; v < NPRIM; ++v) G[v][c] = (V2[v] - V1[v] + V4[v] - V3[v]) * 0.25;
}

// Diffusive_Flux (Lib_Diffusive.f90:10-52): face between cells 1 and 2 along
// direction a (1-based), tangential stencils 3-6 along b and 7-10 along c
void Diffusive_Flux(const orc_domain* D, const double* normal, double area, const double* P1, const double* P2,
                    const double* P3, const double* P4, const double* P5, const double* P6, const double* P7,
                    const double* P8, const double* P9, const double* P10, const double* M1, const double* M2,
                    double* Res1, double* Res2, int a, int b, int c) {
  const Thermo& t = D->th;
  double G[NPRIM][3];
  for (int v = 0; v < NPRIM; ++v) G[v][0] = G[v][1] = G[v][2] = 0.0;
  double rho1, R1, rho2, R2;
  co_rotot_Rtot(t, P1[0], rho1, R1);
  double T1 = P1[NP] / (rho1 * R1);
  co_rotot_Rtot(t, P2[0], rho2, R2);
  double T2 = P2[NP] / (rho2 * R2);
  G[0][a - 1] = P2[0] / rho2 - P1[0] / rho1;
  G[NP][a - 1] = T2 - T1;
  for (int v = NU; v <= NW; ++v) G[v][a - 1] = P2[v] - P1[v];
  Tangential_Gradient(t, P3, P4, P5, P6, G, b - 1);
  Tangential_Gradient(t, P7, P8, P9, P10, G, c - 1);
  double M[9];
  for (int q = 0; q < 9; ++q) M[q] = 0.5 * (M1[q] + M2[q]);
  grad_matmul(G, M);
  double Prim[NPRIM];
  for (int v = 0; v < NPRIM; ++v) Prim[v] = 0.5 * (P1[v] + P2[v]);
  double Flux[NPRIM];
  Compute_Diffusive_Flux(D, Prim, G, area, normal, Flux);
  for (int v = 0; v < NPRIM; ++v) {
    Res1[v] = Res1[v] - Flux[v];
    Res2[v] = Res2[v] + Flux[v];
  }
}

// BC_Connection_Visc (Lib_BC_Fluxes_Connection.f90:117-224).  The ghost stencil
// Pg(:,1) is the first ghost layer; Pg(:,3:6) are the source block's cells
// that Fill_BC_Ghost_Connection (Lib_Ghost.f90:405-460) picks with d11..d22.
void BC_Connection_Visc(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk, const Block& bs, int Is,
                        int Js, int Ks, int Fs, int d11, int d12, int d21, int d22) {
  const Thermo& t = D->th;
  int dir, fi, fj, fk;
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const int modfm2 = 1 - 2 * (Fm % 2);
  const int Ig = Im - G(Fm, 1), Jg = Jm - G(Fm, 2), Kg = Km - G(Fm, 3);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  const double area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  double M[9];
  for (int q = 0; q < 9; ++q) M[q] = 0.5 * ((&blk.M_(1, 1, Im, Jm, Km))[q] + (&blk.M_(1, 1, Ig, Jg, Kg))[q]);
  int i1, j1, k1, i2, j2, k2, i3, j3, k3, i4, j4, k4;
  if (Fs <= 2) {
    i1 = Is; j1 = Js - d11; k1 = Ks - d12; i2 = Is; j2 = Js + d11; k2 = Ks + d12;
    i3 = Is; j3 = Js - d21; k3 = Ks - d22; i4 = Is; j4 = Js + d21; k4 = Ks + d22;
  } else if (Fs <= 4) {
    i1 = Is - d11; j1 = Js; k1 = Ks - d12; i2 = Is + d11; j2 = Js; k2 = Ks + d12;
    i3 = Is - d21; j3 = Js; k3 = Ks - d22; i4 = Is + d21; j4 = Js; k4 = Ks + d22;
  } else {
    i1 = Is - d11; j1 = Js - d12; k1 = Ks; i2 = Is + d11; j2 = Js + d12; k2 = Ks;
    i3 = Is - d21; j3 = Js - d22; k3 = Ks; i4 = Is + d21; j4 = Js + d22; k4 = Ks;
  }
  const double* Prim_loc = blk.Pc(Im, Jm, Km);
  const double* Prim_ghost = blk.Pc(Ig, Jg, Kg);
  double Vl[NPRIM], Vip[NPRIM], Vim[NPRIM], Vjp[NPRIM], Vjm[NPRIM], Vkp[NPRIM], Vkm[NPRIM];
  double Vg[NPRIM], Vg3[NPRIM], Vg4[NPRIM], Vg5[NPRIM], Vg6[NPRIM];
  visc_vars(t, Prim_loc, Vl);
  visc_vars(t, blk.Pc(Im + 1, Jm, Km), Vip);
  visc_vars(t, blk.Pc(Im - 1, Jm, Km), Vim);
  visc_vars(t, blk.Pc(Im, Jm + 1, Km), Vjp);
  visc_vars(t, blk.Pc(Im, Jm - 1, Km), Vjm);
  visc_vars(t, blk.Pc(Im, Jm, Km + 1), Vkp);
  visc_vars(t, blk.Pc(Im, Jm, Km - 1), Vkm);
  visc_vars(t, Prim_ghost, Vg);
  visc_vars(t, &bs.P[NPRIM * bs.cell(i1, j1, k1)], Vg3);
  visc_vars(t, &bs.P[NPRIM * bs.cell(i2, j2, k2)], Vg4);
  visc_vars(t, &bs.P[NPRIM * bs.cell(i3, j3, k3)], Vg5);
  visc_vars(t, &bs.P[NPRIM * bs.cell(i4, j4, k4)], Vg6);
  double Gl[NPRIM][3], Gg[NPRIM][3];
  for (int v = 0; v < NPRIM; ++v) {
    const double across_l = (Vg[v] - Vl[v]) * (double)modfm2;
    const double across_g = (Vl[v] - Vg[v]) * (double)(-modfm2);
    const double g34 = (Vg4[v] - Vg3[v]) * 0.5, g56 = (Vg6[v] - Vg5[v]) * 0.5;
    if (Fm <= 2) {
      Gl[v][0] = across_l; Gl[v][1] = (Vjp[v] - Vjm[v]) * 0.5; Gl[v][2] = (Vkp[v] - Vkm[v]) * 0.5;
      Gg[v][0] = across_g; Gg[v][1] = g34; Gg[v][2] = g56;
    } else if (Fm <= 4) {
      Gl[v][0] = (Vip[v] - Vim[v]) * 0.5; Gl[v][1] = across_l; Gl[v][2] = (Vkp[v] - Vkm[v]) * 0.5;
      Gg[v][0] = g34; Gg[v][1] = across_g; Gg[v][2] = g56;
    } else {
      Gl[v][0] = (Vip[v] - Vim[v]) * 0.5; Gl[v][1] = (Vjp[v] - Vjm[v]) * 0.5; Gl[v][2] = across_l;
      Gg[v][0] = g34; Gg[v][1] = g56; Gg[v][2] = across_g;
    }
  }
  grad_matmul(Gl, M);
  grad_matmul(Gg, M);
  double Prim[NPRIM];
  for (int v = 0; v < NPRIM; ++v) Prim[v] = (Prim_loc[v] + Prim_ghost[v]) * 0.5;
  double Fl[NPRIM], Fg[NPRIM];
  Compute_Diffusive_Flux(D, Prim, Gl, area, Normal, Fl);
  Compute_Diffusive_Flux(D, Prim, Gg, area, Normal, Fg);
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] - 0.5 * (double)modfm2 * (Fl[v] + Fg[v]);
}

// BC_Symmetry_Visc (Lib_BC_Fluxes_Symmetry.f90:128-247), no RSM
void BC_Symmetry_Visc(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk) {
  int dir, fi, fj, fk;
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const int modfm2 = 1 - 2 * (Fm % 2);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  const double Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  const double* M = &blk.M_(1, 1, Im, Jm, Km);
  const double mil = D->cfg.mu, mie = 0.0;
  auto vel = [&](int i, int j, int k, double* V) {
    const double* p = blk.Pc(i, j, k);
    V[0] = p[NU]; V[1] = p[NV]; V[2] = p[NW];
  };
  double V1[3], V3[3], V4[3], V7[3], V8[3];
  int a, b, c;
  vel(Im, Jm, Km, V1);
  if (Fm <= 2) {
    vel(Im, Jm - 1, Km, V3); vel(Im, Jm + 1, Km, V4); vel(Im, Jm, Km - 1, V7); vel(Im, Jm, Km + 1, V8);
    a = 0; b = 1; c = 2;
  } else if (Fm <= 4) {
    vel(Im - 1, Jm, Km, V3); vel(Im + 1, Jm, Km, V4); vel(Im, Jm, Km - 1, V7); vel(Im, Jm, Km + 1, V8);
    a = 1; b = 0; c = 2;
  } else {
    vel(Im - 1, Jm, Km, V3); vel(Im + 1, Jm, Km, V4); vel(Im, Jm - 1, Km, V7); vel(Im, Jm + 1, Km, V8);
    a = 2; b = 0; c = 1;
  }
  auto mirror = [&](const double* V, double* W) {
    const double dn = V[0] * Normal[0] + V[1] * Normal[1] + V[2] * Normal[2];
    for (int q = 0; q < 3; ++q) W[q] = V[q] - 2.0 * dn * Normal[q];
  };
  double V2[3], V5[3], V6[3], V9[3], V10[3];
  mirror(V1, V2); mirror(V3, V5); mirror(V4, V6); mirror(V7, V9); mirror(V8, V10);
  double Gr[NPRIM][3];
  for (int v = 0; v < NPRIM; ++v) Gr[v][0] = Gr[v][1] = Gr[v][2] = 0.0;
  for (int q = 0; q < 3; ++q) {
    Gr[NU + q][a] = (V2[q] - V1[q]) * (double)modfm2;
    Gr[NU + q][b] = (V4[q] - V3[q] + V6[q] - V5[q]) * 0.25;
    Gr[NU + q][c] = (V8[q] - V7[q] + V10[q] - V9[q]) * 0.25;
  }
  grad_matmul(Gr, M);
  double Gv[3][3];
  vel_grad(Gr, Gv);
  double Stress[3];
  stress_vector(Gv, Normal, mil, mie, Stress);
  double Vel[3];
  for (int q = 0; q < 3; ++q) Vel[q] = 0.5 * (V1[q] + V2[q]);
  double Flux[NPRIM] = {0.0, 0.0, 0.0, 0.0, 0.0};
  Flux[NU] = Area * Stress[0];
  Flux[NV] = Area * Stress[1];
  Flux[NW] = Area * Stress[2];
  Flux[NP] = Area * (Vel[0] * Stress[0] + Vel[1] * Stress[1] + Vel[2] * Stress[2]);
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = NU; v <= NP; ++v) r[v] = r[v] - (double)modfm2 * Flux[v];
}

// the wall routines' common part: velocity gradient across the face from the
// no-slip wall (Gradient(nu:nw, Dir) = Prim(nu:nw) * modfm3), the given
// temperature gradient across it, then matmul and the stress
inline void wall_stress(const orc_domain* D, const double* Prim, int dir, int modfm3, double Tgrad, const double* M,
                        const double* Normal, double G[NPRIM][3], double* Stress) {
  for (int v = 0; v < NPRIM; ++v) G[v][0] = G[v][1] = G[v][2] = 0.0;
  for (int v = NU; v <= NW; ++v) G[v][dir - 1] = Prim[v] * (double)modfm3;
  G[NP][dir - 1] = Tgrad;
  grad_matmul(G, M);
  double Gv[3][3];
  vel_grad(G, Gv);
  stress_vector(Gv, Normal, D->cfg.mu, 0.0, Stress);
}

// BC_Wall_Heat (Lib_BC_Fluxes_Wall_Heat.f90:13-116): prescribed heat flux qw
void BC_Wall_Heat(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk, double Heat_Flux) {
  int dir, fi, fj, fk;
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const int modfm = Fm % 2, modfm2 = 1 - 2 * modfm, modfm3 = 2 * (2 * modfm - 1);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  const double Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  const double* M = &blk.M_(1, 1, Im, Jm, Km);
  const double* Prim = blk.Pc(Im, Jm, Km);
  const double kl = D->cfg.kappa;
  const double mdotn = M[(dir - 1) + 0] * Normal[0] + M[(dir - 1) + 3] * Normal[1] + M[(dir - 1) + 6] * Normal[2];
  const double Tgrad = -Heat_Flux / (2.0 * kl * mdotn) * (double)modfm2;
  double G[NPRIM][3], Stress[3];
  wall_stress(D, Prim, dir, modfm3, Tgrad, M, Normal, G, Stress);
  double Flux[NPRIM] = {0.0, 0.0, 0.0, 0.0, 0.0};
  Flux[NU] = Stress[0] * Area;
  Flux[NV] = Stress[1] * Area;
  Flux[NW] = Stress[2] * Area;
  Flux[NP] = Area * Heat_Flux;
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] - (double)modfm2 * Flux[v];
}

// BC_Wall_Temperature (Lib_BC_Fluxes_Wall_Temperature.f90:12-100): wall at T_wall
void BC_Wall_Temperature(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk, double T_wall) {
  const Thermo& t = D->th;
  int dir, fi, fj, fk;
  Face_Index(Fm, Im, Jm, Km, dir, fi, fj, fk);
  const int modfm = Fm % 2, modfm2 = 1 - 2 * modfm, modfm3 = 2 * (2 * modfm - 1);
  const double* Normal = &blk.fN[dir - 1][3 * blk.face(dir, fi, fj, fk)];
  const double Area = blk.fA[dir - 1][blk.face(dir, fi, fj, fk)];
  const double* M = &blk.M_(1, 1, Im, Jm, Km);
  const double* Prim = blk.Pc(Im, Jm, Km);
  double rho, Rgas;
  co_rotot_Rtot(t, Prim[0], rho, Rgas);
  const double T = Prim[NP] / (rho * Rgas);
  const double kl = D->cfg.kappa;
  double G[NPRIM][3], Stress[3];
  wall_stress(D, Prim, dir, modfm3, (T - T_wall) * (double)modfm3, M, Normal, G, Stress);
  double Flux[NPRIM] = {0.0, 0.0, 0.0, 0.0, 0.0};
  Flux[NU] = Stress[0] * Area;
  Flux[NV] = Stress[1] * Area;
  Flux[NW] = Stress[2] * Area;
  Flux[NP] = Area * kl * (G[NP][0] * Normal[0] + G[NP][1] * Normal[1] + G[NP][2] * Normal[2]);
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] - (double)modfm2 * Flux[v];
}

void add_bc_flux(Block& blk, int Im, int Jm, int Km, int modfm2, const double* Flux) {
  double* r = blk.Rc(Im, Jm, Km);
  for (int v = 0; v < NPRIM; ++v) r[v] = r[v] + (double)modfm2 * Flux[v];
}

// BC_Inlet_StagnCond, Lib_BC_Fluxes_Inflow.f90:19-75 (no rotating frame).
// data: T0, p0, alpha, beta, rel_fac.  False when BC_Sign*Un >= 0.
bool BC_Inlet_StagnCond(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk, const double* data) {
  InflowGeo g = Setup_Inflow_Geometry(D, Im, Jm, Km, Fm, blk);
  if (g.BC_Sign * g.Un >= 0.0) return false;
  double alpha, beta;
  inflow_direction(g.Normal, data[2], data[3], alpha, beta);
  double Flux[NPRIM];
  Stagn_Inflow(D->th, g, alpha, beta, data[0], data[1], data[4], Flux);
  add_bc_flux(blk, Im, Jm, Km, g.modfm2, Flux);
  return true;
}

// BC_Inlet_MassFlux_T0 (403, :81-159) and BC_Inlet_MassFlux_T (404,
// :165-236): the mass flux g through the face at the boundary cell's
// pressure, with the total (403) or static (404) temperature.  data: T0 or T,
// g, alpha, beta, rel_fac.  False when BC_Sign*Un >= 0.
bool BC_Inlet_MassFlux(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk, const double* data,
                       bool total) {
  const Thermo& t = D->th;
  InflowGeo g = Setup_Inflow_Geometry(D, Im, Jm, Km, Fm, blk);
  if (g.BC_Sign * g.Un >= 0.0) return false;
  double alpha, beta, b_Vec[3], E1, E2;
  inflow_direction(g.Normal, data[2], data[3], alpha, beta);
  inflow_E(g.Normal, g.t_Vec, alpha, beta, b_Vec, E1, E2);
  const double BC_T = data[0], BC_g = data[1];
  double Rgas3 = 0.0 + 1.0 * t.R;
  double p3 = g.Bound[NP];
  double T3;
  if (total) {
    double cp3 = 0.0 + 1.0 * t.cp;
    double X = BC_g * Rgas3 / p3, Y = p3 / (BC_g * Rgas3);
    T3 = (-cp3 + std::sqrt(cp3 * cp3 + 2.0 * cp3 * BC_T * (X * X))) * (Y * Y);
  } else {
    T3 = BC_T;
  }
  double rho3 = p3 / (Rgas3 * T3);
  double Un3 = BC_g / rho3;
  double Ut3 = Un3 * E1, Ub3 = Un3 * E2;
  double Face[NPRIM];
  Face[0] = rho3 * 1.0;
  for (int q = 0; q < 3; ++q) Face[NU + q] = Un3 * g.Normal[q] + Ut3 * g.t_Vec[q] + Ub3 * b_Vec[q];
  Face[NP] = p3;
  double Flux[NPRIM];
  Flux_from_Face(t, Face, rho3, Rgas3, g.Area, g.Normal, Flux);
  add_bc_flux(blk, Im, Jm, Km, g.modfm2, Flux);
  return true;
}

// update, Series_Data_m.f90:55-86: linear interpolation in a time table;
// a periodic table first wraps time into [t_1, t_n) (Fortran MODULO of
// reals, restated as fmod plus the period when the signs differ).  The
// reference leaves the value undefined before t_1; here it is v_1.
double series_update(const orc_domain::Series& S, double time) {
  const size_t n = S.t.size();
  double t_ = time;
  if (S.periodic) {
    double period = S.t[n - 1] - S.t[0];
    if (period > 0.0) {
      double a = t_ - S.t[0];
      double m = std::fmod(a, period);
      if (m != 0.0 && ((m < 0.0) != (period < 0.0))) m = m + period;
      t_ = S.t[0] + m;
    }
  }
  if (t_ == S.t[0]) return S.v[0];
  for (size_t i = 1; i < n; ++i)
    if (t_ > S.t[i - 1] && t_ <= S.t[i]) return (S.v[i] - S.v[i - 1]) / (S.t[i] - S.t[i - 1]) * (t_ - S.t[i - 1]) + S.v[i - 1];
  if (t_ > S.t[n - 1]) return S.v[n - 1];
  return S.v[0];
}

// BC_FarField, Lib_BC_Fluxes_FarField.f90:19-73 (no rotating frame): the
// back-pressure outflow where the boundary cell leaves the domain, the total
// conditions where it enters (its angles are used as given).  data: T0, p0,
// p_back, alpha, beta, rel_fac.
void BC_FarField(const orc_domain* D, int Im, int Jm, int Km, int Fm, Block& blk, const double* data) {
  InflowGeo g = Setup_Inflow_Geometry(D, Im, Jm, Km, Fm, blk);
  double Flux[NPRIM];
  if (g.BC_Sign * g.Un >= 0.0)
    Outflow(D->th, g.Bound, g.BC_Sign, g.Un, g.Normal, g.Area, data[2], Flux);
  else
    Stagn_Inflow(D->th, g, data[3], data[4], data[0], data[1], data[5], Flux);
  add_bc_flux(blk, Im, Jm, Km, g.modfm2, Flux);
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

orc_domain* orc_create(const orc_config* cfg, int nthreads) {
  orc_domain* d = new orc_domain();
  d->cfg = *cfg;
  d->th.gamma = cfg->gamma;
  d->th.R = cfg->rgas;
  d->th.cp = cfg->gamma * cfg->rgas / (cfg->gamma - 1.0);
  d->th.cv = cfg->rgas / (cfg->gamma - 1.0);
  d->nthreads = nthreads > 0 ? nthreads : 1;
  if (d->cfg.res_diter <= 0) d->cfg.res_diter = 1;
  return d;
}

void orc_destroy(orc_domain* d) { delete d; }

int orc_add_block(orc_domain* d, int ni, int nj, int nk, const double* node) {
  if (ni < 1 || nj < 1 || nk < 1 || !node) return ORC_ERR_INVALID;
  Block b;
  b.ni = ni; b.nj = nj; b.nk = nk;
  b.sx = ni + 2 * GC; b.sy = nj + 2 * GC; b.sz = nk + 2 * GC;
  size_t nc = (size_t)b.sx * b.sy * b.sz;
  b.node.assign(node, node + 3 * (size_t)(ni + 1) * (nj + 1) * (nk + 1));
  b.P.assign(NPRIM * nc, 0.0);
  b.PO.assign(NPRIM * nc, 0.0);
  b.R.assign(NPRIM * nc, 0.0);
  b.M.assign(9 * nc, 0.0);
  b.dl.assign(3 * nc, 0.0);
  b.vol.assign(nc, 0.0);
  b.fN[0].assign(3 * (size_t)(ni + 1) * nj * nk, 0.0); b.fA[0].assign((size_t)(ni + 1) * nj * nk, 0.0);
  b.fN[1].assign(3 * (size_t)ni * (nj + 1) * nk, 0.0); b.fA[1].assign((size_t)ni * (nj + 1) * nk, 0.0);
  b.fN[2].assign(3 * (size_t)ni * nj * (nk + 1), 0.0); b.fA[2].assign((size_t)ni * nj * (nk + 1), 0.0);
  b.dtlocal.assign((size_t)ni * nj * nk, 0.0);
  b.beta.assign((size_t)ni * nj * nk, 1.0);
  d->blk.push_back(std::move(b));
  return ORC_OK;
}

int orc_set_bcs(orc_domain* d, const int32_t* rec, const double* data, int nbound) {
  int nb = (int)d->blk.size();
  size_t expect = 0;
  for (auto& b : d->blk) expect += 2 * ((size_t)b.nj * b.nk + (size_t)b.ni * b.nk + (size_t)b.ni * b.nj);
  if ((size_t)nbound != expect) return ORC_ERR_INVALID;                  // Check_BC, IO_BC.f90:123
  d->bc.resize(nbound);
  d->n_bf.assign(6 * nb, 0);
  int lastkey = -1;
  for (int q = 0; q < nbound; ++q) {
    const int32_t* r = rec + 15 * (size_t)q;
    BCrec& e = d->bc[q];
    e.b = r[0]; e.i = r[1]; e.j = r[2]; e.k = r[3]; e.f = r[4]; e.type = r[5];
    e.bs = r[6]; e.is = r[7]; e.js = r[8]; e.ks = r[9]; e.fs = r[10];
    e.d11 = r[11]; e.d12 = r[12]; e.d21 = r[13]; e.d22 = r[14];
    for (int c = 0; c < 6; ++c) e.data[c] = data ? data[6 * (size_t)q + c] : 0.0;
    if (e.b < 1 || e.b > nb || e.f < 1 || e.f > 6) return ORC_ERR_INVALID;
    int key = (e.b - 1) * 6 + (e.f - 1);
    if (key < lastkey) return ORC_ERR_INVALID;     // BC_Fluxes relies on (block, face) order
    lastkey = key;
    d->n_bf[key] += 1;
    switch (e.type) {
      case 0: case 101: case 201: case 300: case 400: case 401: case 403: case 404: case 405: case 406: case 407:
        break;
      case 301: case 302:   // walls: prescribed heat flux (data[0] = qw) / temperature (data[0] = Tw)
        break;
      case 402:
        if (!(e.data[1] >= 0.0 && e.data[1] < (double)d->series.size() && e.data[1] == std::floor(e.data[1])))
          return ORC_ERR_INVALID;
        break;
      default: return ORC_ERR_UNSUPPORTED;
    }
    if (e.type == 101 || e.type == 201) {
      if (e.bs < 1 || e.bs > nb || e.fs < 1 || e.fs > 6) return ORC_ERR_INVALID;
    }
  }
  return ORC_OK;
}

int orc_add_series(orc_domain* d, const double* time, const double* value, int n, int periodic) {
  if (!d || !time || !value || n < 1) return -ORC_ERR_INVALID;
  orc_domain::Series S;
  S.t.assign(time, time + n);
  S.v.assign(value, value + n);
  S.periodic = periodic != 0;
  d->series.push_back(std::move(S));
  return (int)d->series.size() - 1;
}

double orc_series_eval(const orc_domain* d, int id, double time) {
  if (!d || id < 0 || id >= (int)d->series.size()) return 0.0;
  return series_update(d->series[id], time);
}

int orc_setup_metrics(orc_domain* d) {
  if (d->blk.empty()) return ORC_ERR_INVALID;
  // Check_Mesh_Type, Lib_Metrics.f90:13-66
  Block& b1 = d->blk[0];
  if (d->cfg.ndir > 0) d->ndir = d->cfg.ndir;
  else if (b1.nk > 1) d->ndir = 3;
  else if (b1.nj == 1) d->ndir = 1;
  else d->ndir = 2;
  d->delthe = 0.0;
  if (d->ndir == 2 && b1.nj >= 1) {
    Vec3 a = b1.nd(0, 1, 0), bb = b1.nd(0, 1, 1), c = b1.nd(0, b1.nj, 0), e = b1.nd(0, b1.nj, 1);
    double t1 = std::atan2(bb.c[2], bb.c[1]) - std::atan2(a.c[2], a.c[1]);
    double t2 = std::atan2(e.c[2], e.c[1]) - std::atan2(c.c[2], c.c[1]);
    double r0 = std::sqrt(a.c[1] * a.c[1] + a.c[2] * a.c[2]);
    double r1 = std::sqrt(bb.c[1] * bb.c[1] + bb.c[2] * bb.c[2]);
    if ((t1 - t2) < 1e-5 && r0 > 1e-10 && std::fabs(r0 - r1) < 1e-5 * r0) d->delthe = t1;
  }
  if (d->delthe != 0.0) return ORC_ERR_UNSUPPORTED;   // axisymmetric meshes: out of scope
  bool ok = true;
  for (auto& b : d->blk) {
    for (int k = 1; k <= b.nk; ++k)
      for (int j = 1; j <= b.nj; ++j)
        for (int i = 1; i <= b.ni; ++i)
          ok &= cmt_store(b, i, j, k, b.nd(i - 1, j - 1, k - 1), b.nd(i - 1, j - 1, k), b.nd(i - 1, j, k - 1),
                          b.nd(i - 1, j, k), b.nd(i, j - 1, k - 1), b.nd(i, j - 1, k), b.nd(i, j, k - 1),
                          b.nd(i, j, k));
    Compute_Norm_Area(b);
  }
  for (auto& e : d->bc) {
    Block& bm = d->blk[e.b - 1];
    switch (e.type) {
      case 101:
        ok &= BC_Connect_Metrics(e.i, e.j, e.k, e.f, bm, e.is, e.js, e.ks, e.fs, d->blk[e.bs - 1], e.d11, e.d12,
                                 e.d21, e.d22);
        break;
      case 300: BC_Symmetry_Metrics(e.i, e.j, e.k, e.f, bm); break;
      default: ok &= BC_Extrapolate_Metrics(d, e.i, e.j, e.k, e.f, bm); break;
    }
  }
  return ok ? ORC_OK : ORC_ERR_METRICS;
}

static int check_block(const orc_domain* d, int b) {
  return (b >= 1 && b <= (int)d->blk.size()) ? ORC_OK : ORC_ERR_INVALID;
}

int orc_set_prim(orc_domain* d, int b, const double* P) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  Block& B = d->blk[b - 1];
  std::memcpy(B.P.data(), P, B.P.size() * sizeof(double));
  return ORC_OK;
}
int orc_get_prim(const orc_domain* d, int b, double* P) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  const Block& B = d->blk[b - 1];
  std::memcpy(P, B.P.data(), B.P.size() * sizeof(double));
  return ORC_OK;
}
int orc_set_prim_old(orc_domain* d, int b, const double* PO) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  Block& B = d->blk[b - 1];
  std::memcpy(B.PO.data(), PO, B.PO.size() * sizeof(double));
  return ORC_OK;
}
int orc_get_residual(const orc_domain* d, int b, double* R) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  const Block& B = d->blk[b - 1];
  std::memcpy(R, B.R.data(), B.R.size() * sizeof(double));
  return ORC_OK;
}
int orc_get_dtlocal(const orc_domain* d, int b, double* dt) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  const Block& B = d->blk[b - 1];
  std::memcpy(dt, B.dtlocal.data(), B.dtlocal.size() * sizeof(double));
  return ORC_OK;
}
int orc_set_dtlocal(orc_domain* d, int b, const double* dt) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  Block& B = d->blk[b - 1];
  std::memcpy(B.dtlocal.data(), dt, B.dtlocal.size() * sizeof(double));
  return ORC_OK;
}
int orc_get_metrics(const orc_domain* d, int b, double* vol, double* dl, double* M) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  const Block& B = d->blk[b - 1];
  if (vol) std::memcpy(vol, B.vol.data(), B.vol.size() * sizeof(double));
  if (dl) std::memcpy(dl, B.dl.data(), B.dl.size() * sizeof(double));
  if (M) std::memcpy(M, B.M.data(), B.M.size() * sizeof(double));
  return ORC_OK;
}
int orc_get_faces(const orc_domain* d, int b, int dir, double* N, double* A) {
  if (check_block(d, b) || dir < 1 || dir > 3) return ORC_ERR_INVALID;
  const Block& B = d->blk[b - 1];
  if (N) std::memcpy(N, B.fN[dir - 1].data(), B.fN[dir - 1].size() * sizeof(double));
  if (A) std::memcpy(A, B.fA[dir - 1].data(), B.fA[dir - 1].size() * sizeof(double));
  return ORC_OK;
}

// Replaces the block's metrics (tests: precomputed metrics handed to the
// device must be the ones both sides step with).  Same layouts as the getters.
int orc_set_metrics(orc_domain* d, int b, const double* vol, const double* dl, const double* M) {
  if (check_block(d, b)) return ORC_ERR_INVALID;
  Block& B = d->blk[b - 1];
  if (vol) std::memcpy(B.vol.data(), vol, B.vol.size() * sizeof(double));
  if (dl) std::memcpy(B.dl.data(), dl, B.dl.size() * sizeof(double));
  if (M) std::memcpy(B.M.data(), M, B.M.size() * sizeof(double));
  return ORC_OK;
}
int orc_set_faces(orc_domain* d, int b, int dir, const double* N, const double* A) {
  if (check_block(d, b) || dir < 1 || dir > 3) return ORC_ERR_INVALID;
  Block& B = d->blk[b - 1];
  if (N) std::memcpy(B.fN[dir - 1].data(), N, B.fN[dir - 1].size() * sizeof(double));
  if (A) std::memcpy(B.fA[dir - 1].data(), A, B.fA[dir - 1].size() * sizeof(double));
  return ORC_OK;
}

// Fill_Ghost_Cell, Lib_Ghost.f90:11-137 (single rank: every block is local).
int orc_fill_ghost_cell(orc_domain* d) {
  int n = (int)d->bc.size();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(d->nthreads)
#endif
  for (int q = 0; q < n; ++q) {
    const BCrec& e = d->bc[q];
    Block& bm = d->blk[e.b - 1];
    switch (e.type) {
      case 101: case 201:
        Ghost_Connection(e.i, e.j, e.k, e.f, bm, e.is, e.js, e.ks, e.fs, d->blk[e.bs - 1]);
        break;
      case 300: Ghost_Symmetry(e.i, e.j, e.k, e.f, bm); break;
      case 0: case 401: case 402: case 403: case 404: case 405: case 406: case 407: case 420:
        Ghost_ZG_Extrapolate(e.i, e.j, e.k, e.f, bm);
        break;
      default: Ghost_Extrapolate(e.i, e.j, e.k, e.f, bm); break;
    }
  }
  return ORC_OK;
}

// Fluxes / Fluxes_blk, Mod_Fluxes.f90:10-209 (convective part, SD off).
int orc_fluxes(orc_domain* d) {
  for (int bi = 0; bi < (int)d->blk.size(); ++bi) {
    Block& B = d->blk[bi];
    const int n1 = B.ni, n2 = B.nj, n3 = B.nk;
#ifdef _OPENMP
#pragma omp parallel num_threads(d->nthreads)
#endif
    {
#ifdef _OPENMP
#pragma omp for collapse(3)
#endif
      for (int k = 1; k <= n3; ++k)
        for (int j = 1; j <= n2; ++j)
          for (int i = 1; i <= n1; ++i) {
            double* r = B.Rc(i, j, k);
            for (int v = 0; v < NPRIM; ++v) r[v] = 0.0;
            B.beta[B.inner(i, j, k)] = 1.0;
          }
      // Shock-detector, Mod_Fluxes.f90:78-85
      if (sd_any(d)) {
#ifdef _OPENMP
#pragma omp for collapse(3)
#endif
        for (int k = 1; k <= n3; ++k)
          for (int j = 1; j <= n2; ++j)
            for (int i = 1; i <= n1; ++i)
              B.beta[B.inner(i, j, k)] = SD_Tramel(B.Pc(i, j, k)[NP], B.Pc(i - 1, j, k)[NP], B.Pc(i + 1, j, k)[NP],
                                                   B.Pc(i, j - 1, k)[NP], B.Pc(i, j + 1, k)[NP],
                                                   B.Pc(i, j, k - 1)[NP], B.Pc(i, j, k + 1)[NP]);
      }
      // i faces (:89-99)
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
      for (int k = 1; k <= n3; ++k)
        for (int j = 1; j <= n2; ++j)
          for (int i = 1; i <= n1 - 1; ++i) {
            double dls[4] = {B.dl_(1, i - 1, j, k), B.dl_(1, i, j, k), B.dl_(1, i + 1, j, k), B.dl_(1, i + 2, j, k)};
            size_t f = B.face(1, i, j, k);
            if (!Convective_Flux(d, dls, &B.fN[0][3 * f], B.fA[0][f], B.Pc(i - 1, j, k), B.Pc(i, j, k),
                                 B.Pc(i + 1, j, k), B.Pc(i + 2, j, k), B.Rc(i, j, k), B.Rc(i + 1, j, k), B.beta[B.inner(i, j, k)]))
              d->fail(ORC_ERR_INTERFACE_STATE, bi + 1, i, j, k);
          }
      if (d->cfg.model > 0) {   // diffusive i faces (:101-126)
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
        for (int k = 1; k <= n3; ++k)
          for (int j = 1; j <= n2; ++j)
            for (int i = 1; i <= n1 - 1; ++i) {
              size_t f = B.face(1, i, j, k);
              Diffusive_Flux(d, &B.fN[0][3 * f], B.fA[0][f], B.Pc(i, j, k), B.Pc(i + 1, j, k), B.Pc(i, j - 1, k),
                             B.Pc(i, j + 1, k), B.Pc(i + 1, j - 1, k), B.Pc(i + 1, j + 1, k), B.Pc(i, j, k - 1),
                             B.Pc(i, j, k + 1), B.Pc(i + 1, j, k - 1), B.Pc(i + 1, j, k + 1), &B.M_(1, 1, i, j, k),
                             &B.M_(1, 1, i + 1, j, k), B.Rc(i, j, k), B.Rc(i + 1, j, k), 1, 2, 3);
            }
      }
      // j faces (:129-139)
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
      for (int k = 1; k <= n3; ++k)
        for (int i = 1; i <= n1; ++i)
          for (int j = 1; j <= n2 - 1; ++j) {
            double dls[4] = {B.dl_(2, i, j - 1, k), B.dl_(2, i, j, k), B.dl_(2, i, j + 1, k), B.dl_(2, i, j + 2, k)};
            size_t f = B.face(2, i, j, k);
            if (!Convective_Flux(d, dls, &B.fN[1][3 * f], B.fA[1][f], B.Pc(i, j - 1, k), B.Pc(i, j, k),
                                 B.Pc(i, j + 1, k), B.Pc(i, j + 2, k), B.Rc(i, j, k), B.Rc(i, j + 1, k), B.beta[B.inner(i, j, k)]))
              d->fail(ORC_ERR_INTERFACE_STATE, bi + 1, i, j, k);
          }
      if (d->cfg.model > 0) {   // diffusive j faces (:141-166)
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
        for (int k = 1; k <= n3; ++k)
          for (int i = 1; i <= n1; ++i)
            for (int j = 1; j <= n2 - 1; ++j) {
              size_t f = B.face(2, i, j, k);
              Diffusive_Flux(d, &B.fN[1][3 * f], B.fA[1][f], B.Pc(i, j, k), B.Pc(i, j + 1, k), B.Pc(i - 1, j, k),
                             B.Pc(i + 1, j, k), B.Pc(i - 1, j + 1, k), B.Pc(i + 1, j + 1, k), B.Pc(i, j, k - 1),
                             B.Pc(i, j, k + 1), B.Pc(i, j + 1, k - 1), B.Pc(i, j + 1, k + 1), &B.M_(1, 1, i, j, k),
                             &B.M_(1, 1, i, j + 1, k), B.Rc(i, j, k), B.Rc(i, j + 1, k), 2, 1, 3);
            }
      }
      // k faces (:169-179)
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
      for (int j = 1; j <= n2; ++j)
        for (int i = 1; i <= n1; ++i)
          for (int k = 1; k <= n3 - 1; ++k) {
            double dls[4] = {B.dl_(3, i, j, k - 1), B.dl_(3, i, j, k), B.dl_(3, i, j, k + 1), B.dl_(3, i, j, k + 2)};
            size_t f = B.face(3, i, j, k);
            if (!Convective_Flux(d, dls, &B.fN[2][3 * f], B.fA[2][f], B.Pc(i, j, k - 1), B.Pc(i, j, k),
                                 B.Pc(i, j, k + 1), B.Pc(i, j, k + 2), B.Rc(i, j, k), B.Rc(i, j, k + 1), B.beta[B.inner(i, j, k)]))
              d->fail(ORC_ERR_INTERFACE_STATE, bi + 1, i, j, k);
          }
      if (d->cfg.model > 0) {   // diffusive k faces (:181-206)
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
        for (int j = 1; j <= n2; ++j)
          for (int i = 1; i <= n1; ++i)
            for (int k = 1; k <= n3 - 1; ++k) {
              size_t f = B.face(3, i, j, k);
              Diffusive_Flux(d, &B.fN[2][3 * f], B.fA[2][f], B.Pc(i, j, k), B.Pc(i, j, k + 1), B.Pc(i - 1, j, k),
                             B.Pc(i + 1, j, k), B.Pc(i - 1, j, k + 1), B.Pc(i + 1, j, k + 1), B.Pc(i, j - 1, k),
                             B.Pc(i, j + 1, k), B.Pc(i, j - 1, k + 1), B.Pc(i, j + 1, k + 1), &B.M_(1, 1, i, j, k),
                             &B.M_(1, 1, i, j, k + 1), B.Rc(i, j, k), B.Rc(i, j, k + 1), 3, 1, 2);
            }
      }
    }
  }
  return d->err;
}

// BC_Fluxes, Mod_BC_Fluxes.f90:10-218: in order of block and face.
int orc_bc_fluxes(orc_domain* d) {
  int upper = 0;
  int nb = (int)d->blk.size();
  for (int b = 1; b <= nb; ++b)
    for (int f = 1; f <= 6; ++f) {
      int lower = upper;
      upper = upper + d->n_bf[(b - 1) * 6 + (f - 1)];
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(d->nthreads)
#endif
      for (int q = lower; q < upper; ++q) {
        const BCrec& e = d->bc[q];
        Block& bm = d->blk[e.b - 1];
        switch (e.type) {
          case 101: case 201:
            BC_Connection_Eul(d, e.i, e.j, e.k, e.f, bm);
            if (d->cfg.model > 0)
              BC_Connection_Visc(d, e.i, e.j, e.k, e.f, bm, d->blk[e.bs - 1], e.is, e.js, e.ks, e.fs, e.d11, e.d12,
                                 e.d21, e.d22);
            break;
          case 300:
            BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            if (d->cfg.model > 0) BC_Symmetry_Visc(d, e.i, e.j, e.k, e.f, bm);
            break;
          case 301:   // Mod_BC_Fluxes.f90:87-95 (no rotating frame)
            BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            if (d->cfg.model > 0) BC_Wall_Heat(d, e.i, e.j, e.k, e.f, bm, e.data[0]);
            break;
          case 302:   // Mod_BC_Fluxes.f90:97-104
            BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            if (d->cfg.model > 0) BC_Wall_Temperature(d, e.i, e.j, e.k, e.f, bm, e.data[0]);
            break;
          case 400: BC_Extrapolation(d, e.i, e.j, e.k, e.f, bm); break;
          case 405:
            if (!BC_Inlet_Supersonic(d, e.i, e.j, e.k, e.f, bm, e.data)) BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            break;
          case 406:
            if (!BC_Outflow(d, e.i, e.j, e.k, e.f, bm, e.data)) BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            break;
          case 401:
            if (!BC_Inlet_StagnCond(d, e.i, e.j, e.k, e.f, bm, e.data)) BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            break;
          case 403: case 404:
            if (!BC_Inlet_MassFlux(d, e.i, e.j, e.k, e.f, bm, e.data, e.type == 403))
              BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            break;
          case 407: BC_FarField(d, e.i, e.j, e.k, e.f, bm, e.data); break;
          case 402: {
            // p0 from the time table at the domain time (Mod_BC_Fluxes.f90:129-140)
            double dd[6] = {e.data[0], series_update(d->series[(size_t)e.data[1]], d->time), e.data[2], e.data[3],
                            e.data[4], e.data[5]};
            if (!BC_Inlet_StagnCond(d, e.i, e.j, e.k, e.f, bm, dd)) BC_Symmetry_Eul(d, e.i, e.j, e.k, e.f, bm);
            break;
          }
          default: break;
        }
      }
    }
  return d->err;
}

// Residual_Smoothing, Lib_IRS.f90:14-39: per direction, the residual's first
// ghost layer (Ghost_Residual_Extrapolation :130-187: 101 copies the source
// cell, every other type the boundary cell), then per block two Jacobi
// sweeps of R* = R + beta (R*(-1) - 2 R* + R*(+1)) along that direction
// (Residual_Smoothing_Blk :42-103).
static void residual_smoothing(orc_domain* d, double beta) {
  const int njacobi = 2;
  for (int dir = 1; dir <= d->ndir; ++dir) {
    for (const BCrec& e : d->bc) {
      Block& B = d->blk[e.b - 1];
      int ig = e.i - G(e.f, 1), jg = e.j - G(e.f, 2), kg = e.k - G(e.f, 3);
      const double* src = (e.type == 101) ? d->blk[e.bs - 1].Rc(e.is, e.js, e.ks) : B.Rc(e.i, e.j, e.k);
      double* dst = B.Rc(ig, jg, kg);
      for (int v = 0; v < NPRIM; ++v) dst[v] = src[v];
    }
    const int di = dir == 1, dj = dir == 2, dk = dir == 3;
    for (Block& B : d->blk) {
      std::vector<double> Rs(B.R), Rsn(B.R.size());
      for (int it = 1; it <= njacobi; ++it) {
        for (int k = 1; k <= B.nk; ++k)
          for (int j = 1; j <= B.nj; ++j)
            for (int i = 1; i <= B.ni; ++i) {
              const double* r = B.Rc(i, j, k);
              const double* rm = &Rs[NPRIM * B.cell(i - di, j - dj, k - dk)];
              const double* rp = &Rs[NPRIM * B.cell(i + di, j + dj, k + dk)];
              double* o = &Rsn[NPRIM * B.cell(i, j, k)];
              for (int v = 0; v < NPRIM; ++v) o[v] = (r[v] + beta * (rm[v] + rp[v])) / (1.0 + 2.0 * beta);
            }
        for (int k = 1; k <= B.nk; ++k)
          for (int j = 1; j <= B.nj; ++j)
            for (int i = 1; i <= B.ni; ++i)
              for (int v = 0; v < NPRIM; ++v) Rs[NPRIM * B.cell(i, j, k) + v] = Rsn[NPRIM * B.cell(i, j, k) + v];
      }
      for (int k = 1; k <= B.nk; ++k)
        for (int j = 1; j <= B.nj; ++j)
          for (int i = 1; i <= B.ni; ++i)
            for (int v = 0; v < NPRIM; ++v) B.Rc(i, j, k)[v] = Rs[NPRIM * B.cell(i, j, k) + v];
    }
  }
}

// Compute_Prim_Residual, Lib_Newstate.f90:255-302 (one calorically perfect
// species): the conservative residual of a cell turned, in place, into the
// increment of its primitives over dt.
static void prim_residual(const Thermo& t, const double* prim, double* res, double dt, double volume,
                          double strangcoeff) {
  double rho, Rgas;
  co_rotot_Rtot(t, prim[0], rho, Rgas);
  double temperature = prim[NP] / (rho * Rgas);
  double inv_volume = 1.0 / volume;
  double inv_rhovolume = inv_volume / rho;
  double velocity[3] = {prim[NU], prim[NV], prim[NW]};
  res[0] = -res[0] * inv_volume;
  double dwrotot = res[0];
  for (int q = 0; q < 3; ++q) res[NU + q] = -res[NU + q] * inv_rhovolume - velocity[q] / rho * dwrotot;
  double dwE = -res[NP] * inv_volume;
  double dwroe = dwE - rho * (velocity[0] * res[NU] + velocity[1] * res[NV] + velocity[2] * res[NW]) -
                 0.5 * dwrotot * (velocity[0] * velocity[0] + velocity[1] * velocity[1] + velocity[2] * velocity[2]);
  double eiroi = (t.cp * temperature - t.R * temperature) * res[0];
  double cv = prim[0] * (t.cp - t.R);
  double dwTemp = (dwroe - eiroi) / cv;
  res[NP] = t.R * (temperature * res[0] + prim[0] * dwTemp);
  for (int v = 0; v < NPRIM; ++v) res[v] = res[v] * dt * strangcoeff;
}

// RK_Newstate => Newstate_Conservative / Newstate_Primitive, Lib_Newstate.f90
int orc_rk_newstate(orc_domain* d, int irk) {
  static const double RKcoeff[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0 / 3.0}};  // Lib_RK.f90:8-11
  const int n_rk = d->cfg.n_rk;
  const double c = RKcoeff[n_rk - 1][irk - 1];
  const double strangcoeff = 1.0;
  const Thermo& t = d->th;
  const bool prim_mode = d->cfg.integration == ORC_INT_PRIM;
  if (d->cfg.irs_beta > 0.0 && prim_mode) {
    // Newstate_Primitive with IRS, Lib_Newstate.f90:195-231: every residual
    // to primitive increments, smooth, then RK_stage and Check_And_Fix_State
    for (Block& B : d->blk)
      for (int k = 1; k <= B.nk; ++k)
        for (int j = 1; j <= B.nj; ++j)
          for (int i = 1; i <= B.ni; ++i)
            prim_residual(t, B.Pc(i, j, k), B.Rc(i, j, k), B.dtlocal[B.inner(i, j, k)], B.vol_(i, j, k), strangcoeff);
    residual_smoothing(d, d->cfg.irs_beta);
    for (int bi = 0; bi < (int)d->blk.size(); ++bi) {
      Block& B = d->blk[bi];
      for (int k = 1; k <= B.nk; ++k)
        for (int j = 1; j <= B.nj; ++j)
          for (int i = 1; i <= B.ni; ++i) {
            double* prim = B.Pc(i, j, k);
            const double* primold = B.POc(i, j, k);
            const double* res = B.Rc(i, j, k);
            for (int v = 0; v < NPRIM; ++v) {
              double r_ = (prim[v] - primold[v] + res[v]) * c;
              prim[v] = primold[v] + r_;
            }
            bool nan = false;
            for (int v = 0; v < NPRIM; ++v) nan |= std::isnan(prim[v]);
            if (nan || prim[NP] < 0.0) d->fail(ORC_ERR_NAN_OR_NEG_P, bi + 1, i, j, k);
            if (prim[0] < 1e-20) prim[0] = 1e-20;
          }
    }
    return d->err;
  }
  if (d->cfg.irs_beta > 0.0 && !prim_mode) {
    // Newstate_Conservative with IRS, Lib_Newstate.f90:40-72: scale every
    // residual (Scale_Residual_Cons), smooth, then Update_State_Cons_IRS
    for (Block& B : d->blk)
      for (int k = 1; k <= B.nk; ++k)
        for (int j = 1; j <= B.nj; ++j)
          for (int i = 1; i <= B.ni; ++i) {
            double* res = B.Rc(i, j, k);
            double dt = B.dtlocal[B.inner(i, j, k)];
            double volume = B.vol_(i, j, k);
            for (int v = 0; v < NPRIM; ++v) res[v] = -(res[v] / volume * dt * strangcoeff);
          }
    residual_smoothing(d, d->cfg.irs_beta);
    for (int bi = 0; bi < (int)d->blk.size(); ++bi) {
      Block& B = d->blk[bi];
      for (int k = 1; k <= B.nk; ++k)
        for (int j = 1; j <= B.nj; ++j)
          for (int i = 1; i <= B.ni; ++i) {
            double* prim = B.Pc(i, j, k);
            const double* primold = B.POc(i, j, k);
            const double* res = B.Rc(i, j, k);
            double consold[NPRIM], cons[NPRIM];
            prim2cons(t, primold, consold);
            prim2cons(t, prim, cons);
            for (int v = 0; v < NPRIM; ++v) {
              double r_ = (cons[v] - consold[v] + res[v]) * c;
              cons[v] = consold[v] + r_;
            }
            cons2prim(t, cons, prim);
            bool nan = false;
            for (int v = 0; v < NPRIM; ++v) nan |= std::isnan(prim[v]);
            if (nan || prim[NP] < 0.0) d->fail(ORC_ERR_NAN_OR_NEG_P, bi + 1, i, j, k);
            if (prim[0] < 1e-20) prim[0] = 1e-20;
          }
    }
    return d->err;
  }
  for (int bi = 0; bi < (int)d->blk.size(); ++bi) {
    Block& B = d->blk[bi];
#ifdef _OPENMP
#pragma omp parallel for collapse(3) schedule(static) num_threads(d->nthreads)
#endif
    for (int k = 1; k <= B.nk; ++k)
      for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i) {
          double* prim = B.Pc(i, j, k);
          const double* primold = B.POc(i, j, k);
          double* res = B.Rc(i, j, k);
          double dt = B.dtlocal[B.inner(i, j, k)];
          double volume = B.vol_(i, j, k);
          if (!prim_mode) {
            // Compute_Cons_NoIRS :134-160
            for (int v = 0; v < NPRIM; ++v) res[v] = -(res[v] / volume * dt * strangcoeff);
            double consold[NPRIM], cons[NPRIM];
            prim2cons(t, primold, consold);
            prim2cons(t, prim, cons);
            for (int v = 0; v < NPRIM; ++v) {        // RK_stage, Lib_RK.f90:15-27
              double r_ = (cons[v] - consold[v] + res[v]) * c;
              cons[v] = consold[v] + r_;
            }
            double rho, Rgas;
            co_rotot_Rtot(t, prim[0], rho, Rgas);
            double temperature = prim[NP] / (rho * Rgas);
            (void)temperature;                        // T_guess: closed-form cons2prim
            cons2prim(t, cons, prim);
          } else {
            // Compute_And_Update_Prim :305-315: Compute_Prim_Residual, then RK_Stage
            prim_residual(t, prim, res, dt, volume, strangcoeff);
            for (int v = 0; v < NPRIM; ++v) {
              double r_ = (prim[v] - primold[v] + res[v]) * c;
              prim[v] = primold[v] + r_;
            }
          }
          // Check_And_Fix_State :323-356
          bool nan = false;
          for (int v = 0; v < NPRIM; ++v) nan |= std::isnan(prim[v]);
          if (nan || prim[NP] < 0.0) d->fail(ORC_ERR_NAN_OR_NEG_P, bi + 1, i, j, k);
          if (prim[0] < 1e-20) prim[0] = 1e-20;
        }
  }
  return d->err;
}

int orc_copy_state(orc_domain* d) {   // Copy_State, Mod_Explicit.f90:149-170
  for (auto& B : d->blk) {
#ifdef _OPENMP
#pragma omp parallel for collapse(3) num_threads(d->nthreads)
#endif
    for (int k = 1; k <= B.nk; ++k)
      for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i) {
          const double* p = B.Pc(i, j, k);
          double* po = B.POc(i, j, k);
          for (int v = 0; v < NPRIM; ++v) po[v] = p[v];
        }
  }
  return ORC_OK;
}

// Compute_dt, Mod_dt.f90:10-106 (Euler: CFL only).
int orc_compute_dt(orc_domain* d, double* dtglobal_out) {
  double dtglobal = d->dtglobal;
  const Thermo& t = d->th;
  const double cfl = d->cfg.cfl;
  const int ndir = d->ndir;
  for (auto& B : d->blk) {
    double dtg = dtglobal;
#ifdef _OPENMP
#pragma omp parallel for collapse(3) reduction(min : dtg) num_threads(d->nthreads)
#endif
    for (int k = 1; k <= B.nk; ++k)
      for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i) {
          const double* p = B.Pc(i, j, k);
          double rho, Rgas;
          co_rotot_Rtot(t, p[0], rho, Rgas);
          double Sound = f_ss(t, p[0], p[NP], rho, Rgas);
          double dtmin = 1e8;
          double vel[3] = {p[NU], p[NV], p[NW]};
          for (int dd = 1; dd <= ndir; ++dd) {
            double met[3] = {B.M_(dd, 1, i, j, k), B.M_(dd, 2, i, j, k), B.M_(dd, 3, i, j, k)};
            double nrm = norm2(met[0], met[1], met[2]);
            double versor[3] = {met[0] / nrm, met[1] / nrm, met[2] / nrm};
            double vel_ = std::fabs(dot3(vel, versor));
            double lambda = vel_ + Sound;
            double dt = B.dl_(dd, i, j, k) / lambda * cfl;
            dtmin = std::min(dt, dtmin);
          }
          if (d->cfg.model > 0) {   // VNN condition, Mod_dt.f90:87-103 (laminar: mi = 0 + mil)
            const double mi = 0.0 + d->cfg.mu;
            for (int dd = 1; dd <= ndir; ++dd) {
              const double dlv = B.dl_(dd, i, j, k);
              double dt = (rho * (dlv * dlv) * d->cfg.vnn) / mi;
              dtmin = std::min(dt, dtmin);
            }
          }
          double dtcell = dtmin;
          if (d->iter < d->cfg.ramp_iter) dtcell = dtcell * (double)d->iter / (double)d->cfg.ramp_iter;
          B.dtlocal[B.inner(i, j, k)] = dtcell;
          dtg = std::min(dtcell, dtg);
        }
    dtglobal = dtg;
  }
  d->dtglobal = dtglobal;
  if (dtglobal_out) *dtglobal_out = dtglobal;
  return ORC_OK;
}

int orc_set_global_dt(orc_domain* d) {   // Set_Global_dt, Mod_dt.f90:110-130
  for (auto& B : d->blk) std::fill(B.dtlocal.begin(), B.dtlocal.end(), d->dtglobal);
  return ORC_OK;
}

// Explicit_Step, Mod_Explicit.f90:10-97 (no Strang, no sources, no coupling hook).
int orc_explicit_step(orc_domain* d, double* dtglobal, double* time) {
  d->iter = d->iter + 1;
  d->iter_from_call = d->iter_from_call + 1;
  d->dtglobal = 1e5;
  orc_compute_dt(d, nullptr);
  if (d->cfg.time_accurate) {
    orc_set_global_dt(d);
    d->time = d->time + d->dtglobal;
  }
  orc_copy_state(d);
  for (int i_rk = 1; i_rk <= d->cfg.n_rk; ++i_rk) {
    orc_fill_ghost_cell(d);
    orc_fluxes(d);
    orc_bc_fluxes(d);
    orc_rk_newstate(d, i_rk);
    if (d->err) break;
  }
  if (dtglobal) *dtglobal = d->dtglobal;
  if (time) *time = d->time;
  return d->err;
}

// Compute_Residual, Mod_Diagnostic.f90:13-50, summed over blocks.
int orc_compute_residual(const orc_domain* d, double* total) {
  for (int q = 0; q < NRES; ++q) total[q] = 0.0;
  for (const auto& B : d->blk) {
    double residuo[NRES] = {0, 0, 0, 0, 0};
    for (int k = 1; k <= B.nk; ++k)
      for (int j = 1; j <= B.nj; ++j)
        for (int i = 1; i <= B.ni; ++i) {
          const double* pn = &B.P[NPRIM * B.cell(i, j, k)];
          const double* po = &B.PO[NPRIM * B.cell(i, j, k)];
          double resn[NRES];
          resn[0] = std::fabs(pn[0] - po[0]);
          for (int v = 1; v < NRES; ++v) resn[v] = std::fabs(pn[v] - po[v]);
          for (int v = 0; v < NRES; ++v) residuo[v] = residuo[v] + resn[v] * resn[v];
        }
    for (int v = 0; v < NRES; ++v) total[v] = total[v] + residuo[v];
  }
  return ORC_OK;
}

void orc_set_time(orc_domain* d, double time, int iter) {
  d->time = time;
  d->iter = iter;
}
double orc_get_time(const orc_domain* d) { return d->time; }
void orc_set_dtglobal(orc_domain* d, double dtglobal) { d->dtglobal = dtglobal; }

int orc_last_error(const orc_domain* d, int* b, int* i, int* j, int* k) {
  if (b) *b = d->eb;
  if (i) *i = d->ei;
  if (j) *j = d->ej;
  if (k) *k = d->ek;
  return d->err;
}

double orc_limiter(int limiter, double x, double y) { return rlimiter(limiter, x, y); }

void orc_riemann(const orc_domain* d, const double* left, const double* right, const double* normal,
                 double* flux) {
  bool bad = false;
  RState L = make_state(d->th, left, bad);
  RState R = make_state(d->th, right, bad);
  RFlux F = Riemann(d, L, R, normal[0], normal[1], normal[2]);
  flux[0] = F.r; flux[1] = F.u; flux[2] = F.v; flux[3] = F.w; flux[4] = F.E;
}

}  // extern "C"
