// physics_fast.cuh -- FP64 and mixed FP32/FP64 face physics: the same
// algorithm as physics_exact.cuh, restated for speed.
//
// FP64 ("fp64" precision): the single-species calorically perfect algebra is
// simplified where it is an identity in exact arithmetic (rho_s/rho = 1,
// R_roe = R, gamma_roe = gamma, cv_roe T_roe - sum_ei = 0, h = gamma/(gamma-1)
// p/rho), divisions and square roots become reciprocals / reciprocal square
// roots refined by Newton-Raphson from the hardware seed, and the compiler
// contracts multiply-adds.  Branch-free, so independent faces interleave.
// Results stay within ~1e-14 relative of the reference arithmetic; the
// tests hold them to the 1e-12 normwise bar.
//
// Mixed ("mixed" precision): the limited slopes and the Riemann solver's wave
// structure (sound speeds, Roe averages, signal speeds, star state) run in
// FP32 with single-instruction reciprocals; the upwind physical flux and the
// interface states stay FP64, so the FP32 rounding only touches the small
// dissipative part of each face flux.
#pragma once

#include "common.cuh"

namespace mose {
namespace fast {

// ---- reciprocal / reciprocal square root ------------------------------------
// Seed from the hardware approximation of the leading bits, then ONE
// third-order (Householder) correction, which cubes the seed's relative
// error d: with e = 1 - x r (= d),
//   1/x       = r (1 + e + e^2 + ...)          -> r + r (e + e^2)
//   1/sqrt(x) = y (1 + e/2 + 3 e^2 / 8 + ...)  with e = 1 - x y^2
// (Householder, The Numerical Treatment of a Single Nonlinear Equation,
// 1970; Muller et al., Handbook of Floating-Point Arithmetic, ch. 4).  A seed
// good to 2^-18 or better leaves the cubic term below 2^-54, so the result is
// within about one ulp; the accuracy is checked on the device against IEEE
// division and square root.  Valid for normal, finite, positive x (rcp: any
// normal x).
__device__ __forceinline__ double rcp(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  const double e = fma(-x, r, 1.0);
  return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ double rsqrt_(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x * y, y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}
// sqrt(x) = x rsqrt(x) with one residual correction; sqrt(0) = 0.
__device__ __forceinline__ double sqrt_(double x) {
  double y = rsqrt_(x);
  double s = x * y;
  double e = fma(-s, s, x);          // x - s^2
  s = fma(0.5 * y, e, s);
  return x > 0.0 ? s : 0.0;
}
__device__ __forceinline__ double div_(double a, double b) { return a * rcp(b); }
// Sign tests on the high word, on the integer pipe instead of the FP64 one
// (the stage kernels are bound by the FP64 pipe): sgn_neg(x) for x < 0 or
// -0 (or a NaN with the sign bit set), pos_(x) for x > 0 (or a positive NaN).
__device__ __forceinline__ bool sgn_neg(double x) { return __double2hiint(x) < 0; }
__device__ __forceinline__ bool pos_(double x) { return __double_as_longlong(x) > 0; }
// sqrt(x) = x rsqrt(x) without the residual correction (about 1.5 ulp): the
// sound speeds of the Riemann solver, where that is far inside the bar
__device__ __forceinline__ double sqrt1_(double x) { return pos_(x) ? x * rsqrt_(x) : 0.0; }

// ---- limiters: phi(r) x with r = y/(x + 1e-30), one reciprocal each --------
// The rational limiters are rewritten over a common denominator, which is
// positive whenever x + 1e-30 != 0 (the only x the reference divides by).
template <int LIM>
__device__ __forceinline__ double limiter(double x, double y) {
  if constexpr (LIM == 1) {            // minmod
    double r = (fabs(x) > fabs(y)) ? y : x;
    return (x * y < 0.0) ? 0.0 : r;
  } else if constexpr (LIM == 2) {     // van Leer: x (y sgn(x') + |y|) / (|x'| + |y|)
    const double xp = x + 1e-30;
    const double num = y * copysign(1.0, xp) + fabs(y);
    return (x * num) * rcp(fabs(xp) + fabs(y));
  } else if constexpr (LIM == 3) {     // van Albada: x (y^2 + y x') / (x'^2 + y^2)
    const double xp = x + 1e-30;
    const double num = y * (y + xp);
    return (x * num) * rcp(fma(xp, xp, y * y));
  } else if constexpr (LIM == 4) {     // MC
    const double ru = y * rcp(x + 1e-30);
    return fmax(0.0, fmin(fmin(2.0 * ru, 0.5 * (1.0 + ru)), 2.0)) * x;
  } else if constexpr (LIM == 5) {     // superbee
    const double ru = y * rcp(x + 1e-30);
    return fmax(fmax(0.0, fmin(2.0 * ru, 1.0)), fmin(ru, 2.0)) * x;
  } else {
    return 0.0;
  }
}

// ---- FP32 building blocks ---------------------------------------------------
// Single-instruction approximations (relative error about 2^-22 / 2^-23):
// the FP32 Riemann solve is an approximation of the FP64 one by design, and
// its error against the FP64 oracle is measured, not assumed.
__device__ __forceinline__ float frcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float frsq(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
// sqrt(x) for x > 0 (x rsqrt(x))
__device__ __forceinline__ float fsqrtp(float x) { return x * frsq(x); }

// FP32 limiters.  The denominator is floored at FLT_MIN: where it would be
// zero the numerator is zero too, and 0 * (1 / FLT_MIN) = 0.
template <int LIM>
__device__ __forceinline__ float limiter32(float x, float y) {
  constexpr float kMin = 1.17549435e-38f;
  if constexpr (LIM == 1) {
    float r = (fabsf(x) > fabsf(y)) ? y : x;
    return (x * y < 0.0f) ? 0.0f : r;
  } else if constexpr (LIM == 2) {
    const float xp = x + 1e-30f;
    const float num = y * copysignf(1.0f, xp) + fabsf(y);
    return (x * num) * frcp(fmaxf(fabsf(xp) + fabsf(y), kMin));
  } else if constexpr (LIM == 3) {
    const float xp = x + 1e-30f;
    const float num = y * (y + xp);
    return (x * num) * frcp(fmaxf(fmaf(xp, xp, y * y), kMin));
  } else if constexpr (LIM == 4) {
    const float ru = y * frcp(x + 1e-30f);
    return fmaxf(0.0f, fminf(fminf(2.0f * ru, 0.5f * (1.0f + ru)), 2.0f)) * x;
  } else if constexpr (LIM == 5) {
    const float ru = y * frcp(x + 1e-30f);
    return fmaxf(fmaxf(0.0f, fminf(2.0f * ru, 1.0f)), fminf(ru, 2.0f)) * x;
  } else {
    return 0.0f;
  }
}
template <int LIM>
__device__ __forceinline__ float4 limiter32x4(float4 x, float4 y) {
  return make_float4(limiter32<LIM>(x.x, y.x), limiter32<LIM>(x.y, y.y), limiter32<LIM>(x.z, y.z),
                     limiter32<LIM>(x.w, y.w));
}

struct GasF {
  double gamma, gm1, gcp;       // gamma, gamma - 1, gamma / (gamma - 1)
  double igm1;                  // 1 / (gamma - 1)
};
__device__ __forceinline__ GasF gasf(const Gas& g) {
  GasF f;
  f.gamma = g.gamma;
  f.gm1 = g.gm1;
  f.gcp = g.gcp;
  f.igm1 = g.igm1;
  return f;
}

template <int NV>
__device__ __forceinline__ double un(const double* q, const double* n) {
  if constexpr (NV == 5) return q[1] * n[0] + q[2] * n[1] + q[3] * n[2];
  else return q[1] * n[0] + q[2] * n[1];
}
template <int NV>
__device__ __forceinline__ double v2(const double* q) {
  if constexpr (NV == 5) return q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  else return q[1] * q[1] + q[2] * q[2];
}

// Batten HLLC (Lib_Riemann_HLL.f90:147-258) in FP64, branch free: the side
// and the star correction are selected, not branched to.
template <int NV>
__device__ __forceinline__ void hllc(const GasF& g, const double* L, const double* R, const double* n, double* F) {
  constexpr int P = NV - 1;
  const double rl = L[0], rr = R[0];
  const double rsl = rsqrt_(rl), rsr = rsqrt_(rr);
  const double srL = rl * rsl, srR = rr * rsr;          // sqrt(rho)
  const double irl = rsl * rsl, irr = rsr * rsr;        // 1/rho
  const double unl = un<NV>(L, n), unr = un<NV>(R, n);
  const double pol = L[P] * irl, por = R[P] * irr;      // p/rho
  const double aL = sqrt1_(g.gamma * pol), aR = sqrt1_(g.gamma * por);
  const double h0l = fma(g.gcp, pol, 0.5 * v2<NV>(L));
  const double h0r = fma(g.gcp, por, 0.5 * v2<NV>(R));
  const double isr = rcp(srL + srR);
  const double wl = srL * isr, wr = srR * isr;
  double ur[3];
  ur[0] = fma(wr, R[1], wl * L[1]);
  ur[1] = fma(wr, R[2], wl * L[2]);
  ur[2] = 0.0;
  if constexpr (NV == 5) ur[2] = fma(wr, R[3], wl * L[3]);
  const double h0_roe = fma(wr, h0r, wl * h0l);
  const double vel2 = ur[0] * ur[0] + ur[1] * ur[1] + ur[2] * ur[2];
  const double a_roe = sqrt1_(g.gm1 * fma(-0.5, vel2, h0_roe));
  const double un_roe = (NV == 5) ? ur[0] * n[0] + ur[1] * n[1] + ur[2] * n[2] : ur[0] * n[0] + ur[1] * n[1];
  // min(0, unl - aL, un_roe - a_roe) and max(0, unr + aR, un_roe + a_roe),
  // the comparisons with 0 as sign tests
  const double t1 = unl - aL, t4 = unr + aR;
  const double S1 = fmin(sgn_neg(t1) ? t1 : 0.0, un_roe - a_roe);
  const double S4 = fmax(sgn_neg(t4) ? 0.0 : t4, un_roe + a_roe);
  const double ml = rl * (S1 - unl), mr = rr * (S4 - unr);
  const double idn = rcp(ml - mr);
  const double Sstar = (R[P] - L[P] + ml * unl - mr * unr) * idn;
  // upwind side K: left when S1 >= 0 or Sstar >= 0 (a -0 takes the other
  // branch, to which the flux is continuous)
  const bool left = !sgn_neg(S1) || !sgn_neg(Sstar);
  const double* K = left ? L : R;
  const double rk = left ? rl : rr, unk = left ? unl : unr, h0k = left ? h0l : h0r;
  const double SK = left ? S1 : S4;
  const double pk = K[P];
  const double e0k = h0k - pk * (left ? irl : irr);
  F[0] = rk * unk;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = fma(F[0], K[1 + d], pk * n[d]);
  F[P] = F[0] * h0k;
  // star correction, applied when K's outer wave is subsonic in the face frame
  const bool corr = left ? sgn_neg(S1) : pos_(S4);
  const double mk = left ? ml : mr;                        // rho_K (S_K - un_K)
  const double pstar = fma(rl * (unl - S1), unl - Sstar, L[P]);
  const double inv = rcp(SK - Sstar);
  const double dp = pstar - pk;
  const double c0 = SK * (mk * inv - rk);                  // S_K (U*_1 - rho_K)
  double c[5];
  c[0] = c0;
  for (int d = 0; d < NV - 2; ++d) c[1 + d] = SK * (fma(mk, K[1 + d], dp * n[d]) * inv - rk * K[1 + d]);
  c[P] = SK * ((mk * e0k - pk * unk + pstar * Sstar) * inv - rk * e0k);
  for (int v = 0; v < NV; ++v) F[v] = corr ? F[v] + c[v] : F[v];
}

// AUSM+ (Lib_Riemann_AUSM.f90:150-238) in FP64.
template <int NV>
__device__ __forceinline__ void ausmp(const GasF& g, const double* L, const double* R, const double* n, double* F) {
  constexpr int P = NV - 1;
  const double beta = 0.125, alpha = 0.1875;
  const double irl = rcp(L[0]), irr = rcp(R[0]);
  const double unl = un<NV>(L, n), unr = un<NV>(R, n);
  const double pol = L[P] * irl, por = R[P] * irr;
  const double H_L = fma(g.gcp, pol, 0.5 * v2<NV>(L));
  const double H_R = fma(g.gcp, por, 0.5 * v2<NV>(R));
  const double a_half = sqrt_(g.gamma * sqrt_(pol * por));   // sqrt(aL aR)
  const double ia = rcp(a_half);
  const double ML = unl * ia, MR = unr * ia;
  const double mL2 = (ML * ML - 1.0), mR2 = (MR * MR - 1.0);
  const double sub_Mp = fma(0.25 * (ML + 1.0), ML + 1.0, beta * mL2 * mL2);
  const double sub_pp = fma(0.25 * (ML + 1.0) * (ML + 1.0), 2.0 - ML, alpha * ML * mL2 * mL2);
  const double sub_Mm = -fma(0.25 * (MR - 1.0), MR - 1.0, beta * mR2 * mR2);
  const double sub_pm = fma(0.25 * (MR - 1.0) * (MR - 1.0), 2.0 + MR, -alpha * MR * mR2 * mR2);
  const bool sl = fabs(ML) < 1.0, sr = fabs(MR) < 1.0;
  const double MplusL = sl ? sub_Mp : 0.5 * (ML + fabs(ML));
  const double pplusL = sl ? sub_pp : 0.5 * (1.0 + copysign(1.0, ML));
  const double MminusR = sr ? sub_Mm : 0.5 * (MR - fabs(MR));
  const double pminusR = sr ? sub_pm : 0.5 * (1.0 - copysign(1.0, MR));
  const double Mhalf = MplusL + MminusR;
  const double phalf = fma(pplusL, L[P], pminusR * R[P]);
  const double mdotp = L[0] * a_half * 0.5 * (Mhalf + fabs(Mhalf));
  const double mdotm = R[0] * a_half * 0.5 * (Mhalf - fabs(Mhalf));
  F[0] = mdotp + mdotm;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = fma(mdotp, L[1 + d], fma(mdotm, R[1 + d], n[d] * phalf));
  F[P] = fma(mdotp, H_L, mdotm * H_R);
}

// ---- mixed: FP32 wave structure, FP64 upwind flux ----------------------------
template <int NV>
__device__ __forceinline__ void hllc_mixed(const GasF& g, const double* L, const double* R, const double* n,
                                           double* F) {
  constexpr int P = NV - 1;
  const float gam = (float)g.gamma, gm1 = (float)g.gm1;
  float l[5], r[5], nf[3];
  for (int v = 0; v < NV; ++v) { l[v] = (float)L[v]; r[v] = (float)R[v]; }
  for (int d = 0; d < 3; ++d) nf[d] = (float)n[d];
  const float rsl = rsqrtf(l[0]), rsr = rsqrtf(r[0]);
  const float srL = l[0] * rsl, srR = r[0] * rsr;
  const float irl = rsl * rsl, irr = rsr * rsr;
  float unl = l[1] * nf[0] + l[2] * nf[1], unr = r[1] * nf[0] + r[2] * nf[1];
  float vl2 = l[1] * l[1] + l[2] * l[2], vr2 = r[1] * r[1] + r[2] * r[2];
  if constexpr (NV == 5) {
    unl += l[3] * nf[2]; unr += r[3] * nf[2];
    vl2 += l[3] * l[3]; vr2 += r[3] * r[3];
  }
  const float pol = l[P] * irl, por = r[P] * irr;
  const float aL = sqrtf(gam * pol), aR = sqrtf(gam * por);
  const float gcp = (float)g.gcp;
  const float h0l = fmaf(gcp, pol, 0.5f * vl2), h0r = fmaf(gcp, por, 0.5f * vr2);
  const float isr = __frcp_rn(srL + srR);
  const float wl = srL * isr, wr = srR * isr;
  float ur0 = fmaf(wr, r[1], wl * l[1]), ur1 = fmaf(wr, r[2], wl * l[2]), ur2 = 0.0f;
  if constexpr (NV == 5) ur2 = fmaf(wr, r[3], wl * l[3]);
  const float h0_roe = fmaf(wr, h0r, wl * h0l);
  const float a_roe = sqrtf(fmaxf(gm1 * fmaf(-0.5f, ur0 * ur0 + ur1 * ur1 + ur2 * ur2, h0_roe), 0.0f));
  const float un_roe = ur0 * nf[0] + ur1 * nf[1] + ur2 * nf[2];
  const float S1 = fminf(fminf(0.0f, unl - aL), un_roe - a_roe);
  const float S4 = fmaxf(fmaxf(0.0f, unr + aR), un_roe + a_roe);
  const float ml = l[0] * (S1 - unl), mr = r[0] * (S4 - unr);
  const float Sstar = __fdividef(r[P] - l[P] + ml * unl - mr * unr, ml - mr);
  const bool left = (S1 >= 0.0f) || (Sstar >= 0.0f);
  // FP64 physical flux of the upwind state
  const double* K = left ? L : R;
  const double unK = (NV == 5) ? K[1] * n[0] + K[2] * n[1] + K[3] * n[2] : K[1] * n[0] + K[2] * n[1];
  const double iK = 1.0 / K[0];
  const double pK = K[P];
  const double h0K = fma(g.gcp, pK * iK, 0.5 * v2<NV>(K));
  F[0] = K[0] * unK;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = fma(F[0], K[1 + d], pK * n[d]);
  F[P] = F[0] * h0K;
  // FP32 star correction S_K (U*_K - U_K)
  const bool corr = left ? (S1 < 0.0f) : (S4 > 0.0f);
  const float SK = left ? S1 : S4;
  const float* k = left ? l : r;
  const float mk = left ? ml : mr, unk = left ? unl : unr, rk = k[0];
  const float pstar = fmaf(l[0] * (unl - S1), unl - Sstar, l[P]);
  const float inv = __frcp_rn(SK - Sstar);
  const float dp = pstar - k[P];
  const float e0k = (left ? h0l : h0r) - k[P] * (left ? irl : irr);
  float c[5];
  c[0] = SK * (mk * inv - rk);
  for (int d = 0; d < NV - 2; ++d) c[1 + d] = SK * (fmaf(mk, k[1 + d], dp * nf[d]) * inv - rk * k[1 + d]);
  c[P] = SK * ((mk * e0k - k[P] * unk + pstar * Sstar) * inv - rk * e0k);
  for (int v = 0; v < NV; ++v) F[v] = corr ? F[v] + (double)c[v] : F[v];
}

template <int NV>
__device__ __forceinline__ void ausmp_mixed(const GasF& g, const double* L, const double* R, const double* n,
                                            double* F) {
  constexpr int P = NV - 1;
  const float beta = 0.125f, alpha = 0.1875f;
  float l[5], r[5], nf[3];
  for (int v = 0; v < NV; ++v) { l[v] = (float)L[v]; r[v] = (float)R[v]; }
  for (int d = 0; d < 3; ++d) nf[d] = (float)n[d];
  const float irl = __frcp_rn(l[0]), irr = __frcp_rn(r[0]);
  float unl = l[1] * nf[0] + l[2] * nf[1], unr = r[1] * nf[0] + r[2] * nf[1];
  if constexpr (NV == 5) { unl += l[3] * nf[2]; unr += r[3] * nf[2]; }
  const float a_half = sqrtf((float)g.gamma * sqrtf(l[P] * irl * r[P] * irr));
  const float ia = __frcp_rn(a_half);
  const float ML = unl * ia, MR = unr * ia;
  const float mL2 = ML * ML - 1.0f, mR2 = MR * MR - 1.0f;
  const bool sl = fabsf(ML) < 1.0f, sr = fabsf(MR) < 1.0f;
  const float MplusL = sl ? fmaf(0.25f * (ML + 1.0f), ML + 1.0f, beta * mL2 * mL2) : 0.5f * (ML + fabsf(ML));
  const float pplusL = sl ? fmaf(0.25f * (ML + 1.0f) * (ML + 1.0f), 2.0f - ML, alpha * ML * mL2 * mL2)
                          : 0.5f * (1.0f + copysignf(1.0f, ML));
  const float MminusR = sr ? -fmaf(0.25f * (MR - 1.0f), MR - 1.0f, beta * mR2 * mR2) : 0.5f * (MR - fabsf(MR));
  const float pminusR = sr ? fmaf(0.25f * (MR - 1.0f) * (MR - 1.0f), 2.0f + MR, -alpha * MR * mR2 * mR2)
                           : 0.5f * (1.0f - copysignf(1.0f, MR));
  const float Mhalf = MplusL + MminusR;
  // mass fluxes and pressure in FP32, the transported quantities in FP64
  const double mdotp = (double)(l[0] * a_half * 0.5f * (Mhalf + fabsf(Mhalf)));
  const double mdotm = (double)(r[0] * a_half * 0.5f * (Mhalf - fabsf(Mhalf)));
  const double phalf = (double)pplusL * L[P] + (double)pminusR * R[P];
  const double H_L = fma(g.gcp, L[P] / L[0], 0.5 * v2<NV>(L));
  const double H_R = fma(g.gcp, R[P] / R[0], 0.5 * v2<NV>(R));
  F[0] = mdotp + mdotm;
  for (int d = 0; d < NV - 2; ++d) F[1 + d] = fma(mdotp, L[1 + d], fma(mdotm, R[1 + d], n[d] * phalf));
  F[P] = fma(mdotp, H_L, mdotm * H_R);
}

// ---- complete FP32 face solves (2-D: states (rho, u, v, p), normal (nx, ny)) --
struct GasF32 {
  float gamma, gm1, gcp;   // gamma, gamma - 1, gamma / (gamma - 1)
};
__device__ __forceinline__ GasF32 gasf32(const Gas& g) {
  GasF32 f;
  f.gamma = (float)g.gamma;
  f.gm1 = (float)g.gm1;
  f.gcp = (float)g.gcp;
  return f;
}

// Batten HLLC (Lib_Riemann_HLL.f90:147-258) in FP32, flux per unit area.
// The star correction S_K (U*_K - U_K) is added with the factor S_K folded
// into a select, so the solve is branch free.
__device__ __forceinline__ void hllc32(const GasF32& g, float4 L, float4 R, float nx, float ny, float* F) {
  const float rsl = frsq(L.x), rsr = frsq(R.x);
  const float srL = L.x * rsl, srR = R.x * rsr;            // sqrt(rho)
  const float irl = rsl * rsl, irr = rsr * rsr;            // 1 / rho
  const float unl = fmaf(L.y, nx, L.z * ny), unr = fmaf(R.y, nx, R.z * ny);
  const float pol = L.w * irl, por = R.w * irr;            // p / rho
  const float aL = fsqrtp(g.gamma * pol), aR = fsqrtp(g.gamma * por);
  const float h0l = fmaf(g.gcp, pol, 0.5f * fmaf(L.y, L.y, L.z * L.z));
  const float h0r = fmaf(g.gcp, por, 0.5f * fmaf(R.y, R.y, R.z * R.z));
  const float isr = frcp(srL + srR);
  const float wl = srL * isr, wr = srR * isr;
  const float ur0 = fmaf(wr, R.y, wl * L.y), ur1 = fmaf(wr, R.z, wl * L.z);
  const float h0_roe = fmaf(wr, h0r, wl * h0l);
  const float a2 = g.gm1 * fmaf(-0.5f, fmaf(ur0, ur0, ur1 * ur1), h0_roe);
  const float a_roe = fsqrtp(fmaxf(a2, 1.17549435e-38f));
  const float un_roe = fmaf(ur0, nx, ur1 * ny);
  const float S1 = fminf(fminf(0.0f, unl - aL), un_roe - a_roe);
  const float S4 = fmaxf(fmaxf(0.0f, unr + aR), un_roe + a_roe);
  const float ml = L.x * (S1 - unl), mr = R.x * (S4 - unr);
  const float Sstar = (R.w - L.w + ml * unl - mr * unr) * frcp(ml - mr);
  const bool left = (S1 >= 0.0f) || (Sstar >= 0.0f);
  const float rk = left ? L.x : R.x, uk = left ? L.y : R.y, vk = left ? L.z : R.z, pk = left ? L.w : R.w;
  const float unk = left ? unl : unr, h0k = left ? h0l : h0r, irk = left ? irl : irr;
  const float SK = left ? S1 : S4, mk = left ? ml : mr;
  const float m = rk * unk;
  F[0] = m;
  F[1] = fmaf(m, uk, pk * nx);
  F[2] = fmaf(m, vk, pk * ny);
  F[3] = m * h0k;
  // star correction, applied when K's outer wave is subsonic in the face frame
  const bool corr = left ? (S1 < 0.0f) : (S4 > 0.0f);
  const float sc = corr ? SK : 0.0f;
  const float pstar = fmaf(L.x * (unl - S1), unl - Sstar, L.w);
  const float inv = frcp(SK - Sstar);
  const float dp = pstar - pk;
  const float e0k = h0k - pk * irk;
  F[0] = fmaf(sc, fmaf(mk, inv, -rk), F[0]);
  F[1] = fmaf(sc, fmaf(fmaf(mk, uk, dp * nx), inv, -rk * uk), F[1]);
  F[2] = fmaf(sc, fmaf(fmaf(mk, vk, dp * ny), inv, -rk * vk), F[2]);
  F[3] = fmaf(sc, fmaf(fmaf(mk, e0k, fmaf(-pk, unk, pstar * Sstar)), inv, -rk * e0k), F[3]);
}

// AUSM+ (Lib_Riemann_AUSM.f90:150-238) in FP32, flux per unit area.
__device__ __forceinline__ void ausmp32(const GasF32& g, float4 L, float4 R, float nx, float ny, float* F) {
  const float beta = 0.125f, alpha = 0.1875f;
  const float irl = frcp(L.x), irr = frcp(R.x);
  const float unl = fmaf(L.y, nx, L.z * ny), unr = fmaf(R.y, nx, R.z * ny);
  const float pol = L.w * irl, por = R.w * irr;
  const float a_half = fsqrtp(g.gamma * fsqrtp(pol * por));   // sqrt(aL aR)
  const float ia = frcp(a_half);
  const float ML = unl * ia, MR = unr * ia;
  const float mL2 = fmaf(ML, ML, -1.0f), mR2 = fmaf(MR, MR, -1.0f);
  const bool sl = fabsf(ML) < 1.0f, sr = fabsf(MR) < 1.0f;
  const float lp1 = ML + 1.0f, rm1 = MR - 1.0f;
  const float MplusL = sl ? fmaf(0.25f * lp1, lp1, beta * mL2 * mL2) : 0.5f * (ML + fabsf(ML));
  const float pplusL = sl ? fmaf(0.25f * lp1 * lp1, 2.0f - ML, alpha * ML * mL2 * mL2)
                          : 0.5f * (1.0f + copysignf(1.0f, ML));
  const float MminusR = sr ? -fmaf(0.25f * rm1, rm1, beta * mR2 * mR2) : 0.5f * (MR - fabsf(MR));
  const float pminusR = sr ? fmaf(0.25f * rm1 * rm1, 2.0f + MR, -alpha * MR * mR2 * mR2)
                           : 0.5f * (1.0f - copysignf(1.0f, MR));
  const float Mhalf = MplusL + MminusR;
  const float phalf = fmaf(pplusL, L.w, pminusR * R.w);
  const float mp = L.x * a_half * 0.5f * (Mhalf + fabsf(Mhalf));
  const float mm = R.x * a_half * 0.5f * (Mhalf - fabsf(Mhalf));
  const float HL = fmaf(g.gcp, pol, 0.5f * fmaf(L.y, L.y, L.z * L.z));
  const float HR = fmaf(g.gcp, por, 0.5f * fmaf(R.y, R.y, R.z * R.z));
  F[0] = mp + mm;
  F[1] = fmaf(mp, L.y, fmaf(mm, R.y, nx * phalf));
  F[2] = fmaf(mp, L.z, fmaf(mm, R.z, ny * phalf));
  F[3] = fmaf(mp, HL, mm * HR);
}

// ---- FP32 solvers over NV-variable arrays -----------------------------------
// hllc32 / ausmp32 above for (rho, u, ..., p) arrays of NV values and a
// three-component normal (the 3-D sweeps of the mixed precision).  The upwind
// side is chosen per value with selects, so the arrays stay in registers.
template <int NV>
__device__ __forceinline__ float un32(const float* q, const float* n) {
  if constexpr (NV == 5) return fmaf(q[1], n[0], fmaf(q[2], n[1], q[3] * n[2]));
  else return fmaf(q[1], n[0], q[2] * n[1]);
}
template <int NV>
__device__ __forceinline__ float v2_32(const float* q) {
  if constexpr (NV == 5) return fmaf(q[1], q[1], fmaf(q[2], q[2], q[3] * q[3]));
  else return fmaf(q[1], q[1], q[2] * q[2]);
}

template <int NV>
__device__ __forceinline__ void hllc32n(const GasF32& g, const float* L, const float* R, const float* n, float* F) {
  constexpr int P = NV - 1, D = NV - 2;
  const float rsl = frsq(L[0]), rsr = frsq(R[0]);
  const float srL = L[0] * rsl, srR = R[0] * rsr;          // sqrt(rho)
  const float irl = rsl * rsl, irr = rsr * rsr;            // 1 / rho
  const float unl = un32<NV>(L, n), unr = un32<NV>(R, n);
  const float pol = L[P] * irl, por = R[P] * irr;          // p / rho
  const float aL = fsqrtp(g.gamma * pol), aR = fsqrtp(g.gamma * por);
  const float h0l = fmaf(g.gcp, pol, 0.5f * v2_32<NV>(L));
  const float h0r = fmaf(g.gcp, por, 0.5f * v2_32<NV>(R));
  const float isr = frcp(srL + srR);
  const float wl = srL * isr, wr = srR * isr;
  float vel2 = 0.0f, un_roe = 0.0f;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float ur = fmaf(wr, R[1 + d], wl * L[1 + d]);
    vel2 = fmaf(ur, ur, vel2);
    un_roe = fmaf(ur, n[d], un_roe);
  }
  const float h0_roe = fmaf(wr, h0r, wl * h0l);
  const float a2 = g.gm1 * fmaf(-0.5f, vel2, h0_roe);
  const float a_roe = fsqrtp(fmaxf(a2, 1.17549435e-38f));
  const float S1 = fminf(fminf(0.0f, unl - aL), un_roe - a_roe);
  const float S4 = fmaxf(fmaxf(0.0f, unr + aR), un_roe + a_roe);
  const float ml = L[0] * (S1 - unl), mr = R[0] * (S4 - unr);
  const float Sstar = (R[P] - L[P] + ml * unl - mr * unr) * frcp(ml - mr);
  const bool left = (S1 >= 0.0f) || (Sstar >= 0.0f);
  const float rk = left ? L[0] : R[0], pk = left ? L[P] : R[P];
  const float unk = left ? unl : unr, h0k = left ? h0l : h0r, irk = left ? irl : irr;
  const float SK = left ? S1 : S4, mk = left ? ml : mr;
  const float m = rk * unk;
  // star correction, applied when K's outer wave is subsonic in the face frame
  const bool corr = left ? (S1 < 0.0f) : (S4 > 0.0f);
  const float sc = corr ? SK : 0.0f;
  const float pstar = fmaf(L[0] * (unl - S1), unl - Sstar, L[P]);
  const float inv = frcp(SK - Sstar);
  const float dp = pstar - pk;
  const float e0k = h0k - pk * irk;
  F[0] = fmaf(sc, fmaf(mk, inv, -rk), m);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float uk = left ? L[1 + d] : R[1 + d];
    F[1 + d] = fmaf(sc, fmaf(fmaf(mk, uk, dp * n[d]), inv, -rk * uk), fmaf(m, uk, pk * n[d]));
  }
  F[P] = fmaf(sc, fmaf(fmaf(mk, e0k, fmaf(-pk, unk, pstar * Sstar)), inv, -rk * e0k), m * h0k);
}

template <int NV>
__device__ __forceinline__ void ausmp32n(const GasF32& g, const float* L, const float* R, const float* n, float* F) {
  constexpr int P = NV - 1, D = NV - 2;
  const float beta = 0.125f, alpha = 0.1875f;
  const float irl = frcp(L[0]), irr = frcp(R[0]);
  const float unl = un32<NV>(L, n), unr = un32<NV>(R, n);
  const float pol = L[P] * irl, por = R[P] * irr;
  const float a_half = fsqrtp(g.gamma * fsqrtp(pol * por));   // sqrt(aL aR)
  const float ia = frcp(a_half);
  const float ML = unl * ia, MR = unr * ia;
  const float mL2 = fmaf(ML, ML, -1.0f), mR2 = fmaf(MR, MR, -1.0f);
  const bool sl = fabsf(ML) < 1.0f, sr = fabsf(MR) < 1.0f;
  const float lp1 = ML + 1.0f, rm1 = MR - 1.0f;
  const float MplusL = sl ? fmaf(0.25f * lp1, lp1, beta * mL2 * mL2) : 0.5f * (ML + fabsf(ML));
  const float pplusL = sl ? fmaf(0.25f * lp1 * lp1, 2.0f - ML, alpha * ML * mL2 * mL2)
                          : 0.5f * (1.0f + copysignf(1.0f, ML));
  const float MminusR = sr ? -fmaf(0.25f * rm1, rm1, beta * mR2 * mR2) : 0.5f * (MR - fabsf(MR));
  const float pminusR = sr ? fmaf(0.25f * rm1 * rm1, 2.0f + MR, -alpha * MR * mR2 * mR2)
                           : 0.5f * (1.0f - copysignf(1.0f, MR));
  const float Mhalf = MplusL + MminusR;
  const float phalf = fmaf(pplusL, L[P], pminusR * R[P]);
  const float mp = L[0] * a_half * 0.5f * (Mhalf + fabsf(Mhalf));
  const float mm = R[0] * a_half * 0.5f * (Mhalf - fabsf(Mhalf));
  const float HL = fmaf(g.gcp, pol, 0.5f * v2_32<NV>(L));
  const float HR = fmaf(g.gcp, por, 0.5f * v2_32<NV>(R));
  F[0] = mp + mm;
#pragma unroll
  for (int d = 0; d < D; ++d) F[1 + d] = fmaf(mp, L[1 + d], fmaf(mm, R[1 + d], n[d] * phalf));
  F[P] = fmaf(mp, HL, mm * HR);
}

// ---- state update (Newstate_Conservative restated, one species) -----------
// U = (rho, rho u, ..., p/(gamma-1) + rho |u|^2 / 2); p = (gamma-1)(E - rho |u|^2 / 2)
template <int NV>
__device__ __forceinline__ bool rk_update(const GasF& g, double* Q, const double* QO, const double* R, double dtv,
                                          double c, bool first_stage) {
  constexpr int P = NV - 1;
  double U[NV], U0[NV];
  U[0] = Q[0];
  for (int d = 0; d < NV - 2; ++d) U[1 + d] = Q[0] * Q[1 + d];
  U[P] = fma(Q[P], g.igm1, 0.5 * Q[0] * v2<NV>(Q));
  if (first_stage) {
    for (int v = 0; v < NV; ++v) U[v] = fma(-R[v] * dtv, c, U[v]);
  } else {
    U0[0] = QO[0];
    for (int d = 0; d < NV - 2; ++d) U0[1 + d] = QO[0] * QO[1 + d];
    U0[P] = fma(QO[P], g.igm1, 0.5 * QO[0] * v2<NV>(QO));
    for (int v = 0; v < NV; ++v) U[v] = fma(fma(-R[v], dtv, U[v] - U0[v]), c, U0[v]);
  }
  const double ir = rcp(U[0]);
  Q[0] = U[0];
  double ke = 0.0;
  for (int d = 0; d < NV - 2; ++d) {
    Q[1 + d] = U[1 + d] * ir;
    ke = fma(U[1 + d], Q[1 + d], ke);
  }
  Q[P] = g.gm1 * fma(-0.5, ke, U[P]);
  // A NaN in any conserved variable reaches p (through 1/rho, the velocities
  // or E), so one test finds NaN or p < 0 (Lib_Newstate.f90:334-338): as an
  // unsigned integer, every bit pattern above +inf is a negative number or a
  // NaN (-0 excepted, which is not below 0).
  const unsigned long long pb = (unsigned long long)__double_as_longlong(Q[P]);
  const bool bad = pb > 0x7ff0000000000000ULL && pb != 0x8000000000000000ULL;
  if (Q[0] < 1e-20) Q[0] = 1e-20;
  return !bad;
}

}  // namespace fast
}  // namespace mose
