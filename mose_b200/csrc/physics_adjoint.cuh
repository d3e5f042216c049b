// physics_adjoint.cuh -- reverse-mode (adjoint) forms of the 2-D face physics:
// the limiters' partial derivatives, Batten HLLC (Lib_Riemann_HLL.f90:147-258,
// the single-species algebra of physics_fast.cuh) and the primitive <->
// conservative maps of Newstate_Conservative (Lib_Newstate.f90:134-160).
// Divisions and square roots use the refined hardware reciprocal and
// reciprocal square root of physics_fast.cuh (about one ulp): a derivative
// needs no more than that.
//
// Each *_vjp function recomputes its forward values (kept in registers) and
// then walks the operations in reverse, accumulating the adjoint of every
// input from the adjoint of the outputs: one forward plus one reverse sweep,
// no tape.  Branches (min/max selections, the HLLC upwind side and the star
// correction switch) follow the forward's choice, which is the derivative of
// the piecewise-smooth forward wherever it is differentiable.
#pragma once

#include "common.cuh"
#include "physics_fast.cuh"

namespace mose {
namespace adj {

// phi(x, y) of the reference limiters (x the downwind, y the upwind slope:
// Lib_Limiters.f90:35-75 with r = y / (x + 1e-30)) and its partials.
template <int LIM>
__device__ __forceinline__ double limiter_grad(double x, double y, double* dx, double* dy) {
  if constexpr (LIM == 1) {   // minmod: 0 if x y < 0, else the smaller |.| (ties -> x)
    if (x * y < 0.0) { *dx = 0.0; *dy = 0.0; return 0.0; }
    if (fabs(x) > fabs(y)) { *dx = 0.0; *dy = 1.0; return y; }
    *dx = 1.0; *dy = 0.0; return x;
  } else if constexpr (LIM == 2) {   // van Leer: x (y sg + |y|) / (|x'| + |y|)
    const double xp = x + 1e-30, sg = copysign(1.0, xp), sy = copysign(1.0, y);
    const double N = y * sg + fabs(y), D = fabs(xp) + fabs(y);
    const double iD = fast::rcp(D);
    *dx = N * iD - x * N * sg * iD * iD;
    *dy = x * (sg + sy) * iD - x * N * sy * iD * iD;
    return x * N * iD;
  } else if constexpr (LIM == 3) {   // van Albada: x (y^2 + y x') / (x'^2 + y^2)
    const double xp = x + 1e-30;
    const double N = y * (y + xp), D = xp * xp + y * y;
    const double iD = fast::rcp(D);
    *dx = N * iD + x * y * iD - 2.0 * x * N * xp * iD * iD;
    *dy = x * (2.0 * y + xp) * iD - 2.0 * x * N * y * iD * iD;
    return x * N * iD;
  } else {
    *dx = 0.0; *dy = 0.0;
    return 0.0;
  }
}

// HLLC flux per unit area F(L, R; n) of 2-D states (rho, u, v, p), and the
// adjoint: given Fb = dJ/dF, Lb += dJ/dL and Rb += dJ/dR.
__device__ __forceinline__ void hllc_vjp(double gam, double gcp, double gm1, const double* L, const double* R,
                                         double nx, double ny, const double* Fb, double* F, double* Lb, double* Rb) {
  // ---- forward ------------------------------------------------------------
  const double rl = L[0], ul = L[1], vl = L[2], pl = L[3];
  const double rr = R[0], ur = R[1], vr = R[2], pr = R[3];
  const double rsl = fast::rsqrt_(rl), rsr = fast::rsqrt_(rr);
  const double srL = rl * rsl, srR = rr * rsr;
  const double irl = rsl * rsl, irr = rsr * rsr;
  const double unl = ul * nx + vl * ny, unr = ur * nx + vr * ny;
  const double pol = pl * irl, por = pr * irr;
  const double raL = fast::rsqrt_(gam * pol), raR = fast::rsqrt_(gam * por);
  const double aL = gam * pol * raL, aR = gam * por * raR;
  const double h0l = gcp * pol + 0.5 * (ul * ul + vl * vl);
  const double h0r = gcp * por + 0.5 * (ur * ur + vr * vr);
  const double isr = fast::rcp(srL + srR);
  const double wl = srL * isr, wr = srR * isr;
  const double ur0 = wr * ur + wl * ul, ur1 = wr * vr + wl * vl;
  const double h0roe = wr * h0r + wl * h0l;
  const double vel2 = ur0 * ur0 + ur1 * ur1;
  const double X = gm1 * (h0roe - 0.5 * vel2);
  const double raroe = X > 0.0 ? fast::rsqrt_(X) : 0.0;
  const double a_roe = X * raroe;
  const double unroe = ur0 * nx + ur1 * ny;
  // S1 = min(min(0, unl - aL), unroe - a_roe); S4 = max(max(0, unr + aR), unroe + a_roe)
  const double s1a = unl - aL, s1b = unroe - a_roe;
  const double m1 = fmin(0.0, s1a);
  const double S1 = fmin(m1, s1b);
  const int s1w = (S1 == s1b && s1b < m1) ? 2 : (m1 == s1a && s1a < 0.0) ? 1 : 0;   // active argument
  const double s4a = unr + aR, s4b = unroe + a_roe;
  const double m4 = fmax(0.0, s4a);
  const double S4 = fmax(m4, s4b);
  const int s4w = (S4 == s4b && s4b > m4) ? 2 : (m4 == s4a && s4a > 0.0) ? 1 : 0;
  const double ml = rl * (S1 - unl), mr = rr * (S4 - unr);
  const double idn = fast::rcp(ml - mr);
  const double num = pr - pl + ml * unl - mr * unr;
  const double Sstar = num * idn;
  const bool left = (S1 >= 0.0) || (Sstar >= 0.0);
  const double rk = left ? rl : rr, uk = left ? ul : ur, vk = left ? vl : vr, pk = left ? pl : pr;
  const double unk = left ? unl : unr, h0k = left ? h0l : h0r, irk = left ? irl : irr;
  const double SK = left ? S1 : S4, mk = left ? ml : mr;
  const double F0 = rk * unk;
  F[0] = F0;
  F[1] = F0 * uk + pk * nx;
  F[2] = F0 * vk + pk * ny;
  F[3] = F0 * h0k;
  const bool corr = left ? (S1 < 0.0) : (S4 > 0.0);
  const double a1 = unl - S1, a2 = unl - Sstar;
  const double pstar = rl * a1 * a2 + pl;
  const double inv = fast::rcp(SK - Sstar);
  const double dp = pstar - pk;
  const double e0k = h0k - pk * irk;
  const double t1 = mk * uk + dp * nx, t2 = mk * vk + dp * ny, t3 = mk * e0k - pk * unk + pstar * Sstar;
  if (corr) {
    F[0] += SK * (mk * inv - rk);
    F[1] += SK * (t1 * inv - rk * uk);
    F[2] += SK * (t2 * inv - rk * vk);
    F[3] += SK * (t3 * inv - rk * e0k);
  }
  // ---- reverse ------------------------------------------------------------
  double rkb = 0, ukb = 0, vkb = 0, pkb = 0, unkb = 0, h0kb = 0, irkb = 0, SKb = 0, mkb = 0;
  double pstarb = 0, Sstarb = 0, invb = 0, dpb = 0, e0kb = 0;
  if (corr) {
    const double c0b = Fb[0], c1b = Fb[1], c2b = Fb[2], c3b = Fb[3];
    SKb += c0b * (mk * inv - rk) + c1b * (t1 * inv - rk * uk) + c2b * (t2 * inv - rk * vk) +
           c3b * (t3 * inv - rk * e0k);
    mkb += c0b * SK * inv;
    invb += SK * (c0b * mk + c1b * t1 + c2b * t2 + c3b * t3);
    rkb -= SK * (c0b + c1b * uk + c2b * vk + c3b * e0k);
    ukb -= c1b * SK * rk;
    vkb -= c2b * SK * rk;
    e0kb -= c3b * SK * rk;
    const double t1b = c1b * SK * inv, t2b = c2b * SK * inv, t3b = c3b * SK * inv;
    mkb += t1b * uk + t2b * vk + t3b * e0k;
    ukb += t1b * mk;
    vkb += t2b * mk;
    dpb += t1b * nx + t2b * ny;
    e0kb += t3b * mk;
    pkb -= t3b * unk;
    unkb -= t3b * pk;
    pstarb += t3b * Sstar;
    Sstarb += t3b * pstar;
  }
  // e0k = h0k - pk irk ; dp = pstar - pk ; inv = 1 / (SK - Sstar)
  h0kb += e0kb;
  pkb -= e0kb * irk;
  irkb -= e0kb * pk;
  pstarb += dpb;
  pkb -= dpb;
  {
    const double t = -invb * inv * inv;
    SKb += t;
    Sstarb -= t;
  }
  // pstar = rl a1 a2 + pl
  double rlb = 0, ulb = 0, vlb = 0, plb = 0, rrb = 0, urb = 0, vrb = 0, prb = 0;
  double unlb = 0, unrb = 0, S1b = 0, S4b = 0;
  rlb += pstarb * a1 * a2;
  plb += pstarb;
  {
    const double a1b = pstarb * rl * a2, a2b = pstarb * rl * a1;
    unlb += a1b + a2b;
    S1b -= a1b;
    Sstarb -= a2b;
  }
  // physical flux of the upwind side
  {
    double F0b = Fb[0] + Fb[1] * uk + Fb[2] * vk + Fb[3] * h0k;
    ukb += Fb[1] * F0;
    vkb += Fb[2] * F0;
    pkb += Fb[1] * nx + Fb[2] * ny;
    h0kb += Fb[3] * F0;
    rkb += F0b * unk;
    unkb += F0b * rk;
  }
  // selection of the upwind side
  double h0lb = 0, h0rb = 0, irlb = 0, irrb = 0, mlb = 0, mrb = 0;
  if (left) {
    rlb += rkb; ulb += ukb; vlb += vkb; plb += pkb; unlb += unkb; h0lb += h0kb; irlb += irkb; S1b += SKb; mlb += mkb;
  } else {
    rrb += rkb; urb += ukb; vrb += vkb; prb += pkb; unrb += unkb; h0rb += h0kb; irrb += irkb; S4b += SKb; mrb += mkb;
  }
  // Sstar = num idn ; idn = 1 / (ml - mr)
  {
    const double numb = Sstarb * idn;
    const double idnb = Sstarb * num;
    prb += numb;
    plb -= numb;
    mlb += numb * unl;
    unlb += numb * ml;
    mrb -= numb * unr;
    unrb -= numb * mr;
    const double t = -idnb * idn * idn;
    mlb += t;
    mrb -= t;
  }
  // ml = rl (S1 - unl) ; mr = rr (S4 - unr)
  rlb += mlb * (S1 - unl);
  S1b += mlb * rl;
  unlb -= mlb * rl;
  rrb += mrb * (S4 - unr);
  S4b += mrb * rr;
  unrb -= mrb * rr;
  // wave speed estimates
  double aLb = 0, aRb = 0, unroeb = 0, a_roeb = 0;
  if (s1w == 1) { unlb += S1b; aLb -= S1b; }
  else if (s1w == 2) { unroeb += S1b; a_roeb -= S1b; }
  if (s4w == 1) { unrb += S4b; aRb += S4b; }
  else if (s4w == 2) { unroeb += S4b; a_roeb += S4b; }
  // Roe state
  double ur0b = unroeb * nx, ur1b = unroeb * ny;
  double h0roeb = 0, vel2b = 0;
  {
    const double Xb = a_roeb * 0.5 * raroe;
    h0roeb += Xb * gm1;
    vel2b -= Xb * gm1 * 0.5;
  }
  ur0b += 2.0 * ur0 * vel2b;
  ur1b += 2.0 * ur1 * vel2b;
  double wlb = 0, wrb = 0;
  wrb += h0roeb * h0r + ur0b * ur + ur1b * vr;
  wlb += h0roeb * h0l + ur0b * ul + ur1b * vl;
  h0rb += h0roeb * wr;
  h0lb += h0roeb * wl;
  urb += ur0b * wr;
  ulb += ur0b * wl;
  vrb += ur1b * wr;
  vlb += ur1b * wl;
  double srLb = wlb * isr, srRb = wrb * isr;
  {
    const double isrb = wlb * srL + wrb * srR;
    const double t = -isrb * isr * isr;
    srLb += t;
    srRb += t;
  }
  // enthalpies and sound speeds
  double polb = h0lb * gcp, porb = h0rb * gcp;
  ulb += h0lb * ul;
  vlb += h0lb * vl;
  urb += h0rb * ur;
  vrb += h0rb * vr;
  polb += aLb * gam * 0.5 * raL;
  porb += aRb * gam * 0.5 * raR;
  plb += polb * irl;
  irlb += polb * pl;
  prb += porb * irr;
  irrb += porb * pr;
  // normal velocities
  ulb += unlb * nx;
  vlb += unlb * ny;
  urb += unrb * nx;
  vrb += unrb * ny;
  // 1/rho and sqrt(rho)
  rlb += -irlb * irl * irl + srLb * 0.5 * rsl;
  rrb += -irrb * irr * irr + srRb * 0.5 * rsr;
  Lb[0] += rlb; Lb[1] += ulb; Lb[2] += vlb; Lb[3] += plb;
  Rb[0] += rrb; Rb[1] += urb; Rb[2] += vrb; Rb[3] += prb;
}

// Primitive -> conservative (rho, rho u, rho v, p/(gamma-1) + rho |u|^2/2):
// P_b += J^T U_b.
__device__ __forceinline__ void p2u_vjp(double igm1, const double* P, const double* Ub, double* Pb) {
  const double r = P[0], u = P[1], v = P[2];
  Pb[0] += Ub[0] + Ub[1] * u + Ub[2] * v + Ub[3] * 0.5 * (u * u + v * v);
  Pb[1] += Ub[1] * r + Ub[3] * r * u;
  Pb[2] += Ub[2] * r + Ub[3] * r * v;
  Pb[3] += Ub[3] * igm1;
}
// Conservative -> primitive at the primitive state P (= the map's output):
// U_b = J^T P_b.
__device__ __forceinline__ void u2p_vjp(double gm1, const double* P, const double* Pb, double* Ub) {
  const double r = P[0], u = P[1], v = P[2];
  const double ir = fast::rcp(r);
  Ub[0] = Pb[0] - Pb[1] * u * ir - Pb[2] * v * ir + Pb[3] * gm1 * 0.5 * (u * u + v * v);
  Ub[1] = Pb[1] * ir - Pb[3] * gm1 * u;
  Ub[2] = Pb[2] * ir - Pb[3] * gm1 * v;
  Ub[3] = Pb[3] * gm1;
}

}  // namespace adj
}  // namespace mose
