// stage2d.cuh -- fused residual + RK-stage kernel for 2-D blocks (and 1-D run
// as 2-D with nj = 1), one launch per RK stage over every block.
//
// Work decomposition: an item is a strip of STRIP_W = T-2 cell columns of one
// block and a run of rows.  Thread t owns column c = c0 - 1 + t (one column of
// halo on each side), so per row:
//   * every thread forms the limited i-slope of its cell (T-2 cells + 2 halo);
//   * threads 0..T-2 each form ONE i-face flux F(c+1/2);
//   * threads 1..T-2 update their cell.
// The j direction is marched: each thread keeps its column's last j-slope,
// limited slope and lower j-face flux in registers, so every j-face flux is
// formed once per strip.  Each interior face flux is therefore computed once
// (plus one halo face per strip side); the reference computes the same flux
// with the same operations (Mod_Fluxes.f90:89-139), so results match it
// bit for bit, and do not depend on the decomposition.  The i-face and
// j-face Riemann solves of a row are issued together, without a barrier or a
// branch between them, so the two independent FP64 chains overlap.
//
// Residual accumulation keeps the reference order per cell: the interior
// face sweeps first (i-, i+, j-, j+: Mod_Fluxes.f90:89-179), then the
// boundary-face contributions in face order 1..6 (BC_Fluxes walks the
// bc list by block and face, Mod_BC_Fluxes.f90:52-216).
//
// The arithmetic is a policy: PolExact (the reference's operation order),
// PolFast (FP64 restated for speed) or PolMixed (FP32 wave structure).
// Boundary-face fluxes always use the reference-exact formulas.
#pragma once

#include "arena.cuh"
#include "physics_exact.cuh"
#include "physics_fast.cuh"

namespace mose {

__device__ __forceinline__ void report(DevError* e, int code, int b, int i, int j, int k) {
  if (atomicCAS(&e->code, 0, code) == 0) {
    e->b = b + 1; e->i = i + 1; e->j = j + 1; e->k = k + 1;
  }
}

// Face-flux add mask: which components a boundary contribution adds.
enum : int { ADD_ALL = 0, ADD_MOMENTUM = 1, ADD_NONE = 2 };

// Flux of a block-boundary face of type code w (not BC_CONN / BC_NONE).
// Q = boundary cell, Qi = first interior cell, dlB/dlI their dl along the
// face direction.  face = 1..6.  Returns the add mask.
template <int RIE, int LIM, int NV>
__device__ __noinline__ int boundary_flux(const StageArgs& a, int w, const double* Q, const double* Qi, double dlB,
                                          double dlI, const double* n, double area, int face, double* F) {
  const Gas& g = a.g;
  int code = bc_code(w);
  const double s = (double)(1 - 2 * (face % 2));
  if (code == BC_EXTRAP) {
    ex::bc_extrapolation<NV>(g, Q, n, area, F);
    return ADD_ALL;
  }
  if (code == BC_SUPIN) {
    double Un = ex::dot_vel<NV>(Q, n);
    if (!(s * Un >= 0.0)) {
      ex::bc_supersonic_inflow<RIE, LIM, NV>(g, Q, Qi, a.bcp[bc_param(w)], n, area, face, F);
      return ADD_ALL;
    }
  } else if (code == BC_OUTFLOW) {
    double Un = ex::dot_vel<NV>(Q, n);
    if (!(s * Un < 0.0)) {
      ex::bc_outflow<NV>(g, Q, Un, n, area, a.bcp[bc_param(w)].pback, face, F);
      return ADD_ALL;
    }
  }
  // BC_SYM, and the symmetry fallback of 405 / 406 (Mod_BC_Fluxes.f90:168,173)
  ex::bc_symmetry<RIE, LIM, NV>(g, Q, Qi, dlB, dlI, n, area, face, F);
  return ADD_MOMENTUM;
}

// Newstate_Conservative for one cell (Lib_Newstate.f90:134-160); returns the
// new primitives in Q.  first_stage: P == PO, so U - U0 is an exact zero.
template <int NV>
__device__ __forceinline__ bool rk_update(const Gas& g, double* Q, const double* QO, const double* R,
                                          double vol, double dt, double c, bool first_stage) {
  constexpr int P = NV - 1;
  double U[NV], U0[NV];
  ex::prim2cons<NV>(g, Q, U);
  if (first_stage) {
    for (int v = 0; v < NV; ++v) {
      double r = -(R[v] / vol * dt);
      double r_ = (0.0 + r) * c;
      U[v] = U[v] + r_;
    }
  } else {
    ex::prim2cons<NV>(g, QO, U0);
    for (int v = 0; v < NV; ++v) {
      double r = -(R[v] / vol * dt);
      double r_ = (U[v] - U0[v] + r) * c;
      U[v] = U0[v] + r_;
    }
  }
  ex::cons2prim<NV>(g, U, Q);
  bool bad = false;
  for (int v = 0; v < NV; ++v) bad |= isnan(Q[v]);
  bad |= (Q[P] < 0.0);
  if (Q[0] < 1e-20) Q[0] = 1e-20;
  return !bad;
}

// ---- arithmetic policies ---------------------------------------------------
// slope(dq, l, il): first difference over the cell-centre distance l (il = 1/l)
// lim(x, y): limited slope phi(y/x) x
// face(...): interface flux times area; false if check_gas_state rejects
// update(...): Newstate_Conservative
template <int RIE, int LIM>
struct PolExact {
  static constexpr bool kFast = false;
  static constexpr bool kCompensated = false;
  __device__ static double inv_len(double l) { return 0.0; }
  __device__ static double slope(double dq, double l, double) { return dq / l; }
  __device__ static double lim(double x, double y) { return ex::limiter<LIM>(x, y); }
  template <int NV>
  __device__ static bool face(const Gas& g, const double* QL, const double* QR, const double* n, double A,
                              double* F) {
    return ex::face_flux<RIE, NV>(g, QL, QR, n, A, F);
  }
  template <int NV>
  __device__ static bool update(const Gas& g, double* Q, const double* QO, const double* R, double vol, double dt,
                                double c, bool first) {
    return rk_update<NV>(g, Q, QO, R, vol, dt, c, first);
  }
};

template <int RIE, int LIM, bool MIXED>
struct PolFast {
  static constexpr bool kFast = true;
  static constexpr bool kCompensated = MIXED;
  __device__ static double inv_len(double l) { return fast::rcp(l); }
  __device__ static double slope(double dq, double, double il) { return dq * il; }
  __device__ static double lim(double x, double y) {
    if constexpr (MIXED) return (double)fast::limiter32<LIM>((float)x, (float)y);
    else return fast::limiter<LIM>(x, y);
  }
  template <int NV>
  __device__ static bool face(const Gas& g, const double* QL, const double* QR, const double* n, double A,
                              double* F) {
    constexpr int P = NV - 1;
    bool ok = (QL[0] > 0.0 && QL[P] > 0.0 && QR[0] > 0.0 && QR[P] > 0.0);
    const fast::GasF gf = fast::gasf(g);
    if constexpr (RIE == 0) {
      if constexpr (MIXED) fast::hllc_mixed<NV>(gf, QL, QR, n, F);
      else fast::hllc<NV>(gf, QL, QR, n, F);
    } else if constexpr (RIE == 1) {
      if constexpr (MIXED) fast::ausmp_mixed<NV>(gf, QL, QR, n, F);
      else fast::ausmp<NV>(gf, QL, QR, n, F);
    } else {
      double aL = ex::sound(g, QL[0], QL[P]), aR = ex::sound(g, QR[0], QR[P]);
      ex::riemann<RIE, NV>(g, QL, aL, QR, aR, n, F);
    }
    for (int v = 0; v < NV; ++v) F[v] = F[v] * A;
    return ok;
  }
  template <int NV>
  __device__ static bool update(const Gas& g, double* Q, const double* QO, const double* R, double vol, double dt,
                                double c, bool first) {
    return fast::rk_update<NV>(fast::gasf(g), Q, QO, R, dt * fast::rcp(vol), c, first);
  }
};

// Residual of one cell: plain left-to-right sums (the reference's), or
// Neumaier-compensated FP64 sums of the face-flux differences.
template <int NV, bool COMP>
struct ResAcc {
  double s[NV], c[NV];
  __device__ void init() {
    for (int v = 0; v < NV; ++v) { s[v] = 0.0; c[v] = 0.0; }
  }
  __device__ void add(int v, double x) {
    if constexpr (COMP) {
      double t = s[v] + x;
      c[v] += (fabs(s[v]) >= fabs(x)) ? (s[v] - t) + x : (x - t) + s[v];
      s[v] = t;
    } else {
      s[v] = s[v] + x;
    }
  }
  __device__ double get(int v) const {
    if constexpr (COMP) return s[v] + c[v];
    else return s[v];
  }
};

template <int NV, bool COMP>
__device__ __forceinline__ void add_bc(ResAcc<NV, COMP>& R, const double* F, double sgn, int mask) {
  if (mask == ADD_ALL) {
    for (int v = 0; v < NV; ++v) R.add(v, sgn * F[v]);
  } else if (mask == ADD_MOMENTUM) {
    for (int v = 1; v < NV - 1; ++v) R.add(v, sgn * F[v]);
  }
}

// Minimum resident CTAs per SM the register allocation is sized for.
#ifndef MOSE_STAGE_MIN_CTAS
#define MOSE_STAGE_MIN_CTAS 3
#endif

// MODE: 0 = fused (residual + RK update, writes Pn), 1 = residual only (writes R).
template <class PH, int RIE, int LIM, bool UNI, int MODE>
__global__ void __launch_bounds__(STRIP_T, MOSE_STAGE_MIN_CTAS) k_stage2d(StageArgs a) {
  constexpr int NV = 4;
  constexpr int T = STRIP_T;
  __shared__ double sP[NV][T + 2];
  __shared__ double sDL[T + 2];
  __shared__ double sSig[NV][T];
  __shared__ double sF[NV][T];
  __shared__ int sMask[T];
  const int t = threadIdx.x;

  for (int it = blockIdx.x; it < a.nitems; it += gridDim.x) {
    const int4 item = a.items[it];
    const int b = item.x, c0 = item.y, j0 = item.z, j1 = item.w;
    const BlockDesc& d = a.blk[b];
    const int ni = d.ni, nj = d.nj, px = d.px;
    const long long vs = d.vstride;
    const double* Pc = a.Pc + d.sbase;
    const long long mb = d.mbase;
    const int c = c0 - 1 + t;
    const int cend = min(c0 + STRIP_W, ni);
    const bool colok = (c <= ni + 1);
    const bool has_face = (t < T - 1) && (c <= cend - 1);
    const bool has_cell = (t >= 1) && (c < cend);
    // column used for this thread's loads (threads past the block read its last ghost column)
    const int cl = min(c, ni + 1);
    auto off = [&](int cc, int jj) -> long long { return (long long)(jj + GW) * px + (cc + GW); };
    // uniform metric constants
    double u_dlx = 0, u_dly = 0, u_nx[3] = {0, 0, 0}, u_ny[3] = {0, 0, 0}, u_Ax = 0, u_Ay = 0, u_vol = 0;
    double u_ilx = 0, u_ily = 0;
    if constexpr (UNI) {
      u_dlx = d.u_dl[0]; u_dly = d.u_dl[1];
      for (int q = 0; q < 3; ++q) { u_nx[q] = d.u_n[0][q]; u_ny[q] = d.u_n[1][q]; }
      u_Ax = d.u_A[0]; u_Ay = d.u_A[1]; u_vol = d.u_vol;
      u_ilx = PH::inv_len(0.5 * (u_dlx + u_dlx));
      u_ily = PH::inv_len(0.5 * (u_dly + u_dly));
    }
    auto dlx_at = [&](int cc, int jj) -> double {
      if constexpr (UNI) return u_dlx; else return a.m.dl[3 * mb + 0 * vs + off(cc, jj)];
    };
    auto dly_at = [&](int cc, int jj) -> double {
      if constexpr (UNI) return u_dly; else return a.m.dl[3 * mb + 1 * vs + off(cc, jj)];
    };
    // 1/l for l = 0.5 (dl_a + dl_b)
    auto ilen = [&](double l, double u_il) -> double {
      if constexpr (!PH::kFast) return 0.0;
      else if constexpr (UNI) return u_il;
      else return PH::inv_len(l);
    };
    auto face_at = [&](int dir, int cc, int jj, double* n) -> double {
      if constexpr (UNI) {
        const double* un = dir == 0 ? u_nx : u_ny;
        n[0] = un[0]; n[1] = un[1]; n[2] = un[2];
        return dir == 0 ? u_Ax : u_Ay;
      } else {
        const double* f = a.m.face + 12 * mb + (4 * dir) * vs + off(cc, jj);
        n[0] = f[0]; n[1] = f[vs]; n[2] = f[2 * vs];
        return f[3 * vs];
      }
    };
    auto loadQ = [&](int cc, int jj, double* q) {
      const long long o = off(cc, jj);
#pragma unroll
      for (int v = 0; v < NV; ++v) q[v] = Pc[v * vs + o];
    };
    const bool jwork = has_cell;   // columns that own cells march in j
    const int cj = jwork ? c : max(0, min(c, ni - 1));   // in-block column for the march of idle threads

    // ---- j-march preamble: slopes and the j-face below the first row -------
    double q0[NV], q1[NV], sig0[NV], shalf[NV], Gm[NV];
    int Gmask = ADD_ALL;
    double dy0 = 0, dy1 = 0;
    {
      double qm2[NV], qm1[NV];
      loadQ(cj, j0 - 2, qm2);
      loadQ(cj, j0 - 1, qm1);
      loadQ(cj, j0, q0);
      loadQ(cj, j0 + 1, q1);
      double dym2 = dly_at(cj, j0 - 2), dym1 = dly_at(cj, j0 - 1);
      dy0 = dly_at(cj, j0); dy1 = dly_at(cj, j0 + 1);
      double la = 0.5 * (dym2 + dym1), lb = 0.5 * (dym1 + dy0), lc = 0.5 * (dy0 + dy1);
      double ila = ilen(la, u_ily), ilb = ilen(lb, u_ily), ilc = ilen(lc, u_ily);
      double sigm1[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double sa = PH::slope(qm1[v] - qm2[v], la, ila);
        double sb = PH::slope(q0[v] - qm1[v], lb, ilb);
        double sc = PH::slope(q1[v] - q0[v], lc, ilc);
        sigm1[v] = PH::lim(sb, sa);
        sig0[v] = PH::lim(sc, sb);
        shalf[v] = sc;
      }
      double n[3];
      double A = face_at(1, cj, j0, n);
      double QL[NV], QR[NV];
      double lm = 0.5 * dym1, lp = 0.5 * dy0;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        QL[v] = qm1[v] + sigm1[v] * lm;
        QR[v] = q0[v] - sig0[v] * lp;
      }
      bool ok = PH::template face<NV>(a.g, QL, QR, n, A, Gm);
      if (!ok && jwork && j0 > 0) report(a.err, 4, b, c, j0, 0);
      if (j0 == 0 && jwork) {
        int w = a.bcw[d.bcoff[2] + c];
        if (bc_code(w) == BC_NONE) {
          for (int v = 0; v < NV; ++v) Gm[v] = 0.0;
          Gmask = ADD_NONE;
        } else if (bc_code(w) != BC_CONN) {
          Gmask = boundary_flux<RIE, LIM, NV>(a, w, q0, q1, dy0, dy1, n, A, 3, Gm);
        }
      }
    }

    for (int j = j0; j < j1; ++j) {
      // ---- rows in: own column of row j+2 (march), row j into shared memory --
      double q2[NV];
      loadQ(cj, j + 2, q2);
      const double dy2 = dly_at(cj, j + 2);
      __syncthreads();   // previous row's readers of sP / sSig / sF are done
      if (colok) {
        if (jwork) {
#pragma unroll
          for (int v = 0; v < NV; ++v) sP[v][t + 1] = q0[v];
        } else {
          double q[NV];
          loadQ(cl, j, q);
#pragma unroll
          for (int v = 0; v < NV; ++v) sP[v][t + 1] = q[v];
        }
        sDL[t + 1] = dlx_at(cl, j);
      }
      if (t == 0) {
        double q[NV];
        loadQ(c0 - 2, j, q);
#pragma unroll
        for (int v = 0; v < NV; ++v) sP[v][0] = q[v];
        sDL[0] = dlx_at(c0 - 2, j);
      }
      if (t == T - 1 && c0 + T - 1 <= ni + 1) {
        double q[NV];
        loadQ(c0 + T - 1, j, q);
#pragma unroll
        for (int v = 0; v < NV; ++v) sP[v][T + 1] = q[v];
        sDL[T + 1] = dlx_at(c0 + T - 1, j);
      }
      __syncthreads();
      // ---- limited slopes: i of row j (shared), j of row j+1 (marched) -------
      double sig1[NV], sup[NV];
      {
        const double lu = 0.5 * (dy1 + dy2);
        const double ilu = ilen(lu, u_ily);
        const double lmn = 0.5 * (sDL[t] + sDL[t + 1]);
        const double lpl = 0.5 * (sDL[t + 1] + sDL[t + 2]);
        const double ilmn = ilen(lmn, u_ilx), ilpl = ilen(lpl, u_ilx);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          sup[v] = PH::slope(q2[v] - q1[v], lu, ilu);
          sig1[v] = PH::lim(sup[v], shalf[v]);
          double sm = PH::slope(sP[v][t + 1] - sP[v][t], lmn, ilmn);
          double sp = PH::slope(sP[v][t + 2] - sP[v][t + 1], lpl, ilpl);
          sSig[v][t] = PH::lim(sp, sm);
        }
      }
      __syncthreads();
      // ---- face fluxes: F(c+1/2, j) and G(c, j+1/2), issued together ---------
      double F[NV], Gp[NV];
      int mask = ADD_ALL, Gpmask = ADD_ALL;
      {
        double nf[3], ng[3];
        const double Af = face_at(0, min(c + 1, ni + 1), j, nf);
        const double Ag = face_at(1, cj, j + 1, ng);
        double QLf[NV], QRf[NV], QLg[NV], QRg[NV];
        const double lmf = 0.5 * sDL[t + 1], lpf = 0.5 * sDL[min(t + 2, T + 1)];
        const double lmg = 0.5 * dy0, lpg = 0.5 * dy1;
        const int tn = min(t + 1, T - 1);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          QLf[v] = sP[v][t + 1] + sSig[v][t] * lmf;
          QRf[v] = sP[v][min(t + 2, T + 1)] - sSig[v][tn] * lpf;
          QLg[v] = q0[v] + sig0[v] * lmg;
          QRg[v] = q1[v] - sig1[v] * lpg;
        }
        const bool okf = PH::template face<NV>(a.g, QLf, QRf, nf, Af, F);
        const bool okg = PH::template face<NV>(a.g, QLg, QRg, ng, Ag, Gp);
        const bool lowb = (c == -1), highb = (c == ni - 1);
        if (!okf && has_face && !lowb && !highb) report(a.err, 4, b, c, j, 0);
        if (!okg && jwork && j < nj - 1) report(a.err, 4, b, c, j, 0);
        // boundary faces: the reference's BC_Fluxes formulas override
        if (has_face && (lowb || highb)) {
          const int w = a.bcw[d.bcoff[lowb ? 0 : 1] + j];
          if (bc_code(w) == BC_NONE) {
            for (int v = 0; v < NV; ++v) F[v] = 0.0;
            mask = ADD_NONE;
          } else if (bc_code(w) != BC_CONN) {
            double Q[NV], Qi[NV];
            const int tb = lowb ? t + 2 : t + 1, ti = lowb ? t + 3 : t;   // boundary / interior column
            for (int v = 0; v < NV; ++v) { Q[v] = sP[v][tb]; Qi[v] = sP[v][ti]; }
            mask = boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, sDL[tb], sDL[ti], nf, Af, lowb ? 1 : 2, F);
          }
        }
        if (jwork && j == nj - 1) {
          const int w = a.bcw[d.bcoff[3] + c];
          if (bc_code(w) == BC_NONE) {
            for (int v = 0; v < NV; ++v) Gp[v] = 0.0;
            Gpmask = ADD_NONE;
          } else if (bc_code(w) != BC_CONN) {
            double qin[NV];
            loadQ(c, j - 1, qin);
            Gpmask = boundary_flux<RIE, LIM, NV>(a, w, q0, qin, dy0, dly_at(c, j - 1), ng, Ag, 4, Gp);
          }
        }
      }
      if (has_face) {
#pragma unroll
        for (int v = 0; v < NV; ++v) sF[v][t] = F[v];
        sMask[t] = mask;
      }
      __syncthreads();
      if (has_cell) {
        ResAcc<NV, PH::kCompensated> R;
        R.init();
        const bool bi0 = (c == 0), bi1 = (c == ni - 1), bj0 = (j == 0), bj1 = (j == nj - 1);
        double Fm[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) Fm[v] = sF[v][t - 1];
        if (!bi0) for (int v = 0; v < NV; ++v) R.add(v, -Fm[v]);
        if (!bi1) for (int v = 0; v < NV; ++v) R.add(v, F[v]);
        if (!bj0) for (int v = 0; v < NV; ++v) R.add(v, -Gm[v]);
        if (!bj1) for (int v = 0; v < NV; ++v) R.add(v, Gp[v]);
        if (bi0) add_bc<NV>(R, Fm, -1.0, sMask[t - 1]);
        if (bi1) add_bc<NV>(R, F, 1.0, mask);
        if (bj0) add_bc<NV>(R, Gm, -1.0, Gmask);
        if (bj1) add_bc<NV>(R, Gp, 1.0, Gpmask);
        double Rv[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) Rv[v] = R.get(v);
        const long long o = off(c, j);
        if constexpr (MODE == 1) {
          double* Rb = a.R + d.sbase;
#pragma unroll
          for (int v = 0; v < NV; ++v) Rb[v * vs + o] = Rv[v];
        } else {
          double vol;
          if constexpr (UNI) vol = u_vol; else vol = a.m.vol[mb + o];
          double dt = a.time_accurate ? *a.dtg : a.dtl[mb + o];
          double Q[NV], QO[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) Q[v] = q0[v];
          const bool first = (a.irk == 1);
          if (!first) {
            const double* Po = a.Po + d.sbase;
#pragma unroll
            for (int v = 0; v < NV; ++v) QO[v] = Po[v * vs + o];
          }
          bool ok = PH::template update<NV>(a.g, Q, QO, Rv, vol, dt, a.c_rk, first);
          if (!ok) report(a.err, 5, b, c, j, 0);
          double* Pn = a.Pn + d.sbase;
#pragma unroll
          for (int v = 0; v < NV; ++v) Pn[v * vs + o] = Q[v];
        }
      }
      // ---- advance the j-march ----------------------------------------------
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        q0[v] = q1[v]; q1[v] = q2[v];
        sig0[v] = sig1[v]; shalf[v] = sup[v]; Gm[v] = Gp[v];
      }
      Gmask = Gpmask;
      dy0 = dy1; dy1 = dy2;
    }
    __syncthreads();
  }
}

}  // namespace mose
