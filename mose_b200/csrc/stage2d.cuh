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
// bit for bit, and do not depend on the decomposition.
//
// Residual accumulation keeps the reference order per cell: the interior
// face sweeps first (i-, i+, j-, j+: Mod_Fluxes.f90:89-179), then the
// boundary-face contributions in face order 1..6 (BC_Fluxes walks the
// bc list by block and face, Mod_BC_Fluxes.f90:52-216).
#pragma once

#include "arena.cuh"
#include "physics_exact.cuh"

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
__device__ __forceinline__ int boundary_flux(const StageArgs& a, int w, const double* Q, const double* Qi,
                                             double dlB, double dlI, const double* n, double area, int face,
                                             double* F) {
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

template <int NV>
__device__ __forceinline__ void add_bc(double* R, const double* F, double sgn, int mask) {
  if (mask == ADD_ALL) {
    for (int v = 0; v < NV; ++v) R[v] = R[v] + sgn * F[v];
  } else if (mask == ADD_MOMENTUM) {
    for (int v = 1; v < NV - 1; ++v) R[v] = R[v] + sgn * F[v];
  }
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

// MODE: 0 = fused (residual + RK update, writes Pn), 1 = residual only (writes R).
template <int RIE, int LIM, bool UNI, int MODE>
__global__ void __launch_bounds__(STRIP_T, 2) k_stage2d(StageArgs a) {
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
    const bool has_sig = (c <= cend);
    const bool has_face = (t < T - 1) && (c <= cend - 1);
    const bool has_cell = (t >= 1) && (c < cend);
    auto off = [&](int cc, int jj) -> long long { return (long long)(jj + GW) * px + (cc + GW); };
    // uniform metric constants
    double u_dlx = 0, u_dly = 0, u_nx[3] = {0, 0, 0}, u_ny[3] = {0, 0, 0}, u_Ax = 0, u_Ay = 0, u_vol = 0;
    if constexpr (UNI) {
      u_dlx = d.u_dl[0]; u_dly = d.u_dl[1];
      for (int q = 0; q < 3; ++q) { u_nx[q] = d.u_n[0][q]; u_ny[q] = d.u_n[1][q]; }
      u_Ax = d.u_A[0]; u_Ay = d.u_A[1]; u_vol = d.u_vol;
    }
    auto dlx_at = [&](int cc, int jj) -> double {
      if constexpr (UNI) return u_dlx; else return a.m.dl[3 * mb + 0 * vs + off(cc, jj)];
    };
    auto dly_at = [&](int cc, int jj) -> double {
      if constexpr (UNI) return u_dly; else return a.m.dl[3 * mb + 1 * vs + off(cc, jj)];
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

    // ---- j-march preamble: slopes and the j-face below the first row -------
    double q0[NV], q1[NV], sig0[NV], shalf[NV], Gm[NV];
    int Gmask = ADD_ALL;
    double dy0 = 0, dy1 = 0;
    if (jwork) {
      double qm2[NV], qm1[NV];
      loadQ(c, j0 - 2, qm2);
      loadQ(c, j0 - 1, qm1);
      loadQ(c, j0, q0);
      loadQ(c, j0 + 1, q1);
      double dym2 = dly_at(c, j0 - 2), dym1 = dly_at(c, j0 - 1);
      dy0 = dly_at(c, j0); dy1 = dly_at(c, j0 + 1);
      double la = 0.5 * (dym2 + dym1), lb = 0.5 * (dym1 + dy0), lc = 0.5 * (dy0 + dy1);
      double sigm1[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double sa = (qm1[v] - qm2[v]) / la;
        double sb = (q0[v] - qm1[v]) / lb;
        double sc = (q1[v] - q0[v]) / lc;
        sigm1[v] = ex::limiter<LIM>(sb, sa);
        sig0[v] = ex::limiter<LIM>(sc, sb);
        shalf[v] = sc;
      }
      double n[3];
      double A = face_at(1, c, j0, n);
      int w = (j0 == 0) ? a.bcw[d.bcoff[2] + c] : (BC_CONN);
      if (j0 > 0 || bc_code(w) == BC_CONN) {
        double QL[NV], QR[NV];
        double lm = 0.5 * dym1, lp = 0.5 * dy0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          QL[v] = qm1[v] + sigm1[v] * lm;
          QR[v] = q0[v] - sig0[v] * lp;
        }
        bool ok = ex::face_flux<RIE, NV>(a.g, QL, QR, n, A, Gm);
        if (!ok && j0 > 0) report(a.err, 4, b, c, j0, 0);
      } else if (bc_code(w) != BC_NONE) {
        Gmask = boundary_flux<RIE, LIM, NV>(a, w, q0, q1, dy0, dy1, n, A, 3, Gm);
      } else {
        for (int v = 0; v < NV; ++v) Gm[v] = 0.0;
        Gmask = ADD_NONE;
      }
    }

    for (int j = j0; j < j1; ++j) {
      // ---- j-march: slope above, limited slope of row j+1, face j+1/2 ------
      double Gp[NV];
      int Gpmask = ADD_ALL;
      double sig1[NV], sup[NV], q2[NV];
      double dy2 = 0;
      if (jwork) {
        loadQ(c, j + 2, q2);
        dy2 = dly_at(c, j + 2);
        double lu = 0.5 * (dy1 + dy2);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          sup[v] = (q2[v] - q1[v]) / lu;
          sig1[v] = ex::limiter<LIM>(sup[v], shalf[v]);
        }
        double n[3];
        double A = face_at(1, c, j + 1, n);
        int w = (j == nj - 1) ? a.bcw[d.bcoff[3] + c] : (BC_CONN);
        if (j < nj - 1 || bc_code(w) == BC_CONN) {
          double QL[NV], QR[NV];
          double lm = 0.5 * dy0, lp = 0.5 * dy1;
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            QL[v] = q0[v] + sig0[v] * lm;
            QR[v] = q1[v] - sig1[v] * lp;
          }
          bool ok = ex::face_flux<RIE, NV>(a.g, QL, QR, n, A, Gp);
          if (!ok && j < nj - 1) report(a.err, 4, b, c, j, 0);
        } else if (bc_code(w) != BC_NONE) {
          // face 4: boundary cell j = nj-1, interior neighbour j-1
          double qin[NV];
          loadQ(c, j - 1, qin);
          Gpmask = boundary_flux<RIE, LIM, NV>(a, w, q0, qin, dy0, dly_at(c, j - 1), n, A, 4, Gp);
        } else {
          for (int v = 0; v < NV; ++v) Gp[v] = 0.0;
          Gpmask = ADD_NONE;
        }
      }

      // ---- i direction on row j ---------------------------------------------
      __syncthreads();   // previous row's readers of sP / sF are done
      if (colok) {
        if (jwork) {
#pragma unroll
          for (int v = 0; v < NV; ++v) sP[v][t + 1] = q0[v];
        } else {
          double q[NV];
          loadQ(c, j, q);
#pragma unroll
          for (int v = 0; v < NV; ++v) sP[v][t + 1] = q[v];
        }
        sDL[t + 1] = dlx_at(c, j);
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
      if (has_sig) {
        double lmn = 0.5 * (sDL[t] + sDL[t + 1]);
        double lpl = 0.5 * (sDL[t + 1] + sDL[t + 2]);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          double sm = (sP[v][t + 1] - sP[v][t]) / lmn;
          double sp = (sP[v][t + 2] - sP[v][t + 1]) / lpl;
          sSig[v][t] = ex::limiter<LIM>(sp, sm);
        }
      }
      __syncthreads();
      if (has_face) {
        // face c+1/2, stored with cell c+1
        double n[3];
        double A = face_at(0, c + 1, j, n);
        double F[NV];
        int mask = ADD_ALL;
        const bool lowb = (c == -1), highb = (c == ni - 1);
        int w = BC_CONN;
        if (lowb) w = a.bcw[d.bcoff[0] + j];
        else if (highb) w = a.bcw[d.bcoff[1] + j];
        if (bc_code(w) == BC_CONN) {
          double QL[NV], QR[NV];
          double lm = 0.5 * sDL[t + 1], lp = 0.5 * sDL[t + 2];
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            QL[v] = sP[v][t + 1] + sSig[v][t] * lm;
            QR[v] = sP[v][t + 2] - sSig[v][t + 1] * lp;
          }
          bool ok = ex::face_flux<RIE, NV>(a.g, QL, QR, n, A, F);
          if (!ok && !lowb && !highb) report(a.err, 4, b, c, j, 0);
        } else if (bc_code(w) == BC_NONE) {
          for (int v = 0; v < NV; ++v) F[v] = 0.0;
          mask = ADD_NONE;
        } else if (lowb) {
          // face 1 of cell 0: boundary cell = column 0 (sP index t+2), interior = column 1 (t+3)
          double Q[NV], Qi[NV];
          for (int v = 0; v < NV; ++v) { Q[v] = sP[v][t + 2]; Qi[v] = sP[v][t + 3]; }
          mask = boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, sDL[t + 2], sDL[t + 3], n, A, 1, F);
        } else {
          // face 2 of cell ni-1: boundary = column ni-1 (t+1), interior = ni-2 (t)
          double Q[NV], Qi[NV];
          for (int v = 0; v < NV; ++v) { Q[v] = sP[v][t + 1]; Qi[v] = sP[v][t]; }
          mask = boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, sDL[t + 1], sDL[t], n, A, 2, F);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) sF[v][t] = F[v];
        sMask[t] = mask;
      }
      __syncthreads();
      if (has_cell) {
        double R[NV];
        double Fm[NV], Fp[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) { Fm[v] = sF[v][t - 1]; Fp[v] = sF[v][t]; R[v] = 0.0; }
        const bool bi0 = (c == 0), bi1 = (c == ni - 1), bj0 = (j == 0), bj1 = (j == nj - 1);
        if (!bi0) for (int v = 0; v < NV; ++v) R[v] = R[v] - Fm[v];
        if (!bi1) for (int v = 0; v < NV; ++v) R[v] = R[v] + Fp[v];
        if (!bj0) for (int v = 0; v < NV; ++v) R[v] = R[v] - Gm[v];
        if (!bj1) for (int v = 0; v < NV; ++v) R[v] = R[v] + Gp[v];
        if (bi0) add_bc<NV>(R, Fm, -1.0, sMask[t - 1]);
        if (bi1) add_bc<NV>(R, Fp, 1.0, sMask[t]);
        if (bj0) add_bc<NV>(R, Gm, -1.0, Gmask);
        if (bj1) add_bc<NV>(R, Gp, 1.0, Gpmask);
        const long long o = off(c, j);
        if constexpr (MODE == 1) {
          double* Rb = a.R + d.sbase;
#pragma unroll
          for (int v = 0; v < NV; ++v) Rb[v * vs + o] = R[v];
        } else {
          double vol;
          if constexpr (UNI) vol = u_vol; else vol = a.m.vol[mb + o];
          double dt = a.time_accurate ? *a.dtg : a.dtl[mb + o];
          double Q[NV], QO[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) Q[v] = sP[v][t + 1];
          const bool first = (a.irk == 1);
          if (!first) {
            const double* Po = a.Po + d.sbase;
#pragma unroll
            for (int v = 0; v < NV; ++v) QO[v] = Po[v * vs + o];
          }
          bool ok = rk_update<NV>(a.g, Q, QO, R, vol, dt, a.c_rk, first);
          if (!ok) report(a.err, 5, b, c, j, 0);
          double* Pn = a.Pn + d.sbase;
#pragma unroll
          for (int v = 0; v < NV; ++v) Pn[v * vs + o] = Q[v];
        }
      }
      // ---- advance the j-march ----------------------------------------------
      if (jwork) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          q0[v] = q1[v]; q1[v] = q2[v];
          sig0[v] = sig1[v]; shalf[v] = sup[v]; Gm[v] = Gp[v];
        }
        Gmask = Gpmask;
        dy0 = dy1; dy1 = dy2;
      }
    }
    __syncthreads();
  }
}

}  // namespace mose
