// adjoint.cu -- discrete adjoint of the 2-D explicit step (HLLC with minmod,
// van Leer or van Albada; time-accurate SSP-RK; general metrics).
//
// One RK stage is P_s = U2P(U0 + c ((U(P_{s-1}) - U0) - R(P_{s-1}) dt / vol))
// with U0 = U(P^n) (Lib_Newstate.f90:134-160, Lib_RK.f90:15-27).  Its
// adjoint, given lam = dJ/dP_s:
//   lam_V = J_U2P(P_s)^T lam                         (k_adj_pre)
//   dJ/dP_{s-1} += J_P2U(P_{s-1})^T (c lam_V)          (k_adj_pre)
//   dJ/dP^n     += J_P2U(P^n)^T ((1 - c) lam_V)        (k_adj_pre)
//   lam_R = -(dt / vol) c lam_V ;  dJ/ddt += sum R . (-(c / vol) lam_V)
//   dJ/dP_{s-1} += (dR/dP_{s-1})^T lam_R               (faces, gather, ghosts)
// The residual's transpose is face-local: every face recomputes its flux
// from its four-cell stencil, runs the reverse sweep of HLLC, the limiter
// and the reconstruction with the face-flux adjoint lam_R(left) -
// lam_R(right), and stores the four stencil cells' contributions; a per-cell
// gather then sums the (up to eight) contributions of a cell, so nothing is
// accumulated with atomics and the result does not depend on scheduling.
// Boundary faces (a few per thousand) use central-difference Jacobians of
// the reference boundary formulas (405 also in the inflow Mach); connection
// faces run the interior face's reverse sweep over the ghost stencil.  The
// ghost fill (Lib_Ghost.f90) is transposed face by face.  The global CFL dt
// of the step (Mod_dt.f90) contributes through its argmin cell.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "physics_adjoint.cuh"
#include "stage2d.cuh"

namespace mose {

namespace {

constexpr int NV = 4;

__device__ __forceinline__ long long off(const BlockDesc& d, int i, int j) { return cell_off2(d, i, j); }

// dl along dir of cell o (metric arrays)
__device__ __forceinline__ double dl_at(const MetricArgs& m, const BlockDesc& d, int dir, long long o) {
  return m.dl[3 * d.mbase + dir * d.vstride + o];
}
__device__ __forceinline__ double face_at(const MetricArgs& m, const BlockDesc& d, int dir, long long o, double* n) {
  const long long vs = d.vstride;
  const double* f = m.face + 12 * d.mbase + (4 * dir) * vs + o;
  n[0] = f[0]; n[1] = f[vs]; n[2] = f[2 * vs];
  return f[3 * vs];
}

// Reverse sweep of one face: stencil q[0..3] (cells c-1 .. c+2 along the
// direction, the face between q[1] and q[2]), dl[0..3], face normal n, area
// A; Fb the adjoint of the area-scaled face flux.  Returns the flux (area
// scaled) in F and the stencil cells' adjoint contributions in C[4][NV].
template <int LIM>
__device__ __forceinline__ void face_vjp(const Gas& g, const double q[4][NV], const double* dl, const double* n,
                                         double A, const double* Fb, double* F, double C[4][NV]) {
  const double ila = fast::rcp(0.5 * (dl[0] + dl[1])), ilb = fast::rcp(0.5 * (dl[1] + dl[2])),
               ilc = fast::rcp(0.5 * (dl[2] + dl[3]));
  double QL[NV], QR[NV], dsLx[NV], dsLy[NV], dsRx[NV], dsRy[NV];
  for (int v = 0; v < NV; ++v) {
    const double sa = (q[1][v] - q[0][v]) * ila, sb = (q[2][v] - q[1][v]) * ilb, sc = (q[3][v] - q[2][v]) * ilc;
    const double sL = adj::limiter_grad<LIM>(sb, sa, &dsLx[v], &dsLy[v]);
    const double sR = adj::limiter_grad<LIM>(sc, sb, &dsRx[v], &dsRy[v]);
    QL[v] = q[1][v] + sL * (0.5 * dl[1]);
    QR[v] = q[2][v] - sR * (0.5 * dl[2]);
  }
  double Fa[NV], Fu[NV], QLb[NV] = {0, 0, 0, 0}, QRb[NV] = {0, 0, 0, 0};
  for (int v = 0; v < NV; ++v) Fa[v] = Fb[v] * A;
  adj::hllc_vjp(g.gamma, g.gcp, g.gm1, QL, QR, n[0], n[1], Fa, Fu, QLb, QRb);
  for (int v = 0; v < NV; ++v) F[v] = Fu[v] * A;
  for (int v = 0; v < NV; ++v) {
    for (int s = 0; s < 4; ++s) C[s][v] = 0.0;
    C[1][v] += QLb[v];
    C[2][v] += QRb[v];
    const double sLb = QLb[v] * (0.5 * dl[1]), sRb = -QRb[v] * (0.5 * dl[2]);
    // sL = phi(sb, sa): sb = (q2 - q1) / lb, sa = (q1 - q0) / la
    const double sbb = sLb * dsLx[v] + sRb * dsRy[v];   // sb also feeds sR as its upwind slope
    const double sab = sLb * dsLy[v];
    const double scb = sRb * dsRx[v];
    C[2][v] += sbb * ilb; C[1][v] -= sbb * ilb;
    C[1][v] += sab * ila; C[0][v] -= sab * ila;
    C[3][v] += scb * ilc; C[2][v] -= scb * ilc;
  }
}

}  // namespace

// ---- per-cell pre-step ---------------------------------------------------------
// lam (adjoint of P_s) -> lamR = -(dt/vol) c lam_V, wdt = -(c/vol) lam_V,
// lam_loc = J_P2U(P_{s-1})^T c lam_V, lam_n += J_P2U(P^n)^T (1-c) lam_V.
// lamG == nullptr: the stage output's adjoint is lam; else it is the later
// stage's lam_loc + lamG (that stage's k_adj_combine, folded in here)
__global__ void k_adj_pre(const BlockDesc* blk, int b, MetricArgs m, Gas g, const double* Ps, const double* Pprev,
                          const double* Pn, const double* lam, const double* lamG, double* lamR, double* wdt,
                          double* lam_loc, double* lam_n, double c, const double* dtg) {
  const BlockDesc& d = blk[b];
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= d.ni || j >= d.nj) return;
  const long long vs = d.vstride, o = d.sbase + off(d, i, j), om = d.mbase + off(d, i, j);
  double P[NV], L[NV], V[NV];
  for (int v = 0; v < NV; ++v) {
    P[v] = Ps[o + v * vs];
    L[v] = lamG ? lam_loc[o + v * vs] + lamG[o + v * vs] : lam[o + v * vs];
  }
  adj::u2p_vjp(g.gm1, P, L, V);
  const double vol = m.vol[om], dt = *dtg;
  double Q[NV], Ub[NV], loc[NV] = {0, 0, 0, 0}, acc[NV] = {0, 0, 0, 0};
  for (int v = 0; v < NV; ++v) {
    Ub[v] = c * V[v];
    lamR[o + v * vs] = -(dt / vol) * Ub[v];
    wdt[o + v * vs] = -Ub[v] / vol;
  }
  for (int v = 0; v < NV; ++v) Q[v] = Pprev[o + v * vs];
  adj::p2u_vjp(g.igm1, Q, Ub, loc);
  for (int v = 0; v < NV; ++v) { Q[v] = Pn[o + v * vs]; Ub[v] = (1.0 - c) * V[v]; }
  adj::p2u_vjp(g.igm1, Q, Ub, acc);
  for (int v = 0; v < NV; ++v) {
    lam_loc[o + v * vs] = loc[v];
    lam_n[o + v * vs] += acc[v];
  }
}

// ---- interior faces, both directions in one launch (dir = blockIdx.z) --------------
// Face between cells (i, j) and its dir-neighbour, stored at (i, j): the four
// stencil contributions in C (16 planes per direction) and the flux in F.
template <int LIM>
__global__ void k_adj_faces(const BlockDesc* blk, int b, MetricArgs m, Gas g, const double* P, const double* lamR,
                            double* Cx, double* Fx, double* Cy, double* Fy) {
  const int dir = blockIdx.z;
  double* C = dir ? Cy : Cx;
  double* F = dir ? Fy : Fx;
  const BlockDesc& d = blk[b];
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  const int di = dir == 0, dj = dir == 1;
  if (i >= d.ni - di || j >= d.nj - dj) return;   // interior faces only
  const long long vs = d.vstride;
  double q[4][NV], dl[4];
  for (int s = 0; s < 4; ++s) {
    const long long o = off(d, i + di * (s - 1), j + dj * (s - 1));
    for (int v = 0; v < NV; ++v) q[s][v] = P[d.sbase + o + v * vs];
    dl[s] = dl_at(m, d, dir, o);
  }
  const long long oc = off(d, i, j), on = off(d, i + di, j + dj);
  double n[3], Fb[NV], Fv[NV], Cc[4][NV];
  const double A = face_at(m, d, dir, on, n);
  for (int v = 0; v < NV; ++v) Fb[v] = lamR[d.sbase + oc + v * vs] - lamR[d.sbase + on + v * vs];
  face_vjp<LIM>(g, q, dl, n, A, Fb, Fv, Cc);
  const long long base = 16 * d.mbase + oc;
  for (int s = 0; s < 4; ++s)
    for (int v = 0; v < NV; ++v) C[base + (4 * s + v) * vs] = Cc[s][v];
  for (int v = 0; v < NV; ++v) F[4 * d.mbase + oc + v * vs] = Fv[v];
}

// ---- boundary faces ------------------------------------------------------------
// One thread per boundary face cell of faces 1..4 (list: block, face, cell
// index along the face, bc-table entry).  Stores the face term's adjoint
// contributions to the four cells along the face normal (slots in increasing
// index: -2..1 on a low face, n-2..n+1 on a high face), the face term itself
// (already signed and masked, as added to the boundary cell's residual) and
// dJ/dMach of a 405 face.
template <int RIE, int LIM>
__global__ void k_adj_bc(StageArgs a, const int4* list, int nlist, const double* lamR, double* Cb, double* Fbc,
                         double* dmach) {
  // thread (q, col): entry q of the list; col 0..7 the input (Q then Qi, 4
  // each) of a finite-difference column, col 8 the face term itself, the
  // inflow Mach column and the connection faces
  const long long tq = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int q = (int)(tq / 9), col = (int)(tq % 9);
  if (q >= nlist) return;
  const int4 e = list[q];
  const int b = e.x, f = e.y, idx = e.z, ent = e.w;
  const BlockDesc& d = a.blk[b];
  const int dir = (f - 1) / 2;
  const bool high = (f % 2) == 0;
  const int i = dir == 0 ? (high ? d.ni - 1 : 0) : idx, j = dir == 1 ? (high ? d.nj - 1 : 0) : idx;
  const int di = dir == 0, dj = dir == 1;
  const long long vs = d.vstride;
  const double sgn = high ? 1.0 : -1.0;
  const int w = a.bcw[d.bcoff[f - 1] + idx];
  const int code = bc_code(w);
  const long long ob = off(d, i, j);
  double Lr[NV];
  for (int v = 0; v < NV; ++v) Lr[v] = lamR[d.sbase + ob + v * vs];
  // stencil cells along the normal, increasing index: t = -2..1 (low) or -1..2 (high) from the boundary cell
  auto cell = [&](int s) { const int t = high ? s - 1 : s - 2; return off(d, i + di * t, j + dj * t); };
  double n[3];
  const double A = face_at(a.m, d, dir, high ? off(d, i + di, j + dj) : ob, n);
  double* Cq = Cb + (size_t)ent * 16;
  if (code == BC_NONE || code == BC_CONN) {
    if (col != 8) return;
    double out[4][NV], Fout[NV];
    for (int s = 0; s < 4; ++s)
      for (int v = 0; v < NV; ++v) out[s][v] = 0.0;
    for (int v = 0; v < NV; ++v) Fout[v] = 0.0;
    if (code == BC_CONN) {
      double qq[4][NV], dl[4], Fb[NV], Fv[NV];
      for (int s = 0; s < 4; ++s) {
        const long long o = cell(s);
        for (int v = 0; v < NV; ++v) qq[s][v] = a.Pc[d.sbase + o + v * vs];
        dl[s] = dl_at(a.m, d, dir, o);
      }
      for (int v = 0; v < NV; ++v) Fb[v] = sgn * Lr[v];
      face_vjp<LIM>(a.g, qq, dl, n, A, Fb, Fv, out);
      for (int v = 0; v < NV; ++v) Fout[v] = sgn * Fv[v];
    }
    for (int s = 0; s < 4; ++s)
      for (int v = 0; v < NV; ++v) Cq[4 * s + v] = out[s][v];
    for (int v = 0; v < NV; ++v) Fbc[(size_t)ent * 4 + v] = Fout[v];
    return;
  }
  // central-difference Jacobian of the reference boundary formula in
  // (Q, Qi) = (boundary cell, first interior cell), and in the inflow Mach
  const int sb = high ? 1 : 2, si = high ? 0 : 3;   // slots of the boundary / interior cell
  double Q[NV], Qi[NV], Fv[NV];
  for (int v = 0; v < NV; ++v) { Q[v] = a.Pc[d.sbase + cell(sb) + v * vs]; Qi[v] = a.Pc[d.sbase + cell(si) + v * vs]; }
  const double dlB = dl_at(a.m, d, dir, cell(sb)), dlI = dl_at(a.m, d, dir, cell(si));
  const int mask = boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, dlB, dlI, n, A, f, Fv);
  double Fb[NV];
  for (int v = 0; v < NV; ++v) {
    const double keep = (mask == ADD_ALL || (mask == ADD_MOMENTUM && v >= 1 && v < NV - 1)) ? 1.0 : 0.0;
    Fb[v] = sgn * keep * Lr[v];
    if (col == 8) Fbc[(size_t)ent * 4 + v] = sgn * keep * Fv[v];
  }
  if (col < 8) {
    const int side = col / NV, k = col % NV;
    double* X = side == 0 ? Q : Qi;
    const double x0 = X[k], h = 1e-6 * fmax(fabs(x0), 1e-3);
    double Fp[NV], Fm[NV];
    X[k] = x0 + h;
    boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, dlB, dlI, n, A, f, Fp);
    X[k] = x0 - h;
    boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, dlB, dlI, n, A, f, Fm);
    double sacc = 0.0;
    for (int v = 0; v < NV; ++v) sacc += Fb[v] * (Fp[v] - Fm[v]) / (2.0 * h);
    // slots: the boundary cell's column k, the interior cell's column k; the
    // other two slots are zero
    Cq[4 * (side == 0 ? sb : si) + k] = sacc;
    if (side == 0) {
      const int z0 = high ? 2 : 0, z1 = high ? 3 : 1;   // the two cells off this face's stencil
      Cq[4 * z0 + k] = 0.0;
      Cq[4 * z1 + k] = 0.0;
    }
    return;
  }
  double dm = 0.0;
  if (code == BC_SUPIN) {
    BcParam p = a.bcp[bc_param(w)];
    const double M0 = p.mach, h = 1e-6 * fmax(fabs(M0), 1e-3);
    double Fp[NV], Fm[NV];
    p.mach = M0 + h;
    ex::bc_supersonic_inflow<RIE, LIM, NV>(a.g, Q, Qi, p, n, A, f, Fp);
    p.mach = M0 - h;
    ex::bc_supersonic_inflow<RIE, LIM, NV>(a.g, Q, Qi, p, n, A, f, Fm);
    // only where boundary_flux takes the inflow branch (its test !(s Un >= 0))
    const double Un = ex::dot_vel<NV>(Q, n), s405 = (double)(1 - 2 * (f % 2));
    if (!(s405 * Un >= 0.0))
      for (int v = 0; v < NV; ++v) dm += Fb[v] * (Fp[v] - Fm[v]) / (2.0 * h);
  }
  dmach[ent] += dm;
}

// ---- gather ------------------------------------------------------------------------
// Ghosted cells: lamG = sum of the interior-face contributions that reach the
// cell; interior cells also form R . wdt of the interior faces (dt partial).
__global__ void k_adj_gather(const BlockDesc* blk, int b, const double* Cx, const double* Cy, const double* Fx,
                             const double* Fy, const double* __restrict__ Cb, const double* __restrict__ Fbc,
                             const double* wdt, double* lamG, double* dtpart) {
  const BlockDesc& d = blk[b];
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) - GW, j = (int)blockIdx.y - GW;
  if (i >= d.ni + GW || j >= d.nj + GW) return;
  const long long vs = d.vstride, oc = off(d, i, j);
  double acc[NV] = {0, 0, 0, 0};
  // x faces between (f, j) and (f + 1, j), f = 0..ni-2: cell i is slot s = i - f + 1
  if (j >= 0 && j < d.nj)
    for (int s = 0; s < 4; ++s) {
      const int f = i - s + 1;
      if (f < 0 || f > d.ni - 2) continue;
      const long long base = 16 * d.mbase + off(d, f, j);
      for (int v = 0; v < NV; ++v) acc[v] += Cx[base + (4 * s + v) * vs];
    }
  if (i >= 0 && i < d.ni)
    for (int s = 0; s < 4; ++s) {
      const int f = j - s + 1;
      if (f < 0 || f > d.nj - 2) continue;
      const long long base = 16 * d.mbase + off(d, i, f);
      for (int v = 0; v < NV; ++v) acc[v] += Cy[base + (4 * s + v) * vs];
    }
  // then the boundary faces' stencil contributions (k_adj_bc), faces 1..4 in
  // order: face f's entry idx touches the four cells along its normal, slot s
  // (the boundary cell is slot 2 on a low face, 1 on a high one)
  double bsum[4];
  int nbs = 0;
  if (Cb != nullptr && (i < 2 || i >= d.ni - 2 || j < 2 || j >= d.nj - 2))
    for (int f = 1; f <= 4; ++f) {
      const int dir = (f - 1) / 2;
      const bool high = (f % 2) == 0;
      const int x = dir == 0 ? i : j, idx = dir == 0 ? j : i, n = dir == 0 ? d.ni : d.nj;
      const int s = high ? x - n + 2 : x + 2;
      if (s < 0 || s > 3 || idx < 0 || idx >= d.bcn[f - 1]) continue;
      const size_t ent = (size_t)(d.bcoff[f - 1] + idx);
      for (int v = 0; v < NV; ++v) acc[v] += Cb[ent * 16 + 4 * s + v];
      if (s == (high ? 1 : 2)) {
        double sum = 0.0;
        for (int v = 0; v < NV; ++v) sum += Fbc[ent * 4 + v] * wdt[d.sbase + oc + v * vs];
        bsum[nbs++] = sum;
      }
    }
  for (int v = 0; v < NV; ++v) lamG[d.sbase + oc + v * vs] = acc[v];
  if (i >= 0 && i < d.ni && j >= 0 && j < d.nj) {
    double R[NV] = {0, 0, 0, 0};
    const long long o4 = 4 * d.mbase;
    if (i > 0) for (int v = 0; v < NV; ++v) R[v] -= Fx[o4 + off(d, i - 1, j) + v * vs];
    if (i < d.ni - 1) for (int v = 0; v < NV; ++v) R[v] += Fx[o4 + oc + v * vs];
    if (j > 0) for (int v = 0; v < NV; ++v) R[v] -= Fy[o4 + off(d, i, j - 1) + v * vs];
    if (j < d.nj - 1) for (int v = 0; v < NV; ++v) R[v] += Fy[o4 + oc + v * vs];
    double s = 0.0;
    for (int v = 0; v < NV; ++v) s += R[v] * wdt[d.sbase + oc + v * vs];
    double dp = dtpart[d.mbase + oc] + s;
    for (int q = 0; q < nbs; ++q) dp = dp + bsum[q];
    dtpart[d.mbase + oc] = dp;
  }
}

// Transpose of Fill_Ghost_Cell for the ghost records of one face.
__global__ void k_adj_ghostT(const BlockDesc* blk, const GhostRec* __restrict__ recs, const int* __restrict__ ids,
                             int n, MetricArgs m, double* lamG) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const GhostRec e = recs[ids[q]];
  const BlockDesc& d = blk[e.b];
  const int dir = (e.f - 1) / 2;
  const int gi = (e.f == 1) ? 1 : (e.f == 2) ? -1 : 0;
  const int gj = (e.f == 3) ? 1 : (e.f == 4) ? -1 : 0;
  const long long vs = d.vstride;
  double* Lb = lamG + d.sbase;
  auto at = [&](int g) { return off(d, e.i - gi * g, e.j - gj * g); };   // g > 0 ghost, g <= 0 interior
  // every branch loads what it reads before it stores: the ghost cells and
  // the cells they feed are distinct, so the accesses are independent
  if (e.type == BC_CONN) {
    const BlockDesc& s = blk[e.bs];
    const int si = (e.fs == 1) ? 1 : (e.fs == 2) ? -1 : 0;
    const int sj = (e.fs == 3) ? 1 : (e.fs == 4) ? -1 : 0;
    double* Ls = lamG + s.sbase;
    long long od[GW], os[GW];
    double lg[GW][NV], ls[GW][NV];
    for (int g = 1; g <= GW; ++g) {
      od[g - 1] = at(g);
      os[g - 1] = off(s, e.is + si * (g - 1), e.js + sj * (g - 1));
      for (int v = 0; v < NV; ++v) {
        lg[g - 1][v] = Lb[v * vs + od[g - 1]];
        ls[g - 1][v] = Ls[v * s.vstride + os[g - 1]];
      }
    }
    for (int g = 0; g < GW; ++g)
      for (int v = 0; v < NV; ++v) {
        Ls[v * s.vstride + os[g]] = ls[g][v] + lg[g][v];
        Lb[v * vs + od[g]] = 0.0;
      }
  } else if (e.type == BC_SYM) {
    // first ghost = the boundary cell with its velocity mirrored in the wall
    const int fi = e.i + (e.f == 2), fj = e.j + (e.f == 4);
    const double* fp = m.face + 12 * d.mbase + (4 * dir) * vs + off(d, fi, fj);
    const double nx = fp[0], ny = fp[vs];
    const long long og = at(1), ob = at(0);
    const double lr = Lb[og], lu = Lb[vs + og], lv = Lb[2 * vs + og], lp = Lb[3 * vs + og];
    double b[NV];
    for (int v = 0; v < NV; ++v) b[v] = Lb[v * vs + ob];
    // u' = u - 2 (u.n) n  (transpose of I - 2 n n^T is itself)
    const double dotl = lu * nx + lv * ny;
    Lb[ob] = b[0] + lr;
    Lb[vs + ob] = b[1] + (lu - 2.0 * dotl * nx);
    Lb[2 * vs + ob] = b[2] + (lv - 2.0 * dotl * ny);
    Lb[3 * vs + ob] = b[3] + lp;
    for (int g = 1; g <= GW; ++g)
      for (int v = 0; v < NV; ++v) Lb[v * vs + at(g)] = 0.0;
  } else if (e.type == BC_EXTRAP) {
    // forward: P(g) = 3 P(g-1) - 3 P(g-2) + P(g-3), g = 1, 2 in order;
    // reverse g = 2 then g = 1 on the five cells g = 2 .. -2
    for (int v = 0; v < NV; ++v) {
      double L[5];
      for (int t = 0; t < 5; ++t) L[t] = Lb[v * vs + at(2 - t)];   // L[t] is cell g = 2 - t
      for (int g = GW; g >= 1; --g) {
        const int t = 2 - g;
        const double l = L[t];
        L[t] = 0.0;
        L[t + 1] += 3.0 * l;
        L[t + 2] -= 3.0 * l;
        L[t + 3] += l;
      }
      for (int t = 0; t < 5; ++t) Lb[v * vs + at(2 - t)] = L[t];
    }
  } else {   // zero gradient (0, 405, 406, ...)
    const long long ob = at(0);
    for (int v = 0; v < NV; ++v) {
      double acc = Lb[v * vs + ob];
      for (int g = 1; g <= GW; ++g) acc += Lb[v * vs + at(g)];
      Lb[v * vs + ob] = acc;
      for (int g = 1; g <= GW; ++g) Lb[v * vs + at(g)] = 0.0;
    }
  }
}

// lam_out = (lam_loc + lamG on interior cells, 0 on ghosts) + lam_n: the
// step's first stage and the direct terms of P^n.
__global__ void k_adj_combine(const BlockDesc* blk, int b, const double* lam_loc, const double* lamG,
                              const double* lam_n, double* lam_out) {
  const BlockDesc& d = blk[b];
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) - GW, j = (int)blockIdx.y - GW;
  if (i >= d.ni + GW || j >= d.nj + GW) return;
  const long long vs = d.vstride, o = d.sbase + off(d, i, j);
  const bool in = i >= 0 && i < d.ni && j >= 0 && j < d.nj;
  for (int v = 0; v < NV; ++v) {
    const double x = in ? lam_loc[o + v * vs] + lamG[o + v * vs] : 0.0;
    lam_out[o + v * vs] = x + lam_n[o + v * vs];
  }
}

// Deterministic sum of n values: pass 1, one partial per CTA over a fixed
// strided subset; pass 2, one CTA sums the partials into *out (+= when
// accumulate).  Fixed grid and fixed tree: the same bits every run.
constexpr int kSumCtas = 296;
// Up to two independent sums in one launch pair: sum blockIdx.y reads
// job[blockIdx.y] and writes its partials at part + blockIdx.y * kSumCtas.
struct SumJobs {
  const double* x[2];
  long long n[2];
  double* out[2];
  int accumulate[2];
};
__global__ void k_sum_partial(SumJobs jb, double* part) {
  __shared__ double s[256];
  const int y = blockIdx.y;
  const double* x = jb.x[y];
  const long long n = jb.n[y];
  double acc = 0.0;
  for (long long q = blockIdx.x * 256LL + threadIdx.x; q < n; q += 256LL * gridDim.x) acc += x[q];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[y * kSumCtas + blockIdx.x] = s[0];
}
__global__ void k_sum_final(SumJobs jb, const double* part) {
  __shared__ double s[256];
  const int y = blockIdx.x;
  double acc = 0.0;
  for (int q = threadIdx.x; q < kSumCtas; q += 256) acc += part[y * kSumCtas + q];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *jb.out[y] = jb.accumulate[y] ? *jb.out[y] + s[0] : s[0];
}

// lam_n[argmin] += (dJ/ddt) d(dt_cell)/dP at the argmin cell.
__global__ void k_adj_dt(const BlockDesc* blk, MetricArgs m, Gas g, const double* P, const unsigned long long* arg,
                         const double* lam_dt, double cfl, int ndir, double* lam_n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const unsigned long long a = *arg;
  if (a == ~0ull) return;
  const int b = (int)(a >> 40);
  const long long o = (long long)(a & ((1ull << 40) - 1));
  const BlockDesc& d = blk[b];
  const long long vs = d.vstride;
  double Q[NV];
  for (int v = 0; v < NV; ++v) Q[v] = P[d.sbase + o + v * vs];
  const double a0 = sqrt(g.gamma * Q[3] / Q[0]);
  double dtmin = 1e300, lam = 1.0, K = 0.0, sdot = 0.0, vx = 0.0, vy = 0.0;
  for (int dd = 0; dd < ndir; ++dd) {
    const double ux = m.vers[9 * d.mbase + (3 * dd + 0) * vs + o], uy = m.vers[9 * d.mbase + (3 * dd + 1) * vs + o];
    const double dot = Q[1] * ux + Q[2] * uy;
    const double l = fabs(dot) + a0, k = m.dl[3 * d.mbase + dd * vs + o] * cfl;
    if (k / l < dtmin) { dtmin = k / l; lam = l; K = k; sdot = copysign(1.0, dot); vx = ux; vy = uy; }
  }
  const double f = -(*lam_dt) * K / (lam * lam);   // dJ/dlambda
  lam_n[d.sbase + o + 0 * vs] += f * (-0.5 * a0 / Q[0]);
  lam_n[d.sbase + o + 1 * vs] += f * sdot * vx;
  lam_n[d.sbase + o + 2 * vs] += f * sdot * vy;
  lam_n[d.sbase + o + 3 * vs] += f * (0.5 * a0 / Q[3]);
}

// Objective J = sum over the face cells of face f of block b of p A, and its
// adjoint (dJ/dp = A on those cells) written into lam (zeroed elsewhere).
__global__ void k_adj_objective(const BlockDesc* blk, int b, int f, MetricArgs m, const double* P, double* terms,
                                double* lam) {
  const BlockDesc& d = blk[b];
  const int dir = (f - 1) / 2;
  const bool high = (f % 2) == 0;
  const int n = dir == 0 ? d.nj : d.ni;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = dir == 0 ? (high ? d.ni - 1 : 0) : q, j = dir == 1 ? (high ? d.nj - 1 : 0) : q;
  const long long o = off(d, i, j), vs = d.vstride;
  double nn[3];
  const double A = face_at(m, d, dir, high ? off(d, i + (dir == 0), j + (dir == 1)) : o, nn);
  terms[q] = P[d.sbase + o + 3 * vs] * A;
  lam[d.sbase + o + 3 * vs] = A;
}

// ---- launchers -----------------------------------------------------------------------
namespace adjl {

static dim3 cells(int ni, int nj, bool ghosted) {
  const int nx = ni + (ghosted ? 2 * GW : 0), ny = nj + (ghosted ? 2 * GW : 0);
  return dim3((nx + 127) / 128, ny);
}

}  // namespace adjl

void adj_pre(const BlockDesc* blk, int b, int ni, int nj, MetricArgs m, Gas g, const double* Ps,
             const double* Pprev, const double* Pn, const double* lam, const double* lamG, double* lamR, double* wdt,
             double* lam_loc, double* lam_n, double c, const double* dtg, cudaStream_t s) {
  k_adj_pre<<<adjl::cells(ni, nj, false), 128, 0, s>>>(blk, b, m, g, Ps, Pprev, Pn, lam, lamG, lamR, wdt, lam_loc,
                                                       lam_n, c, dtg);
}
void adj_faces(const BlockDesc* blk, int b, int ni, int nj, MetricArgs m, Gas g, int lim, const double* P,
               const double* lamR, double* Cx, double* Fx, double* Cy, double* Fy, cudaStream_t s) {
  dim3 grid = adjl::cells(ni, nj, false);
  grid.z = 2;
  switch (lim) {
    case 1: k_adj_faces<1><<<grid, 128, 0, s>>>(blk, b, m, g, P, lamR, Cx, Fx, Cy, Fy); break;
    case 2: k_adj_faces<2><<<grid, 128, 0, s>>>(blk, b, m, g, P, lamR, Cx, Fx, Cy, Fy); break;
    default: k_adj_faces<3><<<grid, 128, 0, s>>>(blk, b, m, g, P, lamR, Cx, Fx, Cy, Fy); break;
  }
}
void adj_bc(const StageArgs& a, int lim, const int4* list, int n, const double* lamR, double* Cb, double* Fbc,
            double* dmach, cudaStream_t s) {
  if (n == 0) return;
  const int grid = (int)((9LL * n + 127) / 128);
  switch (lim) {
    case 1: k_adj_bc<0, 1><<<grid, 128, 0, s>>>(a, list, n, lamR, Cb, Fbc, dmach); break;
    case 2: k_adj_bc<0, 2><<<grid, 128, 0, s>>>(a, list, n, lamR, Cb, Fbc, dmach); break;
    default: k_adj_bc<0, 3><<<grid, 128, 0, s>>>(a, list, n, lamR, Cb, Fbc, dmach); break;
  }
}
void adj_gather(const BlockDesc* blk, int b, int ni, int nj, const double* Cx, const double* Cy,
                const double* Fx, const double* Fy, const double* Cb, const double* Fbc, const double* wdt,
                double* lamG, double* dtpart, cudaStream_t s) {
  k_adj_gather<<<adjl::cells(ni, nj, true), 128, 0, s>>>(blk, b, Cx, Cy, Fx, Fy, Cb, Fbc, wdt, lamG, dtpart);
}
void adj_ghost_transpose(const BlockDesc* blk, const GhostRec* recs, const int* ids, int n, MetricArgs m,
                         double* lamG, cudaStream_t s) {
  if (n == 0) return;
  k_adj_ghostT<<<(n + 127) / 128, 128, 0, s>>>(blk, recs, ids, n, m, lamG);
}
void adj_combine(const BlockDesc* blk, int b, int ni, int nj, const double* lam_loc, const double* lamG,
                 const double* lam_n, double* lam_out, cudaStream_t s) {
  k_adj_combine<<<adjl::cells(ni, nj, true), 128, 0, s>>>(blk, b, lam_loc, lamG, lam_n, lam_out);
}
void adj_sum(const double* x, long long n, double* out, int accumulate, double* scratch, cudaStream_t s) {
  SumJobs jb{{x, nullptr}, {n, 0}, {out, nullptr}, {accumulate, 0}};
  k_sum_partial<<<dim3(kSumCtas, 1), 256, 0, s>>>(jb, scratch);
  k_sum_final<<<1, 256, 0, s>>>(jb, scratch);
}
void adj_sum2(const double* x0, long long n0, double* out0, int acc0, const double* x1, long long n1, double* out1,
              int acc1, double* scratch, cudaStream_t s) {
  SumJobs jb{{x0, x1}, {n0, n1}, {out0, out1}, {acc0, acc1}};
  k_sum_partial<<<dim3(kSumCtas, 2), 256, 0, s>>>(jb, scratch);
  k_sum_final<<<2, 256, 0, s>>>(jb, scratch);
}
int adj_sum_scratch() { return 2 * kSumCtas; }
void adj_dt(const BlockDesc* blk, MetricArgs m, Gas g, const double* P, const unsigned long long* arg,
            const double* lam_dt, double cfl, int ndir, double* lam_n, cudaStream_t s) {
  k_adj_dt<<<1, 32, 0, s>>>(blk, m, g, P, arg, lam_dt, cfl, ndir, lam_n);
}
void adj_objective(const BlockDesc* blk, int b, int f, int n, MetricArgs m, const double* P, double* terms,
                   double* lam, cudaStream_t s) {
  k_adj_objective<<<(n + 127) / 128, 128, 0, s>>>(blk, b, f, m, P, terms, lam);
}

}  // namespace mose
