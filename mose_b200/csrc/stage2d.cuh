// stage2d.cuh -- fused residual + RK-stage kernel for 2-D blocks (and 1-D run
// as 2-D with nj = 1), one launch per RK stage over every block.
//
// Work decomposition.  An item is a strip of cell columns [c0, c1) of one
// block (at most SB_W = 62 columns) and a run of rows [j0, j1).  The CTA is
// SB_X = 64 thread columns by SB_Y = 4 thread rows; thread (tx, ty) sits on
// column c = c0 - 1 + tx (one halo column each side) and on row j0 + 4k + ty
// of batch k.  The CTA marches up the strip one batch of 4 rows at a time:
//   phase A: the limited i-slope of every cell of the batch (halo columns
//            included) and the limited j-slope of the row above each cell;
//   phase B: one i-face flux F(c+1/2) per thread and the j-face flux
//            G(c, j+1/2) above each owned cell;
//   phase C: residual assembly and the RK update of the owned cells.
// The j-slope and the j-face flux of the batch's top row carry into the next
// batch, so every interior face flux is formed once per strip (plus one halo
// face per strip side); the reference forms the same flux with the same
// operations (Mod_Fluxes.f90:89-139), so the exact policy matches it bit for
// bit whatever the decomposition.
//
// Data movement.  State rows stream through a 12-row ring in shared memory
// (three units of 4 rows: two in use, one in flight) with 16-byte cp.async
// copies issued one batch ahead, so DRAM latency overlaps the arithmetic and
// no registers hold prefetched data.  The state at the start of the step (PO)
// for the next batch is prefetched the same way.  Slopes and face fluxes live
// in shared memory; one face solve is live per thread at a time.
//
// Residual accumulation keeps the reference order per cell: the interior
// face sweeps first (i-, i+, j-, j+: Mod_Fluxes.f90:89-179), then the
// boundary-face contributions in face order 1..6 (BC_Fluxes walks the
// bc list by block and face, Mod_BC_Fluxes.f90:52-216).
//
// The arithmetic is a policy: PolExact (the reference's operation order),
// PolFast (FP64 restated for speed) or PolFast<..., true> (mixed).  Boundary
// -face fluxes always use the reference-exact formulas.
//
// Mixed precision on uniform grids (HLLC, AUSM+) runs an FP32 pipeline: each
// staged FP64 row is converted once into an FP32 ring of (rho, u, v, p)
// vectors, and the slopes, limiters, face states and the whole Riemann solve
// are FP32.  The FP32 face fluxes are exact FP64 numbers, so the per-
// direction flux differences F(c+1/2) - F(c-1/2) are formed in FP64 without
// rounding (the difference of two FP32 values is exact in FP64 unless their
// exponents differ by more than 28, where the error is below 2^-53 of the
// larger); the residual is A_i dF + A_j dG, and the RK update runs in FP64
// from the FP64 state.
#pragma once

#include <type_traits>

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
  } else if (code >= BC_STAGIN && code <= BC_FARFIELD) {
    // 401 / 403 / 404 take the inflow formula where the boundary cell enters
    // the domain (its test BC_Sign*Un >= 0 rejects); 407 takes the total
    // conditions there and the back-pressure outflow elsewhere
    // (Mod_BC_Fluxes.f90:119-185, Lib_BC_Fluxes_FarField.f90:53-69)
    const BcParam& bp = a.bcp[bc_param(w)];
    const ex::InGeo G = ex::inflow_geo<NV>(g, Q, n, face);
    if (!(G.sign * G.Un >= 0.0)) {
      if (code == BC_STAGIN || code == BC_FARFIELD) ex::stagn_inflow<NV>(g, Q, G, bp, n, area, F);
      else ex::mass_flux_inflow<NV>(g, Q, bp, n, area, code == BC_MFLUX_T0, F);
      return ADD_ALL;
    }
    if (code == BC_FARFIELD) {
      ex::bc_outflow<NV>(g, Q, G.Un, n, area, bp.pback, face, F);
      return ADD_ALL;
    }
  }
  // BC_SYM, and the symmetry fallback of 401 / 403 / 404 / 405 / 406
  // (Mod_BC_Fluxes.f90:128,148,157,168,173)
  ex::bc_symmetry<RIE, LIM, NV>(g, Q, Qi, dlB, dlI, n, area, face, F);
  return ADD_MOMENTUM;
}

// Compute_Prim_Residual (Lib_Newstate.f90:255-302, one calorically perfect
// species): the conservative residual R of a cell with primitives Q turned,
// in place, into its primitive increment over dt.  In 2-D the reference's
// w terms are exact zeros.
template <int NV>
__device__ __forceinline__ void prim_residual(const Gas& g, const double* Q, double* R, double vol, double dt) {
  constexpr int P = NV - 1;
  const double rho = Q[0];
  const double temperature = Q[P] / (rho * g.R);
  const double inv_volume = 1.0 / vol;
  const double inv_rhovolume = inv_volume / rho;
  R[0] = -R[0] * inv_volume;
  const double dwrotot = R[0];
  for (int d = 0; d < NV - 2; ++d) R[1 + d] = -R[1 + d] * inv_rhovolume - Q[1 + d] / rho * dwrotot;
  const double dwE = -R[P] * inv_volume;
  double vr = Q[1] * R[1] + Q[2] * R[2];
  if constexpr (NV == 5) vr = vr + Q[3] * R[3];
  const double dwroe = dwE - rho * vr - 0.5 * dwrotot * ex::vel_sq<NV>(Q);
  const double eiroi = (g.cp * temperature - g.R * temperature) * R[0];
  const double cv = Q[0] * (g.cp - g.R);
  const double dwTemp = (dwroe - eiroi) / cv;
  R[P] = g.R * (temperature * R[0] + Q[0] * dwTemp);
  for (int v = 0; v < NV; ++v) R[v] = R[v] * dt * 1.0;
}

// RK_Stage on the primitives and Check_And_Fix_State (Lib_RK.f90:15-27,
// Lib_Newstate.f90:323-356): Q = QO + c ((Q - QO) + Rp).  first_stage: QO
// equals Q and is not read (the stage kernels do not load it then).
template <int NV>
__device__ __forceinline__ bool rk_prim_stage(double* Q, const double* QO, const double* Rp, double c,
                                              bool first_stage = false) {
  constexpr int P = NV - 1;
  for (int v = 0; v < NV; ++v) {
    if (first_stage) {
      const double r_ = (0.0 + Rp[v]) * c;
      Q[v] = Q[v] + r_;
    } else {
      const double r_ = (Q[v] - QO[v] + Rp[v]) * c;
      Q[v] = QO[v] + r_;
    }
  }
  bool bad = false;
  for (int v = 0; v < NV; ++v) bad |= isnan(Q[v]);
  bad |= (Q[P] < 0.0);
  if (Q[0] < 1e-20) Q[0] = 1e-20;
  return !bad;
}

// Newstate_Conservative for one cell (Lib_Newstate.f90:134-160), or
// Newstate_Primitive's Compute_And_Update_Prim (:305-315) when g.prim;
// returns the new primitives in Q.  first_stage: P == PO, so U - U0 is an
// exact zero.
template <int NV>
__device__ __forceinline__ bool rk_update(const Gas& g, double* Q, const double* QO, const double* R,
                                          double vol, double dt, double c, bool first_stage) {
  constexpr int P = NV - 1;
  if (g.prim) {
    double Rp[NV];
    for (int v = 0; v < NV; ++v) Rp[v] = R[v];
    prim_residual<NV>(g, Q, Rp, vol, dt);
    return rk_prim_stage<NV>(Q, QO, Rp, c, first_stage);
  }
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

// CFL time step of one cell (Mod_dt.f90:71-85): the minimum over the ndir
// directions of dl_d CFL / (|u . versor_d| + a).  FAST: the restated FP64
// arithmetic (a^2 = gamma p / rho, reciprocals); otherwise the reference's
// operations, so the standalone pass and the fused one agree bit for bit.
template <int NV, bool UNI, bool FAST>
__device__ __forceinline__ double cfl_dt(const Gas& g, const double* Q, const BlockDesc& d, const MetricArgs& m,
                                         long long o, int ndir, double cfl) {
  const long long vs = d.vstride, mb = d.mbase;
  double Sound;
  if constexpr (FAST) Sound = fast::sqrt_(g.gamma * Q[NV - 1] * fast::rcp(Q[0]));
  else Sound = ex::sound(g, Q[0], Q[NV - 1]);
  double dtmin = 1e8;
  for (int dd = 0; dd < ndir; ++dd) {
    double ver[3];
    double dlv;
    if constexpr (UNI) {
      ver[0] = d.u_vers[dd][0]; ver[1] = d.u_vers[dd][1]; ver[2] = d.u_vers[dd][2];
      dlv = d.u_dl[dd];
    } else {
      for (int c = 0; c < 3; ++c) ver[c] = m.vers[9 * mb + (3 * dd + c) * vs + o];
      dlv = m.dl[3 * mb + dd * vs + o];
    }
    const double vel_ = fabs(ex::dot_vel<NV>(Q, ver));
    const double lambda = vel_ + Sound;
    double dt;
    if constexpr (FAST) dt = (dlv * cfl) * fast::rcp(lambda);
    else dt = dlv / lambda * cfl;
    dtmin = fmin(dt, dtmin);
  }
  return dtmin;
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
  static constexpr bool kMixed = false;
  static constexpr bool kFace32 = false;
  __device__ static double inv_len(double l) { return 0.0; }
  __device__ static double slope(double dq, double l, double) { return dq / l; }
  __device__ static double lim(double x, double y) { return ex::limiter<LIM>(x, y); }
  template <int NV>
  __device__ static bool face(const Gas& g, const double* QL, const double* QR, const double* n, double A,
                              double* F, double beta = 1.0) {
    return ex::face_flux<RIE, NV>(g, QL, QR, n, A, F, beta);
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
  static constexpr bool kMixed = MIXED;
  // face states and Riemann solve in FP32 (face32): the mixed precision with
  // a solver that has an FP32 form
  static constexpr bool kFace32 = MIXED && RIE <= 1;
  __device__ static double inv_len(double l) { return fast::rcp(l); }
  __device__ static double slope(double dq, double, double il) { return dq * il; }
  __device__ static double lim(double x, double y) {
    if constexpr (MIXED) return (double)fast::limiter32<LIM>((float)x, (float)y);
    else return fast::limiter<LIM>(x, y);
  }
  template <int NV>
  __device__ static bool face(const Gas& g, const double* QL, const double* QR, const double* n, double A,
                              double* F, double beta = 1.0) {
    constexpr int P = NV - 1;
    // check_gas_state (x > 0) on the integer pipe: x in (0, +inf] as bit
    // patterns, which leaves out -0, negatives and NaNs
    auto pos_fin = [](double x) {
      return (unsigned long long)(__double_as_longlong(x) - 1) < 0x7ff0000000000000ULL;
    };
    bool ok = pos_fin(QL[0]) && pos_fin(QL[P]) && pos_fin(QR[0]) && pos_fin(QR[P]);
    const fast::GasF gf = fast::gasf(g);
    if constexpr (RIE == 0) {
      if constexpr (MIXED) fast::hllc_mixed<NV>(gf, QL, QR, n, F);
      else fast::hllc<NV>(gf, QL, QR, n, F);
    } else if constexpr (RIE == 1) {
      if constexpr (MIXED) fast::ausmp_mixed<NV>(gf, QL, QR, n, F);
      else fast::ausmp<NV>(gf, QL, QR, n, F);
    } else {
      double aL = ex::sound(g, QL[0], QL[P]), aR = ex::sound(g, QR[0], QR[P]);
      ex::riemann<RIE, NV>(g, QL, aL, QR, aR, n, F, beta);
    }
    for (int v = 0; v < NV; ++v) F[v] = F[v] * A;
    return ok;
  }
  // FP32 face states QL, QR (rho, velocity, p): the FP32 solve, its flux per
  // unit area widened to FP64 (exactly) and scaled by the face area
  template <int NV>
  __device__ static bool face32(const Gas& g, const float* QL, const float* QR, const double* n, double A,
                                double* F) {
    constexpr int P = NV - 1;
    const bool ok = (QL[0] > 0.0f && QL[P] > 0.0f && QR[0] > 0.0f && QR[P] > 0.0f);
    const fast::GasF32 gf = fast::gasf32(g);
    const float nf[3] = {(float)n[0], (float)n[1], (float)n[2]};
    float f[NV];
    if constexpr (RIE == 0) fast::hllc32n<NV>(gf, QL, QR, nf, f);
    else fast::ausmp32n<NV>(gf, QL, QR, nf, f);
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = (double)f[v] * A;
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

// ---- shared memory of the batched march --------------------------------------
constexpr int SB_RING = 3 * SB_Y;   // ring rows: three units of SB_Y rows
constexpr int SB_RS = 68;           // ring row stride (doubles): cells c0-2 .. c0+63, 16-byte rows
constexpr int SB_CH = 33;           // 16-byte chunks per ring row (66 cells)
constexpr int SB_OCH = SB_W / 2;    // 16-byte chunks of the owned columns of a PO row

// FP32 pipeline: mixed policy, uniform metrics, a solver with an FP32 form.
template <class PH, int RIE, bool UNI>
constexpr bool stage_fp32_pipeline() {
  return PH::kMixed && UNI && RIE <= 1;
}

// NVR ring planes: the NV state variables, plus dl along i and j with metric
// arrays.  MX: the FP32 pipeline's arrays replace the FP64 slope arrays.  BC:
// the items may touch physical boundary faces (their add masks are kept);
// without, the FP32 pipeline's face fluxes are all FP32 values and are kept
// as such.  Arrays a variant does not use shrink to one element.
template <int NV, int NVR, bool MX, bool BC, bool SDV = false>
struct StageSmem {
  using FluxT = typename std::conditional<MX && !BC, float, double>::type;
  static constexpr int kY = MX ? 1 : SB_Y, kX = MX ? 1 : SB_X, kV = MX ? 1 : NV;
  static constexpr int mY = MX ? SB_Y : 1, mX = MX ? SB_X : 1, mR = MX ? SB_RING : 1, mS = MX ? SB_RS : 1;
  double ring[NVR][SB_RING][SB_RS];
  double po[NV][SB_Y][SB_X];          // PO of the owned cells (column c - c0) of the current batch
  FluxT f[NV][SB_Y][SB_X];            // F(c + 1/2, j)
  FluxT g[NV][SB_Y + 1][SB_X];        // G(c, j0 + r - 1/2): row 0 carried from the previous batch
  int fm[BC ? SB_Y : 1][BC ? SB_X : 1];       // add masks of F / G
  int gm[BC ? SB_Y + 1 : 1][BC ? SB_X : 1];
  double sx[kV][kY][kX];              // limited i-slope of cell (c, j)
  double sy[kV][MX ? 1 : SB_Y + 1][kX];   // limited j-slope of row r: 0 = batch base row (carried)
  float4 r32[mR][mS];                 // FP32 ring of (rho, u, v, p)
  float4 sx32[mY][mX];
  float4 sy32[MX ? SB_Y + 1 : 1][mX];
  double beta[SDV ? SB_Y : 1][SDV ? SB_X : 1];   // shock detector of cell (c, j) (run-time solver kernels)
};

template <bool UNI, bool MX, bool BC, bool SDV = false>
constexpr size_t stage_smem_bytes() {
  return sizeof(StageSmem<4, UNI ? 4 : 6, MX, BC, SDV>);
}

// Minimum resident CTAs per SM of a kernel variant.  Without boundary faces
// the uniform-metric kernels fit three CTAs (80 registers, ~71 KB of shared
// memory); the boundary formulas (a call) and the metric-array ring need two.
template <bool UNI, bool BC>
constexpr int stage_min_ctas() {
  return (UNI && !BC) ? 3 : 2;
}

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// all but the most recent commit group of this thread complete
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ float4 f4_add(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 f4_sub(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
// a + s b
__device__ __forceinline__ float4 f4_fma(float s, float4 b, float4 a) {
  return make_float4(fmaf(s, b.x, a.x), fmaf(s, b.y, a.y), fmaf(s, b.z, a.z), fmaf(s, b.w, a.w));
}


// FP32 CFL dt of one cell of a uniform 2-D block (the FP32 pipeline's fused
// Compute_dt): a relative error near 1e-7 in the global dt moves the solution
// far less than the pipeline's own FP32 flux error.
__device__ __forceinline__ double cfl_dt32(const Gas& g, const double* Q, const BlockDesc& d, int ndir, double cfl) {
  const float r = (float)Q[0], u = (float)Q[1], v = (float)Q[2], p = (float)Q[3];
  const float a = fast::fsqrtp((float)g.gamma * p * fast::frcp(r));
  float dtmin = 1e8f;
  for (int dd = 0; dd < ndir; ++dd) {
    const float lam = fabsf(fmaf(u, (float)d.u_vers[dd][0], v * (float)d.u_vers[dd][1])) + a;
    dtmin = fminf(dtmin, (float)(d.u_dl[dd] * cfl) * fast::frcp(lam));
  }
  return (double)dtmin;
}

// MODE: 0 = fused (residual + RK update, writes Pn), 1 = residual only (writes
// R), 2 = fused and the next step's Compute_dt on the new state (last stage).
// BC: the kernel of the items that touch a physical boundary face (a.items);
// without, the items whose block-edge faces are all connections
// (a.items_nb): no boundary formula, every face flux added whole.  Both add
// a cell's face terms in the same order, so their results are identical.
template <class PH, int RIE, int LIM, bool UNI, int MODE, bool BC>
__global__ void __launch_bounds__(SB_T, stage_min_ctas<UNI, BC>()) k_stage2d(StageArgs a) {
  constexpr int NV = 4;
  constexpr int NVR = UNI ? NV : NV + 2;
  constexpr bool MX = stage_fp32_pipeline<PH, RIE, UNI>();
  // uniform grid, fast arithmetic: the limiters are homogeneous of degree 1,
  // so slopes stay in difference units and the half-cell factor is 1/2
  constexpr bool FU = UNI && PH::kFast;
  // the run-time solver kernels carry the shock detector (SD_Tramel) of
  // Mod_Fluxes.f90:78-85: each face takes its low cell's value (the
  // boundary cell's at a connection on a low face, Lib_BC_Fluxes_Connection
  // .f90:58-62), which scales the limited slopes under MUSCL-SD and goes to
  // the SD Riemann solvers
  constexpr bool SDV = (RIE == 4);
  const bool sd = SDV && a.g.sd != 0, sdl = SDV && (a.g.sd & 1) != 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StageSmem<NV, NVR, MX, BC, SDV>& S = *reinterpret_cast<StageSmem<NV, NVR, MX, BC, SDV>*>(smem_raw);
  const int4* items = BC ? a.items : a.items_nb;
  const int nitems = BC ? a.nitems : a.nitems_nb;
  const int t = threadIdx.x;
  const int tx = t % SB_X, ty = t / SB_X;
  const bool need_po = (MODE != 1) && (a.irk != 1);
  double dtrun = __longlong_as_double(0x7ff0000000000000LL);   // fused dt: running minimum

#pragma unroll 1
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 item = items[it];
    const int b = item.x, c0 = item.y & 0xffff, c1 = item.y >> 16, j0 = item.z, j1 = item.w;
    const BlockDesc& d = a.blk[b];
    const int ni = d.ni, nj = d.nj, px = d.px;
    const long long vs = d.vstride;
    const double* Pc = a.Pc + d.sbase;
    const long long mb = d.mbase;
    const int c = c0 - 1 + tx;
    const bool has_face = (tx < SB_X - 1) && (c <= c1 - 1);   // F(c + 1/2)
    const bool owns = (tx >= 1) && (c < c1);
    const int nbatch = (j1 - j0 + SB_Y - 1) / SB_Y;
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
    // ring access: ring row rr, ring column col (cell c0 - 2 + col)
    auto ringQ = [&](int rr, int col, double* q) {
#pragma unroll
      for (int v = 0; v < NV; ++v) q[v] = S.ring[v][rr][col];
    };
    auto ring_dlx = [&](int rr, int col) -> double {
      if constexpr (UNI) return u_dlx; else return S.ring[NV][rr][col];
    };
    auto ring_dly = [&](int rr, int col) -> double {
      if constexpr (UNI) return u_dly; else return S.ring[NV + 1][rr][col];
    };
    // 1/l for l = 0.5 (dl_a + dl_b)
    auto ilen = [&](double l, double u_il) -> double {
      if constexpr (!PH::kFast) return 0.0;
      else if constexpr (UNI) return u_il;
      else return PH::inv_len(l);
    };
    // limited slope of q between qa (low side) and qb (high side), cell-centre
    // distances la, lb
    auto lslope = [&](double qa, double q, double qb, double la, double lb, double ila, double ilb) -> double {
      if constexpr (FU) return PH::lim(qb - q, q - qa);
      else return PH::lim(PH::slope(qb - q, lb, ilb), PH::slope(q - qa, la, ila));
    };
    // half-cell factor of a face state: 0.5 dl (reference) or 0.5 (difference units)
    auto half = [&](double dl) -> double {
      if constexpr (FU) return 0.5; else return 0.5 * dl;
    };
    // shock detector of the cell at ring row rr, column col (rows rm / rp)
    auto cell_beta = [&](int rm_, int rr_, int rp_, int col_) -> double {
      return ex::sd_tramel2(S.ring[NV - 1][rr_][col_], S.ring[NV - 1][rr_][col_ - 1], S.ring[NV - 1][rr_][col_ + 1],
                            S.ring[NV - 1][rm_][col_], S.ring[NV - 1][rp_][col_]);
    };
    // limited j-slope of the cell at ring row rr (rows rm, rr, rp), ring column col
    auto slope_j = [&](int rm, int rr, int rp, int col, double* s) {
      const double la = 0.5 * (ring_dly(rm, col) + ring_dly(rr, col));
      const double lb = 0.5 * (ring_dly(rr, col) + ring_dly(rp, col));
      const double ila = ilen(la, u_ily), ilb = ilen(lb, u_ily);
#pragma unroll
      for (int v = 0; v < NV; ++v)
        s[v] = lslope(S.ring[v][rm][col], S.ring[v][rr][col], S.ring[v][rp][col], la, lb, ila, ilb);
    };
    // FP32 pipeline: face normals of the uniform block
    const float fnx0 = (float)u_nx[0], fnx1 = (float)u_nx[1], fny0 = (float)u_ny[0], fny1 = (float)u_ny[1];
    const fast::GasF32 g32 = fast::gasf32(a.g);
    auto solve32 = [&](float4 L, float4 R, float nx, float ny, double* F) -> bool {
      float f[4];
      if constexpr (RIE == 0) fast::hllc32(g32, L, R, nx, ny, f);
      else fast::ausmp32(g32, L, R, nx, ny, f);
#pragma unroll
      for (int v = 0; v < NV; ++v) F[v] = (double)f[v];
      return L.x > 0.0f && L.w > 0.0f && R.x > 0.0f && R.w > 0.0f;
    };
    // boundary override in the FP32 pipeline: flux per unit area, mask applied
    auto per_area = [&](double* F, int mask, double iA) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const bool keep = (mask == ADD_ALL) || (mask == ADD_MOMENTUM && v >= 1 && v < NV - 1);
        F[v] = keep ? F[v] * iA : 0.0;
      }
    };

    // the item reads ghost chunks of an edge read in place only when it
    // touches a block edge
    const bool edge_item = a.remap && (c0 == 0 || c1 >= ni || j0 == 0 || j1 >= nj);
    // unit u = rows j0 - 2 + 4u .. + 3 into ring rows 4 (u % 3) ..; each
    // thread copies all planes of its (row, 2-cell chunk) pairs
    auto load_unit = [&](int u) {
      const int slot = (u % 3) * SB_Y;
      const int rbase = j0 - 2 + SB_Y * u;
      if (!edge_item) {
        for (int e = t; e < SB_Y * SB_CH; e += SB_T) {
          const int i = e / SB_CH, q = e - i * SB_CH;
          const int r = rbase + i;
          const int x = c0 + 2 * q;   // padded column of cell c0 - 2 + 2q
          if (r > nj + 1 || x >= px) continue;
          const long long o = (long long)(r + GW) * px + x;
#pragma unroll
          for (int pv = 0; pv < NVR; ++pv) {
            const double* plane = pv < NV ? Pc + pv * vs : a.m.dl + 3 * mb + (pv - NV) * vs;
            cp_async16(&S.ring[pv][slot + i][2 * q], plane + o);
          }
        }
        return;
      }
      for (int e = t; e < SB_Y * SB_CH; e += SB_T) {
        const int i = e / SB_CH, q = e - i * SB_CH;
        const int r = rbase + i;
        const int x = c0 + 2 * q;
        if (r > nj + 1 || x >= px) continue;
        const long long o = (long long)(r + GW) * px + x;
        // the state's source: this block's cells, or, for a ghost chunk of
        // an edge read in place, the source block's cells that
        // Ghost_Connection would copy there (corner chunks stay as they are:
        // no stencil reads them)
        const double* src = Pc + o;
        long long svs = vs;
        const int cell = x - GW;
        const int gc = cell < 0 ? 0 : cell >= ni ? 1 : -1;
        const int gr = r < 0 ? 2 : r >= nj ? 3 : -1;
        const int f = (gc >= 0) == (gr >= 0) ? -1 : (gc >= 0 ? gc : gr);
        if (f >= 0 && d.rm_src[f] >= 0) {
          const BlockDesc& sb = a.blk[d.rm_src[f]];
          const int si = f < 2 ? d.rm_at[f] : cell + d.rm_off[f];
          const int sj = f < 2 ? r + d.rm_off[f] : d.rm_at[f] + (f == 2 ? r : r - nj);
          src = a.Pc + sb.sbase + cell_off2(sb, si, sj);
          svs = sb.vstride;
        }
#pragma unroll
        for (int pv = 0; pv < NVR; ++pv) {
          const double* g = pv < NV ? src + pv * svs : a.m.dl + 3 * mb + (pv - NV) * vs + o;
          cp_async16(&S.ring[pv][slot + i][2 * q], g);
        }
      }
    };
    // FP32 copy of the chunks this thread copied for unit u (after its wait)
    auto convert_unit = [&](int u) {
      if constexpr (MX) {
        const int slot = (u % 3) * SB_Y;
        const int rbase = j0 - 2 + SB_Y * u;
        for (int e = t; e < SB_Y * SB_CH; e += SB_T) {
          const int i = e / SB_CH, q = e - i * SB_CH;
          if (rbase + i > nj + 1 || c0 + 2 * q >= px) continue;
          const int rr = slot + i;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int col = 2 * q + h;
            S.r32[rr][col] = make_float4((float)S.ring[0][rr][col], (float)S.ring[1][rr][col],
                                         (float)S.ring[2][rr][col], (float)S.ring[3][rr][col]);
          }
        }
      }
    };
    // PO of batch kk (rows j0 + 4 kk .., owned columns) into po
    auto load_po = [&](int kk) {
      const double* Po = a.Po + d.sbase;
      const int rbase = j0 + SB_Y * kk;
      constexpr int n = NV * SB_Y * SB_OCH;
      for (int e = t; e < n; e += SB_T) {
        const int v = e / (SB_Y * SB_OCH);
        const int rem = e - v * (SB_Y * SB_OCH);
        const int i = rem / SB_OCH;
        const int q = rem - i * SB_OCH;
        const int r = rbase + i;
        const int x = c0 + GW + 2 * q;   // padded column of cell c0 + 2q
        if (r >= j1 || x >= px) continue;
        cp_async16(&S.po[v][i][2 * q], Po + v * vs + (long long)(r + GW) * px + x);
      }
    };

    // ---- prologue: j-slopes of rows j0-1, j0 and the j-face below row j0 --------
    load_unit(0);
    load_unit(1);
    cp_async_commit();
    cp_async_wait_all();
    convert_unit(0);
    convert_unit(1);
    __syncthreads();
    if (ty < 2 && owns) {
      // ty 0: row j0 - 1 (ring row 1) -> slot 1; ty 1: row j0 (ring row 2) -> slot 0
      if constexpr (MX) {
        const float4 qa = S.r32[ty][tx + 1], q = S.r32[ty + 1][tx + 1], qb = S.r32[ty + 2][tx + 1];
        S.sy32[1 - ty][tx] = fast::limiter32x4<LIM>(f4_sub(qb, q), f4_sub(q, qa));
      } else {
        double s[NV];
        slope_j(ty, ty + 1, ty + 2, tx + 1, s);
#pragma unroll
        for (int v = 0; v < NV; ++v) S.sy[v][1 - ty][tx] = s[v];
      }
    }
    __syncthreads();
    if (ty == 0 && owns) {
      double q0[NV], G[NV], n[3];
      ringQ(2, tx + 1, q0);
      const double A = face_at(1, c, j0, n);
      bool ok;
      if constexpr (MX) {
        const float4 L = f4_fma(0.5f, S.sy32[1][tx], S.r32[1][tx + 1]);
        const float4 R = f4_fma(-0.5f, S.sy32[0][tx], S.r32[2][tx + 1]);
        ok = solve32(L, R, fny0, fny1, G);
      } else {
        double qm[NV], QL[NV], QR[NV];
        ringQ(1, tx + 1, qm);
        const double lm = half(ring_dly(1, tx + 1)), lp = half(ring_dly(2, tx + 1));
        // the face below row j0: row j0 - 1's detector, row j0's on the block's low face
        const double bP = sd ? (j0 == 0 ? cell_beta(1, 2, 3, tx + 1) : cell_beta(0, 1, 2, tx + 1)) : 1.0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const double sLv = sdl ? bP * S.sy[v][1][tx] : S.sy[v][1][tx];
          const double sRv = sdl ? bP * S.sy[v][0][tx] : S.sy[v][0][tx];
          QL[v] = qm[v] + sLv * lm;
          QR[v] = q0[v] - sRv * lp;
        }
        ok = PH::template face<NV>(a.g, QL, QR, n, A, G, bP);
      }
      if (!ok && j0 > 0) report(a.err, 4, b, c, j0, 0);
      int mask = ADD_ALL;
      if (BC && j0 == 0) {
        const int w = a.bcw[d.bcoff[2] + c];
        if (bc_code(w) == BC_NONE) {
          for (int v = 0; v < NV; ++v) G[v] = 0.0;
          mask = ADD_NONE;
        } else if (bc_code(w) != BC_CONN) {
          double q1[NV];
          ringQ(3, tx + 1, q1);
          mask = boundary_flux<RIE, LIM, NV>(a, w, q0, q1, ring_dly(2, tx + 1), ring_dly(3, tx + 1), n, A, 3, G);
          if constexpr (MX) per_area(G, mask, 1.0 / A);
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) S.g[v][SB_Y][tx] = G[v];
      if constexpr (BC) S.gm[SB_Y][tx] = mask;
    }

#pragma unroll 1
    for (int k = 0; k < nbatch; ++k) {
      __syncthreads();   // ring units k, k+1 visible; batch k-1 done with everything
      // two commit groups: this batch's PO (waited for before phase C), then
      // ring unit k + 2 (waited for at the end of the batch)
      if (need_po) load_po(k);
      cp_async_commit();
      if (k + 2 <= nbatch) load_unit(k + 2);
      cp_async_commit();
      const int j = j0 + SB_Y * k + ty;
      const bool rowok = j < j1;
      const int rr = (SB_Y * k + ty + 2) % SB_RING;   // ring row of row j
      const int rm = (rr + SB_RING - 1) % SB_RING;
      const int rp = (rr + 1) % SB_RING, rp2 = (rr + 2) % SB_RING;
      const int col = tx + 1;                         // ring column of cell c

      // ---- phase A: limited slopes ------------------------------------------------
      if (ty == 0 && owns) {   // carry the previous batch's top j-face
#pragma unroll
        for (int v = 0; v < NV; ++v) S.g[v][0][tx] = S.g[v][SB_Y][tx];
        if constexpr (BC) S.gm[0][tx] = S.gm[SB_Y][tx];
      }
      if constexpr (SDV) {
        if (sd && rowok) S.beta[ty][tx] = cell_beta(rm, rr, rp, col);
      }
      if (rowok) {
        if constexpr (MX) {
          const float4 qa = S.r32[rr][col - 1], q = S.r32[rr][col], qb = S.r32[rr][col + 1];
          S.sx32[ty][tx] = fast::limiter32x4<LIM>(f4_sub(qb, q), f4_sub(q, qa));
          if (owns) {
            const float4 q1 = S.r32[rp][col], q2 = S.r32[rp2][col];
            S.sy32[ty + 1][tx] = fast::limiter32x4<LIM>(f4_sub(q2, q1), f4_sub(q1, q));
          }
        } else {
          const double dm = ring_dlx(rr, col - 1), d0 = ring_dlx(rr, col), dp = ring_dlx(rr, col + 1);
          const double la = 0.5 * (dm + d0), lb = 0.5 * (d0 + dp);
          const double ila = ilen(la, u_ilx), ilb = ilen(lb, u_ilx);
#pragma unroll
          for (int v = 0; v < NV; ++v)
            S.sx[v][ty][tx] = lslope(S.ring[v][rr][col - 1], S.ring[v][rr][col], S.ring[v][rr][col + 1], la, lb,
                                     ila, ilb);
          if (owns) {
            double s[NV];
            slope_j(rr, rp, rp2, col, s);
#pragma unroll
            for (int v = 0; v < NV; ++v) S.sy[v][ty + 1][tx] = s[v];
          }
        }
      }
      __syncthreads();

      // ---- phase B: face fluxes -----------------------------------------------------
      if (rowok) {
        if (has_face) {
          double F[NV], n[3];
          const double A = face_at(0, c + 1, j, n);
          bool ok;
          if constexpr (MX) {
            const float4 L = f4_fma(0.5f, S.sx32[ty][tx], S.r32[rr][col]);
            const float4 R = f4_fma(-0.5f, S.sx32[ty][tx + 1], S.r32[rr][col + 1]);
            ok = solve32(L, R, fnx0, fnx1, F);
          } else {
            double QL[NV], QR[NV];
            const double lm = half(ring_dlx(rr, col)), lp = half(ring_dlx(rr, col + 1));
            double bF = 1.0;
            if constexpr (SDV) {
              if (sd) bF = (c == -1) ? S.beta[ty][tx + 1] : S.beta[ty][tx];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const double sLv = sdl ? bF * S.sx[v][ty][tx] : S.sx[v][ty][tx];
              const double sRv = sdl ? bF * S.sx[v][ty][tx + 1] : S.sx[v][ty][tx + 1];
              QL[v] = S.ring[v][rr][col] + sLv * lm;
              QR[v] = S.ring[v][rr][col + 1] - sRv * lp;
            }
            ok = PH::template face<NV>(a.g, QL, QR, n, A, F, bF);
          }
          const bool lowb = (c == -1), highb = (c == ni - 1);
          int mask = ADD_ALL;
          if (!ok && !lowb && !highb) report(a.err, 4, b, c, j, 0);
          if (BC && (lowb || highb)) {
            const int w = a.bcw[d.bcoff[lowb ? 0 : 1] + j];
            if (bc_code(w) == BC_NONE) {
              for (int v = 0; v < NV; ++v) F[v] = 0.0;
              mask = ADD_NONE;
            } else if (bc_code(w) != BC_CONN) {
              double Q[NV], Qi[NV];
              const int cb = lowb ? col + 1 : col, ci = lowb ? col + 2 : col - 1;   // boundary / interior cell
              ringQ(rr, cb, Q);
              ringQ(rr, ci, Qi);
              mask = boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, ring_dlx(rr, cb), ring_dlx(rr, ci), n, A,
                                                 lowb ? 1 : 2, F);
              if constexpr (MX) per_area(F, mask, 1.0 / A);
            }
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) S.f[v][ty][tx] = F[v];
          if constexpr (BC) S.fm[ty][tx] = mask;
        }
        if (owns) {
          double G[NV], n[3];
          const double A = face_at(1, c, j + 1, n);
          bool ok;
          if constexpr (MX) {
            const float4 L = f4_fma(0.5f, S.sy32[ty][tx], S.r32[rr][col]);
            const float4 R = f4_fma(-0.5f, S.sy32[ty + 1][tx], S.r32[rp][col]);
            ok = solve32(L, R, fny0, fny1, G);
          } else {
            double QL[NV], QR[NV];
            const double lm = half(ring_dly(rr, col)), lp = half(ring_dly(rp, col));
            double bG = 1.0;
            if constexpr (SDV) {
              if (sd) bG = S.beta[ty][tx];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const double sLv = sdl ? bG * S.sy[v][ty][tx] : S.sy[v][ty][tx];
              const double sRv = sdl ? bG * S.sy[v][ty + 1][tx] : S.sy[v][ty + 1][tx];
              QL[v] = S.ring[v][rr][col] + sLv * lm;
              QR[v] = S.ring[v][rp][col] - sRv * lp;
            }
            ok = PH::template face<NV>(a.g, QL, QR, n, A, G, bG);
          }
          int mask = ADD_ALL;
          if (!ok && j < nj - 1) report(a.err, 4, b, c, j, 0);
          if (BC && j == nj - 1) {
            const int w = a.bcw[d.bcoff[3] + c];
            if (bc_code(w) == BC_NONE) {
              for (int v = 0; v < NV; ++v) G[v] = 0.0;
              mask = ADD_NONE;
            } else if (bc_code(w) != BC_CONN) {
              double Q[NV], Qi[NV];
              ringQ(rr, col, Q);
              ringQ(rm, col, Qi);
              mask = boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, ring_dly(rr, col), ring_dly(rm, col), n, A, 4, G);
              if constexpr (MX) per_area(G, mask, 1.0 / A);
            }
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) S.g[v][ty + 1][tx] = G[v];
          if constexpr (BC) S.gm[ty + 1][tx] = mask;
        }
      }
      cp_async_wait_prev();   // this thread's copies of this batch's PO
      __syncthreads();

      // ---- phase C: residual and update ---------------------------------------------
      if (rowok && owns) {
        double Rv[NV];
        if constexpr (MX) {
          // exact FP64 differences of the FP32 face fluxes, scaled by the areas
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const double dF = (double)S.f[v][ty][tx] - (double)S.f[v][ty][tx - 1];
            const double dG = (double)S.g[v][ty + 1][tx] - (double)S.g[v][ty][tx];
            Rv[v] = fma(u_Ax, dF, u_Ay * dG);
          }
        } else {
          ResAcc<NV, PH::kCompensated> R;
          R.init();
          const bool bi0 = (c == 0), bi1 = (c == ni - 1), bj0 = (j == 0), bj1 = (j == nj - 1);
          double Fm[NV], Fp[NV], Gm[NV], Gp[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            Fm[v] = S.f[v][ty][tx - 1];
            Fp[v] = S.f[v][ty][tx];
            Gm[v] = S.g[v][ty][tx];
            Gp[v] = S.g[v][ty + 1][tx];
          }
          if (!bi0) for (int v = 0; v < NV; ++v) R.add(v, -Fm[v]);
          if (!bi1) for (int v = 0; v < NV; ++v) R.add(v, Fp[v]);
          if (!bj0) for (int v = 0; v < NV; ++v) R.add(v, -Gm[v]);
          if (!bj1) for (int v = 0; v < NV; ++v) R.add(v, Gp[v]);
          // block-edge faces last, in face order (connections without BC)
          if constexpr (BC) {
            if (bi0) add_bc<NV>(R, Fm, -1.0, S.fm[ty][tx - 1]);
            if (bi1) add_bc<NV>(R, Fp, 1.0, S.fm[ty][tx]);
            if (bj0) add_bc<NV>(R, Gm, -1.0, S.gm[ty][tx]);
            if (bj1) add_bc<NV>(R, Gp, 1.0, S.gm[ty + 1][tx]);
          } else {
            if (bi0) add_bc<NV>(R, Fm, -1.0, ADD_ALL);
            if (bi1) add_bc<NV>(R, Fp, 1.0, ADD_ALL);
            if (bj0) add_bc<NV>(R, Gm, -1.0, ADD_ALL);
            if (bj1) add_bc<NV>(R, Gp, 1.0, ADD_ALL);
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) Rv[v] = R.get(v);
        }
        const long long o = off(c, j);
        if constexpr (MODE == 1) {
          double* Rb = a.R + d.sbase;
#pragma unroll
          for (int v = 0; v < NV; ++v) Rb[v * vs + o] = Rv[v];
        } else {
          double vol;
          if constexpr (UNI) vol = u_vol; else vol = a.m.vol[mb + o];
          const double dt = a.time_accurate ? *a.dtg : a.dtl[mb + o];
          double Q[NV], QO[NV];
          ringQ(rr, col, Q);
          const bool first = (a.irk == 1);
          if (!first) {
#pragma unroll
            for (int v = 0; v < NV; ++v) QO[v] = S.po[v][ty][tx - 1];
          }
          const bool ok = PH::template update<NV>(a.g, Q, QO, Rv, vol, dt, a.c_rk, first);
          if (!ok) report(a.err, 5, b, c, j, 0);
          double* Pn = a.Pn + d.sbase;
#pragma unroll
          for (int v = 0; v < NV; ++v) Pn[v * vs + o] = Q[v];
          if constexpr (MODE == 2) {   // Compute_dt of the next step on the new state
            double dtc;
            if constexpr (MX) dtc = cfl_dt32(a.g, Q, d, a.ndir, a.cfl);
            else dtc = cfl_dt<NV, UNI, PH::kFast>(a.g, Q, d, a.m, o, a.ndir, a.cfl);
            if (a.dt_local) a.dtl[mb + o] = dtc;
            dtrun = fmin(dtrun, dtc);
          }
        }
      }
      if (ty == SB_Y - 1 && owns) {   // carry the top row's j-slope
        if constexpr (MX) {
          S.sy32[0][tx] = S.sy32[SB_Y][tx];
        } else {
#pragma unroll
          for (int v = 0; v < NV; ++v) S.sy[v][0][tx] = S.sy[v][SB_Y][tx];
        }
      }
      cp_async_wait_all();   // this thread's copies of unit k+2
      if (k + 2 <= nbatch) convert_unit(k + 2);
    }
    __syncthreads();   // the next item refills the ring
  }
  if constexpr (MODE == 2) {   // CTA minimum, one atomic
    __shared__ double red[SB_T / 32];
    for (int s = 16; s > 0; s >>= 1) dtrun = fmin(dtrun, __shfl_xor_sync(0xffffffffu, dtrun, s));
    if ((t & 31) == 0) red[t >> 5] = dtrun;
    __syncthreads();
    if (t == 0) {
      double v = red[0];
      for (int w = 1; w < SB_T / 32; ++w) v = fmin(v, red[w]);
      atomicMin(a.dtmin, (unsigned long long)__double_as_longlong(v));
    }
  }
}

}  // namespace mose
