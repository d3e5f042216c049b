// kernels.h -- launchers of the device kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include "arena.cuh"
#include "metrics.cuh"

namespace mose {

void launch_cell_metrics(const BlockDesc* dblk, int b, long long ncell, NodeView nv, MetricArgs m, int nd,
                         int ndir, DevError* err, cudaStream_t s);
void launch_face_metrics(const BlockDesc* dblk, int b, long long nface, NodeView nv, MetricArgs m, int nd, int dir,
                         cudaStream_t s);
// mose_gpu_add_block's precomputed metrics (reference layout, see the header)
// over block b's metric planes; dims = (ni, nj, nk)
void launch_metrics_from_ref(const BlockDesc* dblk, int b, const int* dims, const double* src, MetricArgs m, int nd,
                             int ndir, cudaStream_t s);
void launch_ghost_metrics(const BlockDesc* dblk, const void* recs, int nrec, const NodeView* nodes, MetricArgs m,
                          int nd, int ndir, DevError* err, cudaStream_t s);
void launch_uniform_check(const BlockDesc* dblk, int b, long long ncell, MetricArgs m, int nd, int ndir, int* flags,
                          double* firsts, double tol, cudaStream_t s);
void launch_fill_ghosts(const BlockDesc* dblk, const GhostRec* recs, int nrec, double* P, MetricArgs m, int nd,
                        DevError* err, cudaStream_t s);
void launch_compute_dt(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, MetricArgs m,
                       double* dtl, unsigned long long* dtmin_bits, Gas g, double cfl, int ndir, int nd, int iter,
                       int ramp_iter, int store_local, bool uniform, cudaStream_t s, const int* iterp = nullptr);
void launch_set_global_dt(const BlockDesc* dblk, int nblk, long long maxcell, double* dtl, const double* dtg, int nd,
                          cudaStream_t s);
void launch_step_begin(unsigned long long* dtmin_bits, double dt_start, int* iter, cudaStream_t s);
void launch_step_dt_final(const unsigned long long* dtmin_bits, double* dtg, double* time, int advance_time,
                          cudaStream_t s);
void launch_step_dt_take(unsigned long long* dtmin_bits, double* dtg, double* time, int advance_time, double dt_start,
                         int* iter, cudaStream_t s);
// 402 inlets: p0 of every record from its time table at the device time
// (update, Series_Data_m.f90:55-86), written into its BcParam.
void launch_series_p0(const SeriesRec* recs, int n, const double* tv, const double* time, BcParam* bcp,
                      cudaStream_t s);
// The 3-D shock detector of every cell into the beta plane arena (from the
// stage input P, ghosts filled).
void launch_sd_beta3d(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, double* beta,
                      cudaStream_t s);
// Implicit residual smoothing on 2-D and 3-D blocks (nd), conservative or
// primitive integration.
void launch_irs_scale(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, double* R, MetricArgs m,
                      const double* dtl, const double* dtg, int use_dtg, Gas g, int nd, cudaStream_t s);
void launch_irs_ghost(const IrsCopy* list, int n, double* R, int nd, cudaStream_t s);
void launch_irs_jacobi(const BlockDesc* dblk, int nblk, long long maxcell, const double* R, const double* Rs,
                       double* out, int dir, double beta, int nd, cudaStream_t s);
void launch_irs_update(const BlockDesc* dblk, int nblk, long long maxcell, const double* Pin, const double* PO,
                       const double* R, double* Pout, Gas g, double c, DevError* err, int nd, cudaStream_t s);
void launch_rk_stage(const BlockDesc* dblk, int nblk, long long maxcell, double* P, const double* PO, const double* R,
                     MetricArgs m, const double* dtl, Gas g, double c, int nd, bool uniform, DevError* err,
                     cudaStream_t s);
// The same update from Pin into Pout, dt from *dtg when given, else dtl.
void launch_rk_stage_to(const BlockDesc* dblk, int nblk, long long maxcell, const double* Pin, const double* PO,
                        const double* R, MetricArgs m, const double* dtl, const double* dtg, double* Pout, Gas g,
                        double c, int nd, bool uniform, DevError* err, cudaStream_t s);
// Navier-Stokes residual of 2-D blocks (viscous2d.cu): a.Pc with filled
// ghosts -> a.R, every convective, diffusive and boundary term in the
// reference's order.  False for an unknown limiter.
// (two launches: the interior face fluxes into a.Fv, then each cell's residual)
bool launch_visc_residual2d(const StageArgs& a, int nblk, long long maxcell, int lim, cudaStream_t s);
// Discrete adjoint (2-D, HLLC; adjoint.cu).
void adj_pre(const BlockDesc* blk, int b, int ni, int nj, MetricArgs m, Gas g, const double* Ps, const double* Pprev,
             const double* Pn, const double* lam, const double* lamG, double* lamR, double* wdt, double* lam_loc,
             double* lam_n, double c, const double* dtg, cudaStream_t s);
void adj_faces(const BlockDesc* blk, int b, int ni, int nj, MetricArgs m, Gas g, int lim, const double* P,
               const double* lamR, double* Cx, double* Fx, double* Cy, double* Fy, cudaStream_t s);
void adj_bc(const StageArgs& a, int lim, const int4* list, int n, const double* lamR, double* Cb, double* Fbc,
            double* dmach, cudaStream_t s);
// Cb / Fbc: the boundary faces' stencil contributions and fluxes (k_adj_bc),
// added after the interior faces'; nullptr when the domain has none
void adj_gather(const BlockDesc* blk, int b, int ni, int nj, const double* Cx, const double* Cy, const double* Fx,
                const double* Fy, const double* Cb, const double* Fbc, const double* wdt, double* lamG,
                double* dtpart, cudaStream_t s);
void adj_ghost_transpose(const BlockDesc* blk, const GhostRec* recs, const int* ids, int n, MetricArgs m,
                         double* lamG, cudaStream_t s);
void adj_combine(const BlockDesc* blk, int b, int ni, int nj, const double* lam_loc, const double* lamG,
                 const double* lam_n, double* lam_out, cudaStream_t s);
void adj_sum(const double* x, long long n, double* out, int accumulate, double* scratch, cudaStream_t s);
// two sums in one launch pair, each in the same order as adj_sum's
void adj_sum2(const double* x0, long long n0, double* out0, int acc0, const double* x1, long long n1, double* out1,
              int acc1, double* scratch, cudaStream_t s);
int adj_sum_scratch();
void launch_dt_argmin(const BlockDesc* dblk, int b, int ni, int nj, MetricArgs m, Gas g, const double* P,
                      const double* dtg, double cfl, int ndir, bool uniform, unsigned long long* arg, cudaStream_t s);
void adj_dt(const BlockDesc* blk, MetricArgs m, Gas g, const double* P, const unsigned long long* arg,
            const double* lam_dt, double cfl, int ndir, double* lam_n, cudaStream_t s);
void adj_objective(const BlockDesc* blk, int b, int f, int n, MetricArgs m, const double* P, double* terms,
                   double* lam, cudaStream_t s);

int norms_partial_count(int nblk, long long maxcell);
void launch_residual_norms(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, const double* PO,
                           int nd, double* partial, double* out, cudaStream_t s);
void launch_ref_to_soa(const BlockDesc* dblk, int b, long long n, const double* ref, double* dst, int nv, int nd,
                       cudaStream_t s);
void launch_soa_to_ref(const BlockDesc* dblk, int b, long long n, const double* src, double* ref, int nv, int nd,
                       cudaStream_t s);
void launch_plane_io(const BlockDesc* dblk, int b, long long n, double* arena, double* ref, int nd, int to_ref,
                     cudaStream_t s);
void launch_metrics_to_ref(const BlockDesc* dblk, int b, long long n, MetricArgs m, double* vol, double* dl, int nd,
                           cudaStream_t s);
void launch_faces_to_ref(const BlockDesc* dblk, int b, long long n, MetricArgs m, int dir, double* N, double* A,
                         int nd, cudaStream_t s);

}  // namespace mose

namespace mose {
// Stage kernels: one launcher per (precision p, Riemann solver r) unit.
#define MOSE_STAGE_DECL(p, r) \
  bool launch_stage2d_p##p##_r##r(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s);
MOSE_STAGE_DECL(0, 0) MOSE_STAGE_DECL(0, 1) MOSE_STAGE_DECL(0, 2) MOSE_STAGE_DECL(0, 3) MOSE_STAGE_DECL(0, 4)
MOSE_STAGE_DECL(1, 0) MOSE_STAGE_DECL(1, 1) MOSE_STAGE_DECL(1, 2) MOSE_STAGE_DECL(1, 3) MOSE_STAGE_DECL(1, 4)
MOSE_STAGE_DECL(2, 0) MOSE_STAGE_DECL(2, 1) MOSE_STAGE_DECL(2, 2) MOSE_STAGE_DECL(2, 3) MOSE_STAGE_DECL(2, 4)
#undef MOSE_STAGE_DECL

// mode 0: fused residual + RK update; 1: residual only (exact precision);
// 2: fused, plus the next step's Compute_dt (last RK stage of a fused step).
// Solvers 4.. (HLLE, HLLEM, LLF, PLLF, Hanel, AUSM+-up, AUSM+-up2, HLLC+,
// HLLE++) share one unit per precision that selects the solver at run time
// (Gas::rie); with a shock detector (Gas::sd) every solver runs there.
// 2-D (and 1-D): every solver index (the compute-time units 0-3, the run-time
// unit for the rest) in every precision.  Setup refuses what this rejects,
// so a set-up context always has its stage kernel.
inline bool stage2d_supported(int rie, int prec) { return prec >= 0 && prec <= 2 && rie >= 0 && rie <= 14; }
inline bool launch_stage2d(const StageArgs& a, int nsm, int mode, bool uni, int prec, int rie, int lim,
                           cudaStream_t s) {
  using L = bool (*)(const StageArgs&, int, int, bool, int, cudaStream_t);
  static const L table[3][5] = {
      {launch_stage2d_p0_r0, launch_stage2d_p0_r1, launch_stage2d_p0_r2, launch_stage2d_p0_r3, launch_stage2d_p0_r4},
      {launch_stage2d_p1_r0, launch_stage2d_p1_r1, launch_stage2d_p1_r2, launch_stage2d_p1_r3, launch_stage2d_p1_r4},
      {launch_stage2d_p2_r0, launch_stage2d_p2_r1, launch_stage2d_p2_r2, launch_stage2d_p2_r3, launch_stage2d_p2_r4}};
  if (!stage2d_supported(rie, prec)) return false;
  // the shock detector lives in the run-time solver unit, which serves every solver
  return table[prec][(rie < 4 && a.g.sd == 0) ? rie : 4](a, nsm, mode, uni, lim, s);
}

// 3-D: the k-face march and the plane stage per RK stage; HLLC and AUSM+
// compiled in, every other solver, and every solver under the shock
// detector, through the run-time solver unit (r4); all six limiters.
#define MOSE_STAGE3_DECL(p, r) \
  bool launch_stage3d_p##p##_r##r(const StageArgs& a, int nsm, int mode, bool uni, int lim, cudaStream_t s);
MOSE_STAGE3_DECL(0, 0) MOSE_STAGE3_DECL(0, 1) MOSE_STAGE3_DECL(0, 4) MOSE_STAGE3_DECL(1, 0) MOSE_STAGE3_DECL(1, 1)
MOSE_STAGE3_DECL(1, 4) MOSE_STAGE3_DECL(2, 0) MOSE_STAGE3_DECL(2, 1) MOSE_STAGE3_DECL(2, 4)
#undef MOSE_STAGE3_DECL
inline bool stage3d_supported(int rie, int lim) { return rie >= 0 && rie <= 14 && lim >= 0 && lim <= 5; }
inline bool launch_stage3d(const StageArgs& a, int nsm, int mode, bool uni, int prec, int rie, int lim,
                           cudaStream_t s) {
  using L = bool (*)(const StageArgs&, int, int, bool, int, cudaStream_t);
  static const L table[3][3] = {{launch_stage3d_p0_r0, launch_stage3d_p0_r1, launch_stage3d_p0_r4},
                                {launch_stage3d_p1_r0, launch_stage3d_p1_r1, launch_stage3d_p1_r4},
                                {launch_stage3d_p2_r0, launch_stage3d_p2_r1, launch_stage3d_p2_r4}};
  if (prec < 0 || prec > 2 || !stage3d_supported(rie, lim)) return false;
  return table[prec][(rie <= 1 && a.g.sd == 0) ? rie : 2](a, nsm, mode, uni, lim, s);
}
}  // namespace mose
