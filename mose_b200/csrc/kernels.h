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
void launch_ghost_metrics(const BlockDesc* dblk, const void* recs, int nrec, const NodeView* nodes, MetricArgs m,
                          int nd, int ndir, DevError* err, cudaStream_t s);
void launch_uniform_check(const BlockDesc* dblk, int b, long long ncell, MetricArgs m, int nd, int ndir, int* flags,
                          double* firsts, cudaStream_t s);
void launch_fill_ghosts(const BlockDesc* dblk, const GhostRec* recs, int nrec, double* P, MetricArgs m, int nd,
                        cudaStream_t s);
void launch_compute_dt(const BlockDesc* dblk, int nblk, long long maxcell, const double* P, MetricArgs m,
                       double* dtl, unsigned long long* dtmin_bits, Gas g, double cfl, int ndir, int nd, int iter,
                       int ramp_iter, int store_local, bool uniform, cudaStream_t s);
void launch_set_global_dt(const BlockDesc* dblk, int nblk, long long maxcell, double* dtl, const double* dtg, int nd,
                          cudaStream_t s);
void launch_step_begin(unsigned long long* dtmin_bits, double dt_start, int* iter, cudaStream_t s);
void launch_step_dt_final(const unsigned long long* dtmin_bits, double* dtg, double* time, int advance_time,
                          cudaStream_t s);
void launch_rk_stage(const BlockDesc* dblk, int nblk, long long maxcell, double* P, const double* PO, const double* R,
                     MetricArgs m, const double* dtl, Gas g, double c, int nd, bool uniform, DevError* err,
                     cudaStream_t s);
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
bool launch_stage2d_exact_r0(const StageArgs& a, int grid, int mode, bool uni, int lim, cudaStream_t s);
bool launch_stage2d_exact_r1(const StageArgs& a, int grid, int mode, bool uni, int lim, cudaStream_t s);
bool launch_stage2d_exact_r2(const StageArgs& a, int grid, int mode, bool uni, int lim, cudaStream_t s);
bool launch_stage2d_exact_r3(const StageArgs& a, int grid, int mode, bool uni, int lim, cudaStream_t s);
inline bool launch_stage2d_exact(const StageArgs& a, int grid, int mode, bool uni, int rie, int lim, cudaStream_t s) {
  switch (rie) {
    case 0: return launch_stage2d_exact_r0(a, grid, mode, uni, lim, s);
    case 1: return launch_stage2d_exact_r1(a, grid, mode, uni, lim, s);
    case 2: return launch_stage2d_exact_r2(a, grid, mode, uni, lim, s);
    case 3: return launch_stage2d_exact_r3(a, grid, mode, uni, lim, s);
  }
  return false;
}
}  // namespace mose
