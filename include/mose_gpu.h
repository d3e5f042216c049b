/*
 * mose_gpu.h -- C ABI of the B200 (sm_100a) implementation of MOSE's explicit
 * inviscid residual-and-update path on multi-block structured grids.
 *
 * Plain C types only (ints, doubles, pointers and sizes), so MOSE's Fortran
 * drivers bind it with ISO_C_BINDING (see mose_b200/fortran/mose_gpu_m.f90)
 * and Python binds it with ctypes.  Every entry point returns a status code
 * (MOSE_OK = 0) except the getters noted; mose_gpu_last_error() returns the
 * message of the last failure.
 *
 * Each entry point names the reference routine it replaces (paths relative
 * to the MOSE source tree, src/lib/...).
 *
 * Array layouts crossing this boundary are the reference's own:
 *   node  : Fortran real(8) node(3, 0:ni, 0:nj, 0:nk)
 *   P, R  : Fortran real(8) P(nprim, 1-gc:ni+gc, 1-gc:nj+gc, 1-gc:nk+gc),
 *           nprim = 5 (rho, u, v, w, p), gc = 2
 *   bc    : one record per boundary face cell in bc.txt order (block, face
 *           1..6, cell): int32 b,i,j,k,f,type,bs,is,js,ks,fs,d11,d12,d21,d22
 *           (1-based), plus 6 doubles of type data
 *           401: T0, p0, alpha, beta, rel_fac ; 402: T0, time-table id
 *           (mose_gpu_add_series), alpha, beta, rel_fac ; 403: T0, g, alpha, beta,
 *           rel_fac ; 404: T, g, alpha, beta, rel_fac ; 405: mach, T, p,
 *           alpha, beta, rel_fac ; 406: p_back, rel_fac ; 407: T0, p0,
 *           p_back, alpha, beta, rel_fac (g: mass flux per unit area; the
 *           largest double as alpha or beta is the token 'normal', which
 *           407 does not take; on 2-D domains beta is 0 or 'normal') ;
 *           301: qw ; 302: Tw (walls, see mose_gpu_set_viscous)
 *
 * State is device resident between calls: host P is stale until
 * mose_gpu_download_prim().  A context is not thread safe and owns one
 * CUDA stream.  On 2-D domains (nk = 1) the transfers of P and R read and
 * write only the k = 1 plane of the reference array: the reference never
 * reads its k ghost planes on this path, and w is zero there (the
 * 401 / 403 / 404 inlets leave rounding-level w in the reference: their
 * face velocity sums three vectors whose z parts cancel only to rounding).
 */
#ifndef MOSE_GPU_H
#define MOSE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MOSE_GPU_ABI_VERSION 2

/* Status codes.  The nonzero codes mirror the reference's fatal `stop`s. */
enum {
  MOSE_OK = 0,
  MOSE_ERR_INVALID = 1,            /* bad argument or call order */
  MOSE_ERR_UNSUPPORTED = 2,        /* BC type / solver / geometry not on this path */
  MOSE_ERR_CUDA = 3,               /* CUDA runtime failure, or no sm_100 device */
  MOSE_ERR_INTERFACE_STATE = 4,    /* Lib_Convective.f90:45-50 non-physical interface */
  MOSE_ERR_NAN_OR_NEG_P = 5,       /* Lib_Newstate.f90:334-338 NaN or p < 0 */
  MOSE_ERR_METRICS = 6,            /* Lib_Metrics.f90:286,353 det = 0 or volume <= 0 */
  MOSE_ERR_TIMEOUT = 7,            /* a bounded device wait gave up */
  MOSE_ERR_NOT_READY = 8           /* setup incomplete */
};

/* flux-limiter (Mod_Space.f90:45-70) */
enum {
  MOSE_LIMITER_FIRST_ORDER = 0,
  MOSE_LIMITER_MINMOD = 1,
  MOSE_LIMITER_VANLEER = 2,
  MOSE_LIMITER_VANALBADA = 3,
  MOSE_LIMITER_MC = 4,
  MOSE_LIMITER_SUPERBEE = 5
};

/* riemann-solver (Mod_Riemann.f90:43-112) */
enum {
  MOSE_RIEMANN_HLLC = 0,
  MOSE_RIEMANN_AUSMP = 1,
  MOSE_RIEMANN_SLAU = 2,
  MOSE_RIEMANN_SLAU2 = 3,
  MOSE_RIEMANN_HLLE = 4,       /* 'HLLE'  (Lib_Riemann_HLL.f90:259-317) */
  MOSE_RIEMANN_HLLEM = 5,      /* 'HLLEM' (Lib_Riemann_HLL.f90:23-146) */
  MOSE_RIEMANN_LLF = 6,        /* 'LLF', 'Rusanov' (Lib_Riemann_LF.f90:10-45) */
  MOSE_RIEMANN_PLLF = 7,       /* 'PLLF'  (Lib_Riemann_LF.f90:48-102) */
  MOSE_RIEMANN_HANEL = 8,      /* 'Hanel' (Lib_Riemann_AUSM.f90:48-117) */
  MOSE_RIEMANN_AUSMP_UP = 9,   /* 'AUSM+-up'  (Lib_Riemann_AUSM.f90:273-418), needs Minf */
  MOSE_RIEMANN_AUSMP_UP2 = 10, /* 'AUSM+-up2' (Lib_Riemann_AUSM.f90:455-570), needs Minf */
  MOSE_RIEMANN_HLLC_SD = 11,   /* 'HLLC+'  (Lib_Riemann_HLL.f90:500-534), shock detector */
  MOSE_RIEMANN_HLLE_PP = 12,   /* 'HLLE++' (Lib_Riemann_HLL.f90:320-464), shock detector */
  MOSE_RIEMANN_HLLC_ROT = 13,  /* 'HLLC Rotated' (Lib_Riemann_HLL.f90:672-755) */
  MOSE_RIEMANN_EXACT = 14      /* 'exact' (Lib_Riemann_Godunov.f90:10-224) */
};

/* Arithmetic of the face fluxes and of the fused steps' CFL pass.  In the
 * fused step (mose_gpu_step / mose_gpu_advance) the last RK stage also forms
 * the next step's Compute_dt on the state it writes; the first fused step
 * after any call that changes the state runs the standalone (reference
 * arithmetic) pass instead. */
enum {
  MOSE_PRECISION_FP64_EXACT = 0,   /* the reference's FP64 operation order, no FMA contraction */
  MOSE_PRECISION_FP64 = 1,         /* FP64, FMA-contracted and reciprocal-folded */
  MOSE_PRECISION_MIXED = 2         /* FP32 reconstruction + Riemann, FP64 state/accumulation */
};

/* integration-variables (Mod_Newstate.f90:30-44): 'cons' (Newstate_Conservative)
 * or 'prim' (Newstate_Primitive, Lib_Newstate.f90:168-317; the reference-exact
 * and fp64 precisions, mose_gpu_create refuses it with the mixed one) */
enum { MOSE_INTEGRATION_CONS = 0, MOSE_INTEGRATION_PRIM = 1 };

typedef struct mose_gpu_config {
  int32_t abi_version;     /* MOSE_GPU_ABI_VERSION */
  int32_t n_rk;            /* time-scheme: 1 = euler, 2 = RK2, 3 = RK3 */
  double cfl;              /* cfl */
  int32_t time_accurate;   /* time-accurate */
  int32_t ramp_iter;       /* cfl-rise-threshold */
  int32_t limiter;         /* MOSE_LIMITER_* */
  int32_t riemann;         /* MOSE_RIEMANN_* */
  int32_t integration;     /* MOSE_INTEGRATION_CONS or _PRIM */
  int32_t precision;       /* MOSE_PRECISION_* */
  int32_t ndir;            /* 0: derived from block 1 as Check_Mesh_Type does */
  int32_t nsc;             /* number of species; must be 1 */
  double gamma;            /* ratio of specific heats (calorically perfect gas) */
  double rgas;             /* gas constant */
  int32_t device;          /* CUDA device ordinal */
  int32_t res_diter;       /* res-diter: residual-norm interval of mose_gpu_step */
} mose_gpu_config;

typedef struct mose_gpu_ctx mose_gpu_ctx;

/* Fills cfg with the reference defaults (Register_Numerics.f90:30-72). */
void mose_gpu_default_config(mose_gpu_config* cfg);

/* Context.  Replaces the numerics state bound by Assign_Setup
 * (config/Assign_Setup.f90:41-56). */
int mose_gpu_create(const mose_gpu_config* cfg, mose_gpu_ctx** out);
void mose_gpu_destroy(mose_gpu_ctx* ctx);
const char* mose_gpu_last_error(const mose_gpu_ctx* ctx);
/* Offending (b,i,j,k) of the last device-detected failure (1-based). */
int mose_gpu_error_location(const mose_gpu_ctx* ctx, int32_t* b, int32_t* i, int32_t* j, int32_t* k);

/* Geometry and boundaries.  Blocks are added in order b = 1..nb.
 * node: block_type%node(0:ni, 0:nj, 0:nk)%c(3) in its Fortran memory order
 * (Advanced_Types_m.f90:16).  The device forms the metrics from the nodes at
 * setup, bit for bit as Setup_Metrics does (Mod_Metrics.f90:8-107).
 * metrics (optional, NULL: formed from the nodes) hands in the block's own
 * Setup_Metrics output instead: the block_type arrays allocated by
 * Allocate_Block (driver/Mod_Allocate_Data.f90:105-110), one after another,
 * each in its Fortran memory order, ghost layers included (gc = 2 in every
 * direction; NG = (ni+4)(nj+4)(nk+4)):
 *   vol(1-gc:ni+gc, 1-gc:nj+gc, 1-gc:nk+gc)       NG doubles
 *   dl(...)%c(3)                                  3 NG
 *   M(...)%c(3,3)                                 9 NG
 *   dir(1)%f(0:ni, nj, nk)%(N(3), A)              4 (ni+1) nj nk
 *   dir(2)%f(ni, 0:nj, nk)%(N(3), A)              4 ni (nj+1) nk
 *   dir(3)%f(ni, nj, 0:nk)%(N(3), A)              4 ni nj (nk+1)
 * The device takes vol, dl and the CFL versors M(d,:)/norm2(M(d,:)) of the
 * interior cells (and M(1:2,1:2) for the viscous terms), dl along each
 * boundary's normal in the ghost layers (and M in the first layer), and every
 * face's N and A; the nodes still give the inlet tangents.  The array is
 * copied before the call returns. */
int mose_gpu_add_block(mose_gpu_ctx* ctx, int32_t b, int32_t ni, int32_t nj, int32_t nk,
                       const double* node, const double* metrics);
/* Replaces Read_BCfile (io/IO_BC.f90:136-414) with the parsed records. */
int mose_gpu_set_bcs(mose_gpu_ctx* ctx, const int32_t* rec, const double* data, int32_t nbound);
/* The p0 time table of 402 inlets, replacing time_series_type::initialize
 * (base/Series_Data_m.f90:20-52): n (time, value) pairs, value in the units
 * of p0 (the file's bar times 1e5), periodic or not.  Call before
 * mose_gpu_setup; *id (0, 1, ...) is what a 402 record holds as its second
 * datum in place of the reference's file name.  At every step the device
 * evaluates update(time) (Series_Data_m.f90:55-86) at the step's time. */
int mose_gpu_add_series(mose_gpu_ctx* ctx, const double* time, const double* value, int32_t n, int32_t periodic,
                        int32_t* id);
/* Setup_Metrics (numerics/space/Mod_Metrics.f90:8-107) on the device, then the
 * device tables.  Must follow add_block and set_bcs. */
int mose_gpu_setup(mose_gpu_ctx* ctx);

/* State transfer, reference layout (see above). */
int mose_gpu_upload_prim(mose_gpu_ctx* ctx, int32_t b, const double* P);
int mose_gpu_download_prim(mose_gpu_ctx* ctx, int32_t b, double* P);
int mose_gpu_upload_prim_old(mose_gpu_ctx* ctx, int32_t b, const double* PO);
int mose_gpu_download_residual(mose_gpu_ctx* ctx, int32_t b, double* R);
int mose_gpu_upload_residual(mose_gpu_ctx* ctx, int32_t b, const double* R);
/* dtlocal(1:ni,1:nj,1:nk) */
int mose_gpu_download_dt(mose_gpu_ctx* ctx, int32_t b, double* dt);
int mose_gpu_upload_dt(mose_gpu_ctx* ctx, int32_t b, const double* dt);

/* The phases of Explicit_Step (numerics/time/explicit/Mod_Explicit.f90:40-85). */
/* Compute_dt (numerics/time/Mod_dt.f90:10-106): local dt and global minimum.
 * Starts the minimum from *dtglobal on entry (the reference passes 1d5). */
int mose_gpu_compute_dt(mose_gpu_ctx* ctx, double cfl, int32_t iter, int32_t ramp_iter,
                        double* dtglobal);
/* Set_Global_dt (Mod_dt.f90:110-130). */
int mose_gpu_set_global_dt(mose_gpu_ctx* ctx, double dtglobal);
/* Copy_State (Mod_Explicit.f90:149-170): PO = P. */
int mose_gpu_copy_state(mose_gpu_ctx* ctx);
/* Fill_Ghost_Cell (numerics/space/Lib_Ghost.f90:11-137). */
int mose_gpu_fill_ghosts(mose_gpu_ctx* ctx);
/* Fluxes (numerics/fluxes/Mod_Fluxes.f90:10-209) followed by BC_Fluxes
 * (numerics/fluxes/bc/Mod_BC_Fluxes.f90:10-218): R on the device.  In the
 * reference-exact arithmetic, or in the fp64 precision's when the context
 * computes in it (the mixed precision's phases run the exact arithmetic). */
int mose_gpu_residual(mose_gpu_ctx* ctx);
/* RK_Newstate => Newstate_Conservative (numerics/time/explicit/Lib_Newstate.f90:13-160). */
int mose_gpu_rk_stage(mose_gpu_ctx* ctx, int32_t irk);
/* One whole Explicit_Step (Mod_Explicit.f90:10-113): dt, PO = P, then n_rk
 * fused stages (ghost fill + residual + update in one kernel per stage).
 * Returns dtglobal and the updated time. */
int mose_gpu_step(mose_gpu_ctx* ctx, double* dtglobal, double* time);
/* nsteps Explicit_Steps enqueued back to back with dt kept on the device (no
 * host round trip between steps; replayed from a CUDA graph).  Synchronises
 * once at the end and returns the last dtglobal and time. */
int mose_gpu_advance(mose_gpu_ctx* ctx, int32_t nsteps, double* dtglobal, double* time);
/* Compute_Residual (diagnostic/Mod_Diagnostic.f90:13-50): sums over all
 * blocks of (|d rho|, |du|, |dv|, |dw|, |dp|)^2 between P and PO; total[5]. */
int mose_gpu_residual_norms(mose_gpu_ctx* ctx, double* total);

/* Compute_Residual on caller-owned device arrays, allocating nothing.
 * No counterpart in the reference: it exists for callers that keep P and PO
 * in their own device memory (the reference layout of one block) and cannot
 * let a library call cudaMalloc, because their device memory belongs to
 * another allocator or to a budget fixed at start-up.
 *   P, PO : device pointers, P(5, 1-gc:ni+gc, 1-gc:nj+gc, 1-gc:nk+gc)
 *   total : device pointer to 5 doubles; total += sums of squares of
 *           (|d rho|, |du|, |dv|, |dw|, |dp|) over the interior cells, like
 *           the reference's `total = total + residuo` across blocks
 *   stream: a cudaStream_t (NULL: the legacy default stream)
 * Scratch: a fixed device array of MOSE_NOALLOC_MAX_CHUNKS x 5 doubles
 * (160 KB, held by every GPU that loads the library until exit); a block
 * may hold at most MOSE_NOALLOC_MAX_CHUNKS * MOSE_NOALLOC_CHUNK_CELLS
 * (268,435,456) cells, larger blocks return MOSE_ERR_INVALID with a message
 * in mose_gpu_noalloc_last_error().  The first call on a device looks up the
 * array's address (cudaGetSymbolAddress) with that device current, so make
 * the first call before any stream capture.  Every call shares the array:
 * calls that overlap on the GPU (other streams, other threads) race.  Calls
 * on one stream are ordered and each overwrites what it reads. */
#define MOSE_NOALLOC_MAX_CHUNKS 4096
#define MOSE_NOALLOC_CHUNK_CELLS 65536
int mose_gpu_residual_norms_noalloc(const double* P, const double* PO, int32_t ni, int32_t nj, int32_t nk,
                                    double* total, void* stream);
const char* mose_gpu_noalloc_last_error(void);

int mose_gpu_set_time(mose_gpu_ctx* ctx, double time, int32_t iter);
int mose_gpu_get_time(mose_gpu_ctx* ctx, double* time, int32_t* iter);
/* Waits for the context's stream and reports any device-detected failure. */
int mose_gpu_synchronize(mose_gpu_ctx* ctx);

/* Introspection for tests and the benchmark. */
/* The context's cudaStream_t (as void*), for events or work ordered with it. */
void* mose_gpu_stream(const mose_gpu_ctx* ctx);
/* Runs nsteps fused Explicit_Steps without graph replay, with CUDA events
 * between kernels, and returns the summed device time in ms per kernel class:
 * ms[0] dt pass + step bookkeeping, ms[1] ghost fill, ms[2] stage kernels;
 * launches[c] counts the launches of each class.  Advances the solution. */
int mose_gpu_time_kernels(mose_gpu_ctx* ctx, int32_t nsteps, double* ms, int32_t* launches);
/* 1 when every metric of every block is uniform and the constant-metric
 * kernels are used: bitwise uniform for the exact and fp64 precisions, within
 * 1e-9 relative of each block's first cell for the mixed precision. */
int mose_gpu_uniform_metrics(const mose_gpu_ctx* ctx);
/* Number of kernel launches this context issued since creation. */
int64_t mose_gpu_launch_count(const mose_gpu_ctx* ctx);
/* Device metrics of block b in the reference layout: vol(ghosted cells),
 * dl(3, ghosted cells) along each direction's ghosted line, and face N(3), A
 * over dir(d)%f bounds (see the reference's Mod_Allocate_Data.f90:103-108).
 * Entries the device does not hold are left untouched. */
int mose_gpu_download_metrics(mose_gpu_ctx* ctx, int32_t b, double* vol, double* dl);
int mose_gpu_download_faces(mose_gpu_ctx* ctx, int32_t b, int32_t dir, double* N, double* A);

/* Self-check of the restated FP64 reciprocal, reciprocal square root and
 * square root of the "fp64" and "mixed" precisions over n seeded inputs
 * spread over [2^-60, 2^60) on the current device.  out[0..2]: the largest
 * relative error of 1/x, 1/sqrt(x), sqrt(x) in units of 2^-53 (half an ulp
 * at the top of a binade), measured through exact FMA residuals; out[3]: the
 * largest distance in ulps between the restated sqrt(x) and the correctly
 * rounded one.  No context needed; synchronous. */
int mose_gpu_check_fast_math(int64_t n, uint64_t seed, double* out);

/* ---- Discrete adjoint (2-D, HLLC with minmod / van Leer / van Albada,
 * time-accurate SSP-RK).  The objective is the pressure integral over one
 * block face, J = sum over the face cells of p * A (the wall-pressure
 * convention of Lib_BC_Fluxes.f90:48-72).  The adjoint differentiates the
 * whole Explicit_Step: every RK stage, the boundary fluxes (405 also in the
 * inflow Mach), the ghost fill and the global CFL dt (through its argmin
 * cell). */
/* space-reconstruction = MUSCL-SD (Mod_Space.f90:26-31): the limited slopes of
 * every face scaled by the Tramel shock detector (Lib_Shock_Detector.f90,
 * Lib_Reconstruction.f90:24-25).  The detector also feeds HLLC+ and HLLE++.
 * Call before mose_gpu_setup; 2-D blocks of at least 3 x 3 cells, or 3-D
 * blocks of any size. */
int mose_gpu_set_sd_limiter(mose_gpu_ctx* ctx, int32_t on);

/* irs-beta (Register_Numerics.f90): implicit residual smoothing of every RK
 * stage's residual when beta > 0 (Lib_IRS.f90, Newstate_Conservative's IRS
 * branch Lib_Newstate.f90:40-72); 0 (the default) disables it.  Call before
 * mose_gpu_setup.  2-D and 3-D, exact or fp64 precision: the stage's
 * residual-only kernel in that precision, then the smoothing kernels and the
 * update in the reference's arithmetic. */
int mose_gpu_set_irs_beta(mose_gpu_ctx* ctx, double beta);

/* equations = navier-stokes (Global_m model): model 1 adds the laminar
 * diffusive fluxes of Lib_Diffusive.f90 (Diffusive_Flux, Compute_Diffusive_Flux,
 * called from Mod_Fluxes.f90:101-206 when model > 0), their boundary terms
 * (BC_Connection_Visc for 101 / 201, BC_Symmetry_Visc for 300, BC_Wall_Heat
 * for 301 with qw as the record's first datum, BC_Wall_Temperature for 302
 * with Tw) and the VNN time-step limit (Mod_dt.f90:87-103); model 0 (the
 * default) is the Euler path.  mu and kappa are the laminar viscosity and
 * conductivity (one species, constant-property transport tables, for which
 * FLINT's table interpolation and Wilke mixing return the constants), vnn the
 * von Neumann number.  Call before mose_gpu_setup.  2-D domains, exact
 * precision, conservative integration, no IRS or shock detector; without
 * model 1, 301 and 302 faces are symmetry walls, as in the reference. */
int mose_gpu_set_viscous(mose_gpu_ctx* ctx, int32_t model, double mu, double kappa, double vnn);

/* riemann-options-Minf (Register_Numerics.f90:72), the reference Mach number
 * of AUSM+-up and AUSM+-up2; call before mose_gpu_setup.  Setup rejects
 * those two solvers while it is 0, as Assign_Setup.f90:96-100 does (2-D
 * and 3-D). */
int mose_gpu_set_riemann_minf(mose_gpu_ctx* ctx, double minf);

/* Tiling of the 2-D work list that the persistent stage kernels walk (no
 * counterpart in the reference, whose OpenMP loops have no work list):
 * tiling[0] rows per item (0: the planner's load-balance model), [1] largest
 * strip width in cells (8..62), [2] item order (0: a block's row bands in
 * turn, neighbouring strips side by side; 1: its strips in turn), [3] CTAs
 * per SM of the persistent grid (0: the occupancy limit).  Results do not
 * depend on the tiling: every face flux and cell update is the same
 * arithmetic whichever CTA does it. */
int mose_gpu_set_tiling(mose_gpu_ctx* ctx, const int32_t tiling[4]);
int mose_gpu_get_tiling(const mose_gpu_ctx* ctx, int32_t tiling[4]);
/* Autotuner (no counterpart in the reference): times candidate tilings on
 * the context's own domain, `steps` full steps each from the current state
 * (restored afterwards), keeps the fastest and returns it with its time per
 * step and the default's.  Call after the state is uploaded; 2-D only. */
int mose_gpu_autotune(mose_gpu_ctx* ctx, int32_t steps, int32_t tiling_out[4], double* best_ms_per_step,
                      double* default_ms_per_step);

/* Sets the Mach number of every 405 supersonic-inflow face. */
int mose_gpu_set_inflow_mach(mose_gpu_ctx* ctx, double mach);
/* Runs nsteps fused steps from the current state keeping a checkpoint of the
 * state every `interval` steps (sqrt(nsteps) is the usual choice), and
 * returns J on face `face` (1..4) of block `block` of the final state. */
int mose_gpu_adjoint_forward(mose_gpu_ctx* ctx, int32_t nsteps, int32_t interval, int32_t block, int32_t face,
                             double* J);
/* Reverse sweep of the preceding mose_gpu_adjoint_forward: each checkpoint
 * segment is recomputed (recording its stage inputs) and differentiated
 * back.  Leaves dJ/dP of the initial state in the context's adjoint state
 * (mose_gpu_download_adjoint) and returns dJ/dMach; the state stays the
 * forward run's final state.  The first call with a given interval captures
 * the segment's CUDA graphs on the context's stream (call it outside any
 * stream capture); later calls replay them.  Device memory: 3 * interval + 1
 * state arenas for the segment plus ceil(nsteps / interval) checkpoints. */
int mose_gpu_adjoint_backward(mose_gpu_ctx* ctx, double* dJ_dmach);
/* One step of the adjoint at the current state P^n: the adjoint state goes
 * from lambda^{n+1} (uploaded) to lambda^n = (dP^{n+1}/dP^n)^T lambda^{n+1};
 * *dJ_dmach = lambda^{n+1} . dP^{n+1}/dMach.  The state stays P^n. */
int mose_gpu_adjoint_step(mose_gpu_ctx* ctx, double* dJ_dmach);
/* The adjoint state of block b in the reference layout of P (w entries 0). */
int mose_gpu_upload_adjoint(mose_gpu_ctx* ctx, int32_t b, const double* lam);
int mose_gpu_download_adjoint(mose_gpu_ctx* ctx, int32_t b, double* lam);

#ifdef __cplusplus
}
#endif
#endif /* MOSE_GPU_H */
