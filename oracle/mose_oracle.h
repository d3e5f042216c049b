/*
 * mose_oracle.h -- C API of the CPU oracle for the MOSE explicit inviscid
 * residual-and-update path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against; it is also the CPU baseline that bench.py times.
 * Product code never links, loads or calls it.
 *
 * The oracle is a restatement, in plain C++ with the reference's own data
 * model (Fortran-ordered AoS arrays P(nprim, 1-gc:ni+gc, 1-gc:nj+gc,
 * 1-gc:nk+gc), a face-by-face boundary list in bc.txt order) and the same loop
 * and accumulation order as MOSE's Fortran sources.  Every routine cites the
 * reference file:line it follows.  Build with -ffp-contract=off and without
 * -ffast-math so that each Fortran expression rounds exactly once per
 * operation, left to right.
 */
#ifndef MOSE_ORACLE_H
#define MOSE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_domain orc_domain;

/* Limiters (Lib_Limiters.f90, bound in Mod_Space.f90:45-70). */
enum { ORC_LIM_FIRST_ORDER = 0, ORC_LIM_MINMOD = 1, ORC_LIM_VANLEER = 2,
       ORC_LIM_VANALBADA = 3, ORC_LIM_MC = 4, ORC_LIM_SUPERBEE = 5 };
/* Riemann solvers (Mod_Riemann.f90:43-112). */
enum { ORC_RIE_HLLC = 0, ORC_RIE_AUSMP = 1, ORC_RIE_SLAU = 2, ORC_RIE_SLAU2 = 3,
       ORC_RIE_HLLE = 4, ORC_RIE_HLLEM = 5, ORC_RIE_LLF = 6, ORC_RIE_PLLF = 7,
       ORC_RIE_HANEL = 8, ORC_RIE_AUSMP_UP = 9, ORC_RIE_AUSMP_UP2 = 10,
       ORC_RIE_HLLC_SD = 11, ORC_RIE_HLLE_PP = 12, ORC_RIE_HLLC_ROT = 13, ORC_RIE_EXACT = 14 };
/* Integration variables (Mod_Newstate.f90:30-44). */
enum { ORC_INT_CONS = 0, ORC_INT_PRIM = 1 };

typedef struct orc_config {
  int32_t n_rk;          /* time-scheme: euler=1, RK2=2, RK3=3 */
  double cfl;
  int32_t time_accurate;
  int32_t limiter;
  int32_t riemann;
  int32_t integration;
  int32_t ndir;          /* 0: derive from block 1 (Check_Mesh_Type) */
  double gamma;          /* calorically perfect single species */
  double rgas;
  int32_t ramp_iter;     /* cfl-rise-threshold */
  int32_t res_diter;     /* residual output interval */
  double minf;           /* riemann-options-Minf (AUSM+-up, AUSM+-up2) */
  double irs_beta;       /* irs-beta: implicit residual smoothing when > 0 */
  int32_t sd_limiter;    /* space-reconstruction MUSCL-SD: slopes scaled by the shock detector */
  int32_t model;         /* 0: Euler, 1: laminar Navier-Stokes (Global_m model) */
  double mu;             /* laminar viscosity (constant-property transport table) */
  double kappa;          /* laminar conductivity (constant-property transport table) */
  double vnn;            /* von Neumann number of the viscous time-step limit (Mod_dt.f90:98-103) */
} orc_config;

/* Error codes: mirror the reference's fatal `stop` sites. */
enum { ORC_OK = 0, ORC_ERR_INVALID = 1, ORC_ERR_UNSUPPORTED = 2,
       ORC_ERR_INTERFACE_STATE = 4, ORC_ERR_NAN_OR_NEG_P = 5,
       ORC_ERR_METRICS = 6 };

orc_domain* orc_create(const orc_config* cfg, int nthreads);
void orc_destroy(orc_domain* d);

/* Blocks are added in order b = 1..nb.  node: Fortran (3, 0:ni, 0:nj, 0:nk). */
int orc_add_block(orc_domain* d, int ni, int nj, int nk, const double* node);

/* Boundary list in bc.txt order (block, face 1..6, cell).  rec: nbound x 15
 * int32 (b,i,j,k,f,type,bs,is,js,ks,fs,d11,d12,d21,d22), 1-based.
 * data: nbound x 6 doubles (mach, T, p, alpha, beta, rel_fac) for 405 and
 * (p_back, rel_fac, 0, 0, 0, 0) for 406; may be NULL. */
int orc_set_bcs(orc_domain* d, const int32_t* rec, const double* data, int nbound);
/* Time table of a 402 inlet (time_series_type, Series_Data_m.f90): n pairs
 * (time, value), values already in the units of p0; returns the table's
 * index (>= 0), which a 402 record carries as its second datum, or < 0. */
int orc_add_series(orc_domain* d, const double* time, const double* value, int n, int periodic);
/* update(time) of table id (Series_Data_m.f90:55-86), for tests. */
double orc_series_eval(const orc_domain* d, int id, double time);

/* Setup_Metrics (Mod_Metrics.f90:8-107): interior + ghost metrics. */
int orc_setup_metrics(orc_domain* d);

/* Prim arrays in the reference layout P(5, 1-gc:ni+gc, 1-gc:nj+gc, 1-gc:nk+gc). */
int orc_set_prim(orc_domain* d, int b, const double* P);
int orc_get_prim(const orc_domain* d, int b, double* P);
int orc_set_prim_old(orc_domain* d, int b, const double* PO);
int orc_get_residual(const orc_domain* d, int b, double* R);
int orc_get_dtlocal(const orc_domain* d, int b, double* dt);
int orc_set_dtlocal(orc_domain* d, int b, const double* dt);

/* Metrics access for tests.  vol/dl/M over ghosted cells (Fortran order);
 * faces for direction dir (1..3) over the reference's dir(d)%f bounds. */
int orc_get_metrics(const orc_domain* d, int b, double* vol, double* dl, double* M);
int orc_get_faces(const orc_domain* d, int b, int dir, double* N, double* A);
int orc_set_metrics(orc_domain* d, int b, const double* vol, const double* dl, const double* M);
int orc_set_faces(orc_domain* d, int b, int dir, const double* N, const double* A);

/* The phases of Explicit_Step (Mod_Explicit.f90:40-85). */
int orc_fill_ghost_cell(orc_domain* d);
int orc_fluxes(orc_domain* d);
int orc_bc_fluxes(orc_domain* d);
int orc_rk_newstate(orc_domain* d, int irk);
int orc_copy_state(orc_domain* d);
int orc_compute_dt(orc_domain* d, double* dtglobal);
int orc_set_global_dt(orc_domain* d);
/* One full Explicit_Step; returns dtglobal and time. */
int orc_explicit_step(orc_domain* d, double* dtglobal, double* time);
/* Compute_Residual summed over blocks (Mod_Diagnostic.f90:13-50). */
int orc_compute_residual(const orc_domain* d, double* total);

void orc_set_time(orc_domain* d, double time, int iter);
/* domain%dtglobal: the starting value of Compute_dt's minimum, and the value
 * Set_Global_dt spreads. */
void orc_set_dtglobal(orc_domain* d, double dtglobal);
double orc_get_time(const orc_domain* d);
int orc_last_error(const orc_domain* d, int* b, int* i, int* j, int* k);

/* Scalar kernels exposed for known-answer tests. */
double orc_limiter(int limiter, double x, double y);
void orc_riemann(const orc_domain* d, const double* left, const double* right,
                 const double* normal, double* flux);

#ifdef __cplusplus
}
#endif
#endif
