// common.cuh -- device data model of the MOSE residual/update path on B200.
//
// HBM layout.  Every block owns, inside arenas shared by all blocks:
//   * the state: SoA planes of primitives (rho, u, v, [w,] p), one plane per
//     variable, each plane the block's cells plus two ghost layers in the
//     ACTIVE directions only (i, j in 2-D; i, j, k in 3-D).  Rows are padded to
//     a multiple of 16 doubles; block bases are 256-byte aligned.
//   * metric planes with the same indexing as one state plane: dl along each
//     direction, cell volume, face normal + area of the face on the low side
//     of each cell (face i-1/2 stored at cell i), and the CFL versors.
// In 2-D the reference carries w == 0 exactly (face normals have n_z == 0 on
// planar meshes and the k faces are null), so the device keeps 4 variables.
#pragma once

#include <cstdint>

namespace mose {

constexpr int GW = 2;  // ghost layers (Global_m.f90:17 gc = 2)

// Stage-kernel tiling: a CTA of SB_T threads is SB_X thread columns by SB_Y
// thread rows.  It owns a strip of at most SB_W = SB_X - 2 cell columns (one
// halo column each side) and marches up the strip SB_Y rows per batch.
constexpr int SB_X = 64;
constexpr int SB_Y = 4;
constexpr int SB_T = SB_X * SB_Y;
constexpr int SB_W = SB_X - 2;
// Fused 3-D stage tiling: a CTA of SB_T threads owns T3X x T3Y cells of a
// block's (i, j) plane and marches in k.
constexpr int T3X = 32;
constexpr int T3Y = SB_T / T3X;

// Internal boundary codes (reference bc.txt types in parentheses).
enum BcCode : int {
  BC_NONE = 0,      // (0)   null face: zero-gradient ghosts, no flux
  BC_CONN = 1,      // (101, 201) block connection / periodic
  BC_SYM = 2,       // (300) symmetry / slip wall
  BC_EXTRAP = 3,    // (400) extrapolation
  BC_SUPIN = 4,     // (405) supersonic inflow (M, T, p)
  BC_OUTFLOW = 5,   // (406) outflow with back pressure
  BC_STAGIN = 6,    // (401) inlet, total temperature and pressure
  BC_MFLUX_T0 = 7,  // (403) inlet, total temperature and mass flux
  BC_MFLUX_T = 8,   // (404) inlet, static temperature and mass flux
  BC_FARFIELD = 9,  // (407) ambient: total conditions in, back pressure out
  BC_WALL_Q = 10,   // (301) wall with prescribed heat flux (BcParam::p = qw)
  BC_WALL_T = 11,   // (302) wall at prescribed temperature (BcParam::T = Tw)
};

// Error word written by kernels (first offender wins).
struct DevError {
  int code;
  int b, i, j, k;   // 1-based, reference indexing
};

struct Gas {
  double gamma, R, cp, cv;
  double cpmR;      // 0.5*(cp+cp) - R, as roe_averages forms it
  // constants of the restated (fast) arithmetic, formed once on the host
  double gm1;       // gamma - 1
  double gcp;       // gamma / (gamma - 1)
  double igm1;      // 1 / (gamma - 1)
  // Riemann solver index (MOSE_RIEMANN_*) for the kernels that select the
  // solver at run time, and riemann-options-Minf of AUSM+-up / AUSM+-up2
  int rie;
  double minf;
  // shock detector (SD_Tramel): bit 0 scales the limited slopes (MUSCL-SD),
  // bit 1 feeds the SD Riemann solvers (HLLC+, HLLE++)
  int sd;
  // integration-variables = prim: the exact update advances the primitives
  // (Newstate_Primitive) instead of the conservatives
  int prim;
  // Navier-Stokes (model = 1, laminar): constant transport properties mu and
  // kappa (one species, constant-property tables) and the von Neumann number
  // of the viscous time-step limit
  int model;
  double mu, kappa, vnn;
};

// Source stencil of a viscous connection face cell (2-D, 0-based cells): the
// source block bs, the source cell (is, js) on its face fs, and the
// orientation d11 of the tangential direction (Fill_BC_Ghost_Connection).
struct VConn {
  int bs, is, js, fs, d11;
};

// Per-block descriptor (device resident).
struct BlockDesc {
  int ni, nj, nk;       // interior cells
  int px, py, pz;       // ghosted extents; px padded.  pz = 1 in 2-D.
  long long plane;      // px * py
  long long vstride;    // plane * pz: distance between SoA variable planes
  long long sbase;      // offset of this block in the state arenas (doubles)
  long long mbase;      // offset of this block in the one-plane arenas
  int bcoff[6];         // offset of face f's per-cell BC words in the BC table
  int bcn[6];           // number of face cells on face f
  // Uniform metrics (valid when the context runs the constant-metric kernels)
  double u_dl[3];
  double u_n[3][3];     // face normal per direction
  double u_A[3];        // face area per direction
  double u_vol;
  double u_vers[3][3];  // CFL versor per direction
  // 2-D connection edges read in place (StageArgs::remap): per face f = 1..4
  // (index f - 1) the source block (-1: the ghost layer is filled), and the
  // source cells of the ghost chunks: faces 1 / 2, column rm_at (of the
  // ghost chunk's first cell) and row j + rm_off; faces 3 / 4, column
  // i + rm_off and row rm_at + r (face 3, ghost rows r = -2, -1) or
  // rm_at + r - nj (face 4)
  int rm_src[4];
  int rm_at[4];
  int rm_off[4];
};

// Cell offset inside one plane of block d (i, j, k 0-based, ghosts negative).
__host__ __device__ inline long long cell_off2(const BlockDesc& d, int i, int j) {
  return (long long)(j + GW) * d.px + (i + GW);
}
__host__ __device__ inline long long cell_off3(const BlockDesc& d, int i, int j, int k) {
  return (long long)(k + GW) * d.plane + (long long)(j + GW) * d.px + (i + GW);
}

// BC word: low 8 bits = BcCode, high bits = parameter record index + 1.
__host__ __device__ inline int bc_code(int w) { return w & 0xff; }
__host__ __device__ inline int bc_param(int w) { return (w >> 8) - 1; }

// Parameters of a 401 / 403 / 404 / 405 / 406 / 407 face cell, precomputed
// on the host.  T: the static temperature (404, 405) or the total one (401,
// 403, 407); p: the static pressure (405), the total pressure (401, 407) or
// the mass flux g (403, 404); pback: the back pressure (406, 407).
struct BcParam {
  double mach, T, p, rel_fac;
  double ca, sa, cb, sb;   // cos/sin of the inflow angles (alpha, beta)
  double pback;
  // 401 / 403 / 404 / 407: the face's unit tangent t (a diagonal between two
  // of its nodes) and binormal b = n x t / |n x t|, and the ratios E1, E2 of
  // the t and b velocity components to the normal one that point the inflow
  // along (alpha, beta) (Lib_BC_Fluxes_Inflow.f90:113-129, 404-420)
  double tv[3], bv[3], E1, E2;
};

// One 402 face cell: its BcParam slot, and its time table's (time, value)
// pairs at tv[2 off ..], n pairs, periodic or not (time_series_type,
// Series_Data_m.f90:7-16).
struct SeriesRec {
  int pidx, off, n, periodic;
};

// One first-layer ghost value of the residual for implicit residual
// smoothing (Ghost_Residual_Extrapolation, Lib_IRS.f90:130-187): arena
// offsets of the ghost cell and of its source cell, and their blocks'
// variable strides.
struct IrsCopy {
  long long dst, src, vsd, vss;
};

// One ghost-fill record (Lib_Ghost.f90 dispatch), 0-based cells.
struct GhostRec {
  int type;                 // BcCode of the face
  int b, i, j, k, f;        // boundary cell and face (1..6)
  int bs, is, js, ks, fs;   // connection source
};

// One boundary record for the ghost-metric kernel (1-based reference indices).
struct GhostMetricRec {
  int type;
  int b, I, J, K, F;
  int bs, Is, Js, Ks, Fs, d11, d12, d21, d22;
};

}  // namespace mose
