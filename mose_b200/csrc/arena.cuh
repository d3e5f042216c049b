// arena.cuh -- argument bundles shared by the host driver and the kernels.
#pragma once

#include "common.cuh"

namespace mose {

// Metric arenas (general-metric kernels).  Every plane has the indexing of a
// state plane of its block (offset BlockDesc::mbase * planes).
struct MetricArgs {
  const double* dl;     // 3 planes per block: dl along i, j, k (ghosted along that direction)
  const double* face;   // 12 planes per block: for dir d: nx, ny, nz, A of the low face of each cell
  const double* vol;    // 1 plane
  const double* vers;   // 9 planes: versor of direction d, component q at plane 3 d + q
  // Navier-Stokes only (null otherwise): 4 planes of the 2-D metric tensor
  // M(r, s) = d xi_r / d x_s, r, s = 1, 2, at plane (r - 1) + 2 (s - 1); held
  // for the interior cells and the first ghost layer
  const double* Mt;
};

struct StageArgs {
  const BlockDesc* blk;
  const int4* items;    // (block, first column, first row, last row + 1): items touching a boundary face
  int nitems;
  const int4* items_nb; // items whose block-edge faces are all connections
  int nitems_nb;
  const double* Pc;     // current state arena
  const double* Po;     // state at the start of the step (Copy_State's PO)
  double* Pn;           // next state (fused mode)
  double* R;            // residual arena (residual-only mode)
  double* Hk;           // 3-D: interior k-face flux H(k + 1/2) at cell (i, j, k), a state-shaped arena
  const double* beta;   // 3-D shock detector of every cell (one plane per block), or null
  double* Fv;           // Navier-Stokes: interior face fluxes, 14 planes per block (null otherwise)
  // 2-D: the stage kernels read the ghost cells of remapped connection edges
  // (BlockDesc::rm_*) from their source cells, so their ghost fill is not needed
  int remap;
  MetricArgs m;
  double* dtl;          // local dt plane arena (one plane per block), or null
  const double* dtg;    // device scalar dtglobal (time-accurate)
  const int* bcw;       // boundary words, see bc_code()
  const BcParam* bcp;
  double c_rk;          // RKcoeff(n_rk, irk)
  int irk;
  int time_accurate;
  DevError* err;
  Gas g;
  // Fused Compute_dt of the NEXT step (last RK stage only, else dtmin = null):
  // the CFL dt of every updated cell folds into *dtmin (bit pattern of a
  // positive double); with dt_local each cell's dt is also stored in dtl.
  unsigned long long* dtmin;
  double cfl;
  int ndir;
  int dt_local;
  // 3-D work list in [0]: (block, i0 | j0 << 16, k0, k1) tiles marching k
  const int4* items3[3];
  int nitems3[3];
  // persistent 2-D grid: at most this many CTAs per SM (0: the occupancy limit)
  int grid_cap;
  // Navier-Stokes connection faces: per 101 / 201 face cell the source stencil
  // of its viscous flux (VConn), indexed by the boundary word's parameter
  const int* vconn;
};

}  // namespace mose
