// mose_gpu.cu -- host side of the C ABI declared in include/mose_gpu.h.
//
// One context = one CUDA stream, the device arenas of all blocks, the
// boundary tables and the step graphs.  Setup (metrics, tables) runs on the
// device; after it every entry point only enqueues kernels, except those that
// return values to the host.
#include <cuda_runtime.h>

#include "nvtx.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iterator>
#include <string>
#include <vector>

#include "../../include/mose_gpu.h"
#include "kernels.h"

using namespace mose;

namespace {

struct HostBlock {
  int ni, nj, nk;
  std::vector<double> node;
  std::vector<double> metrics;   // precomputed Setup_Metrics output (reference layout), or empty
};

// Doubles of mose_gpu_add_block's precomputed metrics: vol, dl%c(3), M%c(3,3)
// over the ghosted cells, then the (N(3), A) of the i-, j- and k-faces.
size_t ref_metrics_size(int ni, int nj, int nk) {
  const size_t NG = (size_t)(ni + 4) * (nj + 4) * (nk + 4);
  return 13 * NG + 4 * ((size_t)(ni + 1) * nj * nk + (size_t)ni * (nj + 1) * nk + (size_t)ni * nj * (nk + 1));
}

struct BcRecord {
  int b, i, j, k, f, type, bs, is, js, ks, fs, d11, d12, d21, d22;
  double data[6];
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  ~DevBuf() { release(); }
  // Zero-filled allocation.  The context's stream does not synchronise with
  // the legacy default stream that cudaMemset uses, so wait for the fill
  // before any work on the context's stream can touch the buffer.
  cudaError_t alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e == cudaSuccess) e = cudaMemset(p, 0, count * sizeof(T));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Splits n into parts of nearly equal size, each a multiple of q except the
// last; returns the part boundaries (parts + 1 values).
std::vector<int> split_even(int n, int parts, int q) {
  const int units = (n + q - 1) / q;
  std::vector<int> cut(parts + 1, 0);
  for (int p = 0; p < parts; ++p) {
    const int u = units / parts + (p < units % parts ? 1 : 0);
    cut[p + 1] = std::min(n, cut[p] + u * q);
  }
  cut[parts] = n;
  return cut;
}

// Work items of the 2-D stage kernel: (block, c0 | c1 << 16, j0, j1).
// Every block's columns split into ceil(ni / wmax) strips (wmax <= SB_W) of
// nearly equal width starting on even columns (16-byte aligned row copies);
// its rows into runs of about H rows in whole batches.  order 0 lists a
// block's items row band by row band (neighbouring strips of one band run
// side by side and share their halo columns in L2), order 1 strip by strip.
// H = 0 takes the candidate whose round-robin assignment over the
// persistent grid has the smallest makespan, an item costing its batches
// plus about two for the prologue and the first copies.
std::vector<int4> plan_stage_items(const std::vector<HostBlock>& blocks, int grid, int Hset = 0, int wmax = SB_W,
                                   int order = 0) {
  auto build = [&](int H) {
    std::vector<int4> items;
    for (int b = 0; b < (int)blocks.size(); ++b) {
      const HostBlock& h = blocks[b];
      const int ns = (h.ni + wmax - 1) / wmax;
      const std::vector<int> cc = split_even(h.ni, ns, 2);
      const int nr = std::max(1, (h.nj + H / 2) / H);
      const std::vector<int> rc = split_even(h.nj, std::min(nr, (h.nj + SB_Y - 1) / SB_Y), SB_Y);
      const int nrr = (int)rc.size() - 1;
      for (int o = 0; o < nrr * ns; ++o) {
        const int r = order == 0 ? o / ns : o % nrr, s = order == 0 ? o % ns : o / nrr;
        if (rc[r + 1] > rc[r] && cc[s + 1] > cc[s])
          items.push_back(make_int4(b, cc[s] | (cc[s + 1] << 16), rc[r], rc[r + 1]));
      }
    }
    return items;
  };
  if (Hset > 0) return build(Hset);
  auto makespan = [&](const std::vector<int4>& items) {
    std::vector<long long> load(std::max(1, grid), 0);
    for (size_t i = 0; i < items.size(); ++i)
      load[i % load.size()] += (items[i].w - items[i].z + SB_Y - 1) / SB_Y + 2;
    return *std::max_element(load.begin(), load.end());
  };
  std::vector<int4> best;
  long long best_t = -1;
  for (int H = 16; H <= 512; H += SB_Y) {
    std::vector<int4> items = build(H);
    const long long tm = makespan(items);
    if (best_t < 0 || tm < best_t || (tm == best_t && items.size() < best.size())) {
      best_t = tm;
      best.swap(items);
    }
  }
  return best;
}

// The k-run length of the 3-D work items on a persistent grid of `slots`
// CTAs: the runs of at most L planes that minimise the grid's time, modelled
// as its waves (items over slots, rounded up) times the longest run plus 1.5
// planes of per-item setup (the first plane's copy, the march's extra
// slope).  Ties go to the longer runs.
int choose_k_run(const std::vector<HostBlock>& blocks, int slots) {
  int nkmax = 1;
  for (const HostBlock& h : blocks) nkmax = std::max(nkmax, h.nk);
  int best = nkmax;
  double bcost = 1e300;
  for (int L = nkmax; L >= std::min(4, nkmax); --L) {
    long long n = 0;
    int lmax = 0;
    for (const HostBlock& h : blocks) {
      const int runs = (h.nk + L - 1) / L;
      n += (long long)((h.ni + T3X - 1) / T3X) * ((h.nj + T3Y - 1) / T3Y) * runs;
      lmax = std::max(lmax, (h.nk + runs - 1) / runs);
    }
    const double cost = (double)((n + slots - 1) / slots) * (lmax + 1.5);
    if (cost < bcost - 1e-9) {
      bcost = cost;
      best = L;
    }
  }
  return best;
}

// Work items of the 3-D stage: (block, i0 | j0 << 16, k0, k1), tiles of T3X
// x T3Y cells of the block's (i, j) plane marching k over runs of at most
// run_s planes for the plane stage and run_k planes for the k-face march
// (their grids differ in CTAs per SM).  out[0]: the plane-stage tiles whose
// block-edge faces (the faces 1..6 their cells touch) are all connections;
// out[1]: the other plane-stage tiles; out[2]: the k-face march's tiles.
void plan_3d_items(const std::vector<HostBlock>& blocks, const std::vector<BlockDesc>& desc,
                   const std::vector<int>& bcw, int run_s, int run_k, std::vector<int4> out[3]) {
  for (int q = 0; q < 3; ++q) out[q].clear();
  for (int pass = 0; pass < 2; ++pass) {
    const int L = pass == 0 ? run_s : run_k;
    for (int b = 0; b < (int)blocks.size(); ++b) {
      const HostBlock& h = blocks[b];
      const BlockDesc& d = desc[b];
      const std::vector<int> kc = split_even(h.nk, (h.nk + L - 1) / L, 1);
      for (size_t r = 0; r + 1 < kc.size(); ++r)
        for (int j0 = 0; j0 < h.nj; j0 += T3Y)
          for (int i0 = 0; i0 < h.ni; i0 += T3X) {
            const int k0 = kc[r], k1 = kc[r + 1];
            if (k1 <= k0) continue;
            const int4 it = make_int4(b, i0 | (j0 << 16), k0, k1);
            if (pass == 1) {
              out[2].push_back(it);
              continue;
            }
            const int i1 = std::min(i0 + T3X, h.ni), j1 = std::min(j0 + T3Y, h.nj);
            bool conn = true;
            // face f (1..6) over the index ranges [a0, a1) x [b0, b1) of its
            // words (word index a + na * b)
            auto check = [&](int f, int a0, int a1, int na, int b0, int b1) {
              for (int y = b0; y < b1 && conn; ++y)
                for (int x = a0; x < a1 && conn; ++x) conn = bc_code(bcw[d.bcoff[f - 1] + x + na * y]) == BC_CONN;
            };
            if (i0 == 0) check(1, j0, j1, h.nj, k0, k1);
            if (i1 == h.ni) check(2, j0, j1, h.nj, k0, k1);
            if (j0 == 0) check(3, i0, i1, h.ni, k0, k1);
            if (j1 == h.nj) check(4, i0, i1, h.ni, k0, k1);
            if (k0 == 0) check(5, i0, i1, h.ni, j0, j1);
            if (k1 == h.nk) check(6, i0, i1, h.ni, j0, j1);
            out[conn ? 0 : 1].push_back(it);
          }
    }
  }
}

}  // namespace

struct mose_gpu_ctx {
  mose_gpu_config cfg;
  Gas gas;
  std::string err;
  int devcode = 0, eb = 0, ei = 0, ej = 0, ek = 0;
  // the first failed enqueue that returns no status of its own (a copy
  // inside a step's sequence), reported by the next check_launch
  cudaError_t enq_err = cudaSuccess;
  const char* enq_what = "";
  cudaStream_t stream = nullptr;
  int nsm = 148;
  bool ready = false;
  int ndir = 0, nd = 2, nv = 4;
  bool uniform = false;
  long long launches = 0;

  std::vector<HostBlock> hblk;
  std::vector<BcRecord> bc;
  std::vector<BlockDesc> desc;
  long long marena = 0;      // doubles per one-plane arena
  long long maxcell = 0;

  DevBuf<BlockDesc> d_desc;
  DevBuf<double> state[3];
  DevBuf<double> resid;
  DevBuf<double> hk;          // 3-D: the k-face flux arena of the stage kernels
  DevBuf<double> sdbeta;      // 3-D with the shock detector: beta of every cell (one plane per block)
  DevBuf<double> dl, face, vol, vers, dtl;
  DevBuf<double> Mt;          // Navier-Stokes: 2-D metric tensor planes (null otherwise)
  DevBuf<int> vconn;          // Navier-Stokes: VConn stencils of the connection face cells
  DevBuf<double> vface;       // Navier-Stokes: the interior face fluxes of the residual (14 planes)
  DevBuf<int> bcw;
  DevBuf<BcParam> bcp;
  DevBuf<GhostRec> ghosts;
  // the fill split by kind: connection records as flat (ghost, source) cell
  // copies, one per ghost layer (all of them / those of edges not read in
  // place), and every other record for the record kernel
  DevBuf<IrsCopy> gcopy, gcopy_nc;
  int ngcopy = 0, ngcopy_nc = 0;
  DevBuf<GhostRec> ghosts_other;
  int nghost_other = 0;
  bool remap = false;           // some 2-D connection edge is read in place
  DevBuf<int4> items;
  // implicit residual smoothing (irs-beta > 0): first-layer ghost records of
  // R and two work arenas for the Jacobi sweeps
  double irs_beta = 0.0;
  DevBuf<IrsCopy> irs_list;
  int nirs = 0;
  DevBuf<double> rs1, rs2;
  DevBuf<int4> items_nb;      // 2-D items with no physical boundary face
  int nitems_nb = 0;
  // 2-D work-list tiling (mose_gpu_set_tiling / mose_gpu_autotune): rows per
  // item (0: the planner's model), largest strip width, item order, CTAs per
  // SM (0: the occupancy limit); and the boundary words the planner reads
  int tile_h = 0, tile_w = SB_W, tile_order = 0, tile_ctas = 0;
  std::vector<int> hbcw;
  DevBuf<int4> items3[3];     // 3-D tiles: connection-only, with a physical boundary face, all
  int nitems3[3] = {0, 0, 0};
  DevBuf<double> scal;        // [0] dtglobal, [1] time
  DevBuf<unsigned long long> dtmin;
  DevBuf<int> iterdev;
  DevBuf<DevError> derr;
  DevBuf<double> partial, norms;
  DevBuf<double> staging;     // reference-layout transfers
  int nghost = 0, nitems = 0;
  int cur = 0, po = 0;        // state arena holding P, and PO

  // step graphs per starting arena, [1] with the standalone dt pass forced
  // (the adjoint's forward in a non-exact precision, below)
  cudaGraphExec_t graph[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int graph_kernels[2] = {0, 0};
  // The adjoint's forward and recompute in the fp64 / mixed precisions take
  // every step's dt from the standalone (reference-arithmetic) pass instead
  // of the fused one, so the dt argmin of the reverse sweep finds the cell
  // that set it.
  bool adj_dt_standalone = false;

  // dtmin holds the CFL minimum of state[cur], folded in by the last RK stage
  // of the previous fused step; cleared by every call that changes the state
  bool dt_valid = false;

  double h_time = 0.0;
  int h_iter = 0;

  // ---- discrete adjoint (adjoint.cu) ----
  std::vector<GhostRec> hghost;          // ghost-fill records (host copy)
  bool adj_init = false;
  int adj_nsteps = 0, adj_interval = 0, adj_block = 0, adj_face = 0;
  std::vector<DevBuf<double>> adj_ckpt;  // P^n at steps 0, K, 2K, ...
  // the states of one segment as a chain: adj_seg[3 k + s] is the input of
  // RK stage s + 1 of step k (ghosts filled in place), adj_seg[3 (k + 1)]
  // the state after step k
  std::vector<DevBuf<double>> adj_seg;
  DevBuf<double> adj_dts;                // dt of each step of the segment
  // graphs of a segment's recompute (full segments) and of each reverse step
  // k, valid for the segment length adj_graph_K; the side stream runs the
  // boundary faces and the dt argmin beside the interior faces
  cudaGraphExec_t adj_recgraph = nullptr;
  std::vector<cudaGraphExec_t> adj_rgraph;
  int adj_graph_K = 0, adj_rec_kernels = 0, adj_rev_kernels = 0;
  cudaStream_t adj_aux = nullptr;
  cudaEvent_t adj_fork = nullptr, adj_join = nullptr;
  // 2-D stages with both item lists: the boundary items' launch runs on
  // stage_aux beside the boundary-free items' launch
  cudaStream_t stage_aux = nullptr;
  cudaEvent_t stage_fork = nullptr, stage_join = nullptr;
  DevBuf<double> lam, lam_loc, lam_n, lamR, wdt, lamG, Cx, Cy, Fx, Fy, dtpart, adj_scal, Cb, Fbc, dmach, objt;
  DevBuf<unsigned long long> adj_arg;
  DevBuf<double> adj_sumscr;             // partial sums of the deterministic reductions
  DevBuf<int4> adj_bclist;               // boundary face cells of faces 1..4, grouped by face
  int adj_bcfirst[5] = {0, 0, 0, 0, 0};  // face f's entries: [adj_bcfirst[f-1], adj_bcfirst[f])
  DevBuf<int> adj_gids;                  // ghost records grouped by face
  int adj_gfirst[5] = {0, 0, 0, 0, 0};
  // launches of the ghost transpose: runs of consecutive faces whose records
  // touch disjoint cells, as record ranges
  std::vector<int> adj_gpass;
  bool adj_recorded = false;
  std::vector<BcParam> hbcp;             // 401 / 402 / 403 - 407 parameters (host copy)
  // 402 time tables: (time, value) pairs of every table, and per table its
  // first pair, pair count and periodic flag; per 402 record its SeriesRec
  std::vector<double> hser;
  struct SerIdx { int off, n, periodic; };
  std::vector<SerIdx> hser_idx;
  DevBuf<double> ser_tv;
  DevBuf<SeriesRec> ser_recs;
  int nser = 0;

  MetricArgs margs() const { return MetricArgs{dl.p, face.p, vol.p, vers.p, Mt.p}; }
};

namespace {

int fail(mose_gpu_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CU(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(ctx, MOSE_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                 \
  } while (0)

int check_launch(mose_gpu_ctx* ctx, const char* what) {
  if (ctx->enq_err != cudaSuccess) {
    const cudaError_t q = ctx->enq_err;
    ctx->enq_err = cudaSuccess;
    cudaGetLastError();
    return fail(ctx, MOSE_ERR_CUDA, "%s: %s: %s", what, ctx->enq_what, cudaGetErrorString(q));
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return MOSE_OK;
}

// Reads the device error word; returns a status.
int poll_device_error(mose_gpu_ctx* ctx) {
  DevError h;
  CU(cudaMemcpyAsync(&h, ctx->derr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  if (h.code != 0) {
    ctx->devcode = h.code; ctx->eb = h.b; ctx->ei = h.i; ctx->ej = h.j; ctx->ek = h.k;
    const char* what = h.code == MOSE_ERR_INTERFACE_STATE ? "non-physical interface state"
                       : h.code == MOSE_ERR_NAN_OR_NEG_P   ? "NaN or p<0 after the state update"
                       : h.code == MOSE_ERR_METRICS        ? "metric tensor det=0 or non-positive volume"
                                                           : "device failure";
    return fail(ctx, h.code, "%s at b,i,j,k = %d %d %d %d", what, h.b, h.i, h.j, h.k);
  }
  return MOSE_OK;
}

int bc_code_of(int type) {
  switch (type) {
    case 0: return BC_NONE;
    case 101: case 201: return BC_CONN;
    case 300: return BC_SYM;
    case 400: return BC_EXTRAP;
    case 401: case 402: return BC_STAGIN;   // 402: p0 from its time table, refreshed every step
    case 403: return BC_MFLUX_T0;
    case 404: return BC_MFLUX_T;
    case 405: return BC_SUPIN;
    case 406: return BC_OUTFLOW;
    case 407: return BC_FARFIELD;
    case 301: return BC_WALL_Q;   // walls: the symmetry flux, plus the viscous wall flux with model = 1
    case 302: return BC_WALL_T;
  }
  return -1;
}

// index of a boundary cell along its face (0-based), 2-D and 3-D
int face_index(const HostBlock& h, int f, int i, int j, int k) {
  if (f <= 2) return j + h.nj * k;
  if (f <= 4) return i + h.ni * k;
  return i + h.ni * j;
}

void destroy_adjoint_graphs(mose_gpu_ctx* ctx) {
  if (ctx->adj_recgraph) cudaGraphExecDestroy(ctx->adj_recgraph);
  ctx->adj_recgraph = nullptr;
  for (auto& g : ctx->adj_rgraph)
    if (g) cudaGraphExecDestroy(g);
  ctx->adj_rgraph.clear();
  ctx->adj_graph_K = 0;
}

void destroy_graphs(mose_gpu_ctx* ctx) {
  for (auto& gs : ctx->graph)
    for (auto& g : gs)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  destroy_adjoint_graphs(ctx);
}

}  // namespace

extern "C" {

void mose_gpu_default_config(mose_gpu_config* cfg) {
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->abi_version = MOSE_GPU_ABI_VERSION;
  cfg->n_rk = 1;            // time-scheme = euler
  cfg->cfl = 0.5;
  cfg->time_accurate = 0;
  cfg->ramp_iter = 0;
  cfg->limiter = MOSE_LIMITER_FIRST_ORDER;
  cfg->riemann = MOSE_RIEMANN_HLLC;
  cfg->integration = MOSE_INTEGRATION_CONS;
  cfg->precision = MOSE_PRECISION_FP64_EXACT;
  cfg->ndir = 0;
  cfg->nsc = 1;
  cfg->gamma = 1.4;
  cfg->rgas = 1.0;
  cfg->device = 0;
  cfg->res_diter = 1;
}

int mose_gpu_create(const mose_gpu_config* cfg, mose_gpu_ctx** out) {
  MOSE_NVTX_RANGE("mose_gpu_create");
  mose_gpu_ctx* ctx = nullptr;
  if (!cfg || !out) return MOSE_ERR_INVALID;
  *out = nullptr;
  if (cfg->abi_version != MOSE_GPU_ABI_VERSION) return MOSE_ERR_INVALID;
  // integration-variables = prim runs in the reference-exact and fp64
  // precisions (the mixed precision's FP32 face states are not kept with it)
  if (cfg->integration == MOSE_INTEGRATION_PRIM && cfg->precision == MOSE_PRECISION_MIXED)
    return MOSE_ERR_UNSUPPORTED;
  if (cfg->n_rk < 1 || cfg->n_rk > 3 || cfg->nsc != 1 ||
      (cfg->integration != MOSE_INTEGRATION_CONS && cfg->integration != MOSE_INTEGRATION_PRIM) ||
      cfg->limiter < 0 || cfg->limiter > 5 || cfg->riemann < 0 || cfg->riemann > MOSE_RIEMANN_EXACT ||
      cfg->precision < 0 || cfg->precision > 2 || !(cfg->gamma > 1.0) || !(cfg->rgas > 0.0))
    return MOSE_ERR_UNSUPPORTED;
  ctx = new mose_gpu_ctx();
  ctx->cfg = *cfg;
  if (ctx->cfg.res_diter <= 0) ctx->cfg.res_diter = 1;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device) {
    delete ctx;
    return MOSE_ERR_CUDA;
  }
  cudaDeviceProp prop;
  if (cudaSetDevice(cfg->device) != cudaSuccess || cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess ||
      prop.major != 10) {
    delete ctx;
    return MOSE_ERR_CUDA;   // built for sm_100a only
  }
  ctx->nsm = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stage_aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->stage_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->stage_join, cudaEventDisableTiming) != cudaSuccess) {
    mose_gpu_destroy(ctx);
    return MOSE_ERR_CUDA;
  }
  // thermodynamic constants of the restated FLINT closure
  ctx->gas.gamma = cfg->gamma;
  ctx->gas.R = cfg->rgas;
  ctx->gas.cp = cfg->gamma * cfg->rgas / (cfg->gamma - 1.0);
  ctx->gas.cv = cfg->rgas / (cfg->gamma - 1.0);
  ctx->gas.cpmR = 0.5 * (ctx->gas.cp + ctx->gas.cp) - ctx->gas.R;
  ctx->gas.gm1 = cfg->gamma - 1.0;
  ctx->gas.gcp = cfg->gamma / (cfg->gamma - 1.0);
  ctx->gas.igm1 = 1.0 / (cfg->gamma - 1.0);
  ctx->gas.rie = cfg->riemann;
  ctx->gas.minf = 0.0;
  ctx->gas.sd = (cfg->riemann == MOSE_RIEMANN_HLLC_SD || cfg->riemann == MOSE_RIEMANN_HLLE_PP) ? 2 : 0;
  ctx->gas.prim = cfg->integration == MOSE_INTEGRATION_PRIM ? 1 : 0;
  ctx->gas.model = 0;   // Euler until mose_gpu_set_viscous
  ctx->gas.mu = ctx->gas.kappa = 0.0;
  ctx->gas.vnn = 0.5;
  *out = ctx;
  return MOSE_OK;
}

void mose_gpu_destroy(mose_gpu_ctx* ctx) {
  MOSE_NVTX_RANGE("mose_gpu_destroy");
  if (!ctx) return;
  cudaSetDevice(ctx->cfg.device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->adj_aux) cudaStreamSynchronize(ctx->adj_aux);
  if (ctx->stage_aux) cudaStreamSynchronize(ctx->stage_aux);
  destroy_graphs(ctx);
  if (ctx->adj_fork) cudaEventDestroy(ctx->adj_fork);
  if (ctx->adj_join) cudaEventDestroy(ctx->adj_join);
  if (ctx->adj_aux) cudaStreamDestroy(ctx->adj_aux);
  if (ctx->stage_fork) cudaEventDestroy(ctx->stage_fork);
  if (ctx->stage_join) cudaEventDestroy(ctx->stage_join);
  if (ctx->stage_aux) cudaStreamDestroy(ctx->stage_aux);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* mose_gpu_last_error(const mose_gpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int mose_gpu_error_location(const mose_gpu_ctx* ctx, int32_t* b, int32_t* i, int32_t* j, int32_t* k) {
  if (!ctx) return MOSE_ERR_INVALID;
  if (b) *b = ctx->eb;
  if (i) *i = ctx->ei;
  if (j) *j = ctx->ej;
  if (k) *k = ctx->ek;
  return ctx->devcode;
}

int mose_gpu_add_block(mose_gpu_ctx* ctx, int32_t b, int32_t ni, int32_t nj, int32_t nk, const double* node,
                       const double* metrics) {
  MOSE_NVTX_RANGE("mose_gpu_add_block");
  if (!ctx || !node) return MOSE_ERR_INVALID;
  if (ctx->ready) return fail(ctx, MOSE_ERR_INVALID, "add_block after setup");
  if (b != (int)ctx->hblk.size() + 1) return fail(ctx, MOSE_ERR_INVALID, "blocks must be added in order 1..nb");
  if (ni < 1 || nj < 1 || nk < 1) return fail(ctx, MOSE_ERR_INVALID, "bad block dimensions");
  HostBlock h;
  h.ni = ni; h.nj = nj; h.nk = nk;
  size_t n = 3 * (size_t)(ni + 1) * (nj + 1) * (nk + 1);
  h.node.assign(node, node + n);
  if (metrics) h.metrics.assign(metrics, metrics + ref_metrics_size(ni, nj, nk));
  ctx->hblk.push_back(std::move(h));
  return MOSE_OK;
}

int mose_gpu_add_series(mose_gpu_ctx* ctx, const double* time, const double* value, int32_t n, int32_t periodic,
                        int32_t* id) {
  MOSE_NVTX_RANGE("mose_gpu_add_series");
  if (!ctx || !time || !value || !id || n < 1) return MOSE_ERR_INVALID;
  if (ctx->ready) return fail(ctx, MOSE_ERR_INVALID, "add_series after setup");
  mose_gpu_ctx::SerIdx si{(int)(ctx->hser.size() / 2), n, periodic ? 1 : 0};
  for (int q = 0; q < n; ++q) {
    ctx->hser.push_back(time[q]);
    ctx->hser.push_back(value[q]);
  }
  ctx->hser_idx.push_back(si);
  *id = (int32_t)ctx->hser_idx.size() - 1;
  return MOSE_OK;
}

int mose_gpu_set_bcs(mose_gpu_ctx* ctx, const int32_t* rec, const double* data, int32_t nbound) {
  MOSE_NVTX_RANGE("mose_gpu_set_bcs");
  if (!ctx || !rec) return MOSE_ERR_INVALID;
  if (ctx->ready) return fail(ctx, MOSE_ERR_INVALID, "set_bcs after setup");
  int nb = (int)ctx->hblk.size();
  long long expect = 0;
  for (auto& h : ctx->hblk) expect += 2LL * ((long long)h.nj * h.nk + (long long)h.ni * h.nk + (long long)h.ni * h.nj);
  if (nbound != expect)
    return fail(ctx, MOSE_ERR_INVALID, "boundary records (%d) differ from the block faces (%lld)", nbound, expect);
  // Null (type 0) records of the k faces of single-plane blocks are kept out
  // of the list: such faces are never active (a 3-D domain needs nk > 1 in
  // every block) and a 2-D domain has ni * nj of them per face.
  ctx->bc.clear();
  ctx->bc.reserve(std::min<long long>(nbound, 1LL << 20));
  int lastkey = -1;
  for (int q = 0; q < nbound; ++q) {
    const int32_t* r = rec + 15 * (size_t)q;
    BcRecord e;
    e.b = r[0]; e.i = r[1]; e.j = r[2]; e.k = r[3]; e.f = r[4]; e.type = r[5];
    e.bs = r[6]; e.is = r[7]; e.js = r[8]; e.ks = r[9]; e.fs = r[10];
    e.d11 = r[11]; e.d12 = r[12]; e.d21 = r[13]; e.d22 = r[14];
    for (int c = 0; c < 6; ++c) e.data[c] = data ? data[6 * (size_t)q + c] : 0.0;
    if (e.b < 1 || e.b > nb || e.f < 1 || e.f > 6) return fail(ctx, MOSE_ERR_INVALID, "bad record %d", q + 1);
    const HostBlock& h = ctx->hblk[e.b - 1];
    if (e.i < 1 || e.i > h.ni || e.j < 1 || e.j > h.nj || e.k < 1 || e.k > h.nk)
      return fail(ctx, MOSE_ERR_INVALID, "record %d: cell out of range", q + 1);
    int key = (e.b - 1) * 6 + (e.f - 1);
    if (key < lastkey) return fail(ctx, MOSE_ERR_INVALID, "records must be ordered by block and face");
    lastkey = key;
    if (bc_code_of(e.type) < 0)
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "record %d: bc type %d is not on this path", q + 1, e.type);
    if (e.type == 101 || e.type == 201) {
      if (e.bs < 1 || e.bs > nb || e.fs < 1 || e.fs > 6)
        return fail(ctx, MOSE_ERR_INVALID, "record %d: bad connection", q + 1);
      const HostBlock& s = ctx->hblk[e.bs - 1];
      if (e.is < 1 || e.is > s.ni || e.js < 1 || e.js > s.nj || e.ks < 1 || e.ks > s.nk)
        return fail(ctx, MOSE_ERR_INVALID, "record %d: connection source out of range", q + 1);
    }
    if (e.type == 0 && e.f >= 5 && h.nk == 1) continue;
    ctx->bc.push_back(e);
  }
  return MOSE_OK;
}

// Plans the 2-D work list with the context's tiling and uploads it: an item
// runs the boundary-free kernel when every block-edge face its cells have
// (column -1 / ni, row -1 / nj) is a connection.
static int install_items(mose_gpu_ctx* ctx) {
  std::vector<int4> all = plan_stage_items(ctx->hblk, 3 * ctx->nsm, ctx->tile_h, ctx->tile_w, ctx->tile_order);
  std::vector<int4> items, items_nb;
  for (const int4& it : all) {
    const BlockDesc& d = ctx->desc[it.x];
    const int c0 = it.y & 0xffff, c1 = it.y >> 16, j0 = it.z, j1 = it.w;
    bool conn = true;
    auto check = [&](int f, int lo, int hi) {
      for (int q = lo; q < hi && conn; ++q) conn = bc_code(ctx->hbcw[d.bcoff[f] + q]) == BC_CONN;
    };
    if (c0 == 0) check(0, j0, j1);
    if (c1 == d.ni) check(1, j0, j1);
    if (j0 == 0) check(2, c0, c1);
    if (j1 == d.nj) check(3, c0, c1);
    (conn && ctx->nd == 2 ? items_nb : items).push_back(it);
  }
  ctx->nitems = (int)items.size();
  ctx->nitems_nb = (int)items_nb.size();
  CU(ctx->items.alloc(std::max<size_t>(items.size(), 1)));
  CU(ctx->items_nb.alloc(std::max<size_t>(items_nb.size(), 1)));
  if (!items.empty())
    CU(cudaMemcpyAsync(ctx->items.p, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
  if (!items_nb.empty())
    CU(cudaMemcpyAsync(ctx->items_nb.p, items_nb.data(), items_nb.size() * sizeof(int4), cudaMemcpyHostToDevice,
                       ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return MOSE_OK;
}

int mose_gpu_setup(mose_gpu_ctx* ctx) {
  MOSE_NVTX_RANGE("mose_gpu_setup");
  if (!ctx) return MOSE_ERR_INVALID;
  if (ctx->hblk.empty() || ctx->bc.empty()) return fail(ctx, MOSE_ERR_NOT_READY, "no blocks or no boundary records");
  CU(cudaSetDevice(ctx->cfg.device));
  const int nb = (int)ctx->hblk.size();
  // Check_Mesh_Type (Lib_Metrics.f90:13-66)
  const HostBlock& b1 = ctx->hblk[0];
  if (ctx->cfg.ndir > 0) ctx->ndir = ctx->cfg.ndir;
  else if (b1.nk > 1) ctx->ndir = 3;
  else if (b1.nj == 1) ctx->ndir = 1;
  else ctx->ndir = 2;
  ctx->nd = (ctx->ndir == 3) ? 3 : 2;
  ctx->nv = (ctx->nd == 3) ? 5 : 4;
  if ((ctx->cfg.riemann == MOSE_RIEMANN_AUSMP_UP || ctx->cfg.riemann == MOSE_RIEMANN_AUSMP_UP2) &&
      !(ctx->gas.minf > 0.0))
    return fail(ctx, MOSE_ERR_INVALID, "AUSM+-up solver selected: Minf must be set (mose_gpu_set_riemann_minf)");
  if (ctx->gas.sd && ctx->nd == 2) {
    // the 2-D stage kernel reads the four face neighbours of every cell from
    // its ring (a one-row block, the 1-D cases, reads its j pair from the
    // zero-gradient ghost rows of its null faces: an exact 0, as in the
    // reference); 3-D blocks take the detector from its own pass over the
    // ghosted state
    for (const auto& h : ctx->hblk)
      if (h.ni < 3 || (h.nj < 3 && h.nj != 1))
        return fail(ctx, MOSE_ERR_UNSUPPORTED, "the shock detector needs blocks of at least 3 x 3 cells, or 1-D rows");
  }
  if (ctx->irs_beta > 0.0 && ctx->cfg.precision == MOSE_PRECISION_MIXED)
    return fail(ctx, MOSE_ERR_UNSUPPORTED, "implicit residual smoothing runs in the exact and fp64 precisions");
  if (ctx->gas.model > 0) {
    if (ctx->nd != 2 || ctx->ndir != 2 || ctx->cfg.precision != MOSE_PRECISION_FP64_EXACT ||
        ctx->cfg.integration != MOSE_INTEGRATION_CONS || ctx->irs_beta > 0.0 || ctx->gas.sd != 0)
      return fail(ctx, MOSE_ERR_UNSUPPORTED,
                  "Navier-Stokes runs on 2-D domains in the exact precision, conservative integration, without "
                  "implicit residual smoothing or the shock detector");
    for (int b = 0; b < nb; ++b)
      if (ctx->hblk[b].nj < 3 || ctx->hblk[b].ni < 3)
        return fail(ctx, MOSE_ERR_UNSUPPORTED, "Navier-Stokes: block %d needs at least 3 x 3 cells", b + 1);
  }
  if (ctx->nd == 3 && !stage3d_supported(ctx->cfg.riemann, ctx->cfg.limiter))
    return fail(ctx, MOSE_ERR_UNSUPPORTED, "3-D blocks: no stage kernel for riemann %d, limiter %d",
                ctx->cfg.riemann, ctx->cfg.limiter);
  if (ctx->nd != 3 && !stage2d_supported(ctx->cfg.riemann, ctx->cfg.precision))
    return fail(ctx, MOSE_ERR_UNSUPPORTED, "no stage kernel for riemann %d in precision %d", ctx->cfg.riemann,
                ctx->cfg.precision);
  auto nodeh = [&](const HostBlock& h, int i, int j, int k, int c) {
    return h.node[3 * ((size_t)i + (size_t)(h.ni + 1) * ((size_t)j + (size_t)(h.nj + 1) * k)) + c];
  };
  if (ctx->ndir == 2) {
    double y0 = nodeh(b1, 0, 1, 0, 1), z0 = nodeh(b1, 0, 1, 0, 2), y1 = nodeh(b1, 0, 1, 1, 1), z1 = nodeh(b1, 0, 1, 1, 2);
    double y2 = nodeh(b1, 0, b1.nj, 0, 1), z2 = nodeh(b1, 0, b1.nj, 0, 2), y3 = nodeh(b1, 0, b1.nj, 1, 1),
           z3 = nodeh(b1, 0, b1.nj, 1, 2);
    double t1 = std::atan2(z1, y1) - std::atan2(z0, y0), t2 = std::atan2(z3, y3) - std::atan2(z2, y2);
    double r0 = std::sqrt(y0 * y0 + z0 * z0), r1 = std::sqrt(y1 * y1 + z1 * z1);
    if ((t1 - t2) < 1e-5 && r0 > 1e-10 && std::fabs(r0 - r1) < 1e-5 * r0)
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "axisymmetric 2-D meshes are not on this path");
  }
  // 2-D: planar blocks so that n_z == 0 on i and j faces and w stays 0
  for (int b = 0; b < nb && ctx->nd == 2; ++b) {
    const HostBlock& h = ctx->hblk[b];
    if (h.nk != 1) return fail(ctx, MOSE_ERR_UNSUPPORTED, "mixed 2-D / 3-D blocks");
    for (int j = 0; j <= h.nj; ++j)
      for (int i = 0; i <= h.ni; ++i)
        if (nodeh(h, i, j, 0, 0) != nodeh(h, i, j, 1, 0) || nodeh(h, i, j, 0, 1) != nodeh(h, i, j, 1, 1))
          return fail(ctx, MOSE_ERR_UNSUPPORTED, "block %d is not planar in k", b + 1);
    if (h.ni < 2) return fail(ctx, MOSE_ERR_UNSUPPORTED, "block %d: need ni >= 2", b + 1);
  }
  for (auto& e : ctx->bc) {
    const HostBlock& h = ctx->hblk[e.b - 1];
    if (ctx->nd == 2 && e.f >= 5 && e.type != 0)
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "2-D k faces must be null (type 0), found %d", e.type);
    bool degenerate = (e.f >= 3 && e.f <= 4 && h.nj < 3) || (e.f <= 2 && h.ni < 3) ||
                      (ctx->nd == 3 && e.f >= 5 && h.nk < 3);
    if (degenerate && !(e.type == 0 || e.type == 400 || e.type == 406))
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "bc type %d on a face of a block thinner than 3 cells", e.type);
    // (the token 'normal' resolves to atan(0 / ...) = 0 there: 2-D face normals have n_z = 0)
    if (ctx->nd == 2 && e.type == 405 && e.data[4] != 0.0 && !(e.data[4] >= 0.5 * 1.7976931348623157e308))
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "2-D inflow with a non-zero out-of-plane angle");
    if (ctx->nd == 2 && (e.type >= 401 && e.type <= 404) && e.data[3] != 0.0 &&
        !(e.data[3] >= 0.5 * 1.7976931348623157e308))
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "2-D inflow with a non-zero out-of-plane angle");
    if (e.type == 402 && !(e.data[1] >= 0.0 && e.data[1] < (double)ctx->hser_idx.size() &&
                           e.data[1] == std::floor(e.data[1])))
      return fail(ctx, MOSE_ERR_INVALID, "bc 402: time table %g was not added", e.data[1]);
    // 407 uses its angles as given (Lib_BC_Fluxes_FarField.f90:48-49): the
    // token 'normal' would enter tan() as the largest double
    if (e.type == 407 && (e.data[3] >= 0.5 * 1.7976931348623157e308 || e.data[4] >= 0.5 * 1.7976931348623157e308))
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "bc 407 takes numeric inflow angles, not 'normal'");
    if (ctx->nd == 2 && e.type == 407 && e.data[4] != 0.0)
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "2-D inflow with a non-zero out-of-plane angle");
  }
  for (int b = 0; b < nb && ctx->nd == 3; ++b)
    if (ctx->hblk[b].nk < 1 || ctx->hblk[b].ni >= 65536)
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "block %d: 3-D extents out of range", b + 1);

  // ---- layout ----------------------------------------------------------------
  ctx->desc.assign(nb, BlockDesc{});
  long long mcur = 0;
  ctx->maxcell = 0;
  std::vector<int> bcwords;
  std::vector<BcParam> params;
  for (int b = 0; b < nb; ++b) {
    const HostBlock& h = ctx->hblk[b];
    BlockDesc& d = ctx->desc[b];
    d.ni = h.ni; d.nj = h.nj; d.nk = h.nk;
    d.px = ((h.ni + 2 * GW) + 15) / 16 * 16;
    d.py = h.nj + 2 * GW;
    d.pz = (ctx->nd == 3) ? h.nk + 2 * GW : 1;
    d.plane = (long long)d.px * d.py;
    d.vstride = d.plane * d.pz;
    d.vstride = (d.vstride + 31) / 32 * 32;
    d.mbase = mcur;
    d.sbase = (long long)ctx->nv * mcur;
    mcur += d.vstride;
    ctx->maxcell = std::max(ctx->maxcell, (long long)h.ni * h.nj * h.nk);
    for (int f = 0; f < 6; ++f) {
      d.bcn[f] = (f < 2) ? h.nj * h.nk : (f < 4) ? h.ni * h.nk : h.ni * h.nj;
      d.bcoff[f] = (int)bcwords.size();
      bcwords.resize(bcwords.size() + d.bcn[f], BC_NONE);
    }
  }
  ctx->marena = mcur;
  // 405 records whose direction token is 'normal': their angles follow the
  // face normal (Compute_Inflow_Direction, Lib_BC_Fluxes_Inflow.f90:479-496)
  // and are resolved once the device has formed the face metrics
  struct NormalDir { int pidx, b, f, i, j, k; bool a, be; };
  std::vector<NormalDir> normal_dirs;
  // 401 / 403 / 404 / 407 records: tangent, binormal and direction
  // coefficients, formed from the face normal once the device has it
  struct InletGeo { int pidx, b, f, i, j, k; double alpha, beta; bool raw; };
  std::vector<InletGeo> inlet_geo;
  std::vector<SeriesRec> series_recs;
  std::vector<VConn> vconn;
  for (auto& e : ctx->bc) {
    const BlockDesc& d = ctx->desc[e.b - 1];
    const HostBlock& h = ctx->hblk[e.b - 1];
    int code = bc_code_of(e.type);
    int pidx = -1;
    if (e.type == 405 || e.type == 406) {
      BcParam p{};
      if (e.type == 405) {
        p.mach = e.data[0]; p.T = e.data[1]; p.p = e.data[2]; p.rel_fac = e.data[5];
        double alpha = e.data[3], beta = e.data[4];
        const bool na = alpha >= 0.5 * 1.7976931348623157e308, nb = beta >= 0.5 * 1.7976931348623157e308;
        if (na || nb) normal_dirs.push_back(NormalDir{(int)params.size(), e.b - 1, e.f, e.i - 1, e.j - 1, e.k - 1, na, nb});
        p.ca = std::cos(alpha); p.sa = std::sin(alpha); p.cb = std::cos(beta); p.sb = std::sin(beta);
      } else {
        p.pback = e.data[0]; p.rel_fac = e.data[1];
      }
      pidx = (int)params.size();
      params.push_back(p);
    } else if (e.type >= 401 && e.type <= 407) {
      BcParam p{};
      p.T = e.data[0]; p.p = e.data[1];
      double alpha = e.data[2], beta = e.data[3];
      if (e.type == 407) {
        p.pback = e.data[2]; p.rel_fac = e.data[5];
        alpha = e.data[3]; beta = e.data[4];
      } else {
        p.rel_fac = e.data[4];
      }
      inlet_geo.push_back(InletGeo{(int)params.size(), e.b - 1, e.f, e.i - 1, e.j - 1, e.k - 1, alpha, beta,
                                   e.type == 407});
      if (e.type == 402) {
        const auto& si = ctx->hser_idx[(size_t)e.data[1]];
        series_recs.push_back(SeriesRec{(int)params.size(), si.off, si.n, si.periodic});
        p.p = ctx->hser[2 * (size_t)si.off + 1];    // refreshed from the table before every use
      }
      pidx = (int)params.size();
      params.push_back(p);
    }
    if (e.type == 301 || e.type == 302) {
      BcParam p{};
      if (e.type == 301) p.p = e.data[0];   // qw
      else p.T = e.data[0];                 // Tw
      pidx = (int)params.size();
      params.push_back(p);
    }
    if (ctx->gas.model > 0 && (e.type == 101 || e.type == 201) && e.f <= 4) {
      // the viscous flux's source stencil (Fill_BC_Ghost_Connection); 2-D
      // orientations: d11 = +-1 along the face, d22 = +-1 across k
      if (e.d12 != 0 || e.d21 != 0 || (e.d11 != 1 && e.d11 != -1) || (e.d22 != 1 && e.d22 != -1) || e.fs > 4)
        return fail(ctx, MOSE_ERR_UNSUPPORTED, "Navier-Stokes: connection orientation d11..d22 = %d %d %d %d",
                    e.d11, e.d12, e.d21, e.d22);
      pidx = (int)vconn.size();
      vconn.push_back(VConn{e.bs - 1, e.is - 1, e.js - 1, e.fs, e.d11});
    }
    bcwords[d.bcoff[e.f - 1] + face_index(h, e.f, e.i - 1, e.j - 1, e.k - 1)] = code | ((pidx + 1) << 8);
  }

  // ---- allocation --------------------------------------------------------------
  // Every upload below is a cudaMemcpyAsync on the context's stream: a plain
  // cudaMemcpy from pageable memory may return before its DMA has landed and
  // runs on the legacy default stream, which the context's non-blocking
  // stream does not wait for, so the kernels enqueued next could read the
  // buffer before it is written.
  for (int s = 0; s < 3; ++s)
    if (ctx->state[s].alloc((size_t)ctx->nv * mcur) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (state)");
  if (ctx->resid.alloc((size_t)ctx->nv * mcur) != cudaSuccess || ctx->dl.alloc(3 * (size_t)mcur) != cudaSuccess ||
      ctx->face.alloc(12 * (size_t)mcur) != cudaSuccess || ctx->vol.alloc((size_t)mcur) != cudaSuccess ||
      ctx->vers.alloc(9 * (size_t)mcur) != cudaSuccess || ctx->dtl.alloc((size_t)mcur) != cudaSuccess)
    return fail(ctx, MOSE_ERR_CUDA, "out of device memory (metrics)");
  if (ctx->nd == 3 && ctx->hk.alloc((size_t)ctx->nv * mcur) != cudaSuccess)
    return fail(ctx, MOSE_ERR_CUDA, "out of device memory (k-face arena)");
  if (ctx->nd == 3 && ctx->gas.sd && ctx->sdbeta.alloc((size_t)mcur) != cudaSuccess)
    return fail(ctx, MOSE_ERR_CUDA, "out of device memory (shock detector)");
  if (ctx->gas.model > 0) {
    if (ctx->Mt.alloc(4 * (size_t)mcur) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (metrics)");
    if (ctx->vface.alloc(14 * (size_t)mcur) != cudaSuccess)
      return fail(ctx, MOSE_ERR_CUDA, "out of device memory (viscous face fluxes)");
    CU(cudaMemsetAsync(ctx->Mt.p, 0, 4 * (size_t)mcur * sizeof(double), ctx->stream));
    static_assert(sizeof(VConn) == 5 * sizeof(int), "VConn is five ints");
    CU(ctx->vconn.alloc(5 * std::max<size_t>(vconn.size(), 1)));
    if (!vconn.empty())
      CU(cudaMemcpyAsync(ctx->vconn.p, vconn.data(), vconn.size() * sizeof(VConn), cudaMemcpyHostToDevice,
                         ctx->stream));
  }
  CU(ctx->d_desc.alloc(nb));
  CU(ctx->bcw.alloc(bcwords.size()));
  CU(ctx->bcp.alloc(std::max<size_t>(params.size(), 1)));
  CU(ctx->scal.alloc(4));
  CU(ctx->dtmin.alloc(1));
  CU(ctx->iterdev.alloc(1));
  CU(ctx->derr.alloc(1));
  CU(ctx->norms.alloc(5));
  CU(ctx->partial.alloc(5 * (size_t)norms_partial_count(nb, ctx->maxcell)));
  CU(cudaMemcpyAsync(ctx->d_desc.p, ctx->desc.data(), nb * sizeof(BlockDesc), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->bcw.p, bcwords.data(), bcwords.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  if (!params.empty()) CU(cudaMemcpyAsync(ctx->bcp.p, params.data(), params.size() * sizeof(BcParam), cudaMemcpyHostToDevice, ctx->stream));
  ctx->nser = (int)series_recs.size();
  if (ctx->nser) {
    CU(ctx->ser_recs.alloc(series_recs.size()));
    CU(ctx->ser_tv.alloc(ctx->hser.size()));
    CU(cudaMemcpyAsync(ctx->ser_recs.p, series_recs.data(), series_recs.size() * sizeof(SeriesRec),
                       cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->ser_tv.p, ctx->hser.data(), ctx->hser.size() * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
  }
  ctx->hbcp = params;

  // ---- metrics on the device -------------------------------------------------
  std::vector<DevBuf<double>> dnodes(nb);
  std::vector<NodeView> views(nb);
  for (int b = 0; b < nb; ++b) {
    const HostBlock& h = ctx->hblk[b];
    CU(dnodes[b].alloc(h.node.size()));
    CU(cudaMemcpyAsync(dnodes[b].p, h.node.data(), h.node.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    views[b] = NodeView{dnodes[b].p, h.ni, h.nj, h.nk, ctx->derr.p};
  }
  DevBuf<NodeView> dviews;
  CU(dviews.alloc(nb));
  CU(cudaMemcpyAsync(dviews.p, views.data(), nb * sizeof(NodeView), cudaMemcpyHostToDevice, ctx->stream));
  MetricArgs m = ctx->margs();
  for (int b = 0; b < nb; ++b) {
    const HostBlock& h = ctx->hblk[b];
    long long ncell = (long long)h.ni * h.nj * h.nk;
    launch_cell_metrics(ctx->d_desc.p, b, ncell, views[b], m, ctx->nd, ctx->ndir, ctx->derr.p, ctx->stream);
    for (int dir = 0; dir < ctx->nd; ++dir) {
      long long nf = (long long)(h.ni + (dir == 0)) * (h.nj + (dir == 1)) * (h.nk + (dir == 2));
      launch_face_metrics(ctx->d_desc.p, b, nf, views[b], m, ctx->nd, dir, ctx->stream);
    }
  }
  // ghost metrics per record, in bc order
  std::vector<GhostMetricRec> gm;
  for (auto& e : ctx->bc)
    gm.push_back(GhostMetricRec{e.type, e.b - 1, e.i, e.j, e.k, e.f, e.bs - 1, e.is, e.js, e.ks, e.fs,
                                e.d11, e.d12, e.d21, e.d22});
  // BC_Symmetry_Metrics copies interior metrics: run the other records first
  // is unnecessary (ghosts are never sources), but symmetric records read
  // interior dl which is final after the cell kernel.
  DevBuf<GhostMetricRec> dgm;
  CU(dgm.alloc(gm.size()));
  CU(cudaMemcpyAsync(dgm.p, gm.data(), gm.size() * sizeof(GhostMetricRec), cudaMemcpyHostToDevice, ctx->stream));
  launch_ghost_metrics(ctx->d_desc.p, dgm.p, (int)gm.size(), dviews.p, m, ctx->nd, ctx->ndir, ctx->derr.p, ctx->stream);
  {
    int rc = check_launch(ctx, "metrics");
    if (rc) return rc;
    rc = poll_device_error(ctx);   // metric failures and index self-checks
    if (rc) return rc;
  }
  // precomputed metrics handed to add_block replace the node-derived ones
  for (int b = 0; b < nb; ++b) {
    const HostBlock& h = ctx->hblk[b];
    if (h.metrics.empty()) continue;
    DevBuf<double> src;
    CU(src.alloc(h.metrics.size()));
    CU(cudaMemcpyAsync(src.p, h.metrics.data(), h.metrics.size() * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
    const int dims[3] = {h.ni, h.nj, h.nk};
    launch_metrics_from_ref(ctx->d_desc.p, b, dims, src.p, m, ctx->nd, ctx->ndir, ctx->stream);
    CU(cudaStreamSynchronize(ctx->stream));   // src is freed at the end of this scope
    int rc = check_launch(ctx, "precomputed metrics");
    if (rc) return rc;
  }
  if (!normal_dirs.empty() || !inlet_geo.empty()) {
    // the boundary face's normal (nx, ny, nz planes of its direction), then
    // alpha = atan(N_y / (N_x + 1d-20)), beta = atan(N_z / (N_x + 1d-20)) on
    // the host, as the reference forms them
    auto fetch_normal = [&](int b, int f, int i, int j, int k, double* dst) -> cudaError_t {
      const BlockDesc& d = ctx->desc[b];
      const int dir = (f - 1) / 2;
      const int fi = i + (f == 2), fj = j + (f == 4), fk = k + (f == 6);
      const long long o = (ctx->nd == 3) ? (long long)(fk + GW) * d.plane + (long long)(fj + GW) * d.px + (fi + GW)
                                         : (long long)(fj + GW) * d.px + (fi + GW);
      const double* src = ctx->face.p + 12 * d.mbase + (long long)(4 * dir) * d.vstride + o;
      return cudaMemcpy2DAsync(dst, sizeof(double), src, d.vstride * sizeof(double), sizeof(double), 3,
                               cudaMemcpyDeviceToHost, ctx->stream);
    };
    std::vector<double> nrm(3 * normal_dirs.size()), inrm(3 * inlet_geo.size());
    for (size_t q = 0; q < normal_dirs.size(); ++q) {
      const NormalDir& r = normal_dirs[q];
      CU(fetch_normal(r.b, r.f, r.i, r.j, r.k, &nrm[3 * q]));
    }
    for (size_t q = 0; q < inlet_geo.size(); ++q) {
      const InletGeo& r = inlet_geo[q];
      CU(fetch_normal(r.b, r.f, r.i, r.j, r.k, &inrm[3 * q]));
    }
    CU(cudaStreamSynchronize(ctx->stream));
    for (size_t q = 0; q < normal_dirs.size(); ++q) {
      const NormalDir& r = normal_dirs[q];
      BcParam& p = ctx->hbcp[r.pidx];
      const double* N = &nrm[3 * q];
      if (r.a) {
        const double alpha = std::atan(N[1] / (N[0] + 1e-20));
        p.ca = std::cos(alpha); p.sa = std::sin(alpha);
      }
      if (r.be) {
        const double beta = std::atan(N[2] / (N[0] + 1e-20));
        p.cb = std::cos(beta); p.sb = std::sin(beta);
      }
    }
    for (size_t q = 0; q < inlet_geo.size(); ++q) {
      // Setup_Inflow_Geometry's tangent (Lib_BC_Fluxes_Inflow.f90:537-549):
      // node (Face_i, Face_j, Face_k) less the node one step back along the
      // face's two other directions, normalised; then Compute_Inflow_Direction
      // (:479-496) and the binormal and E1, E2 of :404-420
      const InletGeo& r = inlet_geo[q];
      const HostBlock& h = ctx->hblk[r.b];
      BcParam& p = ctx->hbcp[r.pidx];
      const double* N = &inrm[3 * q];
      // Face_Index in the reference's indexing: cells from 1, nodes from 0
      int ci = r.i + 1, cj = r.j + 1, ck = r.k + 1, di = 0, dj = 0, dk = 0;
      if (r.f <= 2) { ci -= r.f % 2; dj = 1; dk = 1; }
      else if (r.f <= 4) { cj -= r.f % 2; di = 1; dk = 1; }
      else { ck -= r.f % 2; di = 1; dj = 1; }
      double t[3], bv[3];
      for (int c = 0; c < 3; ++c) t[c] = nodeh(h, ci, cj, ck, c) - nodeh(h, ci - di, cj - dj, ck - dk, c);
      const double tmod = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      for (int c = 0; c < 3; ++c) t[c] = t[c] / tmod;
      double alpha = r.alpha, beta = r.beta;
      if (!r.raw) {
        if (alpha >= 0.5 * 1.7976931348623157e308) alpha = std::atan(N[1] / (N[0] + 1e-20));
        if (beta >= 0.5 * 1.7976931348623157e308) beta = std::atan(N[2] / (N[0] + 1e-20));
      }
      bv[0] = N[1] * t[2] - N[2] * t[1];
      bv[1] = N[2] * t[0] - N[0] * t[2];
      bv[2] = N[0] * t[1] - N[1] * t[0];
      const double bmod = std::sqrt(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
      for (int c = 0; c < 3; ++c) bv[c] = bv[c] / bmod;
      const double ta = std::tan(alpha), tb = std::tan(beta);
      const double XA = N[1] - N[0] * ta, XB = t[1] - t[0] * ta, XC = bv[1] - bv[0] * ta;
      const double XD = N[2] - N[0] * tb, XE = t[2] - t[0] * tb, XF = bv[2] - bv[0] * tb;
      const double check = (XC * XE - XF * XB);
      p.E1 = (XF * XA - XC * XD) / check;
      p.E2 = (XD * XB - XE * XA) / check;
      for (int c = 0; c < 3; ++c) { p.tv[c] = t[c]; p.bv[c] = bv[c]; }
    }
    CU(cudaMemcpyAsync(ctx->bcp.p, ctx->hbcp.data(), ctx->hbcp.size() * sizeof(BcParam), cudaMemcpyHostToDevice,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
  }
  // uniformity: bitwise for the exact and fp64 precisions (a last-bit face
  // area difference is ~1e-10 of a residual, above their 1e-12 bar); within
  // 1e-9 relative for the mixed precision, whose FP32 face states carry
  // ~1e-7 relative error, so domains whose nodes were placed by
  // floating-point arithmetic still run the uniform-grid FP32 pipeline
  const double utol = ctx->cfg.precision == MOSE_PRECISION_MIXED ? 1e-9 : 0.0;
  DevBuf<int> flags;
  DevBuf<double> firsts;
  CU(flags.alloc(nb));
  CU(firsts.alloc(25 * (size_t)nb));
  for (int b = 0; b < nb; ++b) {
    const HostBlock& h = ctx->hblk[b];
    long long n = (long long)(h.ni + 4) * (h.nj + 4) * (ctx->nd == 3 ? h.nk + 4 : 1);
    launch_uniform_check(ctx->d_desc.p, b, n, m, ctx->nd, ctx->ndir, flags.p, firsts.p + 25 * b, utol, ctx->stream);
  }
  std::vector<int> hflags(nb);
  std::vector<double> hfirst(25 * (size_t)nb);
  CU(cudaMemcpyAsync(hflags.data(), flags.p, nb * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(hfirst.data(), firsts.p, hfirst.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  {
    int rc = poll_device_error(ctx);
    if (rc) return rc;
  }
  bool uni = true;
  for (int b = 0; b < nb; ++b) uni &= (hflags[b] == 0);
  ctx->uniform = uni;
  for (int b = 0; b < nb; ++b) {
    BlockDesc& d = ctx->desc[b];
    const double* f = &hfirst[25 * (size_t)b];
    for (int h = 0; h < 3; ++h) d.u_dl[h] = f[h];
    for (int dir = 0; dir < 3; ++dir) {
      for (int q = 0; q < 3; ++q) d.u_n[dir][q] = f[3 + 4 * dir + q];
      d.u_A[dir] = f[3 + 4 * dir + 3];
    }
    d.u_vol = f[15];
    for (int dd = 0; dd < 3; ++dd)
      for (int q = 0; q < 3; ++q) d.u_vers[dd][q] = f[16 + 3 * dd + q];
  }
  // ---- connection edges read in place (2-D, inviscid) ----------------------------
  // A block edge whose face cells are all 101 / 201 connections to one source
  // block's opposite face, aligned (the source column, or row, a fixed offset
  // from the face cell's), on an even-sized block with 16-byte-aligned source
  // chunks: the stage kernels read its ghost cells from the source cells
  // Ghost_Connection copies there (Lib_Ghost.f90:140-160), so the fused
  // steps fill only the other ghost records.
  for (BlockDesc& d : ctx->desc)
    for (int f = 0; f < 4; ++f) {
      d.rm_src[f] = -1;
      d.rm_at[f] = 0;
      d.rm_off[f] = 0;
    }
  ctx->remap = false;
  if (ctx->nd == 2 && ctx->gas.model == 0) {
    std::vector<std::vector<const BcRecord*>> recs(4 * (size_t)nb);
    for (const BcRecord& e : ctx->bc)
      if (e.f <= 4) recs[4 * (size_t)(e.b - 1) + (e.f - 1)].push_back(&e);
    for (int b = 0; b < nb; ++b) {
      const HostBlock& h = ctx->hblk[b];
      if (h.ni % 2 != 0) continue;   // the ghost chunk of face 2 starts at cell ni
      for (int f = 0; f < 4; ++f) {
        const std::vector<const BcRecord*>& L = recs[4 * (size_t)b + f];
        if (f >= 2 && h.nj < 3) continue;   // j-faces without a ghost layer
        if ((int)L.size() != (f < 2 ? h.nj : h.ni)) continue;
        const int want_fs = (f == 0) ? 2 : (f == 1) ? 1 : (f == 2) ? 4 : 3;
        bool ok = true;
        int src = -1, at = 0, off = 0;
        for (size_t q = 0; q < L.size() && ok; ++q) {
          const BcRecord& e = *L[q];
          if ((e.type != 101 && e.type != 201) || e.fs != want_fs) {
            ok = false;
            break;
          }
          const int c = f < 2 ? e.j - 1 : e.i - 1, is = e.is - 1, js = e.js - 1;
          const int a_ = f == 0 ? is - 1 : f == 1 ? is : f == 2 ? js + 1 : js;
          const int o_ = f < 2 ? js - c : is - c;
          if (q == 0) {
            src = e.bs - 1;
            at = a_;
            off = o_;
          } else if (e.bs - 1 != src || a_ != at || o_ != off) {
            ok = false;
          }
        }
        // 16-byte source chunks: an even first column
        if (ok && (f < 2 ? at : off) % 2 != 0) ok = false;
        if (!ok) continue;
        BlockDesc& d = ctx->desc[b];
        d.rm_src[f] = src;
        d.rm_at[f] = at;
        d.rm_off[f] = off;
        ctx->remap = true;
      }
    }
  }
  CU(cudaMemcpyAsync(ctx->d_desc.p, ctx->desc.data(), nb * sizeof(BlockDesc), cudaMemcpyHostToDevice, ctx->stream));

  // ---- ghost-fill records (Fill_Ghost_Cell dispatch, Lib_Ghost.f90:50-73) ------
  std::vector<GhostRec> gr;
  for (auto& e : ctx->bc) {
    if ((e.f - 1) / 2 >= ctx->nd) continue;
    const HostBlock& h = ctx->hblk[e.b - 1];
    // faces of degenerate directions have no ghost layer on the device
    if ((e.f == 3 || e.f == 4) && h.nj < 3) continue;
    int t = bc_code_of(e.type);
    if (t == BC_WALL_Q || t == BC_WALL_T) t = BC_EXTRAP;   // walls: Ghost_Extrapolate (the dispatch's default)
    GhostRec g{t, e.b - 1, e.i - 1, e.j - 1, e.k - 1, e.f, e.bs - 1, e.is - 1, e.js - 1, e.ks - 1, e.fs};
    gr.push_back(g);
  }
  ctx->nghost = (int)gr.size();
  ctx->hghost = gr;
  CU(ctx->ghosts.alloc(std::max<size_t>(gr.size(), 1)));
  if (!gr.empty()) CU(cudaMemcpyAsync(ctx->ghosts.p, gr.data(), gr.size() * sizeof(GhostRec), cudaMemcpyHostToDevice, ctx->stream));
  // Ghost_Connection (Lib_Ghost.f90:140-160) as flat copies: ghost g of the
  // boundary cell (i, j, k) on face f takes the source cell (is, js, ks) +
  // guide(fs) (g - 1), g = 1, 2; the copies are static, so their offsets are
  // formed here once instead of per step from the records
  {
    std::vector<IrsCopy> all, ncp;
    std::vector<GhostRec> other;
    auto off = [&](const BlockDesc& d, int i, int j, int k, long long* o) -> bool {
      const bool in = i >= -GW && i < d.ni + GW && j >= -GW && j < d.nj + GW &&
                      (ctx->nd == 2 || (k >= -GW && k < d.nk + GW));
      *o = ctx->nd == 3 ? (long long)(k + GW) * d.plane + (long long)(j + GW) * d.px + (i + GW)
                        : (long long)(j + GW) * d.px + (i + GW);
      return in;
    };
    for (const GhostRec& g : gr)
      if (g.type != BC_CONN) other.push_back(g);
    // record-major, both ghost layers of a cell side by side (they share
    // sectors on the i faces; a layer-major order was slower: 0.176 against
    // 0.102 ms per fill on 8 x 128^3)
    for (const GhostRec& g : gr) {
      if (g.type != BC_CONN) continue;
      const BlockDesc& d = ctx->desc[g.b];
      const BlockDesc& s = ctx->desc[g.bs];
      const int gi = (g.f == 1) ? 1 : (g.f == 2) ? -1 : 0, gj = (g.f == 3) ? 1 : (g.f == 4) ? -1 : 0;
      const int gk = (g.f == 5) ? 1 : (g.f == 6) ? -1 : 0;
      const int si = (g.fs == 1) ? 1 : (g.fs == 2) ? -1 : 0, sj = (g.fs == 3) ? 1 : (g.fs == 4) ? -1 : 0;
      const int sk = (g.fs == 5) ? 1 : (g.fs == 6) ? -1 : 0;
      const bool in_place = g.f <= 4 && ctx->desc[g.b].rm_src[g.f - 1] >= 0;
      for (int l = 1; l <= GW; ++l) {
        long long od, os;
        if (!off(d, g.i - gi * l, g.j - gj * l, g.k - gk * l, &od) ||
            !off(s, g.is + si * (l - 1), g.js + sj * (l - 1), g.ks + sk * (l - 1), &os))
          return fail(ctx, MOSE_ERR_INVALID, "connection record of block %d, face %d: a ghost or source cell "
                      "outside its block", g.b + 1, g.f);
        const IrsCopy c{d.sbase + od, s.sbase + os, d.vstride, s.vstride};
        all.push_back(c);
        if (!in_place) ncp.push_back(c);
      }
    }
    auto upload = [&](DevBuf<IrsCopy>& buf, const std::vector<IrsCopy>& v) -> cudaError_t {
      cudaError_t e = buf.alloc(std::max<size_t>(v.size(), 1));
      if (e == cudaSuccess && !v.empty())
        e = cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(IrsCopy), cudaMemcpyHostToDevice, ctx->stream);
      return e;
    };
    CU(upload(ctx->gcopy, all));
    CU(upload(ctx->gcopy_nc, ncp));
    ctx->ngcopy = (int)all.size();
    ctx->ngcopy_nc = (int)ncp.size();
    ctx->nghost_other = (int)other.size();
    CU(ctx->ghosts_other.alloc(std::max<size_t>(other.size(), 1)));
    if (!other.empty())
      CU(cudaMemcpyAsync(ctx->ghosts_other.p, other.data(), other.size() * sizeof(GhostRec), cudaMemcpyHostToDevice,
                         ctx->stream));
  }


  // ---- implicit residual smoothing: first-layer ghost records of R ----------------
  if (ctx->irs_beta > 0.0) {
    // guide(face, 1:3), faces 1..6
    static const int inward[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    std::vector<IrsCopy> il;
    // 0-based cell (i, j, k) of a block: its offset in the block's planes
    auto cell = [&](const BlockDesc& d, int i, int j, int k) -> long long {
      return ctx->nd == 3 ? (long long)(k + GW) * d.plane + (long long)(j + GW) * d.px + (i + GW)
                          : (long long)(j + GW) * d.px + (i + GW);
    };
    for (auto& e : ctx->bc) {
      if (e.f > 2 * ctx->nd) continue;            // 2-D: no ghost layer across k
      const BlockDesc& d = ctx->desc[e.b - 1];
      const int* g = inward[e.f - 1];
      const int ig = e.i - 1 - g[0], jg = e.j - 1 - g[1], kg = e.k - 1 - g[2];
      const bool conn = e.type == 101;            // 201 takes the zero-gradient branch (Lib_IRS.f90:172-183)
      const BlockDesc& sd = ctx->desc[conn ? e.bs - 1 : e.b - 1];
      const int is = conn ? e.is - 1 : e.i - 1, js = conn ? e.js - 1 : e.j - 1, ks = conn ? e.ks - 1 : e.k - 1;
      IrsCopy c;
      c.dst = d.sbase + cell(d, ig, jg, kg);
      c.src = sd.sbase + cell(sd, is, js, ks);
      c.vsd = d.vstride;
      c.vss = sd.vstride;
      il.push_back(c);
    }
    ctx->nirs = (int)il.size();
    CU(ctx->irs_list.alloc(std::max<size_t>(il.size(), 1)));
    if (!il.empty())
      CU(cudaMemcpyAsync(ctx->irs_list.p, il.data(), il.size() * sizeof(IrsCopy), cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->rs1.alloc((size_t)ctx->nv * mcur) != cudaSuccess || ctx->rs2.alloc((size_t)ctx->nv * mcur) != cudaSuccess)
      return fail(ctx, MOSE_ERR_CUDA, "out of device memory (residual smoothing)");
  }

  // ---- work items for the stage kernel -----------------------------------------
  ctx->hbcw = bcwords;
  {
    int rc = install_items(ctx);
    if (rc) return rc;
  }
  if (ctx->nd == 3) {
    std::vector<int4> it3[3];
    // the plane stage runs three CTAs per SM, the k-face march two
    plan_3d_items(ctx->hblk, ctx->desc, ctx->hbcw, choose_k_run(ctx->hblk, 3 * ctx->nsm),
                  choose_k_run(ctx->hblk, 2 * ctx->nsm), it3);
    for (int q = 0; q < 3; ++q) {
      ctx->nitems3[q] = (int)it3[q].size();
      CU(ctx->items3[q].alloc(std::max<size_t>(it3[q].size(), 1)));
      if (!it3[q].empty())
        CU(cudaMemcpyAsync(ctx->items3[q].p, it3[q].data(), it3[q].size() * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
    }
  }
  ctx->cur = 0;
  ctx->po = 1;
  CU(cudaDeviceSynchronize());
  ctx->ready = true;
  return MOSE_OK;
}

// ---- transfers -----------------------------------------------------------------
static int ensure_staging(mose_gpu_ctx* ctx, size_t n) {
  if (ctx->staging.n < n)
    if (ctx->staging.alloc(n) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (staging)");
  return MOSE_OK;
}

static int prim_io(mose_gpu_ctx* ctx, int32_t b, double* P, int arena, bool upload) {
  if (!ctx || !P) return MOSE_ERR_INVALID;
  if (!ctx->ready) return fail(ctx, MOSE_ERR_NOT_READY, "setup not done");
  if (b < 1 || b > (int)ctx->hblk.size()) return fail(ctx, MOSE_ERR_INVALID, "bad block %d", b);
  CU(cudaSetDevice(ctx->cfg.device));
  const HostBlock& h = ctx->hblk[b - 1];
  // the transferred slab: the whole array in 3-D, the k = 1 plane in 2-D
  long long plane = (long long)(h.ni + 4) * (h.nj + 4);
  long long n = (ctx->nd == 3) ? plane * (h.nk + 4) : plane;
  if (ctx->nd == 2) P += 5 * GW * plane;
  int rc = ensure_staging(ctx, 5 * (size_t)n);
  if (rc) return rc;
  double* dst = (arena == -2) ? ctx->lam.p : (arena < 0) ? ctx->resid.p : ctx->state[arena].p;
  if (arena == -2 && !ctx->lam.p) return fail(ctx, MOSE_ERR_NOT_READY, "no adjoint state yet");
  if (upload) {
    ctx->dt_valid = false;
    CU(cudaMemcpyAsync(ctx->staging.p, P, 5 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    launch_ref_to_soa(ctx->d_desc.p, b - 1, n, ctx->staging.p, dst, ctx->nv, ctx->nd, ctx->stream);
    ctx->launches++;
  } else {
    launch_soa_to_ref(ctx->d_desc.p, b - 1, n, dst, ctx->staging.p, ctx->nv, ctx->nd, ctx->stream);
    ctx->launches++;
    CU(cudaMemcpyAsync(P, ctx->staging.p, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  CU(cudaStreamSynchronize(ctx->stream));
  return check_launch(ctx, "layout conversion");
}

int mose_gpu_upload_prim(mose_gpu_ctx* ctx, int32_t b, const double* P) {
  MOSE_NVTX_RANGE("mose_gpu_upload_prim");
  return prim_io(ctx, b, const_cast<double*>(P), ctx ? ctx->cur : 0, true);
}
int mose_gpu_download_prim(mose_gpu_ctx* ctx, int32_t b, double* P) {
  MOSE_NVTX_RANGE("mose_gpu_download_prim");
  return prim_io(ctx, b, P, ctx ? ctx->cur : 0, false);
}
int mose_gpu_upload_prim_old(mose_gpu_ctx* ctx, int32_t b, const double* PO) {
  MOSE_NVTX_RANGE("mose_gpu_upload_prim_old");
  return prim_io(ctx, b, const_cast<double*>(PO), ctx ? ctx->po : 1, true);
}
int mose_gpu_download_residual(mose_gpu_ctx* ctx, int32_t b, double* R) { return prim_io(ctx, b, R, -1, false); }
int mose_gpu_upload_residual(mose_gpu_ctx* ctx, int32_t b, const double* R) {
  MOSE_NVTX_RANGE("mose_gpu_download_residual");
  return prim_io(ctx, b, const_cast<double*>(R), -1, true);
}

static int dt_io(mose_gpu_ctx* ctx, int32_t b, double* dt, bool upload) {
  if (!ctx || !dt) return MOSE_ERR_INVALID;
  if (!ctx->ready) return fail(ctx, MOSE_ERR_NOT_READY, "setup not done");
  if (b < 1 || b > (int)ctx->hblk.size()) return fail(ctx, MOSE_ERR_INVALID, "bad block %d", b);
  CU(cudaSetDevice(ctx->cfg.device));
  const HostBlock& h = ctx->hblk[b - 1];
  long long n = (long long)h.ni * h.nj * h.nk;
  int rc = ensure_staging(ctx, (size_t)n);
  if (rc) return rc;
  if (upload) {
    ctx->dt_valid = false;
    CU(cudaMemcpyAsync(ctx->staging.p, dt, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    launch_plane_io(ctx->d_desc.p, b - 1, n, ctx->dtl.p, ctx->staging.p, ctx->nd, 0, ctx->stream);
  } else {
    launch_plane_io(ctx->d_desc.p, b - 1, n, ctx->dtl.p, ctx->staging.p, ctx->nd, 1, ctx->stream);
    CU(cudaMemcpyAsync(dt, ctx->staging.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  ctx->launches++;
  CU(cudaStreamSynchronize(ctx->stream));
  return check_launch(ctx, "dt transfer");
}
int mose_gpu_download_dt(mose_gpu_ctx* ctx, int32_t b, double* dt) { return dt_io(ctx, b, dt, false); }
int mose_gpu_upload_dt(mose_gpu_ctx* ctx, int32_t b, const double* dt) {
  MOSE_NVTX_RANGE("mose_gpu_download_dt");
  return dt_io(ctx, b, const_cast<double*>(dt), true);
}

// ---- phases ----------------------------------------------------------------------
static int require_ready(mose_gpu_ctx* ctx) {
  if (!ctx) return MOSE_ERR_INVALID;
  if (!ctx->ready) return fail(ctx, MOSE_ERR_NOT_READY, "setup not done");
  if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "cudaSetDevice");
  return MOSE_OK;
}

int mose_gpu_compute_dt(mose_gpu_ctx* ctx, double cfl, int32_t iter, int32_t ramp_iter, double* dtglobal) {
  MOSE_NVTX_RANGE("mose_gpu_compute_dt");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (!dtglobal) return MOSE_ERR_INVALID;
  ctx->dt_valid = false;
  launch_step_begin(ctx->dtmin.p, *dtglobal, nullptr, ctx->stream);
  launch_compute_dt(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->state[ctx->cur].p, ctx->margs(),
                    ctx->dtl.p, ctx->dtmin.p, ctx->gas, cfl, ctx->ndir, ctx->nd, iter, ramp_iter, 1, ctx->uniform,
                    ctx->stream);
  launch_step_dt_final(ctx->dtmin.p, ctx->scal.p, ctx->scal.p + 1, 0, ctx->stream);
  ctx->launches += 3;
  CU(cudaMemcpyAsync(dtglobal, ctx->scal.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_launch(ctx, "compute_dt");
}

int mose_gpu_set_global_dt(mose_gpu_ctx* ctx, double dtglobal) {
  MOSE_NVTX_RANGE("mose_gpu_set_global_dt");
  int rc = require_ready(ctx);
  if (rc) return rc;
  ctx->dt_valid = false;
  CU(cudaMemcpyAsync(ctx->scal.p, &dtglobal, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  launch_set_global_dt(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->dtl.p, ctx->scal.p, ctx->nd,
                       ctx->stream);
  ctx->launches++;
  CU(cudaStreamSynchronize(ctx->stream));
  return check_launch(ctx, "set_global_dt");
}

int mose_gpu_copy_state(mose_gpu_ctx* ctx) {
  MOSE_NVTX_RANGE("mose_gpu_copy_state");
  int rc = require_ready(ctx);
  if (rc) return rc;
  ctx->dt_valid = false;
  ctx->po = (ctx->cur + 1) % 3;
  CU(cudaMemcpyAsync(ctx->state[ctx->po].p, ctx->state[ctx->cur].p, ctx->state[0].n * sizeof(double),
                     cudaMemcpyDeviceToDevice, ctx->stream));
  return MOSE_OK;
}

static int enqueue_fill(mose_gpu_ctx* ctx, double* P, bool in_place_skipped, cudaStream_t st);

int mose_gpu_fill_ghosts(mose_gpu_ctx* ctx) {
  MOSE_NVTX_RANGE("mose_gpu_fill_ghosts");
  int rc = require_ready(ctx);
  if (rc) return rc;
  ctx->launches += enqueue_fill(ctx, ctx->state[ctx->cur].p, false, ctx->stream);
  return check_launch(ctx, "fill_ghosts");
}

static StageArgs stage_args(mose_gpu_ctx* ctx, int pc, int po, int pn, int irk) {
  static const double RKcoeff[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0 / 3.0}};
  StageArgs a{};
  a.blk = ctx->d_desc.p;
  a.items = ctx->items.p;
  a.nitems = ctx->nitems;
  a.items_nb = ctx->items_nb.p;
  a.nitems_nb = ctx->nitems_nb;
  a.Pc = ctx->state[pc].p;
  a.Po = ctx->state[po].p;
  a.Pn = pn >= 0 ? ctx->state[pn].p : nullptr;
  a.R = ctx->resid.p;
  a.Hk = ctx->hk.p;
  a.beta = ctx->sdbeta.p;
  a.Fv = ctx->vface.p;
  a.remap = ctx->remap ? 1 : 0;
  a.m = ctx->margs();
  a.dtl = ctx->dtl.p;
  a.dtg = ctx->scal.p;
  a.bcw = ctx->bcw.p;
  a.bcp = ctx->bcp.p;
  a.c_rk = RKcoeff[ctx->cfg.n_rk - 1][irk - 1];
  a.irk = irk;
  a.time_accurate = ctx->cfg.time_accurate;
  a.err = ctx->derr.p;
  a.g = ctx->gas;
  for (int q = 0; q < 3; ++q) {
    a.items3[q] = ctx->items3[q].p;
    a.nitems3[q] = ctx->nitems3[q];
  }
  a.grid_cap = ctx->tile_ctas;
  a.vconn = ctx->vconn.p;
  return a;
}

// Fill_Ghost_Cell on state arena P: the connection copies (all of them, or
// with in_place_skipped those of the edges the stage kernels read in place)
// and the other records.  Returns the number of kernels enqueued.
static int enqueue_fill(mose_gpu_ctx* ctx, double* P, bool in_place_skipped, cudaStream_t st) {
  const bool nc = in_place_skipped && ctx->remap;
  const int ncopy = nc ? ctx->ngcopy_nc : ctx->ngcopy;
  launch_irs_ghost(nc ? ctx->gcopy_nc.p : ctx->gcopy.p, ncopy, P, ctx->nd, st);
  launch_fill_ghosts(ctx->d_desc.p, ctx->ghosts_other.p, ctx->nghost_other, P, ctx->margs(), ctx->nd, ctx->derr.p,
                     st);
  return (ncopy > 0) + (ctx->nghost_other > 0);
}

// The ghost layers of the stage input pc (Fill_Ghost_Cell) that the fused
// steps' stage kernels read from memory: every record, less those of the
// connection edges they read in place.  Returns the number of kernels
// enqueued.
static int enqueue_stage_ghosts(mose_gpu_ctx* ctx, int pc) {
  return enqueue_fill(ctx, ctx->state[pc].p, true, ctx->stream);
}

// One RK stage (mode 0 / 2) or one residual evaluation (mode 1) on every
// block: the 2-D kernel, or the 3-D k-face march and plane stage.  Returns
// the kernel count (0: no kernel for this configuration).
static int launch_stage(mose_gpu_ctx* ctx, const StageArgs& a, int mode, int prec, bool uni) {
  if (ctx->nd == 3) {
    int ksd = 0;
    if (ctx->gas.sd) {
      // the shock detector of every cell of the stage input first
      launch_sd_beta3d(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, a.Pc, ctx->sdbeta.p, ctx->stream);
      ksd = 1;
    }
    if (a.nitems3[0] > 0 && a.nitems3[1] > 0) {
      // the k-face march, then the two plane stages side by side (disjoint
      // cells, as the 2-D kernels below): the boundary tiles on stage_aux
      StageArgs ak = a, anb = a, abc = a;
      ak.nitems3[0] = ak.nitems3[1] = 0;
      anb.nitems3[1] = anb.nitems3[2] = 0;
      abc.nitems3[0] = abc.nitems3[2] = 0;
      if (!launch_stage3d(ak, ctx->nsm, mode, uni, prec, ctx->cfg.riemann, ctx->cfg.limiter, ctx->stream)) return 0;
      if (cudaEventRecord(ctx->stage_fork, ctx->stream) != cudaSuccess ||
          cudaStreamWaitEvent(ctx->stage_aux, ctx->stage_fork, 0) != cudaSuccess)
        return 0;
      const bool ok =
          launch_stage3d(abc, ctx->nsm, mode, uni, prec, ctx->cfg.riemann, ctx->cfg.limiter, ctx->stage_aux) &&
          launch_stage3d(anb, ctx->nsm, mode, uni, prec, ctx->cfg.riemann, ctx->cfg.limiter, ctx->stream);
      if (cudaEventRecord(ctx->stage_join, ctx->stage_aux) != cudaSuccess ||
          cudaStreamWaitEvent(ctx->stream, ctx->stage_join, 0) != cudaSuccess)
        return 0;
      return ok ? 3 + ksd : 0;
    }
    return launch_stage3d(a, ctx->nsm, mode, uni, prec, ctx->cfg.riemann, ctx->cfg.limiter, ctx->stream)
               ? ksd + (a.nitems3[2] > 0) + (a.nitems3[0] > 0) + (a.nitems3[1] > 0)
               : 0;
  }
  if (a.nitems > 0 && a.nitems_nb > 0) {
    // The boundary-free items and the boundary items write disjoint cells
    // and meet only in atomics (the fused dt minimum, the error word), so the
    // two persistent launches run side by side: the boundary items on
    // stage_aux, forked from and joined back into the context's stream (also
    // inside graph capture).  Serialised, a small domain paid one item's
    // march twice per stage.
    StageArgs anb = a, abc = a;
    anb.nitems = 0;
    abc.nitems_nb = 0;
    if (cudaEventRecord(ctx->stage_fork, ctx->stream) != cudaSuccess ||
        cudaStreamWaitEvent(ctx->stage_aux, ctx->stage_fork, 0) != cudaSuccess)
      return 0;
    const bool ok = launch_stage2d(abc, ctx->nsm, mode, uni, prec, ctx->cfg.riemann, ctx->cfg.limiter, ctx->stage_aux) &&
                    launch_stage2d(anb, ctx->nsm, mode, uni, prec, ctx->cfg.riemann, ctx->cfg.limiter, ctx->stream);
    // the join is recorded whatever happened, so a capture never ends forked
    if (cudaEventRecord(ctx->stage_join, ctx->stage_aux) != cudaSuccess ||
        cudaStreamWaitEvent(ctx->stream, ctx->stage_join, 0) != cudaSuccess)
      return 0;
    return ok ? 2 : 0;
  }
  return launch_stage2d(a, ctx->nsm, mode, uni, prec, ctx->cfg.riemann, ctx->cfg.limiter, ctx->stream)
             ? (a.nitems > 0) + (a.nitems_nb > 0)
             : 0;
}

static int enqueue_series(mose_gpu_ctx* ctx);

int mose_gpu_residual(mose_gpu_ctx* ctx) {
  MOSE_NVTX_RANGE("mose_gpu_residual");
  int rc = require_ready(ctx);
  if (rc) return rc;
  // the residual phase runs the reference-exact arithmetic, or the fp64
  // precision's restated arithmetic when the context computes in it (the
  // same face physics as its fused stages); 402 tables are read at the
  // caller's domain time (mose_gpu_set_time)
  if (ctx->nser) {
    CU(cudaMemcpyAsync(ctx->scal.p + 1, &ctx->h_time, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    ctx->launches += enqueue_series(ctx);
  }
  StageArgs a = stage_args(ctx, ctx->cur, ctx->po, -1, 1);
  if (ctx->gas.model > 0) {
    if (!launch_visc_residual2d(a, (int)ctx->hblk.size(), ctx->maxcell, ctx->cfg.limiter, ctx->stream))
      return fail(ctx, MOSE_ERR_UNSUPPORTED, "no viscous kernel for limiter %d", ctx->cfg.limiter);
    ctx->launches += 2;
    return check_launch(ctx, "residual");
  }
  // the exact residual-only kernels read the metric arrays; the fp64 ones
  // take the constant metrics of uniform grids like the fused stages
  const bool fp64 = ctx->cfg.precision == MOSE_PRECISION_FP64;
  const int nk = launch_stage(ctx, a, 1, fp64 ? MOSE_PRECISION_FP64 : MOSE_PRECISION_FP64_EXACT,
                              fp64 && ctx->uniform);
  if (!nk) return fail(ctx, MOSE_ERR_UNSUPPORTED, "no kernel for this solver / limiter");
  ctx->launches += nk;
  return check_launch(ctx, "residual");
}

static int enqueue_irs_smoothing(mose_gpu_ctx* ctx);

int mose_gpu_rk_stage(mose_gpu_ctx* ctx, int32_t irk) {
  MOSE_NVTX_RANGE("mose_gpu_rk_stage");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (irk < 1 || irk > ctx->cfg.n_rk) return fail(ctx, MOSE_ERR_INVALID, "irk out of range");
  static const double RKcoeff[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0 / 3.0}};
  ctx->dt_valid = false;
  if (ctx->irs_beta > 0.0) {
    // RK_Newstate with IRS on the residual of mose_gpu_residual, dt from
    // dtlocal (Compute_dt / Set_Global_dt of the phase path)
    const int nb = (int)ctx->hblk.size();
    launch_irs_scale(ctx->d_desc.p, nb, ctx->maxcell, ctx->state[ctx->cur].p, ctx->resid.p, ctx->margs(), ctx->dtl.p,
                     ctx->scal.p, 0, ctx->gas, ctx->nd, ctx->stream);
    ctx->launches += 1 + enqueue_irs_smoothing(ctx);
    launch_irs_update(ctx->d_desc.p, nb, ctx->maxcell, ctx->state[ctx->cur].p, ctx->state[ctx->po].p, ctx->resid.p,
                      ctx->state[ctx->cur].p, ctx->gas, RKcoeff[ctx->cfg.n_rk - 1][irk - 1], ctx->derr.p, ctx->nd,
                      ctx->stream);
    ctx->launches++;
    return check_launch(ctx, "rk_stage");
  }
  launch_rk_stage(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->state[ctx->cur].p, ctx->state[ctx->po].p,
                  ctx->resid.p, ctx->margs(), ctx->dtl.p, ctx->gas, RKcoeff[ctx->cfg.n_rk - 1][irk - 1], ctx->nd,
                  ctx->uniform, ctx->derr.p, ctx->stream);
  ctx->launches++;
  return check_launch(ctx, "rk_stage");
}

// integration-variables = prim in the fp64 precision: each stage is the fp64
// residual kernel and Newstate_Primitive in its own kernel (the fused fp64
// stage kernels carry the conservative update only)
static bool prim_phased(const mose_gpu_ctx* ctx) {
  return ctx->gas.prim != 0 && ctx->cfg.precision == MOSE_PRECISION_FP64;
}
// Time-accurate runs fold the next step's Compute_dt (the CFL minimum) into
// the last RK stage, which holds the new state anyway.  With local time
// stepping each step keeps its standalone pass, so dtlocal always holds the
// dt of the step that used it, as in the reference.
static bool fused_dt(const mose_gpu_ctx* ctx) {
  return ctx->cfg.time_accurate != 0 && ctx->irs_beta == 0.0 && ctx->cfg.ramp_iter <= 0 && ctx->gas.model == 0 &&
         !ctx->adj_dt_standalone && !prim_phased(ctx);
}
static void fuse_next_dt(mose_gpu_ctx* ctx, StageArgs& a) {
  a.dtmin = ctx->dtmin.p;
  a.cfl = ctx->cfg.cfl;
  a.ndir = ctx->ndir;
  a.dt_local = 0;
}

// The standalone Compute_dt pass over state arena s0: dtmin = min over cells,
// starting from 1d5 (Mod_Explicit.f90:44); local dt stored when not time
// accurate.  Returns the number of kernels enqueued.
static int enqueue_dt_pass(mose_gpu_ctx* ctx, int s0) {
  launch_step_begin(ctx->dtmin.p, 1e5, nullptr, ctx->stream);
  // the CFL ramp (cfl-rise-threshold) reads the step's iteration on the
  // device: the completed steps + 1, as Explicit_Step increments iter first
  launch_compute_dt(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->state[s0].p, ctx->margs(), ctx->dtl.p,
                    ctx->dtmin.p, ctx->gas, ctx->cfg.cfl, ctx->ndir, ctx->nd, 0, ctx->cfg.ramp_iter,
                    ctx->cfg.time_accurate ? 0 : 1, ctx->uniform, ctx->stream, ctx->iterdev.p);
  return 2;
}

// Enqueues one fused Explicit_Step starting from state arena s0, whose CFL
// minimum is already in dtmin (the dt pass, or the previous step's last
// stage): publish dtglobal and advance time, then the RK stages; the last
// stage folds in the CFL minimum of the new state for the next step.
// Returns the number of kernels enqueued.
// Residual_Smoothing (Lib_IRS.f90:14-39) of the scaled residual in ctx->resid:
// per direction the first ghost layer, then two Jacobi sweeps (the second
// writes R).  Returns the kernel count.
static int enqueue_irs_smoothing(mose_gpu_ctx* ctx) {
  const size_t bytes = (size_t)ctx->nv * ctx->marena * sizeof(double);
  const int nb = (int)ctx->hblk.size();
  int k = 0;
  for (int dir = 0; dir < ctx->ndir; ++dir) {
    launch_irs_ghost(ctx->irs_list.p, ctx->nirs, ctx->resid.p, ctx->nd, ctx->stream);
    // the Jacobi sweeps read both copies: a failed copy is reported by the
    // step's check_launch instead of smoothing stale data silently
    for (double* dst : {ctx->rs1.p, ctx->rs2.p}) {
      const cudaError_t e = cudaMemcpyAsync(dst, ctx->resid.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
      if (e != cudaSuccess && ctx->enq_err == cudaSuccess) {
        ctx->enq_err = e;
        ctx->enq_what = "IRS residual copy";
      }
    }
    launch_irs_jacobi(ctx->d_desc.p, nb, ctx->maxcell, ctx->resid.p, ctx->rs1.p, ctx->rs2.p, dir, ctx->irs_beta,
                      ctx->nd, ctx->stream);
    launch_irs_jacobi(ctx->d_desc.p, nb, ctx->maxcell, ctx->resid.p, ctx->rs2.p, ctx->resid.p, dir, ctx->irs_beta,
                      ctx->nd, ctx->stream);
    k += (ctx->nirs > 0) + 2;
  }
  return k;
}

// One RK stage with implicit residual smoothing (Newstate_Conservative with
// IRS, Lib_Newstate.f90:40-72): the residual-only stage kernel into
// ctx->resid, Scale_Residual_Cons, the smoothing, Update_State_Cons_IRS from
// arena pc (PO = arena s0) into arena pn.
static int enqueue_irs_stage(mose_gpu_ctx* ctx, int pc, int s0, int pn, int irk) {
  StageArgs a = stage_args(ctx, pc, s0, -1, irk);
  // the residual in the context's arithmetic (exact, or fp64 with the
  // constant metrics of uniform grids); the smoothing and the update in the
  // reference's
  const bool fp64 = ctx->cfg.precision == MOSE_PRECISION_FP64;
  int k = launch_stage(ctx, a, 1, fp64 ? MOSE_PRECISION_FP64 : MOSE_PRECISION_FP64_EXACT, fp64 && ctx->uniform);
  const int nb = (int)ctx->hblk.size();
  launch_irs_scale(ctx->d_desc.p, nb, ctx->maxcell, ctx->state[pc].p, ctx->resid.p, ctx->margs(), ctx->dtl.p,
                   ctx->scal.p, ctx->cfg.time_accurate, ctx->gas, ctx->nd, ctx->stream);
  k += 1 + enqueue_irs_smoothing(ctx);
  launch_irs_update(ctx->d_desc.p, nb, ctx->maxcell, ctx->state[pc].p, ctx->state[s0].p, ctx->resid.p,
                    ctx->state[pn].p, ctx->gas, a.c_rk, ctx->derr.p, ctx->nd, ctx->stream);
  return k + 1;
}

// 402 inlets: p0 from the time tables at the device time (scal[1]), which
// Explicit_Step has already advanced to the end of the step when BC_Fluxes
// reads it (Mod_Explicit.f90:40-48, Mod_BC_Fluxes.f90:129-131).
static int enqueue_series(mose_gpu_ctx* ctx) {
  if (!ctx->nser) return 0;
  launch_series_p0(ctx->ser_recs.p, ctx->nser, ctx->ser_tv.p, ctx->scal.p + 1, ctx->bcp.p, ctx->stream);
  return 1;
}

static int enqueue_step(mose_gpu_ctx* ctx, int s0) {
  int k = 0;
  if (!fused_dt(ctx)) k += enqueue_dt_pass(ctx, s0);
  launch_step_dt_take(ctx->dtmin.p, ctx->scal.p, ctx->scal.p + 1, ctx->cfg.time_accurate, 1e5, ctx->iterdev.p,
                      ctx->stream); ++k;
  k += enqueue_series(ctx);
  int pc = s0;
  for (int irk = 1; irk <= ctx->cfg.n_rk; ++irk) {
    int pn = (irk == 1) ? (s0 + 1) % 3 : (pc == (s0 + 1) % 3 ? (s0 + 2) % 3 : (s0 + 1) % 3);
    k += enqueue_stage_ghosts(ctx, pc);
    if (ctx->irs_beta > 0.0) {
      k += enqueue_irs_stage(ctx, pc, s0, pn, irk);
    } else if (ctx->gas.model > 0 || prim_phased(ctx)) {
      // Navier-Stokes: the residual of every term; primitive integration in
      // fp64: the fp64 residual kernel; then Newstate
      StageArgs a = stage_args(ctx, pc, s0, pn, irk);
      if (ctx->gas.model > 0) {
        launch_visc_residual2d(a, (int)ctx->hblk.size(), ctx->maxcell, ctx->cfg.limiter, ctx->stream);
        ++k;   // the face pass and the cell pass
      } else
        k += launch_stage(ctx, a, 1, MOSE_PRECISION_FP64, ctx->uniform) - 1;
      launch_rk_stage_to(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->state[pc].p, ctx->state[s0].p,
                         ctx->resid.p, ctx->margs(), ctx->dtl.p, ctx->cfg.time_accurate ? ctx->scal.p : nullptr,
                         ctx->state[pn].p, ctx->gas, a.c_rk, ctx->nd, ctx->uniform, ctx->derr.p, ctx->stream);
      k += 2;
    } else {
      StageArgs a = stage_args(ctx, pc, s0, pn, irk);
      if (irk == ctx->cfg.n_rk && fused_dt(ctx)) fuse_next_dt(ctx, a);
      k += launch_stage(ctx, a, a.dtmin ? 2 : 0, ctx->cfg.precision, ctx->uniform);
    }
    pc = pn;
  }
  return k;
}

static int step_final_index(const mose_gpu_ctx* ctx, int s0) {
  int pc = s0;
  for (int irk = 1; irk <= ctx->cfg.n_rk; ++irk)
    pc = (irk == 1) ? (s0 + 1) % 3 : (pc == (s0 + 1) % 3 ? (s0 + 2) % 3 : (s0 + 1) % 3);
  return pc;
}

int mose_gpu_step(mose_gpu_ctx* ctx, double* dtglobal, double* time) {
  MOSE_NVTX_RANGE("mose_gpu_step");
  int rc = require_ready(ctx);
  if (rc) return rc;
  CU(cudaMemcpyAsync(ctx->scal.p + 1, &ctx->h_time, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->iterdev.p, &ctx->h_iter, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  int s0 = ctx->cur;
  if (fused_dt(ctx) && !ctx->dt_valid) ctx->launches += enqueue_dt_pass(ctx, s0);
  ctx->launches += enqueue_step(ctx, s0);
  rc = check_launch(ctx, "step");
  if (rc) return rc;
  ctx->dt_valid = fused_dt(ctx);
  ctx->po = s0;
  ctx->cur = step_final_index(ctx, s0);
  double h[2];
  CU(cudaMemcpyAsync(h, ctx->scal.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  rc = poll_device_error(ctx);
  ctx->h_iter += 1;
  ctx->h_time = h[1];
  if (dtglobal) *dtglobal = h[0];
  if (time) *time = h[1];
  return rc;
}

// Enqueues nsteps graph-replayed steps (one graph per starting arena,
// captured on first use); the device time and iteration are already set.
static int enqueue_graph_steps(mose_gpu_ctx* ctx, int nsteps) {
  if (nsteps > 0 && fused_dt(ctx) && !ctx->dt_valid) ctx->launches += enqueue_dt_pass(ctx, ctx->cur);
  for (int n = 0; n < nsteps; ++n) {
    int s0 = ctx->cur;
    const int gv = ctx->adj_dt_standalone ? 1 : 0;
    if (!ctx->graph[gv][s0]) {
      cudaGraph_t g;
      CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      int k = enqueue_step(ctx, s0);
      CU(cudaStreamEndCapture(ctx->stream, &g));
      if (int rc = check_launch(ctx, "step capture")) {
        cudaGraphDestroy(g);
        return rc;
      }
      CU(cudaGraphInstantiate(&ctx->graph[gv][s0], g, 0));
      cudaGraphDestroy(g);
      ctx->graph_kernels[gv] = k;
    }
    CU(cudaGraphLaunch(ctx->graph[gv][s0], ctx->stream));
    ctx->launches += ctx->graph_kernels[gv];
    ctx->dt_valid = fused_dt(ctx);
    ctx->po = s0;
    ctx->cur = step_final_index(ctx, s0);
  }
  return MOSE_OK;
}

int mose_gpu_advance(mose_gpu_ctx* ctx, int32_t nsteps, double* dtglobal, double* time) {
  MOSE_NVTX_RANGE("mose_gpu_advance");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (nsteps < 0) return MOSE_ERR_INVALID;
  CU(cudaMemcpyAsync(ctx->scal.p + 1, &ctx->h_time, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->iterdev.p, &ctx->h_iter, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  rc = enqueue_graph_steps(ctx, nsteps);
  if (rc) return rc;
  double h[2];
  CU(cudaMemcpyAsync(h, ctx->scal.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  rc = poll_device_error(ctx);
  ctx->h_iter += nsteps;
  ctx->h_time = h[1];
  if (dtglobal) *dtglobal = h[0];
  if (time) *time = h[1];
  return rc;
}

int mose_gpu_residual_norms(mose_gpu_ctx* ctx, double* total) {
  MOSE_NVTX_RANGE("mose_gpu_residual_norms");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (!total) return MOSE_ERR_INVALID;
  launch_residual_norms(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->state[ctx->cur].p,
                        ctx->state[ctx->po].p, ctx->nd, ctx->partial.p, ctx->norms.p, ctx->stream);
  ctx->launches += 2;
  CU(cudaMemcpyAsync(total, ctx->norms.p, 5 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return check_launch(ctx, "residual_norms");
}

int mose_gpu_set_time(mose_gpu_ctx* ctx, double time, int32_t iter) {
  MOSE_NVTX_RANGE("mose_gpu_set_time");
  if (!ctx) return MOSE_ERR_INVALID;
  ctx->h_time = time;
  ctx->h_iter = iter;
  return MOSE_OK;
}

int mose_gpu_get_time(mose_gpu_ctx* ctx, double* time, int32_t* iter) {
  if (!ctx) return MOSE_ERR_INVALID;
  if (time) *time = ctx->h_time;
  if (iter) *iter = ctx->h_iter;
  return MOSE_OK;
}

int mose_gpu_synchronize(mose_gpu_ctx* ctx) {
  MOSE_NVTX_RANGE("mose_gpu_synchronize");
  int rc = require_ready(ctx);
  if (rc) return rc;
  CU(cudaStreamSynchronize(ctx->stream));
  rc = check_launch(ctx, "synchronize");
  if (rc) return rc;
  return poll_device_error(ctx);
}

void* mose_gpu_stream(const mose_gpu_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int mose_gpu_time_kernels(mose_gpu_ctx* ctx, int32_t nsteps, double* ms, int32_t* launches) {
  MOSE_NVTX_RANGE("mose_gpu_time_kernels");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (!ms || !launches || nsteps < 1) return MOSE_ERR_INVALID;
  for (int c = 0; c < 3; ++c) { ms[c] = 0.0; launches[c] = 0; }
  CU(cudaMemcpyAsync(ctx->scal.p + 1, &ctx->h_time, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(ctx->iterdev.p, &ctx->h_iter, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  std::vector<cudaEvent_t> ev;
  std::vector<int> cls;
  auto mark = [&](int c) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, ctx->stream);
    ev.push_back(e);
    cls.push_back(c);
  };
  for (int n = 0; n < nsteps; ++n) {
    int s0 = ctx->cur;
    mark(-1);
    if (!fused_dt(ctx) || !ctx->dt_valid) launches[0] += enqueue_dt_pass(ctx, s0);
    launch_step_dt_take(ctx->dtmin.p, ctx->scal.p, ctx->scal.p + 1, ctx->cfg.time_accurate, 1e5, ctx->iterdev.p,
                        ctx->stream);
    launches[0] += 1 + enqueue_series(ctx);
    mark(0);
    int pc = s0;
    for (int irk = 1; irk <= ctx->cfg.n_rk; ++irk) {
      int pn = (irk == 1) ? (s0 + 1) % 3 : (pc == (s0 + 1) % 3 ? (s0 + 2) % 3 : (s0 + 1) % 3);
      const int ng = enqueue_stage_ghosts(ctx, pc);
      if (ng) {
        mark(1);
        launches[1] += ng;
      }
      StageArgs a = stage_args(ctx, pc, s0, pn, irk);
      if (irk == ctx->cfg.n_rk && fused_dt(ctx)) fuse_next_dt(ctx, a);
      launches[2] += launch_stage(ctx, a, a.dtmin ? 2 : 0, ctx->cfg.precision, ctx->uniform);
      mark(2);
      pc = pn;
    }
    ctx->dt_valid = fused_dt(ctx);
    ctx->po = s0;
    ctx->cur = pc;
  }
  ctx->launches += launches[0] + launches[1] + launches[2];
  CU(cudaStreamSynchronize(ctx->stream));
  rc = check_launch(ctx, "time_kernels");
  for (size_t q = 1; q < ev.size(); ++q) {
    if (cls[q] < 0) continue;
    float t = 0.f;
    cudaEventElapsedTime(&t, ev[q - 1], ev[q]);
    ms[cls[q]] += t;
  }
  for (auto e : ev) cudaEventDestroy(e);
  double h[2];
  CU(cudaMemcpy(h, ctx->scal.p, 2 * sizeof(double), cudaMemcpyDeviceToHost));
  ctx->h_time = h[1];
  ctx->h_iter += nsteps;
  if (rc) return rc;
  return poll_device_error(ctx);
}

int mose_gpu_uniform_metrics(const mose_gpu_ctx* ctx) { return ctx && ctx->uniform ? 1 : 0; }
int64_t mose_gpu_launch_count(const mose_gpu_ctx* ctx) { return ctx ? ctx->launches : -1; }

int mose_gpu_download_metrics(mose_gpu_ctx* ctx, int32_t b, double* vol, double* dl) {
  MOSE_NVTX_RANGE("mose_gpu_download_metrics");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (b < 1 || b > (int)ctx->hblk.size()) return fail(ctx, MOSE_ERR_INVALID, "bad block");
  const HostBlock& h = ctx->hblk[b - 1];
  long long n = (long long)(h.ni + 4) * (h.nj + 4) * (h.nk + 4);
  DevBuf<double> v, l;
  if (vol) CU(v.alloc(n));
  if (dl) CU(l.alloc(3 * n));
  launch_metrics_to_ref(ctx->d_desc.p, b - 1, n, ctx->margs(), v.p, l.p, ctx->nd, ctx->stream);
  ctx->launches++;
  CU(cudaStreamSynchronize(ctx->stream));
  if (vol) CU(cudaMemcpy(vol, v.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  if (dl) CU(cudaMemcpy(dl, l.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
  return check_launch(ctx, "download_metrics");
}

int mose_gpu_download_faces(mose_gpu_ctx* ctx, int32_t b, int32_t dir, double* N, double* A) {
  MOSE_NVTX_RANGE("mose_gpu_download_faces");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (b < 1 || b > (int)ctx->hblk.size() || dir < 1 || dir > ctx->nd) return fail(ctx, MOSE_ERR_INVALID, "bad args");
  const HostBlock& h = ctx->hblk[b - 1];
  int d0 = dir - 1;
  long long n = (long long)(h.ni + (d0 == 0)) * (h.nj + (d0 == 1)) * (h.nk + (d0 == 2));
  DevBuf<double> nn, aa;
  if (N) CU(nn.alloc(3 * n));
  if (A) CU(aa.alloc(n));
  launch_faces_to_ref(ctx->d_desc.p, b - 1, n, ctx->margs(), d0, nn.p, aa.p, ctx->nd, ctx->stream);
  ctx->launches++;
  CU(cudaStreamSynchronize(ctx->stream));
  if (N) CU(cudaMemcpy(N, nn.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
  if (A) CU(cudaMemcpy(A, aa.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  return check_launch(ctx, "download_faces");
}


// ---- discrete adjoint (kernels in adjoint.cu) -------------------------------------
static double rk_coeff(const mose_gpu_ctx* ctx, int irk) {
  static const double RKcoeff[3][3] = {{1.0, 0.0, 0.0}, {1.0, 0.50, 0.0}, {1.0, 0.25, 2.0 / 3.0}};
  return RKcoeff[ctx->cfg.n_rk - 1][irk - 1];
}

// Buffers and work lists of the adjoint, made on first use.
// Splits the face groups first[0..4] into launches: a face joins the current
// launch when none of the cells its entries touch (cells(q) of entry q) is
// touched by the faces already in it, so every cell sees the same updates in
// the same order as with one launch per face.  Returns the entry offsets at
// which launches start, followed by first[4].
static std::vector<int> face_passes(const int first[5],
                                    const std::function<void(int, std::vector<long long>&)>& cells) {
  std::vector<int> pass{first[0]};
  std::vector<long long> in_pass, face, c;
  for (int f = 0; f < 4; ++f) {
    face.clear();
    for (int q = first[f]; q < first[f + 1]; ++q) {
      c.clear();
      cells(q, c);
      face.insert(face.end(), c.begin(), c.end());
    }
    std::sort(face.begin(), face.end());
    face.erase(std::unique(face.begin(), face.end()), face.end());
    bool overlap = false;
    for (long long x : face)
      if (std::binary_search(in_pass.begin(), in_pass.end(), x)) { overlap = true; break; }
    if (overlap) {
      pass.push_back(first[f]);
      in_pass.clear();
    }
    std::vector<long long> u;
    std::merge(in_pass.begin(), in_pass.end(), face.begin(), face.end(), std::back_inserter(u));
    in_pass.swap(u);
  }
  pass.push_back(first[4]);
  return pass;
}

// (block, i, j) as one key; i and j lie within GW of the block.
static long long cell_key(int b, int i, int j) {
  return ((long long)b << 40) | ((long long)(i + 16) << 20) | (long long)(j + 16);
}

static int adj_prepare(mose_gpu_ctx* ctx) {
  if (ctx->adj_init) return MOSE_OK;
  if (ctx->nd != 2) return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: 2-D domains only");
  if (ctx->cfg.riemann != MOSE_RIEMANN_HLLC || ctx->cfg.limiter < 1 || ctx->cfg.limiter > 3)
    return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: HLLC with minmod, van Leer or van Albada");
  if (!ctx->cfg.time_accurate) return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: time-accurate runs only");
  if (ctx->cfg.ramp_iter > 0) return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: no cfl ramp");
  if (ctx->irs_beta > 0.0 || ctx->gas.sd) return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: no IRS or shock detector");
  if (ctx->nser) return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: no time-table (402) inlets");
  if (ctx->gas.prim) return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: conservative integration variables only");
  if (ctx->gas.model > 0) return fail(ctx, MOSE_ERR_UNSUPPORTED, "adjoint: the Euler step only");
  const size_t ns = (size_t)ctx->nv * ctx->marena, m = (size_t)ctx->marena;
  for (DevBuf<double>* b : {&ctx->lam, &ctx->lam_loc, &ctx->lam_n, &ctx->lamR, &ctx->wdt, &ctx->lamG})
    if (b->alloc(ns) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (adjoint)");
  if (ctx->Cx.alloc(16 * m) != cudaSuccess || ctx->Cy.alloc(16 * m) != cudaSuccess || ctx->Fx.alloc(4 * m) != cudaSuccess ||
      ctx->Fy.alloc(4 * m) != cudaSuccess || ctx->dtpart.alloc(m) != cudaSuccess)
    return fail(ctx, MOSE_ERR_CUDA, "out of device memory (adjoint)");
  CU(ctx->adj_scal.alloc(4));
  CU(cudaStreamCreateWithFlags(&ctx->adj_aux, cudaStreamNonBlocking));
  CU(cudaEventCreateWithFlags(&ctx->adj_fork, cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&ctx->adj_join, cudaEventDisableTiming));
  CU(ctx->adj_arg.alloc(1));
  CU(ctx->adj_sumscr.alloc(adj_sum_scratch()));
  // boundary face cells of faces 1..4, grouped by face: one k_adj_bc entry
  // each, whose stencil contributions k_adj_gather adds per cell
  std::vector<int4> list;
  size_t nent = 0, maxface = 1;
  for (const BlockDesc& d : ctx->desc) {
    for (int f = 0; f < 6; ++f) nent = std::max(nent, (size_t)(d.bcoff[f] + d.bcn[f]));
    maxface = std::max(maxface, (size_t)std::max(d.ni, d.nj));
  }
  for (int f = 1; f <= 4; ++f) {
    ctx->adj_bcfirst[f - 1] = (int)list.size();
    for (int b = 0; b < (int)ctx->desc.size(); ++b) {
      const BlockDesc& d = ctx->desc[b];
      for (int idx = 0; idx < d.bcn[f - 1]; ++idx) list.push_back(make_int4(b, f, idx, d.bcoff[f - 1] + idx));
    }
  }
  ctx->adj_bcfirst[4] = (int)list.size();
  CU(ctx->adj_bclist.alloc(std::max<size_t>(list.size(), 1)));
  if (!list.empty())
    CU(cudaMemcpyAsync(ctx->adj_bclist.p, list.data(), list.size() * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
  if (ctx->Cb.alloc(16 * std::max<size_t>(nent, 1)) != cudaSuccess || ctx->Fbc.alloc(4 * std::max<size_t>(nent, 1)) != cudaSuccess ||
      ctx->dmach.alloc(std::max<size_t>(nent, 1)) != cudaSuccess || ctx->objt.alloc(maxface) != cudaSuccess)
    return fail(ctx, MOSE_ERR_CUDA, "out of device memory (adjoint)");
  std::vector<int> gids;
  for (int f = 1; f <= 4; ++f) {
    ctx->adj_gfirst[f - 1] = (int)gids.size();
    for (int q = 0; q < (int)ctx->hghost.size(); ++q)
      if (ctx->hghost[q].f == f) gids.push_back(q);
  }
  ctx->adj_gfirst[4] = (int)gids.size();
  ctx->adj_gpass = face_passes(ctx->adj_gfirst, [&](int q, std::vector<long long>& c) {
    // the cells k_adj_ghostT reads and writes for the record
    const GhostRec& e = ctx->hghost[gids[q]];
    const int gi = (e.f == 1) ? 1 : (e.f == 2) ? -1 : 0;
    const int gj = (e.f == 3) ? 1 : (e.f == 4) ? -1 : 0;
    const int lo = e.type == BC_CONN ? 1 : e.type == BC_EXTRAP ? -GW : 0;
    for (int g = lo; g <= GW; ++g) c.push_back(cell_key(e.b, e.i - gi * g, e.j - gj * g));
    if (e.type == BC_CONN) {
      const int si = (e.fs == 1) ? 1 : (e.fs == 2) ? -1 : 0;
      const int sj = (e.fs == 3) ? 1 : (e.fs == 4) ? -1 : 0;
      for (int g = 1; g <= GW; ++g) c.push_back(cell_key(e.bs, e.is + si * (g - 1), e.js + sj * (g - 1)));
    }
  });
  CU(ctx->adj_gids.alloc(std::max<size_t>(gids.size(), 1)));
  if (!gids.empty())
    CU(cudaMemcpyAsync(ctx->adj_gids.p, gids.data(), gids.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  ctx->adj_init = true;
  return MOSE_OK;
}

static int adj_segment_buffers(mose_gpu_ctx* ctx, int K) {
  const size_t ns = (size_t)ctx->nv * ctx->marena;
  if ((int)ctx->adj_seg.size() < 3 * K + 1) {
    const size_t old = ctx->adj_seg.size();
    ctx->adj_seg.resize(3 * (size_t)K + 1);
    for (size_t q = old; q < ctx->adj_seg.size(); ++q)
      if (ctx->adj_seg[q].alloc(ns) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (segment)");
  }
  if ((int)ctx->adj_dts.n < K) {
    destroy_adjoint_graphs(ctx);   // they hold adj_dts
    if (ctx->adj_dts.alloc(K) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (segment)");
  }
  return MOSE_OK;
}

// Recomputes cnt Explicit_Steps from adj_seg[0] along the chain: the
// standalone Compute_dt of the first state, the fused CFL minimum of each
// later one (the last stage of the step before), every RK stage reading its
// input slot (ghosts filled in place) and writing the next; the steps' dt
// into adj_dts.  Returns the number of kernels enqueued.
static int enqueue_record(mose_gpu_ctx* ctx, int cnt) {
  cudaStream_t st = ctx->stream;
  launch_step_begin(ctx->dtmin.p, 1e5, nullptr, st);
  launch_compute_dt(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->adj_seg[0].p, ctx->margs(), ctx->dtl.p,
                    ctx->dtmin.p, ctx->gas, ctx->cfg.cfl, ctx->ndir, ctx->nd, 0, 0, 0, ctx->uniform, st);
  int kern = 2;
  const int nrk = ctx->cfg.n_rk;
  // the exact precision folds each next dt into the last stage; the others
  // take it from the standalone pass, as their forward did
  const bool fuse_ok = ctx->cfg.precision == MOSE_PRECISION_FP64_EXACT;
  for (int k = 0; k < cnt; ++k) {
    if (k > 0 && !fuse_ok) {
      launch_step_begin(ctx->dtmin.p, 1e5, nullptr, st);
      launch_compute_dt(ctx->d_desc.p, (int)ctx->hblk.size(), ctx->maxcell, ctx->adj_seg[3 * (size_t)k].p,
                        ctx->margs(), ctx->dtl.p, ctx->dtmin.p, ctx->gas, ctx->cfg.cfl, ctx->ndir, ctx->nd, 0, 0, 0,
                        ctx->uniform, st);
      kern += 2;
    }
    launch_step_dt_take(ctx->dtmin.p, ctx->scal.p, ctx->scal.p + 1, ctx->cfg.time_accurate, 1e5, ctx->iterdev.p, st);
    cudaMemcpyAsync(ctx->adj_dts.p + k, ctx->scal.p, sizeof(double), cudaMemcpyDeviceToDevice, st);
    ++kern;
    for (int irk = 1; irk <= nrk; ++irk) {
      double* Pc = ctx->adj_seg[3 * (size_t)k + irk - 1].p;
      kern += enqueue_fill(ctx, Pc, false, st);
      StageArgs a = stage_args(ctx, 0, 0, -1, irk);
      a.Pc = Pc;
      a.Po = ctx->adj_seg[3 * (size_t)k].p;
      a.Pn = ctx->adj_seg[irk == nrk ? 3 * (size_t)(k + 1) : 3 * (size_t)k + irk].p;
      const bool fuse = fuse_ok && irk == nrk && k + 1 < cnt;
      if (fuse) fuse_next_dt(ctx, a);
      kern += launch_stage(ctx, a, fuse ? 2 : 0, ctx->cfg.precision, ctx->uniform);
    }
  }
  return kern;
}

// The adjoint of recorded step k of the chain: ctx->lam holds dJ/dP^{k+1}
// on entry and dJ/dP^k on exit.  dJ/dMach accumulates in adj_scal[1].  The
// boundary faces and the dt argmin run on the side stream, beside the
// interior faces.  Returns the number of kernels enqueued.
static int adj_reverse_step(mose_gpu_ctx* ctx, int k) {
  cudaStream_t st = ctx->stream, aux = ctx->adj_aux;
  const size_t ns = (size_t)ctx->nv * ctx->marena;
  const int nrk = ctx->cfg.n_rk;
  const double* S[4];
  for (int q = 0; q < nrk; ++q) S[q] = ctx->adj_seg[3 * (size_t)k + q].p;
  S[nrk] = ctx->adj_seg[3 * (size_t)(k + 1)].p;
  const double* dtg = ctx->adj_dts.p + k;
  const int nb = (int)ctx->hblk.size(), lim = ctx->cfg.limiter;
  const MetricArgs m = ctx->margs();
  const int nlist = ctx->adj_bcfirst[4];
  int kern = 0;
  cudaMemsetAsync(ctx->lam_n.p, 0, ns * sizeof(double), st);
  cudaMemsetAsync(ctx->dtpart.p, 0, ctx->marena * sizeof(double), st);
  if (nlist) cudaMemsetAsync(ctx->dmach.p, 0, ctx->dmach.n * sizeof(double), st);
  // the step's dt = min over cells of the CFL dt of P^k: its argmin cell
  cudaMemsetAsync(ctx->adj_arg.p, 0xff, sizeof(unsigned long long), st);
  cudaEventRecord(ctx->adj_fork, st);
  cudaStreamWaitEvent(aux, ctx->adj_fork, 0);
  for (int b = 0; b < nb; ++b)
    launch_dt_argmin(ctx->d_desc.p, b, ctx->hblk[b].ni, ctx->hblk[b].nj, m, ctx->gas, S[0], dtg, ctx->cfg.cfl,
                     ctx->ndir, ctx->uniform, ctx->adj_arg.p, aux);
  kern += nb;
  for (int irk = nrk; irk >= 1; --irk) {
    const double* Ps = S[irk];
    const double* Pprev = S[irk - 1];
    const double c = rk_coeff(ctx, irk);
    // the adjoint of stage irk's output: lam for the last stage, else the
    // later stage's lam_loc + lamG
    for (int b = 0; b < nb; ++b)
      adj_pre(ctx->d_desc.p, b, ctx->hblk[b].ni, ctx->hblk[b].nj, m, ctx->gas, Ps, Pprev, S[0], ctx->lam.p,
              irk == nrk ? nullptr : ctx->lamG.p, ctx->lamR.p, ctx->wdt.p, ctx->lam_loc.p, ctx->lam_n.p, c, dtg, st);
    if (nlist) {
      StageArgs a = stage_args(ctx, 0, 0, -1, irk);
      a.Pc = Pprev;
      cudaEventRecord(ctx->adj_fork, st);
      cudaStreamWaitEvent(aux, ctx->adj_fork, 0);
      adj_bc(a, lim, ctx->adj_bclist.p, nlist, ctx->lamR.p, ctx->Cb.p, ctx->Fbc.p, ctx->dmach.p, aux);
      ++kern;
    }
    for (int b = 0; b < nb; ++b)
      adj_faces(ctx->d_desc.p, b, ctx->hblk[b].ni, ctx->hblk[b].nj, m, ctx->gas, lim, Pprev, ctx->lamR.p, ctx->Cx.p,
                ctx->Fx.p, ctx->Cy.p, ctx->Fy.p, st);
    cudaEventRecord(ctx->adj_join, aux);
    cudaStreamWaitEvent(st, ctx->adj_join, 0);
    // interior and boundary faces' contributions, per cell
    for (int b = 0; b < nb; ++b)
      adj_gather(ctx->d_desc.p, b, ctx->hblk[b].ni, ctx->hblk[b].nj, ctx->Cx.p, ctx->Cy.p, ctx->Fx.p, ctx->Fy.p,
                 nlist ? ctx->Cb.p : nullptr, nlist ? ctx->Fbc.p : nullptr, ctx->wdt.p, ctx->lamG.p, ctx->dtpart.p,
                 st);
    for (size_t q = 0; q + 1 < ctx->adj_gpass.size(); ++q) {
      const int n = ctx->adj_gpass[q + 1] - ctx->adj_gpass[q];
      adj_ghost_transpose(ctx->d_desc.p, ctx->ghosts.p, ctx->adj_gids.p + ctx->adj_gpass[q], n, m, ctx->lamG.p, st);
      kern += n > 0;
    }
    kern += 3 * nb;   // pre, faces, gather
  }
  // dJ/ddt of this step; dJ/dMach accumulates over the steps
  if (nlist)
    adj_sum2(ctx->dtpart.p, ctx->marena, ctx->adj_scal.p, 0, ctx->dmach.p, (long long)ctx->dmach.n,
             ctx->adj_scal.p + 1, 1, ctx->adj_sumscr.p, st);
  else
    adj_sum(ctx->dtpart.p, ctx->marena, ctx->adj_scal.p, 0, ctx->adj_sumscr.p, st);
  kern += 2;
  adj_dt(ctx->d_desc.p, m, ctx->gas, S[0], ctx->adj_arg.p, ctx->adj_scal.p, ctx->cfg.cfl, ctx->ndir, ctx->lam_n.p, st);
  // lam = the first stage's lam_loc + lamG, plus the direct terms of P^n
  for (int b = 0; b < nb; ++b)
    adj_combine(ctx->d_desc.p, b, ctx->hblk[b].ni, ctx->hblk[b].nj, ctx->lam_loc.p, ctx->lamG.p, ctx->lam_n.p,
                ctx->lam.p, st);
  return kern + 1 + nb;
}

// (Re)builds the graphs of a K-step segment: the recompute of a full
// segment and the reverse of each of its steps (the same buffers serve
// every segment).
static int adj_graphs(mose_gpu_ctx* ctx, int K) {
  if (ctx->adj_graph_K == K) return MOSE_OK;
  destroy_adjoint_graphs(ctx);
  cudaGraph_t g;
  CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  ctx->adj_rec_kernels = enqueue_record(ctx, K);
  CU(cudaStreamEndCapture(ctx->stream, &g));
  CU(cudaGraphInstantiate(&ctx->adj_recgraph, g, 0));
  cudaGraphDestroy(g);
  ctx->adj_rgraph.assign(K, nullptr);
  for (int k = 0; k < K; ++k) {
    CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->adj_rev_kernels = adj_reverse_step(ctx, k);
    CU(cudaStreamEndCapture(ctx->stream, &g));
    CU(cudaGraphInstantiate(&ctx->adj_rgraph[k], g, 0));
    cudaGraphDestroy(g);
  }
  ctx->adj_graph_K = K;
  return MOSE_OK;
}

int mose_gpu_set_sd_limiter(mose_gpu_ctx* ctx, int32_t on) {
  MOSE_NVTX_RANGE("mose_gpu_set_sd_limiter");
  if (!ctx) return MOSE_ERR_INVALID;
  if (ctx->ready) return fail(ctx, MOSE_ERR_INVALID, "set_sd_limiter: call before mose_gpu_setup");
  ctx->gas.sd = (ctx->gas.sd & ~1) | (on ? 1 : 0);
  return MOSE_OK;
}

int mose_gpu_set_viscous(mose_gpu_ctx* ctx, int32_t model, double mu, double kappa, double vnn) {
  MOSE_NVTX_RANGE("mose_gpu_set_viscous");
  if (!ctx) return MOSE_ERR_INVALID;
  if (ctx->ready) return fail(ctx, MOSE_ERR_INVALID, "set_viscous must precede setup");
  if (model == 0) {
    ctx->gas.model = 0;
    return MOSE_OK;
  }
  if (model != 1) return fail(ctx, MOSE_ERR_UNSUPPORTED, "model %d: only 0 (Euler) and 1 (laminar) are on this path", model);
  if (!(mu > 0.0) || !(kappa >= 0.0) || !(vnn > 0.0) || !std::isfinite(mu) || !std::isfinite(kappa) ||
      !std::isfinite(vnn))
    return fail(ctx, MOSE_ERR_INVALID, "viscous constants: need mu > 0, kappa >= 0, vnn > 0");
  ctx->gas.model = 1;
  ctx->gas.mu = mu;
  ctx->gas.kappa = kappa;
  ctx->gas.vnn = vnn;
  return MOSE_OK;
}

int mose_gpu_set_irs_beta(mose_gpu_ctx* ctx, double beta) {
  MOSE_NVTX_RANGE("mose_gpu_set_irs_beta");
  if (!ctx) return MOSE_ERR_INVALID;
  if (ctx->ready) return fail(ctx, MOSE_ERR_INVALID, "set_irs_beta: call before mose_gpu_setup");
  if (!(beta >= 0.0)) return fail(ctx, MOSE_ERR_INVALID, "set_irs_beta: beta must be >= 0");
  ctx->irs_beta = beta;
  return MOSE_OK;
}

int mose_gpu_set_riemann_minf(mose_gpu_ctx* ctx, double minf) {
  MOSE_NVTX_RANGE("mose_gpu_set_riemann_minf");
  if (!ctx) return MOSE_ERR_INVALID;
  if (ctx->ready) return fail(ctx, MOSE_ERR_INVALID, "set_riemann_minf: call before mose_gpu_setup");
  if (!(minf >= 0.0)) return fail(ctx, MOSE_ERR_INVALID, "set_riemann_minf: Minf must be >= 0");
  ctx->gas.minf = minf;
  return MOSE_OK;
}

int mose_gpu_set_inflow_mach(mose_gpu_ctx* ctx, double mach) {
  MOSE_NVTX_RANGE("mose_gpu_set_inflow_mach");
  int rc = require_ready(ctx);
  if (rc) return rc;
  bool any = false;
  for (auto& e : ctx->bc)
    if (e.type == 405) any = true;
  if (!any) return fail(ctx, MOSE_ERR_INVALID, "no 405 inflow faces");
  // every record with a parameter slot (401 - 407) holds it in bc order;
  // only 405 has a Mach number
  size_t q = 0;
  for (auto& e : ctx->bc) {
    if (e.type == 405) ctx->hbcp[q].mach = mach;
    if (e.type >= 401 && e.type <= 407) ++q;
  }
  CU(cudaMemcpyAsync(ctx->bcp.p, ctx->hbcp.data(), ctx->hbcp.size() * sizeof(BcParam), cudaMemcpyHostToDevice,
                     ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  ctx->dt_valid = false;
  return MOSE_OK;
}

int mose_gpu_adjoint_forward(mose_gpu_ctx* ctx, int32_t nsteps, int32_t interval, int32_t block, int32_t face,
                             double* J) {
  MOSE_NVTX_RANGE("mose_gpu_adjoint_forward");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (nsteps < 1 || interval < 1 || !J) return fail(ctx, MOSE_ERR_INVALID, "adjoint_forward: bad arguments");
  if (block < 1 || block > (int)ctx->hblk.size() || face < 1 || face > 4)
    return fail(ctx, MOSE_ERR_INVALID, "adjoint_forward: objective face must be face 1..4 of a block");
  rc = adj_prepare(ctx);
  if (rc) return rc;
  const size_t ns = (size_t)ctx->nv * ctx->marena;
  const int nck = (nsteps + interval - 1) / interval;
  if ((int)ctx->adj_ckpt.size() < nck) {
    const size_t old = ctx->adj_ckpt.size();
    ctx->adj_ckpt.resize(nck);
    for (size_t q = old; q < ctx->adj_ckpt.size(); ++q)
      if (ctx->adj_ckpt[q].alloc(ns) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (checkpoints)");
  }
  rc = adj_segment_buffers(ctx, interval);
  if (rc) return rc;
  ctx->adj_dt_standalone = ctx->cfg.precision != MOSE_PRECISION_FP64_EXACT;
  for (int mck = 0; mck < nck; ++mck) {
    CU(cudaMemcpyAsync(ctx->adj_ckpt[mck].p, ctx->state[ctx->cur].p, ns * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    const int cnt = std::min(interval, nsteps - mck * interval);
    rc = mose_gpu_advance(ctx, cnt, nullptr, nullptr);
    if (rc) {
      ctx->adj_dt_standalone = false;
      return rc;
    }
  }
  ctx->adj_dt_standalone = false;
  ctx->dt_valid = false;   // the next fused step starts from the standalone pass
  // the objective on the final state
  const BlockDesc& d = ctx->desc[block - 1];
  const int nf = (face <= 2) ? d.nj : d.ni;
  CU(cudaMemsetAsync(ctx->lam.p, 0, ns * sizeof(double), ctx->stream));
  adj_objective(ctx->d_desc.p, block - 1, face, nf, ctx->margs(), ctx->state[ctx->cur].p, ctx->objt.p, ctx->lam.p,
                ctx->stream);
  adj_sum(ctx->objt.p, nf, ctx->adj_scal.p + 2, 0, ctx->adj_sumscr.p, ctx->stream);
  CU(cudaMemcpyAsync(J, ctx->adj_scal.p + 2, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  ctx->adj_nsteps = nsteps;
  ctx->adj_interval = interval;
  ctx->adj_block = block;
  ctx->adj_face = face;
  ctx->adj_recorded = true;
  return check_launch(ctx, "adjoint_forward");
}

int mose_gpu_adjoint_backward(mose_gpu_ctx* ctx, double* dJ_dmach) {
  MOSE_NVTX_RANGE("mose_gpu_adjoint_backward");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (!ctx->adj_recorded) return fail(ctx, MOSE_ERR_INVALID, "adjoint_backward needs a preceding adjoint_forward");
  const size_t ns = (size_t)ctx->nv * ctx->marena;
  const int N = ctx->adj_nsteps, K = ctx->adj_interval, nck = (N + K - 1) / K;
  const double h_time = ctx->h_time;
  rc = adj_graphs(ctx, K);
  if (rc) return rc;
  CU(cudaMemsetAsync(ctx->adj_scal.p + 1, 0, sizeof(double), ctx->stream));
  for (int mck = nck - 1; mck >= 0; --mck) {
    const int cnt = std::min(K, N - mck * K);
    // recompute the segment from its checkpoint along the chain, then its
    // steps in reverse (the state arenas keep the forward run's final state)
    CU(cudaMemcpyAsync(ctx->adj_seg[0].p, ctx->adj_ckpt[mck].p, ns * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    if (cnt == K) {
      CU(cudaGraphLaunch(ctx->adj_recgraph, ctx->stream));
      ctx->launches += ctx->adj_rec_kernels;
    } else {
      ctx->launches += enqueue_record(ctx, cnt);
    }
    for (int k = cnt - 1; k >= 0; --k) {
      CU(cudaGraphLaunch(ctx->adj_rgraph[k], ctx->stream));
      ctx->launches += ctx->adj_rev_kernels;
    }
    rc = check_launch(ctx, "adjoint_backward");
    if (rc) return rc;
  }
  // the forward run's time (the recompute advanced the device clock)
  ctx->h_time = h_time;
  ctx->dt_valid = false;
  double h = 0.0;
  CU(cudaMemcpyAsync(&h, ctx->adj_scal.p + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  rc = poll_device_error(ctx);
  if (dJ_dmach) *dJ_dmach = h;
  ctx->adj_recorded = false;
  return rc;
}

int mose_gpu_adjoint_step(mose_gpu_ctx* ctx, double* dJ_dmach) {
  MOSE_NVTX_RANGE("mose_gpu_adjoint_step");
  int rc = require_ready(ctx);
  if (rc) return rc;
  rc = adj_prepare(ctx);
  if (rc) return rc;
  rc = adj_segment_buffers(ctx, 1);
  if (rc) return rc;
  const size_t ns = (size_t)ctx->nv * ctx->marena;
  const double h_time = ctx->h_time;
  CU(cudaMemsetAsync(ctx->adj_scal.p + 1, 0, sizeof(double), ctx->stream));
  CU(cudaMemcpyAsync(ctx->adj_seg[0].p, ctx->state[ctx->cur].p, ns * sizeof(double), cudaMemcpyDeviceToDevice,
                     ctx->stream));
  ctx->launches += enqueue_record(ctx, 1);
  ctx->launches += adj_reverse_step(ctx, 0);
  // the state arenas still hold P^n
  ctx->h_time = h_time;
  ctx->dt_valid = false;
  double h = 0.0;
  CU(cudaMemcpyAsync(&h, ctx->adj_scal.p + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  rc = poll_device_error(ctx);
  if (dJ_dmach) *dJ_dmach = h;
  return rc ? rc : check_launch(ctx, "adjoint_step");
}

int mose_gpu_upload_adjoint(mose_gpu_ctx* ctx, int32_t b, const double* lam) {
  MOSE_NVTX_RANGE("mose_gpu_upload_adjoint");
  int rc = require_ready(ctx);
  if (rc) return rc;
  rc = adj_prepare(ctx);
  if (rc) return rc;
  return prim_io(ctx, b, const_cast<double*>(lam), -2, true);
}
int mose_gpu_download_adjoint(mose_gpu_ctx* ctx, int32_t b, double* lam) { return prim_io(ctx, b, lam, -2, false); }

// ---- 2-D work-list tiling and its autotuner ------------------------------------
int mose_gpu_get_tiling(const mose_gpu_ctx* ctx, int32_t* tiling) {
  MOSE_NVTX_RANGE("mose_gpu_download_adjoint");
  if (!ctx || !tiling) return MOSE_ERR_INVALID;
  tiling[0] = ctx->tile_h; tiling[1] = ctx->tile_w; tiling[2] = ctx->tile_order; tiling[3] = ctx->tile_ctas;
  return MOSE_OK;
}

static int apply_tiling(mose_gpu_ctx* ctx, int h, int w, int order, int ctas) {
  CU(cudaStreamSynchronize(ctx->stream));
  destroy_graphs(ctx);   // the captured steps hold the old work lists
  ctx->tile_h = h; ctx->tile_w = w; ctx->tile_order = order; ctx->tile_ctas = ctas;
  return install_items(ctx);
}

int mose_gpu_set_tiling(mose_gpu_ctx* ctx, const int32_t* tiling) {
  MOSE_NVTX_RANGE("mose_gpu_set_tiling");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (!tiling) return MOSE_ERR_INVALID;
  if (ctx->nd != 2) return fail(ctx, MOSE_ERR_UNSUPPORTED, "the tiling applies to the 2-D work list");
  if (tiling[0] < 0 || tiling[0] > (1 << 20) || tiling[1] < 8 || tiling[1] > SB_W || tiling[2] < 0 || tiling[2] > 1 ||
      tiling[3] < 0 || tiling[3] > 32)
    return fail(ctx, MOSE_ERR_INVALID, "tiling out of range (rows >= 0, 8 <= width <= %d, order 0/1, ctas 0..32)",
                SB_W);
  return apply_tiling(ctx, tiling[0], tiling[1], tiling[2], tiling[3]);
}

// Times candidate tilings of the 2-D work list on the context's own domain
// and keeps the fastest.  Every trial runs the path mose_gpu_advance runs
// (graph-replayed steps): it restores the state, runs one untimed step, then
// twice `steps` timed steps (CUDA events on the context's stream), keeping
// the faster.  Default-tiling steps come first until the timing has settled
// (a new context runs slower for its first few hundred steps); coordinate search over rows per item, then strip width, item
// order and CTAs per SM, then rows per item again, a candidate replacing
// the best one only when more than 1 % faster; finally the default and the
// best are timed again, alternately, three times, and the best is kept only
// if still more than 1 % faster.  The state is restored at the end.
int mose_gpu_autotune(mose_gpu_ctx* ctx, int32_t steps, int32_t* tiling_out, double* best_ms, double* default_ms) {
  MOSE_NVTX_RANGE("mose_gpu_autotune");
  int rc = require_ready(ctx);
  if (rc) return rc;
  if (ctx->nd != 2) return fail(ctx, MOSE_ERR_UNSUPPORTED, "the autotuner tunes the 2-D work list");
  if (steps < 1) steps = 3;
  CU(cudaStreamSynchronize(ctx->stream));
  const size_t n = (size_t)ctx->nv * ctx->marena;
  DevBuf<double> snap;
  if (snap.alloc(n) != cudaSuccess) return fail(ctx, MOSE_ERR_CUDA, "out of device memory (autotune snapshot)");
  const int cur0 = ctx->cur, po0 = ctx->po;
  const bool valid0 = ctx->dt_valid;
  CU(cudaMemcpyAsync(snap.p, ctx->state[cur0].p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  const long long launches0 = ctx->launches;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  auto restore = [&]() -> int {
    CU(cudaMemcpyAsync(ctx->state[cur0].p, snap.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->scal.p + 1, &ctx->h_time, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->iterdev.p, &ctx->h_iter, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    ctx->cur = cur0;
    ctx->po = po0;
    ctx->dt_valid = false;
    return MOSE_OK;
  };
  auto trial = [&](int h, int w, int order, int ctas, double& ms) -> int {
    int r = apply_tiling(ctx, h, w, order, ctas);
    if (r) return r;
    if ((r = restore())) return r;
    if ((r = enqueue_graph_steps(ctx, 1))) return r;
    ms = 0.0;
    for (int rep = 0; rep < 2; ++rep) {
      CU(cudaEventRecord(e0, ctx->stream));
      if ((r = enqueue_graph_steps(ctx, steps))) return r;
      CU(cudaEventRecord(e1, ctx->stream));
      CU(cudaEventSynchronize(e1));
      float t = 0.0f;
      CU(cudaEventElapsedTime(&t, e0, e1));
      if (rep == 0 || (double)t / steps < ms) ms = (double)t / steps;
    }
    return poll_device_error(ctx);
  };
  int best[4] = {0, SB_W, 0, 0};
  double tbest = 0.0;
  // warm-up with the default tiling until two successive trials agree within
  // 1 % after at least 0.5 s of steps (at most about 4 s): a new context runs
  // slower for its first few hundred steps
  double warm = 0.0, prev = -1.0;
  for (int q = 0; q < 400 && !rc && warm < 4000.0; ++q) {
    rc = trial(best[0], best[1], best[2], best[3], tbest);
    warm += tbest * (2 * steps + 1);
    if (warm >= 500.0 && prev > 0.0 && std::fabs(tbest - prev) <= 0.01 * prev) break;
    prev = tbest;
  }
  static const int Hs[] = {16, 32, 64, 128, 256, 512, 0};
  static const int Ws[] = {SB_W, 46, 30};
  static const int Os[] = {0, 1};
  static const int Cs[] = {0, 2, 1};
  auto sweep = [&](int knob, const int* vals, int nv) -> int {
    for (int q = 0; q < nv && !rc; ++q) {
      int c[4] = {best[0], best[1], best[2], best[3]};
      c[knob] = vals[q];
      if (c[knob] == best[knob]) continue;
      double t = 0.0;
      int r = trial(c[0], c[1], c[2], c[3], t);
      if (r) return r;
      if (t < 0.99 * tbest) {
        tbest = t;
        for (int z = 0; z < 4; ++z) best[z] = c[z];
      }
    }
    return MOSE_OK;
  };
  if (!rc) rc = sweep(0, Hs, 7);
  if (!rc) rc = sweep(1, Ws, 3);
  if (!rc) rc = sweep(2, Os, 2);
  if (!rc) rc = sweep(3, Cs, 3);
  if (!rc) rc = sweep(0, Hs, 7);
  // the decision: default and best measured again, alternately, three times
  double tdef = 0.0, tb = 0.0;
  const bool moved = best[0] != 0 || best[1] != SB_W || best[2] != 0 || best[3] != 0;
  for (int q = 0; q < 3 && !rc; ++q) {
    double t = 0.0;
    rc = trial(0, SB_W, 0, 0, t);
    if (!rc) tdef = (q == 0 || t < tdef) ? t : tdef;
    if (!rc && moved) {
      rc = trial(best[0], best[1], best[2], best[3], t);
      if (!rc) tb = (q == 0 || t < tb) ? t : tb;
    }
  }
  if (!moved || !(tb < 0.99 * tdef)) {
    best[0] = 0; best[1] = SB_W; best[2] = 0; best[3] = 0;
    tb = tdef;
  }
  tbest = tb;
  const double t0 = tdef;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  rc = apply_tiling(ctx, best[0], best[1], best[2], best[3]);
  if (rc) return rc;
  if ((rc = restore())) return rc;
  ctx->dt_valid = false;
  (void)valid0;
  CU(cudaStreamSynchronize(ctx->stream));
  ctx->launches = launches0;   // the trials are not the caller's steps
  if (tiling_out) for (int z = 0; z < 4; ++z) tiling_out[z] = best[z];
  if (best_ms) *best_ms = tbest;
  if (default_ms) *default_ms = t0;
  return MOSE_OK;
}

}  // extern "C"
