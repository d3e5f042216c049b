// stage3d.cuh -- one RK stage (or one residual evaluation) of 3-D blocks in
// two launches over every block: the k-face march (k_kface3d) and the plane
// stage (k_stage3d) that forms the i- and j-faces and updates the cells.
//
// The reference accumulates a cell's residual in a fixed order: the interior
// i-faces (low then high), the interior j-faces, the interior k-faces
// (Mod_Fluxes.f90:89-179), then the boundary faces in face order 1..6
// (BC_Fluxes walks the bc list, Mod_BC_Fluxes.f90:52-216).  The plane stage
// keeps that order with the residual in registers.  Boundary faces are formed
// only for boundary cells: the interior formula with the ghosts for
// connections (101/201, as BC_Connection_Eul does), boundary_flux() for the
// other types.
#pragma once

#include "stage2d.cuh"

namespace mose {
namespace s3 {

constexpr int NV = 5;

__device__ __forceinline__ long long off3(const BlockDesc& d, int i, int j, int k) { return cell_off3(d, i, j, k); }

// dl of cell o along direction dir
template <bool UNI>
__device__ __forceinline__ double dl_at(const StageArgs& a, const BlockDesc& d, int dir, long long o) {
  if constexpr (UNI) return d.u_dl[dir];
  else return a.m.dl[3 * d.mbase + dir * d.vstride + o];
}
// normal and area of the low face along dir of cell o
template <bool UNI>
__device__ __forceinline__ double face_at(const StageArgs& a, const BlockDesc& d, int dir, long long o, double* n) {
  if constexpr (UNI) {
    n[0] = d.u_n[dir][0]; n[1] = d.u_n[dir][1]; n[2] = d.u_n[dir][2];
    return d.u_A[dir];
  } else {
    const long long vs = d.vstride;
    const double* f = a.m.face + 12 * d.mbase + (4 * dir) * vs + o;
    n[0] = f[0]; n[1] = f[vs]; n[2] = f[2 * vs];
    return f[3 * vs];
  }
}
__device__ __forceinline__ void loadQ(const double* P, long long vs, long long o, double* q) {
#pragma unroll
  for (int v = 0; v < NV; ++v) q[v] = P[v * vs + o];
}

// Limited slope of q between qa (low side) and qb (high side) with dl da, d0,
// db along the line (Lib_Reconstruction.f90:10-29 with l = (dl_a + dl_b) / 2).
template <class PH, bool UNI>
__device__ __forceinline__ void lslope(const double* qa, const double* q, const double* qb, double da, double d0,
                                       double db, double* s) {
  constexpr bool FU = UNI && PH::kFast;
  if constexpr (FU) {
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = PH::lim(qb[v] - q[v], q[v] - qa[v]);
  } else {
    const double la = 0.5 * (da + d0), lb = 0.5 * (d0 + db);
    double ila = 0.0, ilb = 0.0;
    if constexpr (PH::kFast) { ila = PH::inv_len(la); ilb = PH::inv_len(lb); }
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = PH::lim(PH::slope(qb[v] - q[v], lb, ilb), PH::slope(q[v] - qa[v], la, ila));
  }
}

// Face flux between cells L (state PL, slope sL, dl dL) and R from the
// reconstructed states; n, A the face metric.  false: check_gas_state rejects.
// beta: the face's shock detector (its low cell's), which scales both slopes
// under MUSCL-SD (sdl, Lib_Reconstruction.f90:24-25) and goes to the SD
// Riemann solvers.
template <class PH, bool UNI>
__device__ __forceinline__ bool face(const Gas& g, const double* PL, const double* sL, double dL, const double* PR,
                                     const double* sR, double dR, const double* n, double A, double* F,
                                     double beta = 1.0, bool sdl = false) {
  constexpr bool FU = UNI && PH::kFast;
  if constexpr (FU && PH::kFace32) {
    // mixed precision on uniform grids: face states and the solve in FP32
    // (slopes in difference units, half-cell offsets of 1/2)
    float QL[NV], QR[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      QL[v] = fmaf((float)sL[v], 0.5f, (float)PL[v]);
      QR[v] = fmaf((float)sR[v], -0.5f, (float)PR[v]);
    }
    return PH::template face32<NV>(g, QL, QR, n, A, F);
  }
  const double hm = FU ? 0.5 : 0.5 * dL, hp = FU ? 0.5 : 0.5 * dR;
  double QL[NV], QR[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double sl = sdl ? beta * sL[v] : sL[v], sr = sdl ? beta * sR[v] : sR[v];
    QL[v] = PL[v] + sl * hm;
    QR[v] = PR[v] - sr * hp;
  }
  return PH::template face<NV>(g, QL, QR, n, A, F, beta);
}

// Boundary-face term of face f (1..6) of boundary cell (i, j, k) of block b:
// returns the add mask and the flux in F (per the reference's BC_Fluxes).
template <class PH, int RIE, int LIM, bool UNI>
__device__ __noinline__ int bc_face(const StageArgs& a, int b, int f, int i, int j, int k, double* F) {
  const BlockDesc& d = a.blk[b];
  const int dir = (f - 1) / 2;
  const bool high = (f % 2) == 0;
  const int idx = (f <= 2) ? j + d.nj * k : (f <= 4) ? i + d.ni * k : i + d.ni * j;
  const int w = a.bcw[d.bcoff[f - 1] + idx];
  const int code = bc_code(w);
  if (code == BC_NONE) return ADD_NONE;
  const double* P = a.Pc + d.sbase;
  const long long vs = d.vstride;
  const int di = dir == 0, dj = dir == 1, dk = dir == 2;
  // cells along the face normal, m = 0 the boundary cell, m > 0 inward
  const int sgn = high ? -1 : 1;
  auto cell = [&](int m) { return off3(d, i + sgn * m * di, j + sgn * m * dj, k + sgn * m * dk); };
  double n[3];
  // the boundary face is the low face of the boundary cell, or of the next cell
  const double A = face_at<UNI>(a, d, dir, high ? off3(d, i + di, j + dj, k + dk) : cell(0), n);
  if (code == BC_CONN) {
    // interior formula across the face with the ghost cells: stencil
    // (-2, -1 | 0, 1) on the low side, (n-2, n-1 | n, n+1) on the high side
    double q[4][NV], dl[4];
    for (int s = 0; s < 4; ++s) {
      // offset from the boundary cell along +dir, low index first: the face
      // lies between stencil cells 1 and 2
      const int t = high ? s - 1 : s - 2;
      const long long o = off3(d, i + di * t, j + dj * t, k + dk * t);
      loadQ(P, vs, o, q[s]);
      dl[s] = dl_at<UNI>(a, d, dir, o);
    }
    double sL[NV], sR[NV];
    lslope<PH, UNI>(q[0], q[1], q[2], dl[0], dl[1], dl[2], sL);
    lslope<PH, UNI>(q[1], q[2], q[3], dl[1], dl[2], dl[3], sR);
    // the shock detector of a connection face is the boundary cell's
    // (Lib_BC_Fluxes_Connection.f90:58-62)
    double bF = 1.0;
    bool sdl = false;
    if constexpr (RIE == 4) {
      if (a.g.sd) bF = a.beta[d.mbase + cell(0)];
      sdl = (a.g.sd & 1) != 0;
    }
    face<PH, UNI>(a.g, q[1], sL, dl[1], q[2], sR, dl[2], n, A, F, bF, sdl);
    return ADD_ALL;
  }
  double Q[NV], Qi[NV];
  loadQ(P, vs, cell(0), Q);
  loadQ(P, vs, cell(1), Qi);
  return boundary_flux<RIE, LIM, NV>(a, w, Q, Qi, dl_at<UNI>(a, d, dir, cell(0)), dl_at<UNI>(a, d, dir, cell(1)), n,
                                     A, f, F);
}

}  // namespace s3

// ---- k-face march ----------------------------------------------------------------
// k_kface3d: each thread marches one (i, j) column of a work item's tile up its
// run of k planes with P(k), P(k + 1), P(k + 2), the k-slopes and the next
// plane's load in registers, and stores the interior k-face flux H(k + 1/2)
// (0 <= k <= nk - 2) at cell (i, j, k) of the k-face arena; a connection face
// at either k end of the block takes the same formula with the ghosts.  No shared memory
// and no barrier: the march is a register pipeline, and the plane stage below
// reads H(k - 1/2) and H(k + 1/2) back as two coalesced loads per cell.  The
// flux is the interior formula of Mod_Fluxes.f90:155-179 (the k loop), so
// the plane stage adds exactly the value the reference adds.  Two CTAs per
// SM: the march holds four states and two slopes across the face, which at
// the three-CTA budget of 80 registers spills to local memory.
template <class PH, int RIE, int LIM, bool UNI>
__global__ void __launch_bounds__(SB_T, 2) k_kface3d(StageArgs a, const int4* items, int nitems) {
  using namespace s3;
  const int t = threadIdx.x, tx = t % T3X, ty = t / T3X;
#pragma unroll 1
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 item = items[it];
    const int b = item.x, i = (item.y & 0xffff) + tx, j = (item.y >> 16) + ty, k0 = item.z;
    const BlockDesc& d = a.blk[b];
    if (ty >= T3Y || i >= d.ni || j >= d.nj) continue;
    // faces k + 1/2 for kb <= k < ke: the interior faces of the run, and a
    // connection face at the block's k = 0 or k = nk end (its ghosts are the
    // source block's cells), stored at the ghost slot k = -1 or at k = nk - 1
    auto conn = [&](int f) { return bc_code(a.bcw[d.bcoff[f - 1] + i + d.ni * j]) == BC_CONN; };
    const int kb = (k0 == 0 && conn(5)) ? -1 : k0;
    const int ke = (item.w == d.nk && conn(6)) ? d.nk : (item.w < d.nk - 1 ? item.w : d.nk - 1);
    if (kb >= ke) continue;
    const long long vs = d.vstride;
    const double* P = a.Pc + d.sbase;
    double* H = a.Hk + d.sbase;
    // the run-time solver kernels carry the shock detector: a face takes its
    // low cell's beta (a connection face at k = 0, the boundary cell's)
    constexpr bool SDV = (RIE == 4);
    const bool sd = SDV && a.g.sd != 0, sdl = SDV && (a.g.sd & 1) != 0;
    double un[3] = {0.0, 0.0, 0.0}, uA = 0.0, udl = 0.0;
    if constexpr (UNI) {
      un[0] = d.u_n[2][0]; un[1] = d.u_n[2][1]; un[2] = d.u_n[2][2];
      uA = d.u_A[2];
      udl = d.u_dl[2];
    }
    auto ok3 = [&](int kk) { return off3(d, i, j, kk); };
    auto dlk = [&](long long o) -> double {
      if constexpr (UNI) return udl; else return a.m.dl[3 * d.mbase + 2 * vs + o];
    };
    double p0[NV], p1[NV], pn[NV], s0[NV];
    double d0, d1;
    {
      double pm[NV];
      loadQ(P, vs, ok3(kb - 1), pm);
      loadQ(P, vs, ok3(kb), p0);
      loadQ(P, vs, ok3(kb + 1), p1);
      const double dm = dlk(ok3(kb - 1));
      d0 = dlk(ok3(kb));
      d1 = dlk(ok3(kb + 1));
      lslope<PH, UNI>(pm, p0, p1, dm, d0, d1, s0);
    }
    loadQ(P, vs, ok3(kb + 2), pn);
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
      double p2[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) p2[v] = pn[v];
      // the next plane's P(k + 2), in flight during this face
      if (k + 1 < ke) loadQ(P, vs, ok3(k + 3), pn);
      const double d2 = dlk(ok3(k + 2));
      double s1[NV], Hf[NV], n[3], A;
      lslope<PH, UNI>(p0, p1, p2, d0, d1, d2, s1);
      if constexpr (UNI) { n[0] = un[0]; n[1] = un[1]; n[2] = un[2]; A = uA; }
      else A = face_at<false>(a, d, 2, ok3(k + 1), n);
      double bF = 1.0;
      if constexpr (SDV) {
        if (sd) bF = a.beta[d.mbase + ok3(k < 0 ? 0 : k)];
      }
      const bool ok = face<PH, UNI>(a.g, p0, s0, d0, p1, s1, d1, n, A, Hf, bF, sdl);
      if (!ok) report(a.err, 4, b, i, j, k);
      const long long o = ok3(k);
#pragma unroll
      for (int v = 0; v < NV; ++v) H[v * vs + o] = Hf[v];
#pragma unroll
      for (int v = 0; v < NV; ++v) { p0[v] = p1[v]; p1[v] = p2[v]; s0[v] = s1[v]; }
      d0 = d1;
      d1 = d2;
    }
  }
}

// ---- plane stage -----------------------------------------------------------------
// k_stage3d: a CTA of T3X x T3Y threads owns a tile of cells (i0 .. i0 + T3X -
// 1, j0 .. j0 + T3Y - 1) of one block and marches up a run of k planes.  Per
// plane it stages the tile and a two-cell halo ring in i and j in shared
// memory, forms the limited i- and j-slopes and every i- and j-face flux of
// the tile (halo faces included) there, then each thread adds its cell's
// terms in the reference's order: interior i-faces, j-faces, the k-faces from
// the k-face arena, then the boundary faces in face order 1..6, and applies
// Newstate (or stores R in residual mode) and the next step's CFL dt.  R
// never goes through HBM.  The next plane's copy is issued once the faces
// are formed, so it lands during the cell updates; with no k-march state in
// registers three CTAs fit on an SM.
constexpr int H3X = T3X + 4, H3Y = T3Y + 4;  // plane region: the tile and two halo cells per side
// Threads of a plane-stage CTA.  The fast policies: one per tile cell (256),
// three CTAs per SM at 80 registers.  The reference-exact policy: 320, so
// that the slope (592 per plane) and face (552) phases take two rounds each
// instead of three, at two CTAs per SM; its IEEE divisions and square roots
// make each round long enough for that to pay (1.07 against 1.02 G
// cell-updates/s on 8 x 128^3, where the fast policies lose 5-8 % with it).
template <class PH>
constexpr int s3_threads() { return PH::kFast ? T3X * T3Y : 320; }

// F32: the mixed policy on uniform grids, whose limited slopes and per-area
// face fluxes are FP32 values: held as such (the face area is applied when a
// cell adds the flux, the same product as before), half the bytes.
template <int NVS, bool UNI, bool F32 = false>
struct Stage3dSmem {
  using T = typename std::conditional<F32, float, double>::type;
  double P[NVS][H3Y][H3X];          // plane k: region cells, corners unused
  double dx[UNI ? 1 : T3Y][UNI ? 1 : H3X];   // dl along i on the tile rows (metric arrays only)
  double dy[UNI ? 1 : H3Y][UNI ? 1 : T3X];   // dl along j on the tile columns
  T sx[NVS][T3Y][T3X + 2];          // limited i-slope of cells i0 - 1 .. i0 + T3X
  T sy[NVS][T3Y + 2][T3X];          // limited j-slope of cells j0 - 1 .. j0 + T3Y
  T F[NVS][T3Y][T3X + 1];           // F(i0 - 1 + x + 1/2) (F32: per unit area)
  T G[NVS][T3Y + 1][T3X];           // G(j0 - 1 + y + 1/2)
  // the block's uniform metrics: dl (3), face normals (3 x 3), areas (3), volume
  double um[16];
};
template <bool UNI, bool F32 = false>
constexpr size_t stage3d_smem_bytes() { return sizeof(Stage3dSmem<5, UNI, F32>); }
// the FP32 shared-memory variant of a policy
template <class PH, bool UNI>
constexpr bool stage3d_f32() { return UNI && PH::kFace32; }

// Items: (block, i0 | j0 << 16, k0, k1).  BC: the items with a physical
// boundary face (the boundary formulas, a call, hold the kernel to two CTAs
// per SM); without, every block-edge face of the items' cells is a
// connection, formed here from the staged ghosts (i, j) or by the k-face
// march (k) and added in its boundary-face position.  Both add a cell's terms
// in the same order, so their results are identical.
template <class PH, bool BC, bool F32>
constexpr int stage3d_min_ctas() { return (BC || !PH::kFast) ? 2 : F32 ? 4 : 3; }

template <class PH, int RIE, int LIM, bool UNI, int MODE, bool BC>
__global__ void __launch_bounds__(s3_threads<PH>(), stage3d_min_ctas<PH, BC, stage3d_f32<PH, UNI>()>())
    k_stage3d(StageArgs a, const int4* items, int nitems) {
  constexpr int S3_T = s3_threads<PH>();
  constexpr bool F32 = stage3d_f32<PH, UNI>();
  using namespace s3;
  extern __shared__ __align__(16) unsigned char smem3[];
  Stage3dSmem<NV, UNI, F32>& S = *reinterpret_cast<Stage3dSmem<NV, UNI, F32>*>(smem3);
  const int t = threadIdx.x, tx = t % T3X, ty = t / T3X;
  constexpr bool SDV = (RIE == 4);   // the shock detector (run-time solver kernels)
  const bool sd = SDV && a.g.sd != 0, sdl = SDV && (a.g.sd & 1) != 0;
  double dtrun = __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll 1
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 item = items[it];
    const int b = item.x, i0 = item.y & 0xffff, j0 = item.y >> 16, k0 = item.z, k1 = item.w;
    const BlockDesc& d = a.blk[b];
    const int ni = d.ni, nj = d.nj, nk = d.nk;
    const long long vs = d.vstride;
    const double* P = a.Pc + d.sbase;
    const int i = i0 + tx, j = j0 + ty;
    const bool mine = ty < T3Y && i < ni && j < nj;
    const double dtg = (MODE != 1 && a.time_accurate) ? *a.dtg : 0.0;
    // the face metric of the low face along dir of cell o: the uniform
    // constants (shared memory) or the metric arrays
    auto facek = [&](int dir, long long o, double* n) -> double {
      if constexpr (UNI) {
        n[0] = S.um[3 + 3 * dir]; n[1] = S.um[4 + 3 * dir]; n[2] = S.um[5 + 3 * dir];
        return S.um[12 + dir];
      } else {
        return face_at<false>(a, d, dir, o, n);
      }
    };
    auto ok3 = [&](int kk) { return off3(d, i, j, kk); };
    // plane kk with 16-byte copies (two cells per copy; the region's rows
    // start on even columns and the padded rows keep every copy inside the
    // block's plane): rows j0 .. j0 + T3Y - 1 over columns i0 - 2 .. i0 + T3X
    // + 1, and columns i0 .. i0 + T3X - 1 over rows j0 - 2, j0 - 1, j0 + T3Y,
    // j0 + T3Y + 1
    auto stage_plane = [&](int kk) {
      constexpr int CA = H3X / 2, CB = T3X / 2;   // chunks per row
      for (int e = t; e < T3Y * CA + 4 * CB; e += S3_T) {
        int cx, ry;
        if (e < T3Y * CA) { cx = 2 * (e % CA); ry = 2 + e / CA; }
        else { const int q = e - T3Y * CA; cx = 2 + 2 * (q % CB); const int r = q / CB; ry = r < 2 ? r : T3Y + r; }
        const int ci = i0 - 2 + cx, cj = j0 - 2 + ry;
        if (ci > ni + 1 || cj > nj + 1) continue;   // beyond a partial tile's ghosts
        const long long o = off3(d, ci, cj, kk);
#pragma unroll
        for (int v = 0; v < NV; ++v) cp_async16(&S.P[v][ry][cx], P + v * vs + o);
      }
      cp_async_commit();
    };
    __syncthreads();   // the previous item's readers are done with the plane and the constants
    if constexpr (UNI) {
      if (t < 3) S.um[t] = d.u_dl[t];
      else if (t < 12) S.um[t] = d.u_n[(t - 3) / 3][(t - 3) % 3];
      else if (t < 15) S.um[t] = d.u_A[t - 12];
      else if (t == 15) S.um[15] = d.u_vol;
    }
    stage_plane(k0);
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
      if constexpr (!UNI) {
        for (int e = t; e < T3Y * H3X + 4 * T3X; e += S3_T) {
          int cx, ry;
          if (e < T3Y * H3X) { cx = e % H3X; ry = 2 + e / H3X; }
          else { const int q = e - T3Y * H3X; cx = 2 + q % T3X; const int r = q / T3X; ry = r < 2 ? r : T3Y + r; }
          const int ci = i0 - 2 + cx, cj = j0 - 2 + ry;
          if (ci > ni + 1 || cj > nj + 1) continue;
          const long long o = off3(d, ci, cj, k);
          if (ry >= 2 && ry < T3Y + 2) S.dx[ry - 2][cx] = a.m.dl[3 * d.mbase + 0 * vs + o];
          if (cx >= 2 && cx < T3X + 2) S.dy[ry][cx - 2] = a.m.dl[3 * d.mbase + 1 * vs + o];
        }
      }
      cp_async_wait_all();   // this thread's copies of plane k
      __syncthreads();       // everyone's copies; the previous plane's cell updates are done with F and G
      auto dxat = [&](int y, int cx) -> double { if constexpr (UNI) return S.um[0]; else return S.dx[y][cx]; };
      auto dyat = [&](int ry, int x) -> double { if constexpr (UNI) return S.um[1]; else return S.dy[ry][x]; };
      // ---- limited slopes: i-slopes of cells i0 - 1 .. i0 + T3X (columns 1 .. T3X + 2),
      //      j-slopes of cells j0 - 1 .. j0 + T3Y (rows 1 .. T3Y + 2)
      // (one index space for both, so the items beyond one per thread spread
      // over different threads)
      constexpr int NSX = T3Y * (T3X + 2), NSY = (T3Y + 2) * T3X;
      for (int e = t; e < NSX + NSY; e += S3_T) {
        double qa[NV], q[NV], qb[NV], sl[NV];
        if (e < NSX) {
          const int x = e % (T3X + 2), y = e / (T3X + 2);
          const int ci = i0 - 1 + x, cj = j0 + y;
          if (ci > ni || cj >= nj) continue;
#pragma unroll
          for (int v = 0; v < NV; ++v) { qa[v] = S.P[v][y + 2][x]; q[v] = S.P[v][y + 2][x + 1]; qb[v] = S.P[v][y + 2][x + 2]; }
          lslope<PH, UNI>(qa, q, qb, dxat(y, x), dxat(y, x + 1), dxat(y, x + 2), sl);
#pragma unroll
          for (int v = 0; v < NV; ++v) S.sx[v][y][x] = (typename Stage3dSmem<NV, UNI, F32>::T)sl[v];
        } else {
          const int e2 = e - NSX;
          const int x = e2 % T3X, y = e2 / T3X;
          const int ci = i0 + x, cj = j0 - 1 + y;
          if (ci >= ni || cj > nj) continue;
#pragma unroll
          for (int v = 0; v < NV; ++v) { qa[v] = S.P[v][y][x + 2]; q[v] = S.P[v][y + 1][x + 2]; qb[v] = S.P[v][y + 2][x + 2]; }
          lslope<PH, UNI>(qa, q, qb, dyat(y, x), dyat(y + 1, x), dyat(y + 2, x), sl);
#pragma unroll
          for (int v = 0; v < NV; ++v) S.sy[v][y][x] = (typename Stage3dSmem<NV, UNI, F32>::T)sl[v];
        }
      }
      __syncthreads();
      // ---- interior face fluxes of the tile: i-faces (i0 - 1 + x) + 1/2, j-faces (j0 - 1 + y) + 1/2
      constexpr int NFX = T3Y * (T3X + 1), NFY = (T3Y + 1) * T3X;
      for (int e = t; e < NFX + NFY; e += S3_T) {
        double PL[NV], PR[NV], sL[NV], sR[NV], F[NV], n[3];
        if (e < NFX) {
          const int x = e % (T3X + 1), y = e / (T3X + 1);
          const int cl = i0 - 1 + x, cj = j0 + y;
          if (cl < (BC ? 0 : -1) || cl > (BC ? ni - 2 : ni - 1) || cj >= nj) continue;
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            PL[v] = S.P[v][y + 2][x + 1]; PR[v] = S.P[v][y + 2][x + 2];
            sL[v] = S.sx[v][y][x]; sR[v] = S.sx[v][y][x + 1];
          }
          // F32: the flux per unit area (an FP32 value, held exactly)
          const double A = F32 ? 1.0 : facek(0, off3(d, cl + 1, cj, k), n);
          if constexpr (F32) facek(0, off3(d, cl + 1, cj, k), n);
          double bF = 1.0;
          if constexpr (SDV) {
            if (sd) bF = a.beta[d.mbase + off3(d, cl < 0 ? 0 : cl, cj, k)];
          }
          const bool ok = face<PH, UNI>(a.g, PL, sL, dxat(y, x + 1), PR, sR, dxat(y, x + 2), n, A, F, bF, sdl);
          if (!ok) report(a.err, 4, b, cl, cj, k);
#pragma unroll
          for (int v = 0; v < NV; ++v) S.F[v][y][x] = (typename Stage3dSmem<NV, UNI, F32>::T)F[v];
        } else {
          const int e2 = e - NFX;
          const int x = e2 % T3X, y = e2 / T3X;
          const int ci = i0 + x, cl = j0 - 1 + y;
          if (ci >= ni || cl < (BC ? 0 : -1) || cl > (BC ? nj - 2 : nj - 1)) continue;
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            PL[v] = S.P[v][y + 1][x + 2]; PR[v] = S.P[v][y + 2][x + 2];
            sL[v] = S.sy[v][y][x]; sR[v] = S.sy[v][y + 1][x];
          }
          // F32: the flux per unit area (an FP32 value, held exactly)
          const double A = F32 ? 1.0 : facek(1, off3(d, ci, cl + 1, k), n);
          if constexpr (F32) facek(1, off3(d, ci, cl + 1, k), n);
          double bF = 1.0;
          if constexpr (SDV) {
            if (sd) bF = a.beta[d.mbase + off3(d, ci, cl < 0 ? 0 : cl, k)];
          }
          const bool ok = face<PH, UNI>(a.g, PL, sL, dyat(y + 1, x), PR, sR, dyat(y + 2, x), n, A, F, bF, sdl);
          if (!ok) report(a.err, 4, b, ci, cl, k);
#pragma unroll
          for (int v = 0; v < NV; ++v) S.G[v][y][x] = (typename Stage3dSmem<NV, UNI, F32>::T)F[v];
        }
      }
      // the cell's own state from the plane, its k-face fluxes and
      // stage-start state from HBM.  The mixed policy issues the HBM loads
      // before the barrier, in flight while the last faces of the plane are
      // formed (2.99 against 2.81 G cell-updates/s on 8 x 128^3); the FP64
      // policies after it, where the 15 loaded values are not live across
      // the barrier and the next plane's copy (16 against 88 B of spills at
      // 80 registers; 3.08 against 2.91 G in fp64)
      const long long o = ok3(k);
      const bool first = (a.irk == 1);
      double p0[NV], Hm[NV], Hp[NV], QO[NV];
      auto load_cell = [&]() {
        const double* Hk = a.Hk + d.sbase;
        if (!BC || k > 0) loadQ(Hk, vs, ok3(k - 1), Hm);
        if (!BC || k < nk - 1) loadQ(Hk, vs, o, Hp);
        if (MODE != 1 && !first) loadQ(a.Po + d.sbase, vs, o, QO);
      };
      if (mine) {
#pragma unroll
        for (int v = 0; v < NV; ++v) p0[v] = S.P[v][ty + 2][tx + 2];
        if constexpr (PH::kMixed) load_cell();
      }
      __syncthreads();   // faces formed, the plane read: the next plane may land
      if (k + 1 < k1) stage_plane(k + 1);
      if (!mine) continue;
      if constexpr (!PH::kMixed) load_cell();
      // ---- the residual of cell (i, j, k) in the reference's order
      ResAcc<NV, PH::kCompensated> R;
      R.init();
      // a face flux as the face solve gave it: F32 holds it per unit area
      auto fx = [&](int v, int x) -> double {
        if constexpr (F32) return (double)S.F[v][ty][x] * S.um[12]; else return S.F[v][ty][x];
      };
      auto gy = [&](int v, int y) -> double {
        if constexpr (F32) return (double)S.G[v][y][tx] * S.um[13]; else return S.G[v][y][tx];
      };
      if (i > 0) for (int v = 0; v < NV; ++v) R.add(v, -fx(v, tx));
      if (i < ni - 1) for (int v = 0; v < NV; ++v) R.add(v, fx(v, tx + 1));
      if (j > 0) for (int v = 0; v < NV; ++v) R.add(v, -gy(v, ty));
      if (j < nj - 1) for (int v = 0; v < NV; ++v) R.add(v, gy(v, ty + 1));
      if (k > 0) for (int v = 0; v < NV; ++v) R.add(v, -Hm[v]);
      if (k < nk - 1) for (int v = 0; v < NV; ++v) R.add(v, Hp[v]);
      // boundary faces in face order 1..6
      if constexpr (!BC) {
        double Fe[NV];
        if (i == 0) {
          for (int v = 0; v < NV; ++v) Fe[v] = fx(v, tx);
          add_bc<NV>(R, Fe, -1.0, ADD_ALL);
        }
        if (i == ni - 1) {
          for (int v = 0; v < NV; ++v) Fe[v] = fx(v, tx + 1);
          add_bc<NV>(R, Fe, 1.0, ADD_ALL);
        }
        if (j == 0) {
          for (int v = 0; v < NV; ++v) Fe[v] = gy(v, ty);
          add_bc<NV>(R, Fe, -1.0, ADD_ALL);
        }
        if (j == nj - 1) {
          for (int v = 0; v < NV; ++v) Fe[v] = gy(v, ty + 1);
          add_bc<NV>(R, Fe, 1.0, ADD_ALL);
        }
        if (k == 0) add_bc<NV>(R, Hm, -1.0, ADD_ALL);
        if (k == nk - 1) add_bc<NV>(R, Hp, 1.0, ADD_ALL);
      } else if (i == 0 || i == ni - 1 || j == 0 || j == nj - 1 || k == 0 || k == nk - 1) {
#pragma unroll 1
        for (int f = 1; f <= 6; ++f) {
          const bool on = (f == 1) ? i == 0 : (f == 2) ? i == ni - 1 : (f == 3) ? j == 0 : (f == 4) ? j == nj - 1
                          : (f == 5) ? k == 0 : k == nk - 1;
          if (!on) continue;
          double F[NV];
          const int mask = bc_face<PH, RIE, LIM, UNI>(a, b, f, i, j, k, F);
          add_bc<NV>(R, F, (f % 2) ? -1.0 : 1.0, mask);
        }
      }
      double Rv[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) Rv[v] = R.get(v);
      if constexpr (MODE == 1) {
        double* Rb = a.R + d.sbase;
#pragma unroll
        for (int v = 0; v < NV; ++v) Rb[v * vs + o] = Rv[v];
      } else {
        double vol;
        if constexpr (UNI) vol = S.um[15]; else vol = a.m.vol[d.mbase + o];
        const double dt = a.time_accurate ? dtg : a.dtl[d.mbase + o];
        const bool ok = PH::template update<NV>(a.g, p0, QO, Rv, vol, dt, a.c_rk, first);
        if (!ok) report(a.err, 5, b, i, j, k);
        double* Pn = a.Pn + d.sbase;
#pragma unroll
        for (int v = 0; v < NV; ++v) Pn[v * vs + o] = p0[v];
        if constexpr (MODE == 2) dtrun = fmin(dtrun, cfl_dt<NV, UNI, PH::kFast>(a.g, p0, d, a.m, o, a.ndir, a.cfl));
      }
    }
  }
  if constexpr (MODE == 2) {
    __shared__ double red[S3_T / 32];
    for (int s = 16; s > 0; s >>= 1) dtrun = fmin(dtrun, __shfl_xor_sync(0xffffffffu, dtrun, s));
    if ((t & 31) == 0) red[t >> 5] = dtrun;
    __syncthreads();
    if (t == 0) {
      double v = red[0];
      for (int w = 1; w < S3_T / 32; ++w) v = fmin(v, red[w]);
      atomicMin(a.dtmin, (unsigned long long)__double_as_longlong(v));
    }
  }
}

}  // namespace mose
