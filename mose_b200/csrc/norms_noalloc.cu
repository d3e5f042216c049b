// norms_noalloc.cu -- Compute_Residual over caller-owned device arrays, with
// its scratch in a fixed device array instead of allocated memory.
//
// For callers that keep P and PO in their own device arrays (the reference
// layout) and cannot let a library call cudaMalloc: their device memory is
// owned by another allocator or by a fixed budget set at start-up.  This
// entry point allocates nothing: its per-chunk partial sums live in
// g_norm_scratch below, which every GPU that loads the library holds until
// the process exits.
#include <cuda_runtime.h>

#include "nvtx.cuh"

#include <cstdio>
#include <mutex>

#include "../../include/mose_gpu.h"

namespace {

constexpr int kMaxPartials = MOSE_NOALLOC_MAX_CHUNKS;   // 4096 chunks
constexpr int kChunk = MOSE_NOALLOC_CHUNK_CELLS;         // 65536 cells per chunk
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// 4096 chunks x 5 sums x 8 B = 160 KB of device memory per GPU.
static __device__ __align__(256) double g_norm_scratch[kMaxPartials * 5];

// Host-side device addresses of g_norm_scratch, one per device ordinal,
// filled the first time a device is used.  The symbol's name in host code is
// only a stand-in for the device array, never a device address.
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

thread_local char g_msg[256] = "";

int fail(int code, const char* msg) {
  std::snprintf(g_msg, sizeof(g_msg), "%s", msg);
  return code;
}

// One CTA per chunk of kChunk interior cells: fixed-order partial sums of
// (|d rho|, |du|, |dv|, |dw|, |dp|)^2 (Mod_Diagnostic.f90:33-37).
__global__ void k_norm_chunks(const double* __restrict__ P, const double* __restrict__ PO, int ni, int nj,
                              long long ncell, double* partial) {
  const long long start = (long long)blockIdx.x * kChunk;
  const long long end = min(start + (long long)kChunk, ncell);
  const int ex = ni + 4, ey = nj + 4;
  double acc[5] = {0, 0, 0, 0, 0};
  for (long long q = start + threadIdx.x; q < end; q += kThreads) {
    int i = (int)(q % ni), j = (int)((q / ni) % nj), k = (int)(q / ((long long)ni * nj));
    long long o = 5 * ((long long)(i + 2) + (long long)ex * ((long long)(j + 2) + (long long)ey * (k + 2)));
    for (int v = 0; v < 5; ++v) {
      double r = fabs(P[o + v] - PO[o + v]);
      acc[v] = acc[v] + r * r;
    }
  }
  __shared__ double red[5][kThreads];
  for (int v = 0; v < 5; ++v) red[v][threadIdx.x] = acc[v];
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int v = 0; v < 5; ++v) red[v][threadIdx.x] = red[v][threadIdx.x] + red[v][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int v = 0; v < 5; ++v) partial[5 * blockIdx.x + v] = red[v][0];
}

// total = total + sum of the chunk partials, in chunk order
// (Mod_Diagnostic.f90:48: total accumulates over blocks).
__global__ void k_norm_finish(const double* partial, int nchunks, double* total) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t[5] = {0, 0, 0, 0, 0};
  for (int c = 0; c < nchunks; ++c)
    for (int v = 0; v < 5; ++v) t[v] = t[v] + partial[5 * c + v];
  for (int v = 0; v < 5; ++v) total[v] = total[v] + t[v];
}

}  // namespace

extern "C" int mose_gpu_residual_norms_noalloc(const double* P, const double* PO, int32_t ni, int32_t nj,
                                               int32_t nk, double* total, void* stream) {
  MOSE_NVTX_RANGE("mose_gpu_residual_norms_noalloc");
  if (!P || !PO || !total) return fail(MOSE_ERR_INVALID, "null array");
  if (ni < 1 || nj < 1 || nk < 1) return fail(MOSE_ERR_INVALID, "bad block dimensions");
  const long long ncell = (long long)ni * nj * nk;
  const long long nchunks = (ncell + kChunk - 1) / kChunk;
  if (nchunks > kMaxPartials) {
    std::snprintf(g_msg, sizeof(g_msg),
                  "block of %lld cells exceeds the no-allocation limit of %lld cells (%d chunks of %d)", ncell,
                  (long long)kMaxPartials * kChunk, kMaxPartials, kChunk);
    return MOSE_ERR_INVALID;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(MOSE_ERR_CUDA, "no current CUDA device");
  double* scratch = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      // first call on this device (it is current): look up the array's
      // address.  The lookup may load the module, which a stream capture in
      // progress does not allow, so a first call inside a capture is refused.
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return fail(MOSE_ERR_INVALID,
                    "the first call on a device must come before any stream capture (it looks up the scratch "
                    "array's address)");
      }
      cudaError_t e = cudaGetSymbolAddress((void**)&g_scratch_addr[dev], g_norm_scratch);
      if (e != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        std::snprintf(g_msg, sizeof(g_msg), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return MOSE_ERR_CUDA;
      }
    }
    scratch = g_scratch_addr[dev];
  }
  k_norm_chunks<<<(unsigned)nchunks, kThreads, 0, s>>>(P, PO, ni, nj, ncell, scratch);
  k_norm_finish<<<1, 32, 0, s>>>(scratch, (int)nchunks, total);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::snprintf(g_msg, sizeof(g_msg), "launch: %s", cudaGetErrorString(e));
    return MOSE_ERR_CUDA;
  }
  return MOSE_OK;
}

extern "C" const char* mose_gpu_noalloc_last_error(void) { return g_msg; }
