// fp64_peak.cu -- issue ceilings of the FP64 operations the stage kernels are
// made of, measured on the current device: fused multiply-add, IEEE division
// and IEEE square root.  The path has no dense contraction, so its compute
// roofline is the FP64 pipe, which no copy or GEMM peak describes.
//
// Each thread runs independent dependency chains (enough in flight per
// scheduler to cover the pipe latency) over a fixed iteration count; the
// values stay bounded, and the result is kept live through one conditional
// store, so nothing is optimised away.  Timed with CUDA events around the
// second of two identical launches.
//
// Measurement only: built into libmose_probe.so beside the product library
// (libmose_gpu.so), whose C ABI does not carry it.
#include <cuda_runtime.h>

#include <cstdint>

// status codes of this probe: 0 = ok, 1 = bad argument, 3 = CUDA failure
// (the values of MOSE_OK, MOSE_ERR_INVALID, MOSE_ERR_CUDA in mose_gpu.h)
enum { MOSE_OK = 0, MOSE_ERR_INVALID = 1, MOSE_ERR_CUDA = 3 };

namespace {

constexpr int kThreads = 256;

// 8 chains of x <- x a + b (a < 1: bounded)
__global__ void k_peak_dfma(double* sink, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) x[c] = 1e-3 * (threadIdx.x + c);
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += x[c];
  if (s == -1.0) sink[0] = s;
}

// 4 chains of x <- a / x (alternates between x and a / x: bounded)
__global__ void k_peak_ddiv(double* sink, int iters, double a) {
  double x[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) x[c] = 1.0 + 1e-3 * (threadIdx.x + c);
#pragma unroll 2
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = a / x[c];
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) s += x[c];
  if (s == -1.0) sink[0] = s;
}

// 4 chains of x <- sqrt(x) + b (converges towards a fixed point: bounded)
__global__ void k_peak_dsqrt(double* sink, int iters, double b) {
  double x[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) x[c] = 2.0 + 1e-3 * (threadIdx.x + c);
#pragma unroll 2
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = sqrt(x[c]) + b;
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) s += x[c];
  if (s == -1.0) sink[0] = s;
}

template <class L>
int time_ms(L launch, float* ms) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return MOSE_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return MOSE_ERR_CUDA;
  }
  launch();   // warm-up: clocks up, module loaded
  cudaEventRecord(e0, 0);
  launch();
  cudaEventRecord(e1, 0);
  int rc = cudaEventSynchronize(e1) == cudaSuccess && cudaGetLastError() == cudaSuccess ? MOSE_OK : MOSE_ERR_CUDA;
  if (rc == MOSE_OK && cudaEventElapsedTime(ms, e0, e1) != cudaSuccess) rc = MOSE_ERR_CUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // namespace

// out[0]: FP64 fused multiply-add, TFLOP/s (two flops each); out[1]: IEEE
// FP64 divisions, G/s; out[2]: IEEE FP64 square roots, G/s; out[3..5]: the
// timed launches' durations in ms.  Synchronous; about 0.1 s.
extern "C" int mose_probe_fp64_peak(int32_t device, double* out) {
  if (!out) return MOSE_ERR_INVALID;
  cudaDeviceProp prop;
  if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess)
    return MOSE_ERR_CUDA;
  double* sink = nullptr;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return MOSE_ERR_CUDA;
  const int grid = prop.multiProcessorCount * 4;   // 1024 threads per SM
  const double threads = (double)grid * kThreads;
  const int it_fma = 1 << 17, it_div = 1 << 12, it_sqrt = 1 << 12;
  float ms[3] = {0.0f, 0.0f, 0.0f};
  int rc = time_ms([&] { k_peak_dfma<<<grid, kThreads>>>(sink, it_fma, 0.999999, 1e-6); }, &ms[0]);
  if (rc == MOSE_OK) rc = time_ms([&] { k_peak_ddiv<<<grid, kThreads>>>(sink, it_div, 1.5); }, &ms[1]);
  if (rc == MOSE_OK) rc = time_ms([&] { k_peak_dsqrt<<<grid, kThreads>>>(sink, it_sqrt, 0.25); }, &ms[2]);
  cudaFree(sink);
  if (rc != MOSE_OK) return rc;
  out[0] = 2.0 * 8.0 * it_fma * threads / (ms[0] * 1e-3) / 1e12;   // FP64 FMA, TFLOP/s (2 flops each)
  out[1] = 4.0 * it_div * threads / (ms[1] * 1e-3) / 1e9;          // IEEE divisions, G/s
  out[2] = 4.0 * it_sqrt * threads / (ms[2] * 1e-3) / 1e9;         // IEEE square roots, G/s
  out[3] = ms[0];
  out[4] = ms[1];
  out[5] = ms[2];
  return MOSE_OK;
}
