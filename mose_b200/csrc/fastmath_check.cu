// fastmath_check.cu -- on-device accuracy check of the restated FP64
// reciprocal, reciprocal square root and square root (physics_fast.cuh).
//
// The relative error of each result is measured exactly through FMA
// residuals, not against another approximation:
//   r ~ 1/x:        1 - x r                    = relative error of r
//   y ~ 1/sqrt(x):  1 - x y^2 (x y split exact) = -2 (relative error of y)
//   s ~ sqrt(x):    x - s^2                     = -2 x (relative error of s)
// and the restated square root is compared bit for bit with the correctly
// rounded one (__dsqrt_rn).
#include <cuda_runtime.h>

#include "nvtx.cuh"

#include <cstdint>
#include <cstring>

#include "../../include/mose_gpu.h"
#include "physics_fast.cuh"

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ void amax(unsigned long long* slot, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_check_fast_math(long long n, uint64_t seed, unsigned long long* out) {
  double e_rcp = 0.0, e_rsq = 0.0, e_sqrt = 0.0, ulp_sqrt = 0.0;
  const double scale = 9007199254740992.0;   // 2^53
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)i));
    const double m = 1.0 + (double)(h >> 11) * (1.0 / 9007199254740992.0);   // [1, 2)
    const int ex = (int)((h & 0x7f) % 120) - 60;                              // [-60, 60)
    const double x = ldexp(m, ex);
    const double r = mose::fast::rcp(x);
    e_rcp = fmax(e_rcp, fabs(fma(-x, r, 1.0)) * scale);
    const double y = mose::fast::rsqrt_(x);
    const double p = x * y, pl = fma(x, y, -p);
    const double ey = fma(-p, y, 1.0) - pl * y;
    e_rsq = fmax(e_rsq, 0.5 * fabs(ey) * scale);
    const double s = mose::fast::sqrt_(x);
    e_sqrt = fmax(e_sqrt, fabs(fma(-s, s, x)) / (2.0 * x) * scale);
    const long long d = __double_as_longlong(s) - __double_as_longlong(__dsqrt_rn(x));
    ulp_sqrt = fmax(ulp_sqrt, (double)(d < 0 ? -d : d));
  }
  amax(out + 0, e_rcp);
  amax(out + 1, e_rsq);
  amax(out + 2, e_sqrt);
  amax(out + 3, ulp_sqrt);
}

}  // namespace

extern "C" int mose_gpu_check_fast_math(int64_t n, uint64_t seed, double* out) {
  MOSE_NVTX_RANGE("mose_gpu_check_fast_math");
  if (n <= 0 || !out) return MOSE_ERR_INVALID;
  unsigned long long* d = nullptr;
  if (cudaMalloc(&d, 4 * sizeof(unsigned long long)) != cudaSuccess) return MOSE_ERR_CUDA;
  int rc = MOSE_OK;
  if (cudaMemset(d, 0, 4 * sizeof(unsigned long long)) != cudaSuccess) rc = MOSE_ERR_CUDA;
  if (rc == MOSE_OK) {
    k_check_fast_math<<<1184, 256>>>(n, seed, d);
    unsigned long long h[4];
    if (cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) rc = MOSE_ERR_CUDA;
    if (rc == MOSE_OK) std::memcpy(out, h, sizeof(h));   // non-negative doubles stored as their bits
  }
  cudaFree(d);
  return rc;
}
