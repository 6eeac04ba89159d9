// Shared definitions for the randomized-PCA kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace scx {

constexpr int kWarp = 32;
constexpr int kMaxK = 128;      // widest sketch (n_components + n_oversamples) of the single-panel kernels
constexpr int kPanel = 128;     // column panel of a wider sketch
constexpr int kMaxKWide = 256;  // widest sketch supported (two panels)

// Padded row stride of the tall (n_obs x k) and gene (n_vars x k) buffers:
// k rounded up to a whole warp so each lane owns ld/32 columns; a sketch
// wider than one panel is padded to whole panels.
inline int64_t padded_k(int64_t k) {
  return k <= kMaxK ? (k + 31) / 32 * 32 : (k + kPanel - 1) / kPanel * kPanel;
}

__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float to_f32(__half x) { return __half2float(x); }

template <typename T> __device__ __forceinline__ T from_f32(float x);
template <> __device__ __forceinline__ float from_f32<float>(float x) { return x; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float x) {
  return __float2bfloat16_rn(x);
}
template <> __device__ __forceinline__ __half from_f32<__half>(float x) { return __float2half_rn(x); }

// FP64 reciprocal and reciprocal square root by Newton-Raphson iteration
// (y <- y (2 - x y) and y <- y (3 - x y^2) / 2; each step doubles the correct
// bits) from a single-precision hardware seed.  The argument is first scaled
// by a power of two into [1, 2) (reciprocal) or [1, 4) (rsqrt), so the seed
// never overflows or underflows; two steps reach double precision.  For the
// short dependent chains of the small eigensolver and Cholesky kernels, where
// the division and square-root library sequences dominate the latency.
// Arguments must be positive, finite and normal.
__device__ __forceinline__ double pow2_int(int k) {  // 2^k for k in [-1022, 1023]
  return __longlong_as_double((long long)(k + 1023) << 52);
}
__device__ __forceinline__ int exponent_of(double x) {  // floor(log2 x) for normal x > 0
  return (int)((__double_as_longlong(x) >> 52) & 0x7ff) - 1023;
}
__device__ __forceinline__ double rcp_nr(double x) {
  const int e = exponent_of(x);
  const double xs = x * pow2_int(-e);  // [1, 2)
  double y = (double)__frcp_rn((float)xs);
  y = y * fma(-xs, y, 2.0);
  y = y * fma(-xs, y, 2.0);
  return y * pow2_int(-e);
}
__device__ __forceinline__ double rsqrt_nr(double x) {
  const int h = exponent_of(x) >> 1;
  const double xs = x * pow2_int(-2 * h);  // [1, 4)
  double y = (double)rsqrtf((float)xs);
  const double hx = 0.5 * xs;
  y = y * fma(-hx, y * y, 1.5);
  y = y * fma(-hx, y * y, 1.5);
  return y * pow2_int(-h);
}

// Opts kernel `kern` in to `smem` bytes of dynamic shared memory.  A refused
// opt-in is returned to the launcher, so the caller sees its cause rather than
// the launch failure that would follow it.
template <typename Kernel>
inline cudaError_t allow_smem(Kernel* kern, size_t smem) {
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// Grid size for a grid-stride loop over `work` items at `per_block` items per
// block: a multiple of the SM count, never more blocks than there is work.
inline int grid_for(int64_t work, int per_block, int num_sms, int blocks_per_sm = 8) {
  int64_t need = (work + per_block - 1) / per_block;
  int64_t cap = (int64_t)num_sms * blocks_per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

}  // namespace scx
