// Shared definitions for the randomized-PCA kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace scx {

constexpr int kWarp = 32;
constexpr int kMaxK = 128;  // widest sketch (n_components + n_oversamples) supported

// Padded row stride of the tall (n_obs x k) and gene (n_vars x k) buffers:
// k rounded up to a whole warp so each lane owns ld/32 columns.
inline int64_t padded_k(int64_t k) { return (k + 31) / 32 * 32; }

__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float to_f32(__half x) { return __half2float(x); }

template <typename T> __device__ __forceinline__ T from_f32(float x);
template <> __device__ __forceinline__ float from_f32<float>(float x) { return x; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float x) {
  return __float2bfloat16_rn(x);
}
template <> __device__ __forceinline__ __half from_f32<__half>(float x) { return __float2half_rn(x); }

// Grid size for a grid-stride loop over `work` items at `per_block` items per
// block: a multiple of the SM count, never more blocks than there is work.
inline int grid_for(int64_t work, int per_block, int num_sms, int blocks_per_sm = 8) {
  int64_t need = (work + per_block - 1) / per_block;
  int64_t cap = (int64_t)num_sms * blocks_per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

}  // namespace scx
