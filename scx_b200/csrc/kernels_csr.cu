// CSR validation and per-row sorting on the device.
//
// The reference validates shards on the host (InvalidShard, scx-gpu/src/
// error.rs) and sorts indices before the GPU call (ensure_csr,
// pyscx/src/accel/pca.rs:900).  Here both run where the matrix lives.
#include "common.cuh"
#include "launch.h"

namespace scx {

template <typename ValT>
__global__ void k_validate_csr(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                               const ValT* __restrict__ val, int64_t n, int64_t g, int64_t nnz,
                               int32_t* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    if (s < 0 || e < s || e > nnz) {
      if (lane == 0) atomicOr(&flags[0], 1);
      continue;
    }
    for (int64_t p = s + lane; p < e; p += 32) {
      const int32_t j = idx[p];
      if (j < 0 || (int64_t)j >= g) atomicOr(&flags[1], 1);
      if (p > s && idx[p - 1] >= j) atomicOr(&flags[2], 1);
      if (!isfinite(to_f32(val[p]))) atomicOr(&flags[3], 1);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (indptr[0] != 0 || indptr[n] != nnz) atomicOr(&flags[0], 1);
  }
}

cudaError_t launch_validate_csr(int dtype, const int64_t* indptr, const int32_t* idx,
                                const void* val, int64_t n, int64_t g, int64_t nnz,
                                int32_t* flags, cudaStream_t st, int num_sms) {
  int grid = grid_for(n * 32 + 32, 256, num_sms, 8);
  note_launches(1);
  switch (dtype) {
    case 0: k_validate_csr<float><<<grid, 256, 0, st>>>(indptr, idx, (const float*)val, n, g, nnz, flags); break;
    case 1: k_validate_csr<__nv_bfloat16><<<grid, 256, 0, st>>>(indptr, idx, (const __nv_bfloat16*)val, n, g, nnz, flags); break;
    default: k_validate_csr<__half><<<grid, 256, 0, st>>>(indptr, idx, (const __half*)val, n, g, nnz, flags); break;
  }
  return cudaGetLastError();
}

// Sort a row by gene: rows up to 1024 entries with a bitonic sort in shared
// memory (one block of 256 threads per row batch); longer rows by a
// single-thread insertion sort (rare for cells x genes data).  Equal genes
// keep both entries (duplicates are summed by every product kernel).
template <typename ValT>
__global__ void k_sort_rows(const int64_t* __restrict__ indptr, int32_t* __restrict__ idx,
                            ValT* __restrict__ val, int64_t n) {
  constexpr int CAP = 1024;
  __shared__ int32_t key[CAP];
  __shared__ ValT vv[CAP];
  for (int64_t row = blockIdx.x; row < n; row += gridDim.x) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    const int len = (int)(e - s);
    if (len <= 1) continue;
    if (len > CAP) {
      if (threadIdx.x == 0) {
        for (int64_t a = s + 1; a < e; ++a) {
          int32_t kj = idx[a];
          ValT kv = val[a];
          int64_t b = a - 1;
          while (b >= s && idx[b] > kj) {
            idx[b + 1] = idx[b];
            val[b + 1] = val[b];
            --b;
          }
          idx[b + 1] = kj;
          val[b + 1] = kv;
        }
      }
      __syncthreads();
      continue;
    }
    int pow2 = 1;
    while (pow2 < len) pow2 <<= 1;
    for (int t = threadIdx.x; t < pow2; t += blockDim.x) {
      key[t] = t < len ? idx[s + t] : INT32_MAX;
      if (t < len) vv[t] = val[s + t];
    }
    __syncthreads();
    for (int size = 2; size <= pow2; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = threadIdx.x; t < pow2; t += blockDim.x) {
          int partner = t ^ stride;
          if (partner > t) {
            bool up = (t & size) == 0;
            int32_t a = key[t], b = key[partner];
            if ((a > b) == up) {
              key[t] = b;
              key[partner] = a;
              if (t < CAP && partner < CAP) {
                ValT tv = vv[t];
                vv[t] = vv[partner];
                vv[partner] = tv;
              }
            }
          }
        }
        __syncthreads();
      }
    }
    for (int t = threadIdx.x; t < len; t += blockDim.x) {
      idx[s + t] = key[t];
      val[s + t] = vv[t];
    }
    __syncthreads();
  }
}

cudaError_t launch_sort_rows(int dtype, const int64_t* indptr, int32_t* idx, void* val, int64_t n,
                             cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  int grid = grid_for(n, 1, num_sms, 8);
  note_launches(1);
  switch (dtype) {
    case 0: k_sort_rows<float><<<grid, 256, 0, st>>>(indptr, idx, (float*)val, n); break;
    case 1: k_sort_rows<__nv_bfloat16><<<grid, 256, 0, st>>>(indptr, idx, (__nv_bfloat16*)val, n); break;
    default: k_sort_rows<__half><<<grid, 256, 0, st>>>(indptr, idx, (__half*)val, n); break;
  }
  return cudaGetLastError();
}

}  // namespace scx
