// Upstream producers of the PCA's input on the device: per-row
// normalize_total + log1p (with an optional explicit per-row factor) and the
// column projection behind mask_var / highly_variable, so a raw-count matrix
// that is already resident never leaves the GPU on its way to the PCA.
//
// Restate normalize_log1p_kernel / normalize_kernel / log1p_kernel /
// row_scale_kernel (scx-gpu/kernels/normalize_log1p.cu:17-140, dispatched by
// gpu_apply_fused_ops, scx-gpu/src/gpu_preprocess.rs:340-391) and the
// sorted-merge column projection of ProjectedShardSource
// (scx-accel/src/projected_source.rs:28-80, scx_engine::project_csr).
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace scx {

// ---------------------------------------------------------------------------
// One warp per row.  The row sum is accumulated in FP64 (lanes strided over
// the row, then a fixed-order butterfly), so the factor target / sum is the
// one the reference's CPU path forms in f64 (scx-engine fused_ops: value_f64
// * factor, rounded to f32, then ln_1p).  A row whose sum is zero is left as
// it is (its scale is undefined and log1p(0) = 0).  The explicit per-row
// factor, when given, multiplies last.  `in` and `out` may be the same array
// (in place): every value is read by the lane that writes it, and a row's
// reads for its sum finish (warp shuffle) before its writes begin.
// ---------------------------------------------------------------------------
__global__ void k_normalize_log1p(const int64_t* __restrict__ indptr, const float* in, float* out, int64_t n,
                                  double target_sum, int do_log1p, const float* __restrict__ row_factor) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    double factor = 1.0;
    bool skip = false;
    if (target_sum > 0.0) {
      double acc = 0.0;
      for (int64_t p = s + lane; p < e; p += 32) acc += (double)in[p];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (acc == 0.0) skip = true;
      else factor = target_sum / acc;
    }
    const float rf = row_factor ? row_factor[row] : 1.f;
    for (int64_t p = s + lane; p < e; p += 32) {
      float v = in[p];
      if (!skip) {
        if (target_sum > 0.0) v = (float)((double)v * factor);
        if (do_log1p) v = log1pf(v);
      }
      if (row_factor) v *= rf;
      out[p] = v;
    }
  }
}

cudaError_t launch_normalize_log1p(const int64_t* indptr, const float* in, float* out, int64_t n,
                                   double target_sum, int do_log1p, const float* row_factor, cudaStream_t st,
                                   int num_sms) {
  if (n == 0) return cudaSuccess;
  k_normalize_log1p<<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(indptr, in, out, n, target_sum, do_log1p,
                                                                      row_factor);
  note_launches(1);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Column projection.  col_map[j] is the new index of input column j, or -1
// when the column is dropped; new indices must increase with j (a sorted
// selection), so a sorted row stays sorted.  Pass 1 counts the kept entries
// per row (one warp per row, ballot counts); an exclusive scan of the counts
// gives the output indptr; pass 2 writes the kept entries in row order, each
// warp compacting 32 entries at a time by ballot prefix.
// ---------------------------------------------------------------------------
__global__ void k_project_count(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx, int64_t n,
                                const int32_t* __restrict__ col_map, int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    int64_t c = 0;
    for (int64_t b = s; b < e; b += 32) {
      const int64_t p = b + lane;
      const bool keep = p < e && __ldg(col_map + __ldg(idx + p)) >= 0;
      c += __popc(__ballot_sync(0xffffffffu, keep));
    }
    if (lane == 0) counts[row] = c;
  }
}

__global__ void k_project_fill(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                               const float* __restrict__ val, int64_t n, const int32_t* __restrict__ col_map,
                               const int64_t* __restrict__ out_ptr, int32_t* __restrict__ out_idx,
                               float* __restrict__ out_val) {
  const int lane = threadIdx.x & 31;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    int64_t o = out_ptr[row];
    for (int64_t b = s; b < e; b += 32) {
      const int64_t p = b + lane;
      const int32_t nj = p < e ? __ldg(col_map + __ldg(idx + p)) : -1;
      const unsigned m = __ballot_sync(0xffffffffu, nj >= 0);
      if (nj >= 0) {
        const int64_t q = o + __popc(m & lanemask_lt);
        out_idx[q] = nj;
        out_val[q] = val[p];
      }
      o += __popc(m);
    }
  }
}

cudaError_t launch_project_count(const int64_t* indptr, const int32_t* idx, int64_t n, const int32_t* col_map,
                                 int64_t* counts, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  k_project_count<<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(indptr, idx, n, col_map, counts);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_project_fill(const int64_t* indptr, const int32_t* idx, const float* val, int64_t n,
                                const int32_t* col_map, const int64_t* out_ptr, int32_t* out_idx, float* out_val,
                                cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  k_project_fill<<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(indptr, idx, val, n, col_map, out_ptr, out_idx,
                                                                   out_val);
  note_launches(1);
  return cudaGetLastError();
}

}  // namespace scx

namespace scx {

// ---------------------------------------------------------------------------
// PFlog (v4) on the device.  Restates pflog_baseline_from_raw
// (scx-accel/src/pflog.rs:122-193) and the lazy Scale{4 alpha} -> Log1p
// source it pairs with: delta = log1p(four_alpha * x) at the stored entries
// and b_i = -(1 / D) sum_j delta_ij in FP64, one warp per row.  flags[0] is
// set by a negative count, flags[1] by a non-finite one (the raw-count guard
// of pflog.rs:47-60, 150-160).
// ---------------------------------------------------------------------------
__global__ void k_pflog_prepare(const int64_t* __restrict__ indptr, const float* __restrict__ x, int64_t n,
                                double four_alpha, double inv_d, float* __restrict__ delta,
                                double* __restrict__ baseline, int32_t* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    double acc = 0.0;
    bool neg = false, bad = false;
    for (int64_t p = s + lane; p < e; p += 32) {
      const float v = x[p];
      if (!isfinite(v)) bad = true;
      else if (v < 0.f) neg = true;
      const double d = log1p(four_alpha * (double)v);
      delta[p] = (float)d;
      acc += d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (__any_sync(0xffffffffu, neg) && lane == 0) atomicOr(flags + 0, 1);
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flags + 1, 1);
    if (lane == 0) baseline[row] = -acc * inv_d;
  }
}

cudaError_t launch_pflog_prepare(const int64_t* indptr, const float* x, int64_t n, int64_t d, double four_alpha,
                                 float* delta, double* baseline, int32_t* flags, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  k_pflog_prepare<<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(indptr, x, n, four_alpha, 1.0 / (double)d,
                                                                    delta, baseline, flags);
  note_launches(1);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The baseline-aware PCA of Z = delta + b 1^T (pflog_pca, scx-accel/src/pca/
// cpu.rs:815-882) runs on an augmented matrix A = [delta | b] with one extra
// column g: Z = A E with E = [I; 1^T], so Z V = A [V; 1^T V] and
// Z^T Q = [I, 1] A^T Q.  The forward product sees the extra row
// V[g] = 1^T V; the transposed product's extra row W[g] = b^T Q is folded into
// every gene's row and cleared.  Both rank-1 terms of the reference's
// streaming_spmm_*_offset (cpu.rs:618-687) come out of the ordinary products.
// ---------------------------------------------------------------------------
template <typename ValT>
__global__ void k_pflog_augment(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                                const ValT* __restrict__ val, int64_t n, int32_t g,
                                const double* __restrict__ baseline, int64_t* __restrict__ aptr,
                                int32_t* __restrict__ aidx, ValT* __restrict__ aval, double* __restrict__ cross) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t base0 = indptr[0];
  for (int64_t row = warp; row < n; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    const int64_t o = s - base0 + row;  // this row's first position in the augmented arrays
    double acc = 0.0;
    for (int64_t p = s + lane; p < e; p += 32) {
      const ValT v = val[p];
      aidx[o + (p - s)] = idx[p];
      aval[o + (p - s)] = v;
      acc += (double)to_f32(v);
    }
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o2);
    if (lane == 0) {
      const double b = baseline[row];
      aidx[o + (e - s)] = g;
      aval[o + (e - s)] = from_f32<ValT>((float)b);
      aptr[row] = o;
      cross[row] = b * acc;  // b_i * rowsum(delta_i), for the total variance
      if (row == n - 1) aptr[n] = o + (e - s) + 1;
    }
  }
}

// V[g][c] = sum_{j < g} V[j][c] (FP64 in gene order, rounded once).
__global__ void k_aug_colsum(float* __restrict__ V, int32_t g, int ld) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ld) return;
  double s = 0.0;
  for (int32_t j = 0; j < g; ++j) s += (double)V[(int64_t)j * ld + c];
  V[(int64_t)g * ld + c] = (float)s;
}

// W[j] += W[g] for j < g, then W[g] = 0 (FP64 gene-side rows of ld).
__global__ void k_aug_fold(double* __restrict__ W, int32_t g, int ld) {
  const int64_t total = (int64_t)g * ld;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x)
    W[t] += W[(int64_t)g * ld + (t % ld)];
}
__global__ void k_aug_clear(double* __restrict__ W, int32_t g, int ld) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ld) W[(int64_t)g * ld + c] = 0.0;
}

template <typename ValT>
static cudaError_t pflog_augment_t(const int64_t* indptr, const int32_t* idx, const void* val, int64_t n, int32_t g,
                                   const double* baseline, int64_t* aptr, int32_t* aidx, void* aval, double* cross,
                                   cudaStream_t st, int num_sms) {
  k_pflog_augment<ValT><<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(
      indptr, idx, static_cast<const ValT*>(val), n, g, baseline, aptr, aidx, static_cast<ValT*>(aval), cross);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_pflog_augment(int dtype, const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                                 int32_t g, const double* baseline, int64_t* aptr, int32_t* aidx, void* aval,
                                 double* cross, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  switch (dtype) {
    case 0: return pflog_augment_t<float>(indptr, idx, val, n, g, baseline, aptr, aidx, aval, cross, st, num_sms);
    case 1:
      return pflog_augment_t<__nv_bfloat16>(indptr, idx, val, n, g, baseline, aptr, aidx, aval, cross, st, num_sms);
    default: return pflog_augment_t<__half>(indptr, idx, val, n, g, baseline, aptr, aidx, aval, cross, st, num_sms);
  }
}

cudaError_t launch_aug_colsum(float* V, int32_t g, int ld, cudaStream_t st) {
  k_aug_colsum<<<(ld + 63) / 64, 64, 0, st>>>(V, g, ld);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_aug_fold(double* W, int32_t g, int ld, cudaStream_t st, int num_sms) {
  k_aug_fold<<<grid_for((int64_t)g * ld, 256, num_sms, 4), 256, 0, st>>>(W, g, ld);
  k_aug_clear<<<(ld + 63) / 64, 64, 0, st>>>(W, g, ld);
  note_launches(2);
  return cudaGetLastError();
}

__global__ void k_rebase_indptr(int64_t* __restrict__ indptr, int64_t n, int64_t base) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    indptr[i] -= base;
}

cudaError_t launch_rebase_indptr(int64_t* indptr, int64_t n, int64_t base, cudaStream_t st, int num_sms) {
  k_rebase_indptr<<<grid_for(n + 1, 256, num_sms, 4), 256, 0, st>>>(indptr, n, base);
  note_launches(1);
  return cudaGetLastError();
}

}  // namespace scx
