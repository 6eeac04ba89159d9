// Sparse-side kernels: per-gene statistics, value transforms, the forward
// product Y = (X - 1 mu^T) V and the transposed product W = X^T Q on the
// CUDA cores (FP32 products, FP32/FP64 accumulation).
//
// Layouts (all device memory):
//   CSR    : int64 indptr[n+1], int32 indices[nnz], values[nnz] (f32/bf16/f16)
//   V      : float [n_vars][ld]   gene-major, ld = k padded to 32, pad = 0
//   Y, Q   : float [n_obs][ld]    cell-major
//   partial: float [n_chunks][n_vars][ld] per-chunk partial X^T Q
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace scx {

// ---------------------------------------------------------------------------
// Per-gene sums and sums of squares (FP64), in a fixed order: the result is
// bit-identical from run to run.  Restates ScxCsr::col_sums_and_sum_sq
// (scx-sparse/src/csr.rs:570-580).
//
// Block b owns the stored entries [b * per, (b + 1) * per) and walks them in
// windows of kStatsWindow entries.  Its kStatsWarps warps share one FP64
// accumulator pair per gene, and warp w owns the genes j with (j - lo) %
// kStatsWarps == w, so no two warps touch one accumulator and no atomics are
// needed.  Each window is read into registers one window ahead (thread t of
// warp w holds the window's 32-entry steps w, w + 4, ...), then bucketed by
// owning warp with a stable partition (ballot counts per step, one scan, a
// scatter into shared memory), so each warp then walks only its own entries,
// in window order.  Inside one 32-entry step of a bucket two lanes may name
// the same gene only across a row boundary (a sorted row holds a gene once);
// the step is cut into runs of strictly increasing gene index, applied one
// after another in lane order.  Every gene's adds therefore happen in entry
// order, whatever the rows look like (unsorted rows and duplicates included).
// Genes beyond the shared-memory accumulator take further passes over the
// block's entries, kStatsPassGenes at a time.  Each block writes one partial
// row pair [sum | sum sq] (n_vars each); reduce_rows_f64 adds the partials in
// block order.
// ---------------------------------------------------------------------------
constexpr int kStatsWarps = 4;
constexpr int kStatsWindow = 1024;
constexpr int kStatsSteps = kStatsWindow / 32;  // 32-entry steps per window
// shared bytes besides the accumulators: the bucketed window (index + value)
// and the per-step bucket offsets
constexpr size_t kStatsWindowBytes = (size_t)kStatsWindow * 8 + (size_t)kStatsSteps * kStatsWarps * 4 + 64;
constexpr int kStatsPassGenes = (int)((kStatsSmemMax - kStatsWindowBytes) / 16);
static_assert(kStatsSteps == 32, "the bucket scan gives one window step to each lane of a warp");
static_assert(kStatsSteps % kStatsWarps == 0, "every warp holds the same number of window steps");

// `value(p, j, first)` gives entry p's value (gene j) as float; `first` is
// true in the first gene pass.
template <typename Value>
__device__ __forceinline__ void col_stats_body(const int32_t* __restrict__ idx, Value value, int64_t nnz, int32_t g,
                                               int32_t pass_genes, int nparts, int block0,
                                               double* __restrict__ partial) {
  extern __shared__ double sm[];  // [2][pass_genes] accumulators, then the bucketed window
  double* acc = sm;
  int32_t* b_idx = reinterpret_cast<int32_t*>(sm + 2 * (int64_t)pass_genes);
  float* b_val = reinterpret_cast<float*>(b_idx + kStatsWindow);
  int32_t* base = reinterpret_cast<int32_t*>(b_val + kStatsWindow);  // [kStatsSteps][kStatsWarps]
  int32_t* qbase = base + kStatsSteps * kStatsWarps;                 // [kStatsWarps + 1]
  constexpr int kPer = kStatsSteps / kStatsWarps;                    // steps per warp
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const unsigned lanemask_le = 0xffffffffu >> (31 - lane);
  // partition block b of nparts owns entries [b per, (b + 1) per); this
  // launch runs blocks block0 .. block0 + gridDim.x - 1 of it
  const int b = block0 + (int)blockIdx.x;
  const int64_t per = (nnz + nparts - 1) / nparts;
  const int64_t s = min(nnz, (int64_t)b * per);
  const int64_t e = min(nnz, s + per);
  double* out = partial + (int64_t)b * 2 * g;
  for (int32_t lo = 0; lo < g; lo += pass_genes) {
    const int32_t gp = min(pass_genes, g - lo);
    for (int i = threadIdx.x; i < 2 * gp; i += blockDim.x) acc[i] = 0.0;
    // step u of this thread is the window's step kStatsWarps u + warp
    int32_t ri[kPer];
    float rv[kPer];
    auto load = [&](int64_t w) {
      const int c = (int)min((int64_t)kStatsWindow, e - w);
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int t = (kStatsWarps * u + warp) * 32 + lane;
        ri[u] = t < c ? __ldg(idx + w + t) : -1;
        rv[u] = t < c ? value(w + t, ri[u], lo == 0) : 0.f;
      }
    };
    if (s < e) load(s);
    for (int64_t w0 = s; w0 < e; w0 += kStatsWindow) {
      // owning warp of each held entry (kStatsWarps: not in this pass)
      int own[kPer];
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int32_t jr = ri[u] - lo;
        own[u] = (ri[u] >= 0 && jr >= 0 && jr < gp) ? jr % kStatsWarps : kStatsWarps;
      }
      __syncthreads();  // the previous window's buckets are consumed (and the accumulators zeroed)
      // per-step bucket sizes
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int step = kStatsWarps * u + warp;
#pragma unroll
        for (int q = 0; q < kStatsWarps; ++q) {
          const unsigned m = __ballot_sync(0xffffffffu, own[u] == q);
          if (lane == 0) base[step * kStatsWarps + q] = __popc(m);
        }
      }
      __syncthreads();
      // exclusive scan over the steps, bucket by bucket (warp 0; lane = step)
      if (warp == 0) {
        int cnt[kStatsWarps], inc[kStatsWarps];
#pragma unroll
        for (int q = 0; q < kStatsWarps; ++q) {
          cnt[q] = base[lane * kStatsWarps + q];
          inc[q] = cnt[q];
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc[q], o);
            if (lane >= o) inc[q] += y;
          }
        }
        int off = 0;
#pragma unroll
        for (int q = 0; q < kStatsWarps; ++q) {
          const int total = __shfl_sync(0xffffffffu, inc[q], 31);
          base[lane * kStatsWarps + q] = off + inc[q] - cnt[q];
          if (lane == 0) qbase[q] = off;
          off += total;
        }
        if (lane == 0) qbase[kStatsWarps] = off;
      }
      __syncthreads();
      // stable scatter into the buckets
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int step = kStatsWarps * u + warp;
        const int q = own[u];
        const unsigned m = __match_any_sync(0xffffffffu, q);
        if (q < kStatsWarps) {
          const int pos = base[step * kStatsWarps + q] + __popc(m & lanemask_lt);
          b_idx[pos] = ri[u] - lo;
          b_val[pos] = rv[u];
        }
      }
      __syncthreads();
      // the next window's loads are in flight while the buckets are applied
      if (w0 + kStatsWindow < e) load(w0 + kStatsWindow);
      const int q0 = qbase[warp], q1 = qbase[warp + 1];
      for (int p0 = q0; p0 < q1; p0 += 32) {
        const int t = p0 + lane;
        const bool in = t < q1;
        const int32_t jr = in ? b_idx[t] : -1;
        const int32_t jl = __shfl_up_sync(0xffffffffu, jr, 1);
        const unsigned starts = __ballot_sync(0xffffffffu, lane > 0 && in && jr <= jl);
        const double x = in ? (double)b_val[t] : 0.0;
        if (starts == 0) {
          if (in) {
            acc[jr] += x;
            acc[gp + jr] += x * x;
          }
          __syncwarp();  // the next step's lanes see these updates
        } else {
          const int run = __popc(starts & lanemask_le);
          const int runs = __popc(starts) + 1;
          for (int r = 0; r < runs; ++r) {
            if (in && run == r) {
              acc[jr] += x;
              acc[gp + jr] += x * x;
            }
            __syncwarp();
          }
        }
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < gp; i += blockDim.x) {
      out[lo + i] = acc[i];
      out[g + lo + i] = acc[gp + i];
    }
    __syncthreads();
  }
}

template <typename ValT>
__global__ void __launch_bounds__(kStatsWarps * 32) k_col_stats(const int32_t* __restrict__ idx,
                                                                const ValT* __restrict__ val, int64_t nnz,
                                                                int32_t g, int32_t pass_genes, int nparts,
                                                                int block0, double* __restrict__ partial) {
  col_stats_body(idx, [&](int64_t p, int32_t, bool) { return to_f32(val[p]); }, nnz, g, pass_genes, nparts, block0,
                 partial);
}

// The value transform of one entry (k_transform_values, below): the working
// value as stored.
template <typename InT, typename OutT>
__device__ __forceinline__ OutT transform_value(InT v, int32_t j, int mode, const double* __restrict__ mu,
                                                const double* __restrict__ inv_std,
                                                const double* __restrict__ cshift, double clip) {
  double x = (double)to_f32(v);
  if (mode != 0) {
    const double is = __ldg(inv_std + j);
    if (mode == 1) {
      double sv = (x - __ldg(mu + j)) * is;
      if (clip > 0.0) sv = fmin(fmax(sv, -clip), clip);
      x = sv - __ldg(cshift + j);
    } else {
      x = x * is;
      if (clip > 0.0) x = fmin(x, clip);
    }
  }
  return from_f32<OutT>((float)x);
}

// out[i] (+)= sum_{b < nparts} part[b * len + i] in FP64.  A block takes 32
// consecutive outputs (one per lane, coalesced); warp w sums the partials
// b = w, w + 8, ... with four loads in flight, and warp 0 adds the eight warp
// sums in warp order: a fixed order, so the result is deterministic.
// With width > 0 the output is a column panel of a wider matrix: element i
// goes to out[(i / width) * ldo + i % width].
// FP32 partials with len a multiple of 4: the same sums (warp w adds the
// parts w, w + 8, ... in that order, warp 0 the eight warp sums), but a lane
// takes four consecutive outputs with one 16-byte load per part, so a block
// step covers 128 outputs.  A pass over many small partials (the segments of a
// batch) is bound by the latency of its steps, not by bandwidth.
__device__ __forceinline__ void reduce_rows_body_f4(const float* __restrict__ part, int nparts, int64_t len,
                                                    double* __restrict__ out, int accumulate, int width, int ldo,
                                                    int blk, int nblk) {
  __shared__ double red4[8][4 * 32 + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (nparts <= 8) {
    // Warp w of the eight would hold part w alone, and warp 0 would add them
    // in warp order: out + p_0 + p_1 + ... .  The same sums, each warp on its
    // own 128 outputs: one step per chunk instead of a block-wide step with
    // most warps idle (the partials of a batch's small segments).
    for (int64_t base = ((int64_t)blk * 8 + w) * 128; base < len; base += (int64_t)nblk * 8 * 128) {
      const int64_t i = base + 4 * lane;
      if (i >= len) continue;
      float4 v[8];
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (b < nparts) v[b] = *reinterpret_cast<const float4*>(part + (int64_t)b * len + i);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t ie = i + e;
        const int64_t oi = width > 0 ? (ie / width) * ldo + ie % width : ie;
        double acc = accumulate ? out[oi] : 0.0;
#pragma unroll
        for (int b = 0; b < 8; ++b)
          if (b < nparts) acc += (double)(e == 0 ? v[b].x : e == 1 ? v[b].y : e == 2 ? v[b].z : v[b].w);
        out[oi] = acc;
      }
    }
    return;
  }
  for (int64_t base = (int64_t)blk * 128; base < len; base += (int64_t)nblk * 128) {
    const int64_t i = base + 4 * lane;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < len) {
      int b = w;
      for (; b + 24 < nparts; b += 32) {
        const float4 v0 = *reinterpret_cast<const float4*>(part + (int64_t)b * len + i);
        const float4 v1 = *reinterpret_cast<const float4*>(part + (int64_t)(b + 8) * len + i);
        const float4 v2 = *reinterpret_cast<const float4*>(part + (int64_t)(b + 16) * len + i);
        const float4 v3 = *reinterpret_cast<const float4*>(part + (int64_t)(b + 24) * len + i);
        acc[0] += (double)v0.x; acc[1] += (double)v0.y; acc[2] += (double)v0.z; acc[3] += (double)v0.w;
        acc[0] += (double)v1.x; acc[1] += (double)v1.y; acc[2] += (double)v1.z; acc[3] += (double)v1.w;
        acc[0] += (double)v2.x; acc[1] += (double)v2.y; acc[2] += (double)v2.z; acc[3] += (double)v2.w;
        acc[0] += (double)v3.x; acc[1] += (double)v3.y; acc[2] += (double)v3.z; acc[3] += (double)v3.w;
      }
      for (; b < nparts; b += 8) {
        const float4 v = *reinterpret_cast<const float4*>(part + (int64_t)b * len + i);
        acc[0] += (double)v.x; acc[1] += (double)v.y; acc[2] += (double)v.z; acc[3] += (double)v.w;
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) red4[w][4 * lane + e] = acc[e];
    __syncthreads();
    if (w == 0 && i < len) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t ie = i + e;
        const int64_t oi = width > 0 ? (ie / width) * ldo + ie % width : ie;
        double s = accumulate ? out[oi] : 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u) s += red4[u][4 * lane + e];
        out[oi] = s;
      }
    }
    __syncthreads();
  }
}

template <typename T>
__device__ __forceinline__ void reduce_rows_body(const T* __restrict__ part, int nparts, int64_t len,
                                                 double* __restrict__ out, int accumulate, int width, int ldo,
                                                 int blk, int nblk) {
  if constexpr (sizeof(T) == 4) {
    if ((len & 3) == 0 && (reinterpret_cast<uintptr_t>(part) & 15) == 0) {
      reduce_rows_body_f4(part, nparts, len, out, accumulate, width, ldo, blk, nblk);
      return;
    }
  }
  __shared__ double red[8][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int64_t base = (int64_t)blk * 32; base < len; base += (int64_t)nblk * 32) {
    const int64_t i = base + lane;
    double acc = 0.0;
    if (i < len) {
      int b = w;
      for (; b + 24 < nparts; b += 32) {
        const double v0 = (double)part[(int64_t)b * len + i];
        const double v1 = (double)part[(int64_t)(b + 8) * len + i];
        const double v2 = (double)part[(int64_t)(b + 16) * len + i];
        const double v3 = (double)part[(int64_t)(b + 24) * len + i];
        acc += v0;
        acc += v1;
        acc += v2;
        acc += v3;
      }
      for (; b < nparts; b += 8) acc += (double)part[(int64_t)b * len + i];
    }
    red[w][lane] = acc;
    __syncthreads();
    if (w == 0 && i < len) {
      const int64_t oi = width > 0 ? (i / width) * ldo + i % width : i;
      double s = accumulate ? out[oi] : 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u) s += red[u][lane];
      out[oi] = s;
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_reduce_rows(const T* __restrict__ part, int nparts, int64_t len,
                                                     double* __restrict__ out, int accumulate, int width = 0,
                                                     int ldo = 0) {
  reduce_rows_body<T>(part, nparts, len, out, accumulate, width, ldo, blockIdx.x, gridDim.x);
}

// One reduction per grid row y (batched segments): the task's part into its G.
__global__ void __launch_bounds__(256) k_reduce_rows_batch(const GramTask* __restrict__ tasks, int nparts,
                                                           int64_t len) {
  const GramTask t = tasks[blockIdx.y];
  reduce_rows_body<double>(t.part, nparts, len, t.G, 0, 0, 0, blockIdx.x, gridDim.x);
}

// One reduction per grid row y with its own part count (the segments of a
// batch); the sums have the bits of k_reduce_rows on the same partials.
template <typename T>
__global__ void __launch_bounds__(256) k_reduce_rows_sum(const SumTask* __restrict__ tasks, int64_t len) {
  const SumTask t = tasks[blockIdx.y];
  reduce_rows_body<T>(static_cast<const T*>(t.part), t.nparts, len, t.out, 0, 0, 0, blockIdx.x, gridDim.x);
}

cudaError_t launch_reduce_rows_batch(int part_dtype_f32, const SumTask* tasks, int ntasks, int64_t len,
                                     cudaStream_t st) {
  if (ntasks <= 0 || len <= 0) return cudaSuccess;
  const dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>((len + 31) / 32, 64)), (unsigned)ntasks);
  note_launches(1);
  if (part_dtype_f32)
    k_reduce_rows_sum<float><<<grid, 256, 0, st>>>(tasks, len);
  else
    k_reduce_rows_sum<double><<<grid, 256, 0, st>>>(tasks, len);
  return cudaGetLastError();
}

cudaError_t launch_reduce_rows_f64_batch(const GramTask* tasks, int ntasks, int nparts, int64_t len, cudaStream_t st,
                                         int num_sms) {
  if (ntasks <= 0) return cudaSuccess;
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((len + 31) / 32, 16));
  note_launches(1);
  k_reduce_rows_batch<<<dim3((unsigned)gx, (unsigned)ntasks), 256, 0, st>>>(tasks, nparts, len);
  (void)num_sms;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Value transform: convert to the compute type, optionally scale and clip.
//   mode 0: p = x
//   mode 1 (scale, centred):   p = clip((x - mu) * inv_std, +-clip) - c_g
//   mode 2 (scale, uncentred): p = min(x * inv_std, clip)
// c_g = clip(-mu * inv_std) is the value every stored zero takes, so the dense
// scaled matrix is P + 1 c^T with P on X's sparsity pattern.
// ---------------------------------------------------------------------------
template <typename InT, typename OutT>
__global__ void k_transform_values(const int32_t* __restrict__ idx, const InT* __restrict__ in,
                                   OutT* __restrict__ out, int64_t nnz, int mode,
                                   const double* __restrict__ mu, const double* __restrict__ inv_std,
                                   const double* __restrict__ cshift, double clip) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz;
       p += (int64_t)gridDim.x * blockDim.x)
    out[p] = transform_value<InT, OutT>(in[p], mode != 0 ? __ldg(idx + p) : 0, mode, mu, inv_std, cshift, clip);
}

// ---------------------------------------------------------------------------
// Forward product Y[i, :] = sum_p x_p V[j_p, :] - mc.  One warp per row; lane
// l owns columns l + 32 c.  Nonzeros are fetched 32 at a time (coalesced) and
// broadcast by shuffle; V rows are read through the read-only cache (V is
// n_vars x ld x 4 bytes, L2-resident).
// Restates spmm_forward_row (scx-accel/src/pca/cpu.rs:1500-1523) with the
// mean correction of forward_mean_prefactor (scx-gpu/src/gpu_pca.rs:218-237).
// ---------------------------------------------------------------------------
template <int C, typename ValT>
__global__ void __launch_bounds__(256) k_spmm_fwd(const int64_t* __restrict__ indptr,
                                                  const int32_t* __restrict__ idx,
                                                  const ValT* __restrict__ val, int64_t n_obs,
                                                  const float* __restrict__ V, int ldv,
                                                  const float* __restrict__ mc,
                                                  float* __restrict__ Y, int ldy) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  float m[C];
#pragma unroll
  for (int c = 0; c < C; ++c) m[c] = mc ? mc[lane + 32 * c] : 0.f;
  for (int64_t row = warp; row < n_obs; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    float acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0.f;
    for (int64_t base = s; base < e; base += 32) {
      const int64_t p = base + lane;
      int32_t j = 0;
      float x = 0.f;
      if (p < e) {
        j = __ldg(idx + p);
        x = to_f32(val[p]);
      }
      const int cnt = (int)min((int64_t)32, e - base);
      int t = 0;
      for (; t + 4 <= cnt; t += 4) {
        int jj[4];
        float xx[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          jj[u] = __shfl_sync(0xffffffffu, j, t + u);
          xx[u] = __shfl_sync(0xffffffffu, x, t + u);
        }
        float vv[4][C];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int c = 0; c < C; ++c) vv[u][c] = __ldg(V + (int64_t)jj[u] * ldv + lane + 32 * c);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int c = 0; c < C; ++c) acc[c] = fmaf(xx[u], vv[u][c], acc[c]);
      }
      for (; t < cnt; ++t) {
        const int jt = __shfl_sync(0xffffffffu, j, t);
        const float xt = __shfl_sync(0xffffffffu, x, t);
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] = fmaf(xt, __ldg(V + (int64_t)jt * ldv + lane + 32 * c), acc[c]);
      }
    }
    float* yr = Y + row * (int64_t)ldy;
#pragma unroll
    for (int c = 0; c < C; ++c) yr[lane + 32 * c] = acc[c] - m[c];
  }
}

// ---------------------------------------------------------------------------
// Row-block pointer table for the transposed product: for row i and gene
// block b, rbp[i * (nb + 1) + b] = offset (from indptr[i]) of the first stored
// entry of row i whose gene is >= b * gb.  Rows must be sorted by gene.
// ---------------------------------------------------------------------------
__global__ void k_row_block_ptr(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                                int64_t n_obs, int nb, int gb, int32_t* __restrict__ rbp) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n_obs; row += nwarps) {
    const int64_t s = indptr[row], e = indptr[row + 1];
    for (int b = lane; b <= nb; b += 32) {
      const int32_t key = b * gb;
      int64_t lo = s, hi = e;  // first position with idx >= key
      while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (__ldg(idx + mid) < key) lo = mid + 1; else hi = mid;
      }
      rbp[row * (nb + 1) + b] = (int32_t)(lo - s);
    }
  }
}

// ---------------------------------------------------------------------------
// Transposed product, CUDA-core path: block (chunk, b) owns genes
// [b*GB, (b+1)*GB) and the rows of one chunk, accumulates W_part[gene, :] in
// shared memory (FP32 shared atomics) and writes one partial.  Partials are
// reduced in fixed chunk order into FP64 by k_reduce_rows.
// Restates spmm_transpose_block (scx-accel/src/pca/cpu.rs:1282-1328).
// ---------------------------------------------------------------------------
template <int C, typename ValT, int GB>
__global__ void __launch_bounds__(512) k_spmm_t(const int64_t* __restrict__ indptr,
                                                const int32_t* __restrict__ idx,
                                                const ValT* __restrict__ val, int64_t n_obs,
                                                int32_t g, const int32_t* __restrict__ rbp, int nb,
                                                int64_t rows_per_chunk,
                                                const float* __restrict__ Q, int ldq,
                                                float* __restrict__ part) {
  constexpr int LD = 32 * C;
  extern __shared__ float acc[];  // [GB][LD]
  const int b = blockIdx.y;
  const int chunk = blockIdx.x;
  for (int i = threadIdx.x; i < GB * LD; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int64_t r0 = (int64_t)chunk * rows_per_chunk;
  const int64_t r1 = min(n_obs, r0 + rows_per_chunk);
  const int g0 = b * GB;
  for (int64_t row = r0 + wid; row < r1; row += nw) {
    const int64_t base_row = indptr[row];
    const int32_t* rb = rbp + row * (nb + 1);
    const int64_t s = base_row + rb[b], e = base_row + rb[b + 1];
    if (s >= e) continue;
    float q[C];
#pragma unroll
    for (int c = 0; c < C; ++c) q[c] = __ldg(Q + row * (int64_t)ldq + lane + 32 * c);
    for (int64_t base = s; base < e; base += 32) {
      const int64_t p = base + lane;
      int32_t j = 0;
      float x = 0.f;
      if (p < e) {
        j = __ldg(idx + p) - g0;
        x = to_f32(val[p]);
      }
      const int cnt = (int)min((int64_t)32, e - base);
      for (int t = 0; t < cnt; ++t) {
        const int jt = __shfl_sync(0xffffffffu, j, t);
        const float xt = __shfl_sync(0xffffffffu, x, t);
        float* a = acc + jt * LD + lane;
#pragma unroll
        for (int c = 0; c < C; ++c) atomicAdd(a + 32 * c, xt * q[c]);
      }
    }
  }
  __syncthreads();
  float* out = part + (int64_t)chunk * g * LD;
  const int ng = min(GB, g - g0);
  for (int i = threadIdx.x; i < ng * LD; i += blockDim.x) out[(int64_t)g0 * LD + i] = acc[i];
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
template <typename ValT>
static cudaError_t col_stats_blocks_t(const int32_t* idx, const void* val, int64_t nnz, int32_t g,
                                      double* partial, int nparts, int block0, int nblocks, cudaStream_t st) {
  if (nblocks <= 0) return cudaSuccess;
  const ValT* v = static_cast<const ValT*>(val);
  const int32_t pass_genes = std::min<int32_t>(g, kStatsPassGenes);
  const size_t smem = (size_t)2 * pass_genes * sizeof(double) + kStatsWindowBytes;
  if (smem > 48 * 1024) {
    if (cudaError_t e = allow_smem(k_col_stats<ValT>, smem); e != cudaSuccess) return e;
  }
  k_col_stats<ValT><<<nblocks, kStatsWarps * 32, smem, st>>>(idx, v, nnz, g, pass_genes, nparts, block0, partial);
  note_launches(1);
  return cudaGetLastError();
}

int64_t col_stats_block_begin(int64_t nnz, int nparts, int b) {
  const int64_t per = (nnz + nparts - 1) / nparts;
  return std::min(nnz, (int64_t)b * per);
}

cudaError_t launch_col_stats_blocks(int dtype, const int32_t* idx, const void* val, int64_t nnz, int32_t g,
                                    double* partial, int nparts, int block0, int nblocks, cudaStream_t st) {
  switch (dtype) {
    case 0: return col_stats_blocks_t<float>(idx, val, nnz, g, partial, nparts, block0, nblocks, st);
    case 1: return col_stats_blocks_t<__nv_bfloat16>(idx, val, nnz, g, partial, nparts, block0, nblocks, st);
    default: return col_stats_blocks_t<__half>(idx, val, nnz, g, partial, nparts, block0, nblocks, st);
  }
}

cudaError_t launch_col_stats_reduce(const double* partial, int nparts, int32_t g, double* out, cudaStream_t st,
                                    int num_sms, int accumulate) {
  k_reduce_rows<double><<<grid_for(2 * g, 256, num_sms), 256, 0, st>>>(partial, nparts, 2 * (int64_t)g, out,
                                                                      accumulate);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_col_stats(int dtype, const int32_t* idx, const void* val, int64_t nnz,
                             int32_t g, double* partial, int nparts, double* out,
                             cudaStream_t st, int num_sms, int accumulate) {
  cudaError_t e = launch_col_stats_blocks(dtype, idx, val, nnz, g, partial, nparts, 0, nparts, st);
  if (e != cudaSuccess) return e;
  return launch_col_stats_reduce(partial, nparts, g, out, st, num_sms, accumulate);
}

template <typename InT>
static cudaError_t transform_in(int out_dtype, const int32_t* idx, const void* in, void* out,
                                int64_t nnz, int mode, const double* mu, const double* inv_std,
                                const double* cshift, double clip, cudaStream_t st, int num_sms) {
  const InT* src = static_cast<const InT*>(in);
  int grid = grid_for(nnz, 256, num_sms);
  note_launches(1);
  switch (out_dtype) {
    case 0: k_transform_values<InT, float><<<grid, 256, 0, st>>>(idx, src, (float*)out, nnz, mode, mu, inv_std, cshift, clip); break;
    case 1: k_transform_values<InT, __nv_bfloat16><<<grid, 256, 0, st>>>(idx, src, (__nv_bfloat16*)out, nnz, mode, mu, inv_std, cshift, clip); break;
    default: k_transform_values<InT, __half><<<grid, 256, 0, st>>>(idx, src, (__half*)out, nnz, mode, mu, inv_std, cshift, clip); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_transform_values(int in_dtype, int out_dtype, const int32_t* idx, const void* in,
                                    void* out, int64_t nnz, int mode, const double* mu,
                                    const double* inv_std, const double* cshift, double clip,
                                    cudaStream_t st, int num_sms) {
  if (nnz == 0) return cudaSuccess;
  switch (in_dtype) {
    case 0: return transform_in<float>(out_dtype, idx, in, out, nnz, mode, mu, inv_std, cshift, clip, st, num_sms);
    case 1: return transform_in<__nv_bfloat16>(out_dtype, idx, in, out, nnz, mode, mu, inv_std, cshift, clip, st, num_sms);
    default: return transform_in<__half>(out_dtype, idx, in, out, nnz, mode, mu, inv_std, cshift, clip, st, num_sms);
  }
}

template <int C, typename ValT>
static cudaError_t fwd_c(const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                         const float* V, int ldv, const float* mc, float* Y, int ldy,
                         cudaStream_t st, int num_sms) {
  int grid = grid_for(n * 32, 256, num_sms, 8);
  note_launches(1);
  k_spmm_fwd<C, ValT><<<grid, 256, 0, st>>>(indptr, idx, static_cast<const ValT*>(val), n, V, ldv,
                                            mc, Y, ldy);
  return cudaGetLastError();
}

template <typename ValT>
static cudaError_t fwd_t(int ld, const int64_t* indptr, const int32_t* idx, const void* val,
                         int64_t n, const float* V, int ldv, const float* mc, float* Y, int ldy,
                         cudaStream_t st, int num_sms) {
  switch (ld) {
    case 32: return fwd_c<1, ValT>(indptr, idx, val, n, V, ldv, mc, Y, ldy, st, num_sms);
    case 64: return fwd_c<2, ValT>(indptr, idx, val, n, V, ldv, mc, Y, ldy, st, num_sms);
    case 96: return fwd_c<3, ValT>(indptr, idx, val, n, V, ldv, mc, Y, ldy, st, num_sms);
    default: return fwd_c<4, ValT>(indptr, idx, val, n, V, ldv, mc, Y, ldy, st, num_sms);
  }
}

cudaError_t launch_spmm_fwd(int dtype, int ld, const int64_t* indptr, const int32_t* idx,
                            const void* val, int64_t n, const float* V, const float* mc,
                            float* Y, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  switch (dtype) {
    case 0: return fwd_t<float>(ld, indptr, idx, val, n, V, ld, mc, Y, ld, st, num_sms);
    case 1: return fwd_t<__nv_bfloat16>(ld, indptr, idx, val, n, V, ld, mc, Y, ld, st, num_sms);
    default: return fwd_t<__half>(ld, indptr, idx, val, n, V, ld, mc, Y, ld, st, num_sms);
  }
}

cudaError_t launch_row_block_ptr(const int64_t* indptr, const int32_t* idx, int64_t n, int nb,
                                 int gb, int32_t* rbp, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  note_launches(1);
  k_row_block_ptr<<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(indptr, idx, n, nb, gb, rbp);
  return cudaGetLastError();
}

template <int C, typename ValT>
static cudaError_t spmm_t_c(const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                            int32_t g, const int32_t* rbp, int nb, int nchunks,
                            int64_t rows_per_chunk, const float* Q, int ldq, float* part,
                            cudaStream_t st) {
  constexpr int GB = kTransposeGeneBlock;
  size_t smem = (size_t)GB * 32 * C * sizeof(float);
  auto kern = k_spmm_t<C, ValT, GB>;
  if (cudaError_t e = allow_smem(kern, smem); e != cudaSuccess) return e;
  dim3 grid(nchunks, nb);
  note_launches(1);
  kern<<<grid, 512, smem, st>>>(indptr, idx, static_cast<const ValT*>(val), n, g, rbp, nb,
                                rows_per_chunk, Q, ldq, part);
  return cudaGetLastError();
}

template <typename ValT>
static cudaError_t spmm_t_t(int ld, const int64_t* indptr, const int32_t* idx, const void* val,
                            int64_t n, int32_t g, const int32_t* rbp, int nb, int nchunks,
                            int64_t rpc, const float* Q, float* part, cudaStream_t st) {
  switch (ld) {
    case 32: return spmm_t_c<1, ValT>(indptr, idx, val, n, g, rbp, nb, nchunks, rpc, Q, ld, part, st);
    case 64: return spmm_t_c<2, ValT>(indptr, idx, val, n, g, rbp, nb, nchunks, rpc, Q, ld, part, st);
    case 96: return spmm_t_c<3, ValT>(indptr, idx, val, n, g, rbp, nb, nchunks, rpc, Q, ld, part, st);
    default: return spmm_t_c<4, ValT>(indptr, idx, val, n, g, rbp, nb, nchunks, rpc, Q, ld, part, st);
  }
}

cudaError_t launch_spmm_t(int dtype, int ld, const int64_t* indptr, const int32_t* idx,
                          const void* val, int64_t n, int32_t g, const int32_t* rbp, int nb,
                          int nchunks, int64_t rows_per_chunk, const float* Q, float* part,
                          cudaStream_t st) {
  switch (dtype) {
    case 0: return spmm_t_t<float>(ld, indptr, idx, val, n, g, rbp, nb, nchunks, rows_per_chunk, Q, part, st);
    case 1: return spmm_t_t<__nv_bfloat16>(ld, indptr, idx, val, n, g, rbp, nb, nchunks, rows_per_chunk, Q, part, st);
    default: return spmm_t_t<__half>(ld, indptr, idx, val, n, g, rbp, nb, nchunks, rows_per_chunk, Q, part, st);
  }
}

cudaError_t launch_reduce_rows_f32(const float* part, int nparts, int64_t len, double* out,
                                   int accumulate, cudaStream_t st, int num_sms) {
  note_launches(1);
  k_reduce_rows<float><<<grid_for(len, 32, num_sms), 256, 0, st>>>(part, nparts, len, out, accumulate);
  return cudaGetLastError();
}

cudaError_t launch_reduce_panel_f32(const float* part, int nparts, int64_t rows, int width, double* out, int ldo,
                                    cudaStream_t st, int num_sms) {
  const int64_t len = rows * width;
  note_launches(1);
  k_reduce_rows<float><<<grid_for(len, 32, num_sms), 256, 0, st>>>(part, nparts, len, out, 0, width, ldo);
  return cudaGetLastError();
}

cudaError_t launch_reduce_rows_f64(const double* part, int nparts, int64_t len, double* out,
                                   int accumulate, cudaStream_t st, int num_sms) {
  note_launches(1);
  k_reduce_rows<double><<<grid_for(len, 32, num_sms), 256, 0, st>>>(part, nparts, len, out, accumulate);
  return cudaGetLastError();
}

}  // namespace scx
