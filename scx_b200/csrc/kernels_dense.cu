// Dense-side kernels of the randomized PCA: tall Gram matrices (FP64
// accumulation), Cholesky + triangular inverse and the symmetric Jacobi
// eigensolver (single block, FP64), right-multiplications by small k x k
// factors, the Rayleigh-Ritz finish, embeddings and the seeded Gaussian test
// matrix.
//
// The small factorisations replace cuSOLVER potrf/trsm (scx-gpu/src/
// cusolver.rs:297-409) and the host faer thin SVD of B (scx-gpu/src/
// gpu_pca.rs:593-611): all of them stay on the device in FP64.
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace scx {

// ---------------------------------------------------------------------------
// Gram partials.  Block b owns a contiguous row range; the 16 x 16 thread grid
// owns output entries (ty + 16 i, tx + 16 j), i <= j < T = ld / 16 (the 16 x 16
// blocks on and above the diagonal, mirrored below it), so the shared row
// reads of a warp hit consecutive banks.  Products of float inputs are
// exact in FP64; accumulation is FP64.
// ---------------------------------------------------------------------------
template <typename T, int LD>
__device__ __forceinline__ void gram_body(const T* __restrict__ A, int64_t n, double* __restrict__ part, int b,
                                          int nb) {
  constexpr int TT = LD / 16;
  constexpr int R = 32;  // rows staged per step
  __shared__ double sh[R][LD];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[TT][TT];
#pragma unroll
  for (int i = 0; i < TT; ++i)
#pragma unroll
    for (int j = 0; j < TT; ++j) acc[i][j] = 0.0;
  double csum = 0.0;
  const int64_t per = (n + nb - 1) / nb;
  const int64_t r0 = (int64_t)b * per;
  const int64_t r1 = min(n, r0 + per);
  for (int64_t base = r0; base < r1; base += R) {
    const int rows = (int)min((int64_t)R, r1 - base);
    for (int t = threadIdx.x; t < R * LD; t += 256) {
      int r = t / LD, c = t % LD;
      sh[r][c] = r < rows ? (double)A[(base + r) * LD + c] : 0.0;
    }
    __syncthreads();
    for (int r = 0; r < rows; ++r) {
      double a[TT], b[TT];
#pragma unroll
      for (int i = 0; i < TT; ++i) a[i] = sh[r][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < TT; ++j) b[j] = sh[r][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < TT; ++i)
#pragma unroll
        for (int j = 0; j < TT; ++j)
          if (i <= j) acc[i][j] = fma(a[i], b[j], acc[i][j]);  // blocks on and above the diagonal
    }
    if (threadIdx.x < LD)
      for (int r = 0; r < rows; ++r) csum += sh[r][threadIdx.x];
    __syncthreads();
  }
  // The Gram is symmetric: block (j, i) below the diagonal is the transpose of
  // block (i, j), whose entry (a, b) is the same FMA chain over the rows with
  // the two factors of each product swapped, which fma rounds identically.
  double* out = part + (int64_t)b * (LD * LD + LD);
#pragma unroll
  for (int i = 0; i < TT; ++i)
#pragma unroll
    for (int j = 0; j < TT; ++j)
      if (i <= j) {
        out[(ty + 16 * i) * LD + tx + 16 * j] = acc[i][j];
        if (i < j) out[(tx + 16 * j) * LD + ty + 16 * i] = acc[i][j];
      }
  if (threadIdx.x < LD) out[LD * LD + threadIdx.x] = csum;
}

template <typename T, int LD>
__global__ void __launch_bounds__(256) k_gram(const T* __restrict__ A, int64_t n, double* __restrict__ part) {
  gram_body<T, LD>(A, n, part, blockIdx.x, gridDim.x);
}

// One FP64 matrix per grid row y (batched segments): partials into the task's part.
template <int LD>
__global__ void __launch_bounds__(256) k_gram_batch(const GramTask* __restrict__ tasks, int64_t n) {
  const GramTask t = tasks[blockIdx.y];
  gram_body<double, LD>(t.A, n, t.part, blockIdx.x, gridDim.x);
}

cudaError_t launch_gram_f64_batch(const GramTask* tasks, int ntasks, int64_t n, int ld, int nparts,
                                  cudaStream_t st, int num_sms) {
  if (ntasks <= 0) return cudaSuccess;
  const dim3 grid((unsigned)nparts, (unsigned)ntasks);
  note_launches(1);
  switch (ld) {
    case 32: k_gram_batch<32><<<grid, 256, 0, st>>>(tasks, n); break;
    case 64: k_gram_batch<64><<<grid, 256, 0, st>>>(tasks, n); break;
    case 96: k_gram_batch<96><<<grid, 256, 0, st>>>(tasks, n); break;
    case 128: k_gram_batch<128><<<grid, 256, 0, st>>>(tasks, n); break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_rows_f64_batch(tasks, ntasks, nparts, (int64_t)ld * ld + ld, st, num_sms);
}

template <typename T>
static cudaError_t gram_t(const T* A, int64_t n, int ld, double* part, int nparts, cudaStream_t st) {
  if (ld > kMaxK) {
    if constexpr (sizeof(T) == 4) return launch_gram_wide_f32(reinterpret_cast<const float*>(A), n, ld, part, nparts, st);
    else return launch_gram_wide_f64(reinterpret_cast<const double*>(A), n, ld, part, nparts, st);
  }
  note_launches(1);
  switch (ld) {
    case 32: k_gram<T, 32><<<nparts, 256, 0, st>>>(A, n, part); break;
    case 64: k_gram<T, 64><<<nparts, 256, 0, st>>>(A, n, part); break;
    case 96: k_gram<T, 96><<<nparts, 256, 0, st>>>(A, n, part); break;
    default: k_gram<T, 128><<<nparts, 256, 0, st>>>(A, n, part); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_gram_f32(const float* A, int64_t n, int ld, double* part, int nparts,
                            cudaStream_t st) {
  return gram_t<float>(A, n, ld, part, nparts, st);
}
cudaError_t launch_gram_f64(const double* A, int64_t n, int ld, double* part, int nparts,
                            cudaStream_t st) {
  return gram_t<double>(A, n, ld, part, nparts, st);
}

// ---------------------------------------------------------------------------
// Cholesky of the leading k x k block of G (ld x ld) and the inverse of its
// factor, one block of T x T threads.  A pivot j fails when its Schur
// complement d_j <= tau * G_jj (the column is numerically dependent on the
// previous ones) or is not finite.  With shift_on_fail the factorisation
// restarts once on G + s I, s = 10 tau max_j G_jj, which always succeeds on
// finite input.
//
// Symmetric Gaussian elimination of the augmented matrix [A | I]: step j
// subtracts (A_ja / d_j) times row j from every row a > j, which turns A's
// upper triangle into D L^T and the identity into X = L^{-1} (unit lower
// triangular), where A = L D L^T.  Then R = D^{1/2} L^T and
// R^{-1} = X^T D^{-1/2}: R_jc = A_jc / sqrt(d_j), R^{-1}_ca = X_ac / sqrt(d_a).
// Every matrix entry lives in a register of its owner, thread (ty, tx) owning
// rows ty + T u and columns tx + T v; one register holds A_ac above the
// diagonal (c >= a) or X_ac below it.  Per step the owners of row j + 1
// publish it (double-buffered rows in shared memory) and the owner of the
// next diagonal entry computes the next pivot's reciprocals, so a step is
// one barrier plus a short dependent chain.
// ---------------------------------------------------------------------------
// With `tasks` set, block b factors the matrix of tasks[b] (many segments'
// factorisations in one launch, one block each) and the pointer arguments are
// ignored.
template <int U, int T>
__global__ void __launch_bounds__(T * T) k_cholesky(const double* __restrict__ G, int k, int ld, double tau,
                                                   int shift_on_fail, double* __restrict__ R,
                                                   double* __restrict__ Rinv, float* __restrict__ Rinv_f,
                                                   int* __restrict__ status, const CholTask* __restrict__ tasks) {
  if (tasks) {
    const CholTask t = tasks[blockIdx.x];
    G = t.G;
    R = t.R;
    Rinv = t.Rinv;
    Rinv_f = t.Rinv_f;
    status = t.status;
  }
  __shared__ double rowA[2][kMaxK], rowX[2][kMaxK];
  __shared__ double pv_rinv[kMaxK], pv_di[kMaxK], dg[kMaxK];
  __shared__ int pv_ok[kMaxK];
  __shared__ double maxdiag_s;
  __shared__ int fail_s;
  constexpr int NT = T * T;
  const int tid = threadIdx.x, tx = tid % T, ty = tid / T;
  for (int j = tid; j < k; j += NT) dg[j] = G[(int64_t)j * ld + j];
  for (int t = tid; t < ld * ld; t += NT) {
    R[t] = 0.0;
    Rinv[t] = 0.0;
    Rinv_f[t] = 0.f;
  }
  __syncthreads();
  if (tid < 32) {
    double m = 0.0;
    for (int j = tid; j < k; j += 32) m = fmax(m, dg[j]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (tid == 0) maxdiag_s = m;
  }
  double shift = 0.0;
  int fail = -1;
  double val[U][U];
  for (int attempt = 0; attempt < 2; ++attempt) {
    // Pivot j from its updated diagonal entry d (called by the entry's owner).
    auto pivot = [&](int j, double d) {
      const bool ok = isfinite(d) && d > 0.0 && (attempt == 1 || d > tau * (dg[j] + shift));
      pv_ok[j] = ok ? 1 : 0;
      if (ok) {
        const double rinv = d >= 1e-300 ? rsqrt_nr(d) : rsqrt(d);
        pv_rinv[j] = rinv;
        pv_di[j] = rinv * rinv;
      }
    };
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int v = 0; v < U; ++v) {
        const int a = ty + T * u, c = tx + T * v;
        double x = 0.0;
        if (a < k && c < k) {
          if (c >= a) x = G[(int64_t)a * ld + c] + (a == c ? shift : 0.0);
        }
        val[u][v] = x;  // X starts as the identity; its unit diagonal is implicit
      }
    if (ty == 0) {
#pragma unroll
      for (int v = 0; v < U; ++v) {
        const int c = tx + T * v;
        if (c < k) {
          rowA[0][c] = val[0][v];
          rowX[0][c] = c == 0 ? 1.0 : 0.0;
        }
      }
    }
    if (tid == 0) {
      fail_s = -1;
      pivot(0, val[0][0]);
    }
    __syncthreads();
    for (int j = 0; j < k; ++j) {
      if (!pv_ok[j]) {  // every thread reads the same flag: uniform exit
        if (tid == 0) fail_s = j;
        break;
      }
      const int b = j & 1;
      const double di = pv_di[j], rj = pv_rinv[j];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int a = ty + T * u;
        if (a == j) {  // row j is final: R_jc = A_jc / sqrt(d_j)
#pragma unroll
          for (int v = 0; v < U; ++v) {
            const int c = tx + T * v;
            if (c >= j && c < k) R[(int64_t)j * ld + c] = val[u][v] * rj;
          }
        }
        if (a > j && a < k) {
          const double m = rowA[b][a] * di;
#pragma unroll
          for (int v = 0; v < U; ++v) {
            const int c = tx + T * v;
            if (c < k) {
              if (c >= a) val[u][v] -= m * rowA[b][c];
              else if (c <= j) val[u][v] -= m * rowX[b][c];
            }
          }
          if (a == j + 1) {  // publish row j + 1 for the next step
#pragma unroll
            for (int v = 0; v < U; ++v) {
              const int c = tx + T * v;
              if (c < k) {
                if (c >= a) rowA[b ^ 1][c] = val[u][v];
                if (c < a) rowX[b ^ 1][c] = val[u][v];
                if (c == a) {
                  rowX[b ^ 1][c] = 1.0;
                  pivot(a, val[u][v]);
                }
              }
            }
          }
        }
      }
      __syncthreads();
    }
    __syncthreads();
    fail = fail_s;
    if (fail < 0) break;
    if (!shift_on_fail || attempt == 1) {
      if (tid == 0) status[0] = -(fail + 1);
      // Leave well-defined (identity) factors so downstream kernels stay finite.
      for (int t = tid; t < ld * ld; t += NT) {
        const int r = t / ld, c = t % ld;
        const double v = (r == c && r < k) ? 1.0 : 0.0;
        R[t] = v;
        Rinv[t] = v;
        Rinv_f[t] = (float)v;
      }
      return;
    }
    if (tid == 0) status[0] += 1;
    shift = 10.0 * tau * fmax(maxdiag_s, 1e-300);
    __syncthreads();
  }
  // R^{-1}_ca = X_ac / sqrt(d_a), c <= a.
#pragma unroll
  for (int u = 0; u < U; ++u)
#pragma unroll
    for (int v = 0; v < U; ++v) {
      const int a = ty + T * u, c = tx + T * v;
      if (a < k && c <= a) {
        const double x = (c == a ? 1.0 : val[u][v]) * pv_rinv[a];
        Rinv[(int64_t)c * ld + a] = x;
        Rinv_f[(int64_t)c * ld + a] = (float)x;
      }
    }
}

cudaError_t launch_cholesky(const double* G, int k, int ld, double tau, int shift_on_fail,
                            double* R, double* Rinv, float* Rinv_f, int* status, cudaStream_t st) {
  if (ld > kMaxK) return launch_cholesky_wide(G, k, ld, tau, shift_on_fail, R, Rinv, Rinv_f, status, st);
  if (k > kMaxK) return cudaErrorInvalidValue;
  note_launches(1);
  // 32 x 32 threads, 2 x 2 entries each for k <= 64 (measured per 60 x 60
  // factor: 51 us, against 61 us for 16 x 16 threads with 4 x 4 entries, and
  // 94 us for 8 warps updating rows of the matrix held in shared memory)
  if (k <= 64)
    k_cholesky<2, 32><<<1, 1024, 0, st>>>(G, k, ld, tau, shift_on_fail, R, Rinv, Rinv_f, status, nullptr);
  else
    k_cholesky<4, 32><<<1, 1024, 0, st>>>(G, k, ld, tau, shift_on_fail, R, Rinv, Rinv_f, status, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_cholesky_batch(const CholTask* tasks, int ntasks, int k, int ld, double tau, int shift_on_fail,
                                  cudaStream_t st) {
  if (k > kMaxK || ld > kMaxK) return cudaErrorInvalidValue;
  if (ntasks <= 0) return cudaSuccess;
  note_launches(1);
  if (k <= 64)
    k_cholesky<2, 32><<<ntasks, 1024, 0, st>>>(nullptr, k, ld, tau, shift_on_fail, nullptr, nullptr, nullptr, nullptr,
                                               tasks);
  else
    k_cholesky<4, 32><<<ntasks, 1024, 0, st>>>(nullptr, k, ld, tau, shift_on_fail, nullptr, nullptr, nullptr, nullptr,
                                               tasks);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Tall x small: Out[i, :cnt] = In[i, :K] * M (K x cnt), 128-row tiles.
// M (zero-padded to OUTB columns) sits in shared memory; row tiles are
// double-buffered in shared memory by cp.async (16-byte copies, rows padded
// by 4 floats), so the next tile streams in while this one is multiplied.
// Thread (ty, tx) of the 16 x 16 grid computes rows ty + 16 i (i < 8) at
// columns 64 h + 4 tx + (0..3): per four k-steps it reads eight float4 of
// its rows (two distinct addresses per warp: broadcast) and 4 OUTB/64
// float4 of M, for 128 OUTB/64 FMAs.  A block loads a tile before it writes
// any of its rows, and only ever writes its own tiles, so Out may alias In.
// Optionally writes the 16-bit image of Out in the same pass: row stride
// 2 ldo, column 2 j = hi = round16(x), 2 j + 1 = round16(x - hi) (fmt 1 =
// bf16, 0 = f16).
// ---------------------------------------------------------------------------
constexpr int kTallRows = 128;

__device__ __forceinline__ void split16(float x, int fmt, uint16_t& h, uint16_t& l) {
  if (fmt) {
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    h = __bfloat16_as_ushort(b);
    l = __bfloat16_as_ushort(__float2bfloat16_rn(x - __bfloat162float(b)));
  } else {
    const __half b = __float2half_rn(x);
    h = __half_as_ushort(b);
    l = __half_as_ushort(__float2half_rn(x - __half2float(b)));
  }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// The matrices of one tall right-multiplication launch.  A task is one
// matrix: In (n x ldi, rows in tiles of 128), Out, the optional image, and M;
// tile0 numbers its first tile in the launch.
// TallOne: one matrix, block b takes the tiles b, b + nb, ...
// TallBatch: every matrix of a batch; block b takes a contiguous range of the
// launch's tiles, so it restages M only where its range crosses into the
// next matrix.
struct TallOne {
  TallTask t;
  int64_t n_tiles;
  __device__ int64_t first() const { return blockIdx.x; }
  __device__ int64_t next(int64_t tile) const { return tile + gridDim.x; }
  __device__ bool valid(int64_t tile) const { return tile < n_tiles; }
  __device__ int task_of(int64_t) const { return 0; }
  __device__ TallTask task(int) const { return t; }
};
struct TallBatch {
  const TallTask* tasks;
  int ntasks;
  int64_t begin, end;  // this block's tiles
  __device__ int64_t first() const { return begin; }
  __device__ int64_t next(int64_t tile) const { return tile + 1; }
  __device__ bool valid(int64_t tile) const { return tile < end; }
  __device__ int task_of(int64_t tile) const {  // the last task whose first tile is <= tile
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].tile0 <= tile) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  __device__ TallTask task(int q) const { return tasks[q]; }
};
__device__ __forceinline__ TallBatch tall_batch(const TallTask* tasks, int ntasks, int64_t total_tiles) {
  return TallBatch{tasks, ntasks, (int64_t)blockIdx.x * total_tiles / gridDim.x,
                   (int64_t)(blockIdx.x + 1) * total_tiles / gridDim.x};
}

template <int OUTB, class Src>
__device__ __forceinline__ void tall_mm_body(const Src& src, int K, int ldi, int ldm, int cnt, int ldo, int fmt) {
  constexpr int H = OUTB / 64;
  constexpr int RPT = kTallRows / 16;  // rows per thread
  extern __shared__ __align__(16) float sm_f[];
  const int KP = K + 4;
  float* Ms = sm_f;  // [K][OUTB]
  float* T0 = sm_f + K * OUTB;
  float* T1 = T0 + kTallRows * KP;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int k4 = K >> 2;
  const bool vec_out = ((cnt & 3) == 0) && ((ldo & 3) == 0);

  auto issue = [&](int64_t tile, float* T) {
    const TallTask tk = src.task(src.task_of(tile));
    const int64_t r0 = (tile - tk.tile0) * kTallRows;
    for (int t = threadIdx.x; t < kTallRows * k4; t += blockDim.x) {
      const int r = t / k4, c4 = t - r * k4;
      float* dst = T + r * KP + 4 * c4;
      if (r0 + r < tk.n) cp_async16(dst, tk.In + (r0 + r) * ldi + 4 * c4);
      else *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };

  int cur = -1;  // the task whose M is staged
  int64_t tile = src.first();
  if (src.valid(tile)) issue(tile, T0);
  cp_async_commit();
  for (int it = 0; src.valid(tile); tile = src.next(tile), ++it) {
    float* T = (it & 1) ? T1 : T0;
    const int64_t next = src.next(tile);
    if (src.valid(next)) issue(next, (it & 1) ? T0 : T1);
    cp_async_commit();
    cp_async_wait1();  // this tile's copies are done (the next tile's may still run)
    const int q = src.task_of(tile);
    const TallTask tk = src.task(q);
    if (q != cur) {  // every thread finished with Ms at the previous tile's last barrier
      for (int t = threadIdx.x; t < K * OUTB; t += blockDim.x) {
        const int l = t / OUTB, o = t % OUTB;
        Ms[t] = o < cnt ? tk.M[l * ldm + o] : 0.f;
      }
      cur = q;
    }
    __syncthreads();
    float acc[RPT][4 * H];
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
      for (int o = 0; o < 4 * H; ++o) acc[i][o] = 0.f;
    for (int l = 0; l < K; l += 4) {
      float4 a[RPT];
#pragma unroll
      for (int i = 0; i < RPT; ++i) a[i] = *reinterpret_cast<const float4*>(T + (ty + 16 * i) * KP + l);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const float4 m = *reinterpret_cast<const float4*>(Ms + (l + u) * OUTB + 64 * h + 4 * tx);
#pragma unroll
          for (int i = 0; i < RPT; ++i) {
            const float x = u == 0 ? a[i].x : u == 1 ? a[i].y : u == 2 ? a[i].z : a[i].w;
            acc[i][4 * h + 0] = fmaf(x, m.x, acc[i][4 * h + 0]);
            acc[i][4 * h + 1] = fmaf(x, m.y, acc[i][4 * h + 1]);
            acc[i][4 * h + 2] = fmaf(x, m.z, acc[i][4 * h + 2]);
            acc[i][4 * h + 3] = fmaf(x, m.w, acc[i][4 * h + 3]);
          }
        }
      }
    }
    const int64_t r0 = (tile - tk.tile0) * kTallRows;
    float* Out = tk.Out;
    uint16_t* img = tk.img;
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const int64_t row = r0 + ty + 16 * i;
      if (row >= tk.n) continue;
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const int col = 64 * h + 4 * tx;
        if (col >= cnt) continue;
        float* out = Out + row * ldo + col;
        const float* v = &acc[i][4 * h];
        if (vec_out) {
          *reinterpret_cast<float4*>(out) = make_float4(v[0], v[1], v[2], v[3]);
          if (img) {
            uint16_t hh[4], ll[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) split16(v[j], fmt, hh[j], ll[j]);
            *reinterpret_cast<uint4*>(img + (row * ldo + col) * 2) =
                make_uint4(hh[0] | ((uint32_t)ll[0] << 16), hh[1] | ((uint32_t)ll[1] << 16),
                           hh[2] | ((uint32_t)ll[2] << 16), hh[3] | ((uint32_t)ll[3] << 16));
          }
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (col + j < cnt) {
              out[j] = v[j];
              if (img) split16(v[j], fmt, img[(row * ldo + col + j) * 2], img[(row * ldo + col + j) * 2 + 1]);
            }
        }
      }
    }
    __syncthreads();  // every thread is done with T (and Ms) before they are refilled
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <int OUTB>
__global__ void __launch_bounds__(256, 2) k_tall_mm(const float* In, int64_t n, int K, int ldi,
                                                    const float* __restrict__ M, int ldm, int cnt, float* Out,
                                                    int ldo, uint16_t* __restrict__ img, int fmt) {
  tall_mm_body<OUTB>(TallOne{TallTask{In, Out, img, M, n, 0}, (n + kTallRows - 1) / kTallRows}, K, ldi, ldm, cnt,
                     ldo, fmt);
}

template <int OUTB>
__global__ void __launch_bounds__(256, 2) k_tall_mm_batch(const TallTask* __restrict__ tasks, int ntasks,
                                                          int64_t total_tiles, int K, int ldi, int ldm, int cnt,
                                                          int ldo, int fmt) {
  tall_mm_body<OUTB>(tall_batch(tasks, ntasks, total_tiles), K, ldi, ldm, cnt, ldo, fmt);
}

// ---------------------------------------------------------------------------
// Y <- Y M at ld 64 for an upper-triangular M (the Cholesky inverse), with the
// optional 16-bit image: output column c takes only rows l <= c of M, half
// the FMAs of the full product.  Warp w computes the column groups w and
// 15 - w (4 columns each: 4 (w + 1) + 4 (16 - w) = 68 terms, the same for
// every warp), lane r the rows r + 32 i (i < 4) of a 128-row tile.  The tile
// is staged as in k_tall_mm (padded rows, cp.async double buffering, loaded
// whole before any of its rows is written, so Out may alias In).  The terms
// dropped are exact zeros, so the result equals the full product's.
// ---------------------------------------------------------------------------
template <class Src>
__device__ __forceinline__ void upper64_body(const Src& src, int fmt) {
  constexpr int K = 64, KP = K + 4;
  extern __shared__ __align__(16) float sm_u[];
  float* Ms = sm_u;                    // [K][K]
  float* T0 = sm_u + K * K;
  float* T1 = T0 + kTallRows * KP;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  auto issue = [&](int64_t tile, float* T) {
    const TallTask tk = src.task(src.task_of(tile));
    const int64_t r0 = (tile - tk.tile0) * kTallRows;
    for (int t = threadIdx.x; t < kTallRows * (K / 4); t += blockDim.x) {
      const int r = t / (K / 4), c4 = t - r * (K / 4);
      float* dst = T + r * KP + 4 * c4;
      if (r0 + r < tk.n) cp_async16(dst, tk.In + (r0 + r) * K + 4 * c4);
      else *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  int cur = -1;  // the task whose M is staged
  int64_t tile = src.first();
  if (src.valid(tile)) issue(tile, T0);
  cp_async_commit();
  for (int it = 0; src.valid(tile); tile = src.next(tile), ++it) {
    float* T = (it & 1) ? T1 : T0;
    const int64_t next = src.next(tile);
    if (src.valid(next)) issue(next, (it & 1) ? T0 : T1);
    cp_async_commit();
    cp_async_wait1();
    const int q = src.task_of(tile);
    const TallTask tk = src.task(q);
    if (q != cur) {  // every thread finished with Ms at the previous tile's last barrier
      for (int t = threadIdx.x; t < K * K; t += blockDim.x) Ms[t] = tk.M[t];
      cur = q;
    }
    __syncthreads();
    const int64_t r0 = (tile - tk.tile0) * kTallRows, n = tk.n;
    float* Out = tk.Out;
    uint16_t* img = tk.img;
    float res[2][16];  // [column group][4 rows x 4 columns]
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int cg = h == 0 ? w : 15 - w;  // column group: columns 4 cg .. 4 cg + 3
      float acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int o = 0; o < 4; ++o) acc[i][o] = 0.f;
      for (int l = 0; l < 4 * (cg + 1); l += 4) {
        float4 a[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = *reinterpret_cast<const float4*>(T + (lane + 32 * i) * KP + l);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float4 m = *reinterpret_cast<const float4*>(Ms + (l + u) * K + 4 * cg);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float x = u == 0 ? a[i].x : u == 1 ? a[i].y : u == 2 ? a[i].z : a[i].w;
            acc[i][0] = fmaf(x, m.x, acc[i][0]);
            acc[i][1] = fmaf(x, m.y, acc[i][1]);
            acc[i][2] = fmaf(x, m.z, acc[i][2]);
            acc[i][3] = fmaf(x, m.w, acc[i][3]);
          }
        }
      }
      res[h][0] = acc[0][0]; res[h][1] = acc[0][1]; res[h][2] = acc[0][2]; res[h][3] = acc[0][3];
#pragma unroll
      for (int i = 1; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) res[h][4 * i + j] = acc[i][j];
    }
    // A lane holds rows of the tile, so storing from registers would put 32
    // rows (32 sectors) in every warp store.  The results go back into T
    // instead, and the tile leaves row-contiguous: each warp store covers two
    // whole 256-byte rows.
    __syncthreads();  // every warp is done reading T
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int cg = h == 0 ? w : 15 - w;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        *reinterpret_cast<float4*>(T + (lane + 32 * i) * KP + 4 * cg) =
            make_float4(res[h][4 * i], res[h][4 * i + 1], res[h][4 * i + 2], res[h][4 * i + 3]);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kTallRows * (K / 4) / 256; ++u) {
      const int f = threadIdx.x + 256 * u;
      const int r = f >> 4, c4 = f & 15;
      const int64_t row = r0 + r;
      if (row >= n) continue;
      const float4 v = *reinterpret_cast<const float4*>(T + r * KP + 4 * c4);
      *reinterpret_cast<float4*>(Out + row * K + 4 * c4) = v;
      if (img) {
        uint16_t hh[4], ll[4];
        split16(v.x, fmt, hh[0], ll[0]);
        split16(v.y, fmt, hh[1], ll[1]);
        split16(v.z, fmt, hh[2], ll[2]);
        split16(v.w, fmt, hh[3], ll[3]);
        *reinterpret_cast<uint4*>(img + (row * K + 4 * c4) * 2) =
            make_uint4(hh[0] | ((uint32_t)ll[0] << 16), hh[1] | ((uint32_t)ll[1] << 16),
                       hh[2] | ((uint32_t)ll[2] << 16), hh[3] | ((uint32_t)ll[3] << 16));
      }
    }
    __syncthreads();  // every thread is done with T before it is refilled
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__global__ void __launch_bounds__(256, 2) k_tall_mm_upper64(const float* In, int64_t n,
                                                            const float* __restrict__ M, float* Out,
                                                            uint16_t* __restrict__ img, int fmt) {
  upper64_body(TallOne{TallTask{In, Out, img, M, n, 0}, (n + kTallRows - 1) / kTallRows}, fmt);
}

__global__ void __launch_bounds__(256, 2) k_tall_mm_upper64_batch(const TallTask* __restrict__ tasks, int ntasks,
                                                                  int64_t total_tiles, int fmt) {
  upper64_body(tall_batch(tasks, ntasks, total_tiles), fmt);
}

static cudaError_t tall_mm_upper64(const float* In, int64_t n, const float* M, float* Out, uint16_t* img, int fmt,
                                   cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  const size_t smem = ((size_t)64 * 64 + 2 * (size_t)kTallRows * 68) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_tall_mm_upper64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int grid = grid_for(n, kTallRows, num_sms, 2);
  note_launches(1);
  k_tall_mm_upper64<<<grid, 256, smem, st>>>(In, n, M, Out, img, fmt);
  return cudaGetLastError();
}

cudaError_t launch_apply_upper64_batch(const TallTask* tasks, int ntasks, int64_t total_tiles, int fmt,
                                       cudaStream_t st, int num_sms) {
  if (ntasks <= 0 || total_tiles <= 0) return cudaSuccess;
  const size_t smem = ((size_t)64 * 64 + 2 * (size_t)kTallRows * 68) * sizeof(float);
  if (cudaError_t e = allow_smem(k_tall_mm_upper64_batch, smem); e != cudaSuccess) return e;
  const int grid = (int)std::min<int64_t>(total_tiles, 2 * (int64_t)num_sms);
  note_launches(1);
  k_tall_mm_upper64_batch<<<grid, 256, smem, st>>>(tasks, ntasks, total_tiles, fmt);
  return cudaGetLastError();
}

cudaError_t launch_embed_batch(const TallTask* tasks, int ntasks, int64_t total_tiles, int ld, int nc,
                               cudaStream_t st, int num_sms) {
  if (ntasks <= 0 || total_tiles <= 0) return cudaSuccess;
  if (ld > 64 || nc > 64 || (ld & 3)) return cudaErrorInvalidValue;  // one 64-column panel, as launch_embed at ld 64
  const size_t smem = ((size_t)ld * 64 + 2 * (size_t)kTallRows * (ld + 4)) * sizeof(float);
  if (cudaError_t e = allow_smem(k_tall_mm_batch<64>, smem); e != cudaSuccess) return e;
  const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(2, (220 * 1024) / smem));
  const int grid = (int)std::min<int64_t>(total_tiles, (int64_t)per_sm * num_sms);
  note_launches(1);
  k_tall_mm_batch<64><<<grid, 256, smem, st>>>(tasks, ntasks, total_tiles, ld, ld, nc, nc, nc, 0);
  return cudaGetLastError();
}

static cudaError_t tall_mm(const float* In, int64_t n, int K, int ldi, const float* M, int ldm, int cnt,
                           float* Out, int ldo, uint16_t* img, int fmt, cudaStream_t st,
                           int num_sms) {
  if (n == 0) return cudaSuccess;
  if ((K & 3) || (ldi & 3)) return cudaErrorInvalidValue;
  const int outb = cnt <= 64 ? 64 : 128;
  const size_t smem = ((size_t)K * outb + 2 * (size_t)kTallRows * (K + 4)) * sizeof(float);
  const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(2, (220 * 1024) / smem));
  const int grid = grid_for(n, kTallRows, num_sms, per_sm);
  note_launches(1);
  if (outb == 64) {
    if (cudaError_t e = allow_smem(k_tall_mm<64>, smem); e != cudaSuccess) return e;
    k_tall_mm<64><<<grid, 256, smem, st>>>(In, n, K, ldi, M, ldm, cnt, Out, ldo, img, fmt);
  } else {
    if (cudaError_t e = allow_smem(k_tall_mm<128>, smem); e != cudaSuccess) return e;
    k_tall_mm<128><<<grid, 256, smem, st>>>(In, n, K, ldi, M, ldm, cnt, Out, ldo, img, fmt);
  }
  return cudaGetLastError();
}

cudaError_t launch_apply_right_f32(const float* In, int64_t n, int ld, const float* M, float* Out,
                                   cudaStream_t st, int num_sms) {
  if (ld > kMaxK) {
    // wider than one panel: in place for an upper-triangular M, else panel by panel into Out
    if (In == Out) return launch_apply_upper_wide(Out, n, ld, M, st, num_sms);
    for (int c0 = 0; c0 < ld; c0 += kPanel) {
      cudaError_t e = launch_tall_mm_wide(In, n, ld, ld, M, ld, c0, kPanel, Out, ld, st, num_sms);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  if (ld == 64) return tall_mm_upper64(In, n, M, Out, nullptr, 0, st, num_sms);
  return tall_mm(In, n, ld, ld, M, ld, ld, Out, ld, nullptr, 0, st, num_sms);
}

cudaError_t launch_apply_right_split(const float* In, int64_t n, int ld, const float* M, float* Out,
                                     uint16_t* img, int fmt, cudaStream_t st, int num_sms) {
  if (ld > kMaxK) return cudaErrorInvalidValue;  // the 16-bit image belongs to the tensor-core path (ld <= 128)
  if (ld == 64) return tall_mm_upper64(In, n, M, Out, img, fmt, st, num_sms);
  return tall_mm(In, n, ld, ld, M, ld, ld, Out, ld, img, fmt, st, num_sms);
}

// ---------------------------------------------------------------------------
// Gene-side FP64 ops: Z = (W - mu s^T) M for a g x LD matrix W and an LD x LD
// M (mu null: Z = W M; Z may be W).  A block of 256 threads stages M once and
// then 64 rows of W at a time; thread (ty, tx) of the 16 x 16 grid owns rows
// ty + 16 i (i < 4) and columns tx + 16 v (v < LD / 16) of the 64-row block,
// so every shared value it reads feeds 4 or LD / 16 FMAs (one value per FMA
// made the kernel shared-memory bound at 256 segments).  Each output is one
// FMA chain over l = 0 .. LD-1 in order.
// ---------------------------------------------------------------------------
// Rows per block step: 16 for one matrix (125 blocks at 2,000 genes, a
// latency-bound launch); 64 when a launch covers the segments of a batch
// (thousands of blocks: fewer, larger steps per staged M).
constexpr int kApplyRows = 16, kApplyRowsBatch = 64;

__host__ __device__ constexpr size_t center_apply_smem(int ld, int rb) {
  return ((size_t)ld * ld + (size_t)rb * (ld + 1)) * sizeof(double);
}

// Block b of nb (of one matrix's grid) takes the row blocks b, b + nb, ...
template <int LD, int kApplyRows>
__device__ __forceinline__ void center_apply_body(const double* W, int64_t g, const double* mu, const double* s,
                                                  const double* M, double* Z, int b, int nb) {
  constexpr int TT = LD / 16, RP = LD + 1;  // odd row stride: rows ty and ty + 1 sit in different banks
  extern __shared__ double sm[];
  double* Ms = sm;             // [LD][LD]
  double* rows = sm + LD * LD;  // [kApplyRows][LD + 1]
  {
    // every load of M in flight before the first shared store: one L2 round
    // trip per block instead of one per element the thread stages
    constexpr int PT = LD * LD / 256;  // elements per thread
    double mv[PT];
#pragma unroll
    for (int u = 0; u < PT; ++u) mv[u] = M[threadIdx.x + 256 * u];
#pragma unroll
    for (int u = 0; u < PT; ++u) Ms[threadIdx.x + 256 * u] = mv[u];
  }
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  for (int64_t j0 = (int64_t)b * kApplyRows; j0 < g; j0 += (int64_t)nb * kApplyRows) {
    __syncthreads();  // M staged; the previous block's rows consumed
    constexpr int RT = kApplyRows * LD / 256;  // row elements per thread
    double wv[RT];
#pragma unroll
    for (int u = 0; u < RT; ++u) {
      const int t = threadIdx.x + 256 * u;
      const int64_t j = j0 + t / LD;
      wv[u] = j < g ? W[j * LD + t % LD] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < RT; ++u) {
      const int t = threadIdx.x + 256 * u;
      const int r = t / LD, c = t % LD;
      const int64_t j = j0 + r;
      double v = wv[u];
      if (j < g && mu) v -= mu[j] * s[c];
      rows[r * RP + c] = v;
    }
    __syncthreads();
    constexpr int RI = kApplyRows / 16;  // rows per thread
    double acc[RI][TT];
#pragma unroll
    for (int i = 0; i < RI; ++i)
#pragma unroll
      for (int v = 0; v < TT; ++v) acc[i][v] = 0.0;
#pragma unroll 4
    for (int l = 0; l < LD; ++l) {
      double a[RI], m[TT];
#pragma unroll
      for (int i = 0; i < RI; ++i) a[i] = rows[(ty + 16 * i) * RP + l];
#pragma unroll
      for (int v = 0; v < TT; ++v) m[v] = Ms[l * LD + tx + 16 * v];
#pragma unroll
      for (int i = 0; i < RI; ++i)
#pragma unroll
        for (int v = 0; v < TT; ++v) acc[i][v] = fma(a[i], m[v], acc[i][v]);
    }
#pragma unroll
    for (int i = 0; i < RI; ++i) {
      const int64_t j = j0 + ty + 16 * i;
      if (j < g)
#pragma unroll
        for (int v = 0; v < TT; ++v) Z[j * LD + tx + 16 * v] = acc[i][v];
    }
  }
}

template <int LD>
__global__ void __launch_bounds__(256) k_center_apply(const double* W, int64_t g, const double* __restrict__ mu,
                                                      const double* __restrict__ s, const double* __restrict__ M,
                                                      double* Z) {
  center_apply_body<LD, kApplyRows>(W, g, mu, s, M, Z, blockIdx.x, gridDim.x);
}

// One matrix per grid row y (batched segments).
template <int LD>
__global__ void __launch_bounds__(256) k_center_apply_batch(const ApplyTask* __restrict__ tasks, int64_t g) {
  const ApplyTask t = tasks[blockIdx.y];
  center_apply_body<LD, kApplyRowsBatch>(t.W, g, t.mu, t.s, t.M, t.Z, blockIdx.x, gridDim.x);
}

template <int LD>
static cudaError_t center_apply_t(const ApplyTask* tasks, int ntasks, const double* W, int64_t g, const double* mu,
                                  const double* s, const double* M, double* Z, cudaStream_t st) {
  if (g <= 0) return cudaSuccess;
  note_launches(1);
  if (tasks) {
    const size_t smem = center_apply_smem(LD, kApplyRowsBatch);
    if (cudaError_t e = allow_smem(k_center_apply_batch<LD>, smem); e != cudaSuccess) return e;
    // up to 16 blocks per matrix (two 64-row steps each at 2,000 genes), M staged once per block
    const int64_t blocks = (g + kApplyRowsBatch - 1) / kApplyRowsBatch;
    const dim3 grid((unsigned)std::min<int64_t>(blocks, 16), (unsigned)ntasks);
    k_center_apply_batch<LD><<<grid, 256, smem, st>>>(tasks, g);
  } else {
    const size_t smem = center_apply_smem(LD, kApplyRows);
    const int64_t blocks = (g + kApplyRows - 1) / kApplyRows;
    if (cudaError_t e = allow_smem(k_center_apply<LD>, smem); e != cudaSuccess) return e;
    k_center_apply<LD><<<(unsigned)std::min<int64_t>(blocks, 160), 256, smem, st>>>(W, g, mu, s, M, Z);
  }
  return cudaGetLastError();
}

static cudaError_t center_apply_ld(const ApplyTask* tasks, int ntasks, const double* W, int64_t g, int ld,
                                   const double* mu, const double* s, const double* M, double* Z, cudaStream_t st) {
  switch (ld) {
    case 32: return center_apply_t<32>(tasks, ntasks, W, g, mu, s, M, Z, st);
    case 64: return center_apply_t<64>(tasks, ntasks, W, g, mu, s, M, Z, st);
    case 96: return center_apply_t<96>(tasks, ntasks, W, g, mu, s, M, Z, st);
    case 128: return center_apply_t<128>(tasks, ntasks, W, g, mu, s, M, Z, st);
    default: return cudaErrorInvalidValue;  // ld is a multiple of 32 up to kMaxK here
  }
}

cudaError_t launch_center_apply_batch(const ApplyTask* tasks, int ntasks, int64_t g, int ld, cudaStream_t st) {
  if (ld > kMaxK) return cudaErrorInvalidValue;
  if (ntasks <= 0) return cudaSuccess;
  return center_apply_ld(tasks, ntasks, nullptr, g, ld, nullptr, nullptr, nullptr, nullptr, st);
}

cudaError_t launch_center_apply(const double* W, int64_t g, int ld, const double* mu,
                                const double* s, const double* M, double* Z, cudaStream_t st) {
  if (ld > kMaxK) return launch_center_apply_wide(W, g, ld, mu, s, M, Z, st);
  return center_apply_ld(nullptr, 0, W, g, ld, mu, s, M, Z, st);
}

cudaError_t launch_apply_right_f64(double* A, int64_t g, int ld, const double* M, cudaStream_t st) {
  return launch_center_apply(A, g, ld, nullptr, nullptr, M, A, st);
}

__global__ void k_round_v(const double* __restrict__ A, int64_t g, int ld, float* __restrict__ Vf) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < g * ld;
       t += (int64_t)gridDim.x * blockDim.x)
    Vf[t] = (float)A[t];
}

__global__ void k_round_v_batch(const RoundTask* __restrict__ tasks, int64_t g, int ld) {
  const RoundTask tk = tasks[blockIdx.y];
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < g * ld;
       t += (int64_t)gridDim.x * blockDim.x)
    tk.Vf[t] = (float)tk.A[t];
}

// mc[c] = sum_j mu_j Vf[j][c], FP64 accumulation, one block per column.
__device__ __forceinline__ void mean_prefactor_body(const float* Vf, int64_t g, int ld, const double* mu,
                                                    float* mc, int c) {
  __shared__ double red[256];
  double acc = 0.0;
  if (mu)
    for (int64_t j = threadIdx.x; j < g; j += blockDim.x) acc += mu[j] * (double)Vf[j * ld + c];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) mc[c] = (float)red[0];
}

__global__ void k_mean_prefactor(const float* __restrict__ Vf, int64_t g, int ld,
                                 const double* __restrict__ mu, float* __restrict__ mc) {
  mean_prefactor_body(Vf, g, ld, mu, mc, blockIdx.x);
}

__global__ void k_mean_prefactor_batch(const RoundTask* __restrict__ tasks, int64_t g, int ld) {
  const RoundTask tk = tasks[blockIdx.y];
  mean_prefactor_body(tk.Vf, g, ld, tk.mu, tk.mc, blockIdx.x);
}

cudaError_t launch_round_v_batch(const RoundTask* tasks, int ntasks, int64_t g, int ld, cudaStream_t st) {
  if (ntasks <= 0) return cudaSuccess;
  note_launches(2);
  const int gx = (int)std::min<int64_t>((g * ld + 255) / 256, 64);
  k_round_v_batch<<<dim3((unsigned)gx, (unsigned)ntasks), 256, 0, st>>>(tasks, g, ld);
  k_mean_prefactor_batch<<<dim3((unsigned)ld, (unsigned)ntasks), 256, 0, st>>>(tasks, g, ld);
  return cudaGetLastError();
}

// A batch's per-segment results gathered into contiguous buffers, so the
// host takes them in three copies instead of four per segment: status[q] =
// the segment's three status words and its tensor-core error word, sigma[q]
// its k singular values, comps[q] its `count` component floats.
__global__ void k_gather_out(const OutTask* __restrict__ tasks, int k, int64_t count, int* __restrict__ status,
                             double* __restrict__ sigma, float* __restrict__ comps) {
  const int q = blockIdx.y;
  const OutTask t = tasks[q];
  if (blockIdx.x == 0) {
    if (threadIdx.x < 3) status[4 * q + threadIdx.x] = t.status[threadIdx.x];
    if (threadIdx.x == 3) status[4 * q + 3] = t.tc_err ? t.tc_err[0] : 0;
    for (int i = threadIdx.x; i < k; i += blockDim.x) sigma[(int64_t)q * k + i] = t.sigma[i];
  }
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x)
    comps[(int64_t)q * count + e] = t.comps[e];
}

cudaError_t launch_gather_out(const OutTask* tasks, int ntasks, int k, int64_t count, int* status, double* sigma,
                              float* comps, cudaStream_t st) {
  if (ntasks <= 0) return cudaSuccess;
  note_launches(1);
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, 16));
  k_gather_out<<<dim3((unsigned)gx, (unsigned)ntasks), 256, 0, st>>>(tasks, k, count, status, sigma, comps);
  return cudaGetLastError();
}

// The four status words of every task set to zero (the start of a batch run).
__global__ void k_zero_status(const OutTask* __restrict__ tasks) {
  if (threadIdx.x < 4) tasks[blockIdx.x].status[threadIdx.x] = 0;
}

cudaError_t launch_zero_status(const OutTask* tasks, int ntasks, cudaStream_t st) {
  if (ntasks <= 0) return cudaSuccess;
  note_launches(1);
  k_zero_status<<<ntasks, 32, 0, st>>>(tasks);
  return cudaGetLastError();
}

// mc = mu^T Vf for every task (the Vf and mu of each; A unused).
cudaError_t launch_mean_prefactor_batch(const RoundTask* tasks, int ntasks, int64_t g, int ld, cudaStream_t st) {
  if (ntasks <= 0) return cudaSuccess;
  note_launches(1);
  k_mean_prefactor_batch<<<dim3((unsigned)ld, (unsigned)ntasks), 256, 0, st>>>(tasks, g, ld);
  return cudaGetLastError();
}

// tasks[q].Vf = src for q = 1 .. ntasks - 1 (count floats, a multiple of 4):
// one segment's test matrix handed to the others of a batch.
__global__ void k_broadcast_v(const float* __restrict__ src, int64_t count4, const RoundTask* __restrict__ tasks) {
  float4* dst = reinterpret_cast<float4*>(tasks[blockIdx.y + 1].Vf);
  const float4* s4 = reinterpret_cast<const float4*>(src);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count4; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = s4[t];
}

cudaError_t launch_broadcast_v(const float* src, int64_t count, const RoundTask* tasks, int ntasks,
                               cudaStream_t st) {
  if (ntasks <= 1 || count <= 0) return cudaSuccess;
  if (count & 3) return cudaErrorInvalidValue;
  note_launches(1);
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((count / 4 + 255) / 256, 32));
  k_broadcast_v<<<dim3((unsigned)gx, (unsigned)(ntasks - 1)), 256, 0, st>>>(src, count / 4, tasks);
  return cudaGetLastError();
}

cudaError_t launch_mean_prefactor(const float* Vf, int64_t g, int ld, const double* mu, float* mc,
                                  cudaStream_t st) {
  note_launches(1);
  k_mean_prefactor<<<ld, 256, 0, st>>>(Vf, g, ld, mu, mc);
  return cudaGetLastError();
}

cudaError_t launch_round_v(const double* A, int64_t g, int ld, const double* mu, float* Vf,
                           float* mc, cudaStream_t st) {
  note_launches(1);
  k_round_v<<<(int)std::min<int64_t>((g * ld + 255) / 256, 1184), 256, 0, st>>>(A, g, ld, Vf);
  return launch_mean_prefactor(Vf, g, ld, mu, mc, st);
}

// ---------------------------------------------------------------------------
// Symmetric eigendecomposition of the k x k block of C (SPD up to rounding:
// C = B^T B) by one-sided (Hestenes) Jacobi on its Cholesky factor.
//   1. C = R^T R (FP64, right-looking, in shared memory; a pivot below
//      1e-300 or 1e-15 of the largest diagonal is clamped there -- those are
//      null directions of C, whose eigenvalues are zero to working accuracy).
//   2. Rotate pairs of columns of R from the right until all columns are
//      mutually orthogonal: R J_1 J_2 ... = U Sigma, V = J_1 J_2 ...; then
//      C = V Sigma^2 V^T, eigenvalue i = |column i|^2.
//   3. V is not accumulated rotation by rotation (that doubles the FP64
//      work of every round): it is recovered once as V = R0^{-1} (R0 V) by
//      back substitution against the Cholesky factor R0, and its columns are
//      renormalised.  Its error is about cond(R0) * 1e-16 = sqrt(cond(C)) *
//      1e-16.
// A round takes the kk/2 disjoint column pairs of a round-robin schedule;
// a half-warp owns one pair (a warp serves two pairs with the same shuffle
// instructions): the cross product p.q is a 16-lane partial reduced by
// shuffles, every lane of the half computes the same rotation, and the half
// rotates its two columns of R and of V.  Column norms are carried in closed
// form (a' = a - t c, b' = b + t c for the rotation that zeroes c) and
// recomputed at the start of every sweep.  Pairs are disjoint, so a round
// needs one block barrier.  Columns are stored contiguously (column-major,
// odd stride) so a column walk is conflict-free.  Stops after a sweep with no
// rotation (|p.q| <= 1e-15 |p| |q| for every pair, or |p.q| <= 1e-150), after
// a sweep whose largest rotation tangent is below 1e-4, or after 40 sweeps.
// Convergence is quadratic: the sweep after one whose largest tangent is t
// rotates by about t^2 / 4 at most (measured on power-iteration sketches of
// the NB synthetic at k = 40 and 60: 3e-2 -> 2e-5 -> 9e-11), so stopping at
// t < 1e-4 leaves every eigenvector within ~1e-9 of the next sweep's, below
// the FP32 resolution of the components and embeddings, and the eigenvalues
// (second order in the rotation) within ~1e-18.  FP64 issue bandwidth (one warp instruction per ~4 cycles per SM
// sub-partition) bounds a round, so the work per round is kept minimal.
// ---------------------------------------------------------------------------
// V (use_eglob) and R (use_rglob) go to the scratch that follows evecs when
// they do not fit shared memory.  With `tasks` set, block b solves tasks[b]
// (one launch for many segments) and C, evals, evecs, sweeps_out are ignored.
template <int NR>  // column entries a lane holds in registers: kk <= 16 NR
__global__ void __launch_bounds__(1024) k_jacobi(const double* __restrict__ C, int k, int ld,
                                                 double* __restrict__ evals, double* __restrict__ evecs,
                                                 int use_eglob, int use_rglob, int* sweeps_out,
                                                 const JacobiTask* __restrict__ tasks) {
  if (tasks) {
    const JacobiTask t = tasks[blockIdx.x];
    C = t.C;
    evals = t.evals;
    evecs = t.evecs;
    sweeps_out = t.sweeps;
  }
  double* Eglob = use_eglob ? evecs + (size_t)ld * ld : nullptr;
  double* Rglob = use_rglob ? evecs + (size_t)ld * ld + (size_t)ld * (ld + 1) : nullptr;
  extern __shared__ double sm[];
  const int kk = (k + 1) & ~1;  // even number of columns; column k (if odd) is a zero dummy
  const int S = kk + 1;
  const int npair = kk / 2, m = kk - 1;
  // R, and V after it, in shared memory when they fit, else in the global
  // scratch the launcher passes (a sketch wider than one panel)
  double* R = Rglob != nullptr ? Rglob : sm;                   // [kk cols][S]: R[c * S + r]
  double* sm_rest = Rglob != nullptr ? sm : sm + kk * S;
  uint16_t* sched = reinterpret_cast<uint16_t*>(sm_rest);      // [m][npair]: p | q << 8
  double* V = (Eglob != nullptr) ? Eglob : sm_rest + (m * npair + 3) / 4;  // [kk cols][S]: R0, then V
  __shared__ double colnorm[kMaxKWide];
  __shared__ int done;
  __shared__ unsigned long long maxt_bits;  // largest |t| of the sweep (non-negative doubles order as integers)
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int hl = lane & 15, half = lane >> 4;  // lane within the half-warp, which half
  const unsigned hmask = half ? 0xffff0000u : 0x0000ffffu;
  // R starts as the upper triangle of C (column-major)
  for (int t = tid; t < kk * S; t += nt) {
    const int c = t / S, r = t - c * S;
    R[t] = (r < k && c < k && r <= c) ? C[r * ld + c] : 0.0;
  }
  for (int t = tid; t < m * npair; t += nt) {
    const int round = t / npair, i = t - round * npair;
    int a, b;
    if (i == 0) { a = round; b = m; }
    else { a = (round + i) % m; b = (round - i + m) % m; }
    sched[t] = (uint16_t)(min(a, b) | (max(a, b) << 8));
  }
  __syncthreads();
  // ---- Cholesky in place (upper triangle, right-looking).  Every thread reads
  // pivot j; the diagonal entry itself is written one step later (by thread
  // 0), when nobody reads it any more. ----
  double dmax = 0.0;
  for (int j = 0; j < k; ++j) dmax = fmax(dmax, R[j * S + j]);
  double prev_diag = 0.0;
  for (int j = 0; j < k; ++j) {
    double d = R[j * S + j];
    if (!(d > 1e-15 * dmax) || !(d > 1e-300)) d = fmax(1e-15 * dmax, 1e-300);
    const double rd = rsqrt_nr(d);
    if (tid == 0 && j > 0) R[(j - 1) * S + (j - 1)] = prev_diag;
    prev_diag = d * rd;
    for (int c = j + 1 + tid; c < k; c += nt) R[c * S + j] *= rd;  // row j, right of the diagonal
    __syncthreads();
    // trailing update: R[a][c] -= R[j][a] R[j][c] for j < a <= c (column c by a
    // warp, row a by a lane)
    for (int c = j + 1 + warp; c < k; c += nw) {
      const double rjc = R[c * S + j];
      for (int a = j + 1 + lane; a <= c; a += 32) R[c * S + a] -= R[a * S + j] * rjc;
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (k > 0) R[(k - 1) * S + (k - 1)] = prev_diag;
    done = 1;
    maxt_bits = 0ull;
  }
  __syncthreads();
  // R0, kept for the back substitution; a unit diagonal for the dummy column
  // (odd k) keeps it invertible
  for (int t = tid; t < kk * S; t += nt) V[t] = (k < kk && t == k * S + k) ? 1.0 : R[t];
  __syncthreads();
  // ---- one-sided Jacobi on the columns of R ----
  int sweep = 0;
  for (; sweep < 40; ++sweep) {
    // column norms from scratch once per sweep (a half-warp per column)
    for (int col = 2 * warp + half; col < kk; col += 2 * nw) {
      double a = 0.0;
      for (int r = hl; r < kk; r += 16) a = fma(R[col * S + r], R[col * S + r], a);
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) a += __shfl_xor_sync(hmask, a, o);
      if (hl == 0) colnorm[col] = a;
    }
    __syncthreads();
    for (int round = 0; round < m; ++round) {
      const uint16_t* pr = sched + round * npair;
      for (int i = 2 * warp + half; i < npair; i += 2 * nw) {
        const int p = pr[i] & 0xff, q = pr[i] >> 8;
        double* rp = R + p * S;
        double* rq = R + q * S;
        // the pair's columns stay in registers from the dot product to the
        // rotation: shared-memory traffic bounds a round, so each column is
        // read once and written once
        double xp[NR], xq[NR];
        double c = 0.0;
#pragma unroll
        for (int u = 0; u < NR; ++u) {
          const int r = hl + 16 * u;
          xp[u] = r < kk ? rp[r] : 0.0;
          xq[u] = r < kk ? rq[r] : 0.0;
          c = fma(xp[u], xq[u], c);
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) c += __shfl_xor_sync(hmask, c, o);
        const double a = colnorm[p], b = colnorm[q];
        if (!(fabs(c) > 1e-150 && c * c > 1e-30 * a * b)) continue;  // uniform over the half-warp
        // t = tan of the angle that zeroes p.q: the smaller root of
        // t^2 + 2 zeta t - 1 = 0, zeta = (b - a) / 2c, written as
        // 2c sgn(tau) / (|tau| + sqrt(tau^2 + 4c^2)) with tau = b - a.  The
        // angle only sets how much of p.q a rotation removes, so t is formed
        // in FP32 (inputs scaled by a power of two into range); the rotation
        // itself stays exactly orthogonal in FP64: cs = 1 / sqrt(1 + t^2),
        // sn = t cs.  Near convergence |t| is tiny and its FP32 relative error
        // leaves a residual below 1e-7 |p.q|, cleared by the next sweep.
        const double sc = pow2_int(-exponent_of(a + b));
        const float tf = (float)((b - a) * sc), cf = (float)(2.0 * c * sc);
        const float den = fabsf(tf) + sqrtf(fmaf(tf, tf, cf * cf));
        const double t = (double)(__fdividef(tf >= 0.f ? cf : -cf, den));
        if (t == 0.0) continue;  // below FP32 resolution: nothing to rotate
        const double cs = rsqrt_nr(fma(t, t, 1.0)), sn = t * cs;
#pragma unroll
        for (int u = 0; u < NR; ++u) {
          const int r = hl + 16 * u;
          if (r < kk) {
            rp[r] = cs * xp[u] - sn * xq[u];
            rq[r] = sn * xp[u] + cs * xq[u];
          }
        }
        if (hl == 0) {
          const double cc = cs * cs, ss = sn * sn, x2 = 2.0 * cs * sn * c;
          colnorm[p] = fma(cc, a, fma(ss, b, -x2));
          colnorm[q] = fma(ss, a, fma(cc, b, x2));
          done = 0;
          atomicMax(&maxt_bits, (unsigned long long)__double_as_longlong(fabs(t)));
        }
      }
      __syncthreads();
    }
    const int converged = done || __longlong_as_double((long long)maxt_bits) < 1e-4;
    __syncthreads();  // every thread has read the flags before they are reset
    if (converged) break;
    if (tid == 0) {
      done = 1;
      maxt_bits = 0ull;
    }
    __syncthreads();
  }
  // eigenvalues: squared column norms of R0 V
  for (int col = 2 * warp + half; col < kk; col += 2 * nw) {
    double a = 0.0;
    for (int r = hl; r < kk; r += 16) a = fma(R[col * S + r], R[col * S + r], a);
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) a += __shfl_xor_sync(hmask, a, o);
    if (hl == 0) colnorm[col] = a;
  }
  // V = R0^{-1} (R0 V): back substitution, one column per thread, then unit columns
  __syncthreads();
  for (int c = tid; c < kk; c += nt) {
    double* rc = R + c * S;  // column c of R0 V, overwritten by column c of V
    for (int r = kk - 1; r >= 0; --r) {
      double x = rc[r];
      for (int j = r + 1; j < kk; ++j) x = fma(-V[j * S + r], rc[j], x);
      rc[r] = x * rcp_nr(V[r * S + r]);
    }
  }
  __syncthreads();
  // unit eigenvector columns (the squared norms of R0 V's columns, the
  // eigenvalues, were taken before the back substitution)
  for (int i = warp; i < kk; i += nw) {
    double a = 0.0;
    for (int r = lane; r < kk; r += 32) a = fma(R[i * S + r], R[i * S + r], a);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    a = __shfl_sync(0xffffffffu, a, 0);
    const double inv = a > 0.0 ? rsqrt_nr(a) : 0.0;
    for (int r = lane; r < kk; r += 32) R[i * S + r] *= inv;
  }
  __syncthreads();
  for (int i = tid; i < k; i += nt) {
    const double v = colnorm[i];
    int rank = 0;
    for (int j = 0; j < k; ++j) {
      const double w = colnorm[j];
      if (w > v || (w == v && j < i)) ++rank;
    }
    evals[rank] = v;
    for (int r = 0; r < ld; ++r) evecs[r * ld + rank] = (r < k) ? R[i * S + r] : 0.0;
  }
  for (int t = tid; t < ld * ld; t += nt) {
    const int c = t % ld;
    if (c >= k) evecs[t] = 0.0;
  }
  if (tid == 0 && sweeps_out) *sweeps_out = sweep;
}

static cudaError_t jacobi_go(const double* C, int k, int ld, double* evals, double* evecs, int* sweeps,
                             const JacobiTask* tasks, int nblocks, cudaStream_t st) {
  const int kk = (k + 1) & ~1;
  const size_t one = (size_t)kk * (kk + 1) * sizeof(double);
  const size_t sched = ((size_t)(kk - 1) * (kk / 2) + 3) / 4 * sizeof(double);
  // V lives in shared memory when both matrices fit, else in the scratch that
  // follows evecs (the plan allocates ld * ld + 2 ld (ld + 1) doubles there),
  // and R too when even one does not fit (a sketch wider than one panel).
  if (kk > 256) return cudaErrorInvalidValue;  // the schedule packs a column pair into 8 + 8 bits
  int use_e = 0, use_r = 0;
  size_t smem = 2 * one + sched;
  if (smem > 200 * 1024) {
    use_e = 1;
    smem = one + sched;
  }
  if (smem > 200 * 1024) {
    use_r = 1;
    smem = sched;
  }
  const int warps = std::min(32, std::max(1, (kk / 2 + 1) / 2));  // one half-warp per column pair
  auto go = [&](auto kern) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    note_launches(1);
    kern<<<nblocks, 32 * warps, smem, st>>>(C, k, ld, evals, evecs, use_e, use_r, sweeps, tasks);
    return cudaGetLastError();
  };
  if (kk <= 64) return go(k_jacobi<4>);
  if (kk <= 128) return go(k_jacobi<8>);
  return go(k_jacobi<16>);
}

cudaError_t launch_jacobi_eig(const double* C, int k, int ld, double* evals, double* evecs,
                              int* sweeps, cudaStream_t st) {
  return jacobi_go(C, k, ld, evals, evecs, sweeps, nullptr, 1, st);
}

cudaError_t launch_jacobi_eig_batch(const JacobiTask* tasks, int ntasks, int k, int ld, cudaStream_t st) {
  if (ntasks <= 0) return cudaSuccess;
  return jacobi_go(nullptr, k, ld, nullptr, nullptr, nullptr, tasks, ntasks, st);
}

// ---------------------------------------------------------------------------
// Rayleigh-Ritz finish: sigma, the components and M_emb from B (g x k, in
// Z), the eigenpairs of B^T B and R2^{-1}.
// ---------------------------------------------------------------------------
// Components c0 .. c0 + ncc - 1 of nc per launch (E's columns staged in
// shared memory); one launch takes them all when E[:, :nc] fits.  Block b of
// nb takes the rows l = b, b + nb, ... of M_emb and the genes j = b, b + nb,
// ... of the components, its 128 threads spread over (row, component) pairs.
// Each output is one FMA chain in index order.
__device__ __forceinline__ void ritz_finish_body(const double* __restrict__ B, int64_t g, int ld, int k, int nc,
                                                 int c0, int ncc, const double* __restrict__ evals,
                                                 const double* __restrict__ E, const double* __restrict__ Rinv2,
                                                 double* __restrict__ sigma, float* __restrict__ comps,
                                                 float* __restrict__ M_emb, int b, int nb) {
  extern __shared__ double sm[];
  double* Es = sm;              // [ld][ncc]: columns c0 .. c0 + ncc - 1 of E
  double* sg = sm + ld * ncc;   // [ncc]
  for (int t = threadIdx.x; t < ld * ncc; t += blockDim.x) {
    const int l = t / ncc, c = t - l * ncc;
    Es[t] = E[l * ld + c0 + c];
  }
  for (int c = threadIdx.x; c < ncc; c += blockDim.x) sg[c] = sqrt(fmax(evals[c0 + c], 0.0));
  __syncthreads();
  if (b == 0 && c0 == 0)
    for (int c = threadIdx.x; c < k; c += blockDim.x) sigma[c] = sqrt(fmax(evals[c], 0.0));
  // M_emb row l = Rinv2[l, :] E[:, :nc] diag(sigma)
  const int64_t rows_m = b < ld ? (ld - 1 - b) / nb + 1 : 0;
  for (int64_t t = threadIdx.x; t < rows_m * ncc; t += blockDim.x) {
    const int l = b + (int)(t / ncc) * nb, c = (int)(t % ncc);
    double acc = 0.0;
    for (int m = 0; m < ld; ++m) acc = fma(Rinv2[l * ld + m], Es[m * ncc + c], acc);
    M_emb[l * nc + c0 + c] = (float)(acc * sg[c]);
  }
  // components[c][j] = (B E)[j][c] / sigma_c
  const int64_t rows_g = b < g ? (g - 1 - b) / nb + 1 : 0;
  for (int64_t t = threadIdx.x; t < rows_g * ncc; t += blockDim.x) {
    const int64_t j = b + (t / ncc) * nb;
    const int c = (int)(t % ncc);
    double acc = 0.0;
    for (int l = 0; l < k; ++l) acc = fma(B[j * ld + l], Es[l * ncc + c], acc);
    comps[(int64_t)(c0 + c) * g + j] = sg[c] > 0.0 ? (float)(acc / sg[c]) : 0.f;
  }
}

__global__ void __launch_bounds__(128) k_ritz_finish(const double* __restrict__ B, int64_t g, int ld, int k,
                                                     int nc, int c0, int ncc, const double* __restrict__ evals,
                                                     const double* __restrict__ E,
                                                     const double* __restrict__ Rinv2, double* __restrict__ sigma,
                                                     float* __restrict__ comps, float* __restrict__ M_emb) {
  ritz_finish_body(B, g, ld, k, nc, c0, ncc, evals, E, Rinv2, sigma, comps, M_emb, blockIdx.x, gridDim.x);
}

// One segment per grid row y (batched segments).
__global__ void __launch_bounds__(128) k_ritz_finish_batch(const RitzTask* __restrict__ tasks, int64_t g, int ld,
                                                           int k, int nc, int c0, int ncc) {
  const RitzTask t = tasks[blockIdx.y];
  ritz_finish_body(t.B, g, ld, k, nc, c0, ncc, t.evals, t.evecs, t.Rinv2, t.sigma, t.comps, t.M_emb, blockIdx.x,
                   gridDim.x);
}

// Components staged per launch, and the launch's shared bytes.
static int ritz_cols(int ld, int nc, size_t* smem) {
  constexpr size_t kStage = 160 * 1024;  // shared bytes for the staged columns of E
  const int ncc = (int)std::max<size_t>(1, std::min<size_t>(nc, kStage / ((size_t)(ld + 1) * sizeof(double))));
  *smem = (size_t)(ld * ncc + ncc) * sizeof(double);
  return ncc;
}

cudaError_t launch_ritz_finish(const double* B, int64_t g, int ld, int k, int nc,
                               const double* evals, const double* evecs, const double* Rinv2,
                               double* sigma, float* components, float* M_emb, cudaStream_t st) {
  size_t smem = 0;
  const int ncc = ritz_cols(ld, nc, &smem);
  if (cudaError_t e = allow_smem(k_ritz_finish, smem); e != cudaSuccess) return e;
  // Few blocks: each stages E once and then takes a run of genes.
  const int grid = (int)std::max<int64_t>(std::min<int64_t>(g, 296), std::min<int64_t>(ld, 296));
  for (int c0 = 0; c0 < nc; c0 += ncc) {
    note_launches(1);
    k_ritz_finish<<<grid, 128, smem, st>>>(B, g, ld, k, nc, c0, std::min(ncc, nc - c0), evals, evecs, Rinv2,
                                           sigma, components, M_emb);
  }
  return cudaGetLastError();
}

cudaError_t launch_ritz_finish_batch(const RitzTask* tasks, int ntasks, int64_t g, int ld, int k, int nc,
                                     cudaStream_t st) {
  if (ntasks <= 0) return cudaSuccess;
  size_t smem = 0;
  const int ncc = ritz_cols(ld, nc, &smem);
  if (cudaError_t e = allow_smem(k_ritz_finish_batch, smem); e != cudaSuccess) return e;
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>(std::max<int64_t>(g, ld), 8));
  for (int c0 = 0; c0 < nc; c0 += ncc) {
    note_launches(1);
    k_ritz_finish_batch<<<dim3((unsigned)gx, (unsigned)ntasks), 128, smem, st>>>(tasks, g, ld, k, nc, c0,
                                                                                  std::min(ncc, nc - c0));
  }
  return cudaGetLastError();
}

// Embeddings U = Q M_emb (n x nc row-major).
cudaError_t launch_embed(const float* Q, int64_t n, int ld, int k, const float* M_emb, int nc,
                         float* U, cudaStream_t st, int num_sms) {
  (void)k;  // rows k..ld-1 of M_emb are zero
  if (ld > kMaxK) {
    for (int c0 = 0; c0 < nc; c0 += kPanel) {
      cudaError_t e = launch_tall_mm_wide(Q, n, ld, ld, M_emb, nc, c0, std::min(kPanel, nc - c0), U, nc, st,
                                          num_sms);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  return tall_mm(Q, n, ld, ld, M_emb, nc, nc, U, nc, nullptr, 0, st, num_sms);
}

// ---------------------------------------------------------------------------
// Seeded Gaussian: Philox4x32-10 (Salmon et al., SC'11) + Box-Muller in FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += W0;
    k1 += W1;
  }
}

__global__ void k_gaussian(uint64_t seed, int64_t n_rows, int64_t n_cols, float* __restrict__ out,
                           int ld_pad) {
  const int64_t total = n_rows * n_cols;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    uint64_t p = (uint64_t)e >> 1;
    uint32_t c[4] = {(uint32_t)p, (uint32_t)(p >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint64_t a = (((uint64_t)c[0] << 32) | c[1]) >> 11;
    uint64_t b = (((uint64_t)c[2] << 32) | c[3]) >> 11;
    double u1 = ((double)a + 0.5) * 0x1.0p-53;
    double u2 = ((double)b + 0.5) * 0x1.0p-53;
    double r = sqrt(-2.0 * log(u1));
    double ang = 2.0 * 3.141592653589793 * u2;
    double z = (e & 1) ? r * sin(ang) : r * cos(ang);
    if (ld_pad > 0) {
      int64_t i = e % n_rows, j = e / n_rows;
      out[i * ld_pad + j] = (float)z;
    } else {
      out[e] = (float)z;
    }
  }
}

cudaError_t launch_gaussian(uint64_t seed, int64_t n_rows, int64_t n_cols, float* out, int ld_pad,
                            cudaStream_t st, int num_sms) {
  int64_t total = n_rows * n_cols;
  if (total == 0) return cudaSuccess;
  note_launches(1);
  k_gaussian<<<grid_for(total, 256, num_sms), 256, 0, st>>>(seed, n_rows, n_cols, out, ld_pad);
  return cudaGetLastError();
}

__global__ void k_colmajor_to_padded(const float* __restrict__ in, int64_t n_rows, int64_t n_cols,
                                     int ld, float* __restrict__ out) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n_rows * ld;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = t / ld, j = t % ld;
    out[t] = j < n_cols ? in[j * n_rows + i] : 0.f;
  }
}

cudaError_t launch_colmajor_to_padded(const float* in, int64_t n_rows, int64_t n_cols, int ld,
                                      float* out, cudaStream_t st, int num_sms) {
  if (n_rows == 0) return cudaSuccess;
  note_launches(1);
  k_colmajor_to_padded<<<grid_for(n_rows * ld, 256, num_sms), 256, 0, st>>>(in, n_rows, n_cols, ld, out);
  return cudaGetLastError();
}

}  // namespace scx
