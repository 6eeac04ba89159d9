// Dense kernels of sketches wider than one 128-column panel (kMaxK < k <=
// kMaxKWide; ld is then 256, two panels).  The operations are those of
// kernels_dense.cu -- tall Gram, Cholesky with its inverse, tall and
// gene-side right-multiplications -- shaped for k x k factors that no longer
// fit one block's registers or shared memory whole.  The reference sizes the
// sketch k = min(n_comps + n_oversamples, n_vars, n_obs) with no cap
// (scx-gpu/src/gpu_pca.rs:433-446); these kernels carry the same algebra past
// 128 columns.  The launchers in kernels_dense.cu dispatch here when ld > 128.
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace scx {

// ---------------------------------------------------------------------------
// Gram tile (ta, tb) of a tall matrix with ld = 2 panels: block b of grid.x
// takes a contiguous row range; part[b][(128 ta + i) ld + 128 tb + j] =
// sum_rows A[r][128 ta + i] A[r][128 tb + j] (FP64 products of the inputs,
// FP64 accumulation), and the diagonal tiles add the column sums of their
// panel.  grid.y enumerates the tiles.  Thread (ty, tx) of the 16 x 16 grid
// owns entries (ty + 16 i, tx + 16 j) as in k_gram.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_gram_tile(const T* __restrict__ A, int64_t n, int ld,
                                                   double* __restrict__ part) {
  constexpr int TT = kPanel / 16;
  constexpr int R = 16;  // rows staged per step
  __shared__ double sa[R][kPanel], sb[R][kPanel];
  const int panels = ld / kPanel;
  const int ta = blockIdx.y / panels, tb = blockIdx.y % panels;
  const int a0 = ta * kPanel, b0 = tb * kPanel;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[TT][TT];
#pragma unroll
  for (int i = 0; i < TT; ++i)
#pragma unroll
    for (int j = 0; j < TT; ++j) acc[i][j] = 0.0;
  double csum = 0.0;
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = (int64_t)blockIdx.x * per;
  const int64_t r1 = min(n, r0 + per);
  for (int64_t base = r0; base < r1; base += R) {
    const int rows = (int)min((int64_t)R, r1 - base);
    for (int t = threadIdx.x; t < R * kPanel; t += 256) {
      const int r = t / kPanel, c = t % kPanel;
      sa[r][c] = r < rows ? (double)A[(base + r) * ld + a0 + c] : 0.0;
      sb[r][c] = r < rows ? (double)A[(base + r) * ld + b0 + c] : 0.0;
    }
    __syncthreads();
    for (int r = 0; r < rows; ++r) {
      double a[TT], b[TT];
#pragma unroll
      for (int i = 0; i < TT; ++i) a[i] = sa[r][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < TT; ++j) b[j] = sb[r][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < TT; ++i)
#pragma unroll
        for (int j = 0; j < TT; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (ta == tb && threadIdx.x < kPanel)
      for (int r = 0; r < rows; ++r) csum += sa[r][threadIdx.x];
    __syncthreads();
  }
  double* out = part + (int64_t)blockIdx.x * ((int64_t)ld * ld + ld);
#pragma unroll
  for (int i = 0; i < TT; ++i)
#pragma unroll
    for (int j = 0; j < TT; ++j) out[(int64_t)(a0 + ty + 16 * i) * ld + b0 + tx + 16 * j] = acc[i][j];
  if (ta == tb && threadIdx.x < kPanel) out[(int64_t)ld * ld + a0 + threadIdx.x] = csum;
}

template <typename T>
static cudaError_t gram_wide_t(const T* A, int64_t n, int ld, double* part, int nparts, cudaStream_t st) {
  if (ld % kPanel != 0 || ld > kMaxKWide) return cudaErrorInvalidValue;
  const int panels = ld / kPanel;
  note_launches(1);
  k_gram_tile<T><<<dim3((unsigned)nparts, (unsigned)(panels * panels)), 256, 0, st>>>(A, n, ld, part);
  return cudaGetLastError();
}

cudaError_t launch_gram_wide_f32(const float* A, int64_t n, int ld, double* part, int nparts, cudaStream_t st) {
  return gram_wide_t<float>(A, n, ld, part, nparts, st);
}
cudaError_t launch_gram_wide_f64(const double* A, int64_t n, int ld, double* part, int nparts, cudaStream_t st) {
  return gram_wide_t<double>(A, n, ld, part, nparts, st);
}

// ---------------------------------------------------------------------------
// Cholesky G = R^T R of the leading k x k block (k <= kMaxKWide) and R^{-1},
// one block of 1024 threads, the working triangle held in R itself (global
// memory, L2-resident).  Right-looking: at step j, row j of the updated upper
// triangle is scaled by 1 / sqrt(d_j) and becomes row j of R; rows a > j take
// the rank-1 update S_ac -= R_ja R_jc (c >= a), one warp per row.  The pivot
// test, the single shifted restart (G + s I, s = 10 tau max_j G_jj) and the
// status protocol are k_cholesky's.  R^{-1} by back substitution, one warp
// per column, the sum over the column's known entries split across lanes.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_cholesky_wide(const double* __restrict__ G, int k, int ld, double tau,
                                                        int shift_on_fail, double* __restrict__ R,
                                                        double* __restrict__ Rinv, float* __restrict__ Rinv_f,
                                                        int* __restrict__ status) {
  __shared__ double dg[kMaxKWide];
  __shared__ double maxdiag_s;
  __shared__ int fail_s;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  for (int j = tid; j < k; j += nt) dg[j] = G[(int64_t)j * ld + j];
  for (int t = tid; t < ld * ld; t += nt) {
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
  for (int attempt = 0; attempt < 2; ++attempt) {
    // R <- upper triangle of G + shift I (zero elsewhere)
    for (int t = tid; t < ld * ld; t += nt) {
      const int r = t / ld, c = t - r * ld;
      R[t] = (r < k && c < k && c >= r) ? G[t] + (r == c ? shift : 0.0) : 0.0;
    }
    if (tid == 0) fail_s = -1;
    __syncthreads();
    for (int j = 0; j < k; ++j) {
      const double d = R[(int64_t)j * ld + j];  // every thread reads the same value: uniform exit
      const bool ok = isfinite(d) && d > 0.0 && (attempt == 1 || d > tau * (dg[j] + shift));
      if (!ok) {
        if (tid == 0) fail_s = j;
        break;
      }
      const double rj = 1.0 / sqrt(d);
      __syncthreads();  // every thread has read d before row j is rescaled
      for (int c = j + tid; c < k; c += nt) R[(int64_t)j * ld + c] *= rj;
      __syncthreads();
      for (int a = j + 1 + warp; a < k; a += nw) {
        const double rja = R[(int64_t)j * ld + a];
        for (int c = a + lane; c < k; c += 32) R[(int64_t)a * ld + c] -= rja * R[(int64_t)j * ld + c];
      }
      __syncthreads();
    }
    __syncthreads();
    const int fail = fail_s;
    if (fail < 0) break;
    if (!shift_on_fail || attempt == 1) {
      if (tid == 0) status[0] = -(fail + 1);
      // well-defined (identity) factors keep the downstream kernels finite
      for (int t = tid; t < ld * ld; t += nt) {
        const int r = t / ld, c = t - r * ld;
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
  // R^{-1} (upper triangular): column c, rows r = c, c - 1, ..., 0:
  // X_cc = 1 / R_cc, X_rc = -(sum_{m = r+1..c} R_rm X_mc) / R_rr.
  for (int c = warp; c < k; c += nw) {
    if (lane == 0) Rinv[(int64_t)c * ld + c] = 1.0 / R[(int64_t)c * ld + c];
    __syncwarp();
    for (int r = c - 1; r >= 0; --r) {
      double s = 0.0;
      for (int m = r + 1 + lane; m <= c; m += 32) s = fma(R[(int64_t)r * ld + m], Rinv[(int64_t)m * ld + c], s);
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) Rinv[(int64_t)r * ld + c] = -s / R[(int64_t)r * ld + r];
      __syncwarp();
    }
  }
  __syncthreads();
  for (int t = tid; t < ld * ld; t += nt) Rinv_f[t] = (float)Rinv[t];
}

cudaError_t launch_cholesky_wide(const double* G, int k, int ld, double tau, int shift_on_fail, double* R,
                                 double* Rinv, float* Rinv_f, int* status, cudaStream_t st) {
  if (k > kMaxKWide || ld > kMaxKWide || k > ld) return cudaErrorInvalidValue;
  note_launches(1);
  k_cholesky_wide<<<1, 1024, 0, st>>>(G, k, ld, tau, shift_on_fail, R, Rinv, Rinv_f, status);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Tall x small, one output panel: Out[i, c0 + o] = sum_{l < K} In[i, l]
// M[l, c0 + o], o < cnt <= 128, K <= kMaxKWide.  M's panel (K x 128, zero past
// cnt) sits in shared memory; rows go in tiles of 32, each staged whole in
// shared memory before any of its rows is written, so Out may alias In as long
// as no later launch reads the columns this one writes.  Thread (ty, tx) of
// the 8 x 32 grid computes rows ty + 8 i (i < 4) at columns 4 tx .. 4 tx + 3.
// ---------------------------------------------------------------------------
constexpr int kWideRows = 32;

__global__ void __launch_bounds__(256) k_tall_mm_wide(const float* In, int64_t n, int K, int ldi,
                                                      const float* __restrict__ M, int ldm, int c0, int cnt,
                                                      float* Out, int ldo) {
  extern __shared__ __align__(16) float smw[];
  float* Ms = smw;                 // [K][kPanel]
  float* Ts = smw + K * kPanel;    // [kWideRows][K + 1]
  const int KP = K + 1;
  for (int t = threadIdx.x; t < K * kPanel; t += blockDim.x) {
    const int l = t / kPanel, o = t - l * kPanel;
    Ms[t] = o < cnt ? M[(int64_t)l * ldm + c0 + o] : 0.f;
  }
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t n_tiles = (n + kWideRows - 1) / kWideRows;
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t r0 = tile * kWideRows;
    const int rows = (int)min((int64_t)kWideRows, n - r0);
    __syncthreads();  // the previous tile is consumed (and M is staged)
    for (int t = threadIdx.x; t < kWideRows * K; t += blockDim.x) {
      const int r = t / K, l = t - r * K;
      Ts[r * KP + l] = r < rows ? In[(r0 + r) * ldi + l] : 0.f;
    }
    __syncthreads();
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int o = 0; o < 4; ++o) acc[i][o] = 0.f;
    for (int l = 0; l < K; ++l) {
      const float4 m = *reinterpret_cast<const float4*>(Ms + l * kPanel + 4 * tx);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float a = Ts[(ty + 8 * i) * KP + l];
        acc[i][0] = fmaf(a, m.x, acc[i][0]);
        acc[i][1] = fmaf(a, m.y, acc[i][1]);
        acc[i][2] = fmaf(a, m.z, acc[i][2]);
        acc[i][3] = fmaf(a, m.w, acc[i][3]);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = ty + 8 * i;
      if (r >= rows) continue;
#pragma unroll
      for (int o = 0; o < 4; ++o)
        if (4 * tx + o < cnt) Out[(r0 + r) * ldo + c0 + 4 * tx + o] = acc[i][o];
    }
  }
}

cudaError_t launch_tall_mm_wide(const float* In, int64_t n, int K, int ldi, const float* M, int ldm, int c0,
                                int cnt, float* Out, int ldo, cudaStream_t st, int num_sms) {
  if (n == 0 || cnt <= 0) return cudaSuccess;
  if (cnt > kPanel || K > kMaxKWide || K <= 0) return cudaErrorInvalidValue;
  const size_t smem = ((size_t)K * kPanel + (size_t)kWideRows * (K + 1)) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_tall_mm_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t n_tiles = (n + kWideRows - 1) / kWideRows;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(n_tiles, num_sms));
  note_launches(1);
  k_tall_mm_wide<<<grid, 256, smem, st>>>(In, n, K, ldi, M, ldm, c0, cnt, Out, ldo);
  return cudaGetLastError();
}

// In[i, :] <- In[i, :] M for an upper-triangular M (ld x ld), in place: the
// panels go right to left, panel p reading only columns < its own end, which
// the panels to its right leave untouched.
cudaError_t launch_apply_upper_wide(float* A, int64_t n, int ld, const float* M, cudaStream_t st, int num_sms) {
  for (int c0 = ld - kPanel; c0 >= 0; c0 -= kPanel) {
    cudaError_t e = launch_tall_mm_wide(A, n, c0 + kPanel, ld, M, ld, c0, kPanel, A, ld, st, num_sms);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Gene-side FP64: Z = (W - mu s^T) M for ld <= kMaxKWide, one thread per
// output column, eight rows per step staged in shared memory (so Z may alias
// W); M is read from global memory (L2-resident).  The sum over l runs in
// index order, as in k_center_apply.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kMaxKWide) k_center_apply_wide(const double* W, int64_t g, int ld,
                                                                 const double* __restrict__ mu,
                                                                 const double* __restrict__ s,
                                                                 const double* __restrict__ M, double* Z) {
  constexpr int RB = 8;
  __shared__ double rows[RB][kMaxKWide];
  const int c = threadIdx.x;
  for (int64_t j0 = (int64_t)blockIdx.x * RB; j0 < g; j0 += (int64_t)gridDim.x * RB) {
    __syncthreads();
    for (int t = threadIdx.x; t < RB * ld; t += blockDim.x) {
      const int r = t / ld, l = t - r * ld;
      const int64_t j = j0 + r;
      double v = 0.0;
      if (j < g) {
        v = W[j * ld + l];
        if (mu) v -= mu[j] * s[l];
      }
      rows[r][l] = v;
    }
    __syncthreads();
    if (c < ld) {
      double acc[RB];
#pragma unroll
      for (int r = 0; r < RB; ++r) acc[r] = 0.0;
      for (int l = 0; l < ld; ++l) {
        const double m = M[(int64_t)l * ld + c];
#pragma unroll
        for (int r = 0; r < RB; ++r) acc[r] = fma(rows[r][l], m, acc[r]);
      }
#pragma unroll
      for (int r = 0; r < RB; ++r)
        if (j0 + r < g) Z[(j0 + r) * ld + c] = acc[r];
    }
  }
}

cudaError_t launch_center_apply_wide(const double* W, int64_t g, int ld, const double* mu, const double* s,
                                     const double* M, double* Z, cudaStream_t st) {
  if (ld > kMaxKWide) return cudaErrorInvalidValue;
  if (g == 0) return cudaSuccess;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((g + 7) / 8, 296));
  note_launches(1);
  k_center_apply_wide<<<grid, kMaxKWide, 0, st>>>(W, g, ld, mu, s, M, Z);
  return cudaGetLastError();
}

}  // namespace scx
