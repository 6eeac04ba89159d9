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
// owns output entries (ty + 16 i, tx + 16 j), i, j < T = ld / 16, so the shared
// row reads of a warp hit consecutive banks.  Products of float inputs are
// exact in FP64; accumulation is FP64.
// ---------------------------------------------------------------------------
template <typename T, int LD>
__global__ void __launch_bounds__(256) k_gram(const T* __restrict__ A, int64_t n,
                                              double* __restrict__ part) {
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
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = (int64_t)blockIdx.x * per;
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
        for (int j = 0; j < TT; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (threadIdx.x < LD)
      for (int r = 0; r < rows; ++r) csum += sh[r][threadIdx.x];
    __syncthreads();
  }
  double* out = part + (int64_t)blockIdx.x * (LD * LD + LD);
#pragma unroll
  for (int i = 0; i < TT; ++i)
#pragma unroll
    for (int j = 0; j < TT; ++j) out[(ty + 16 * i) * LD + tx + 16 * j] = acc[i][j];
  if (threadIdx.x < LD) out[LD * LD + threadIdx.x] = csum;
}

template <typename T>
static cudaError_t gram_t(const T* A, int64_t n, int ld, double* part, int nparts, cudaStream_t st) {
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
// Cholesky of the leading k x k block of G (ld x ld), right-looking, one
// block.  A pivot j fails when its Schur complement d_j <= tau * G_jj (the
// column is numerically dependent on the previous ones) or is not finite.
// With shift_on_fail the factorisation restarts once on G + s I,
// s = 10 tau max_j G_jj, which always succeeds on finite input.
// ---------------------------------------------------------------------------
// One barrier per elimination step: every thread reads the pivot d_j itself,
// the trailing update uses the unscaled row j (A_ac -= A_ja A_jc / d_j), and
// the scaled row j of R goes straight to global memory.  R^{-1} is then
// formed in place row by row from the bottom (row i needs only rows > i),
// one warp per column dot product.
__global__ void __launch_bounds__(1024) k_cholesky(const double* __restrict__ G, int k, int ld, double tau,
                                                   int shift_on_fail, double* __restrict__ R,
                                                   double* __restrict__ Rinv, float* __restrict__ Rinv_f,
                                                   int* __restrict__ status) {
  extern __shared__ double A[];  // [k][k], then tmp[k]
  double* tmp = A + k * k;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  double maxdiag = 0.0;
  for (int j = 0; j < k; ++j) maxdiag = fmax(maxdiag, G[j * ld + j]);
  double shift = 0.0;
  int fail = -1;
  for (int attempt = 0; attempt < 2; ++attempt) {
    for (int t = tid; t < ld * ld; t += nt) R[t] = 0.0;
    for (int t = tid; t < k * k; t += nt) {
      const int r = t / k, c = t % k;
      A[t] = G[r * ld + c] + (r == c ? shift : 0.0);
    }
    __syncthreads();
    fail = -1;
    for (int j = 0; j < k; ++j) {
      const double d = A[j * k + j];
      const double d0 = G[j * ld + j] + shift;
      if (!(isfinite(d) && d > 0.0 && (attempt == 1 || d > tau * d0))) {
        fail = j;  // every thread sees the same pivot: uniform exit
        break;
      }
      const double rinv = rsqrt(d), dinv = 1.0 / d;
      for (int c = j + tid; c < k; c += nt) R[j * ld + c] = A[j * k + c] * rinv;
      const int m = k - j - 1;
      for (int t = tid; t < m * m; t += nt) {
        const int a = j + 1 + t / m, c = j + 1 + t % m;
        if (c >= a) A[a * k + c] -= A[j * k + a] * A[j * k + c] * dinv;
      }
      __syncthreads();
    }
    if (fail < 0) break;
    __syncthreads();
    if (!shift_on_fail || attempt == 1) {
      if (tid == 0) status[0] = -(fail + 1);
      // Leave well-defined (identity) factors so downstream kernels stay finite.
      for (int t = tid; t < ld * ld; t += nt) {
        const int r = t / ld, c = t % ld;
        const double v = (r == c && r < k) ? 1.0 : 0.0;
        R[t] = v;
        Rinv[t] = v;
        Rinv_f[t] = (float)v;
      }
      return;
    }
    if (tid == 0) status[0] += 1;
    shift = 10.0 * tau * fmax(maxdiag, 1e-300);
  }
  __syncthreads();
  // A <- R (upper; lower part ignored), then invert in place from the bottom row up.
  for (int t = tid; t < k * k; t += nt) A[t] = R[(t / k) * ld + (t % k)];
  __syncthreads();
  for (int i = k - 1; i >= 0; --i) {
    for (int c = i + tid; c < k; c += nt) tmp[c] = A[i * k + c];
    __syncthreads();
    for (int c = i + warp; c < k; c += nw) {
      double s = 0.0;
      for (int l = i + 1 + lane; l <= c; l += 32) s += tmp[l] * A[l * k + c];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) A[i * k + c] = ((i == c ? 1.0 : 0.0) - s) / tmp[i];
    }
    __syncthreads();
  }
  for (int t = tid; t < ld * ld; t += nt) {
    const int r = t / ld, c = t % ld;
    const double v = (r < k && c < k && c >= r) ? A[r * k + c] : 0.0;
    Rinv[t] = v;
    Rinv_f[t] = (float)v;
  }
}

cudaError_t launch_cholesky(const double* G, int k, int ld, double tau, int shift_on_fail,
                            double* R, double* Rinv, float* Rinv_f, int* status, cudaStream_t st) {
  size_t smem = (size_t)(k * k + k) * sizeof(double);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_cholesky, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  note_launches(1);
  k_cholesky<<<1, 1024, smem, st>>>(G, k, ld, tau, shift_on_fail, R, Rinv, Rinv_f, status);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Tall x small: Out[i, :cnt] = In[i, :K] * M (K x cnt), one thread per row.
// M (zero-padded to OUTB columns) sits in shared memory and every thread of a
// warp reads the same M entries (broadcast); the row and its OUTB outputs stay
// in registers, so there are four FMAs per shared load.  A thread reads its
// whole row before writing, so Out may alias In.
// ---------------------------------------------------------------------------
template <int OUTB>
__global__ void __launch_bounds__(128) k_tall_mm(const float* In, int64_t n, int K, int ldi,
                                                 const float* __restrict__ M, int ldm, int cnt,
                                                 float* Out, int ldo) {
  extern __shared__ float Ms[];  // [K][OUTB]
  for (int t = threadIdx.x; t < K * OUTB; t += blockDim.x) {
    const int l = t / OUTB, o = t % OUTB;
    Ms[t] = o < cnt ? M[l * ldm + o] : 0.f;
  }
  __syncthreads();
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    float acc[OUTB];
#pragma unroll
    for (int o = 0; o < OUTB; ++o) acc[o] = 0.f;
    const float4* in4 = reinterpret_cast<const float4*>(In + row * ldi);
    for (int l = 0; l < K; l += 4) {
      const float4 x = in4[l >> 2];
      const float xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float4* mr = reinterpret_cast<const float4*>(Ms + (l + u) * OUTB);
#pragma unroll
        for (int o = 0; o < OUTB / 4; ++o) {
          const float4 m = mr[o];
          acc[4 * o + 0] = fmaf(xs[u], m.x, acc[4 * o + 0]);
          acc[4 * o + 1] = fmaf(xs[u], m.y, acc[4 * o + 1]);
          acc[4 * o + 2] = fmaf(xs[u], m.z, acc[4 * o + 2]);
          acc[4 * o + 3] = fmaf(xs[u], m.w, acc[4 * o + 3]);
        }
      }
    }
    float* out = Out + row * ldo;
    if ((cnt & 3) == 0 && (ldo & 3) == 0) {
#pragma unroll
      for (int o = 0; o < OUTB / 4; ++o)
        if (4 * o < cnt)
          reinterpret_cast<float4*>(out)[o] =
              make_float4(acc[4 * o], acc[4 * o + 1], acc[4 * o + 2], acc[4 * o + 3]);
    } else {
#pragma unroll
      for (int o = 0; o < OUTB; ++o)
        if (o < cnt) out[o] = acc[o];
    }
  }
}

static cudaError_t tall_mm(const float* In, int64_t n, int K, int ldi, const float* M, int ldm, int cnt,
                           float* Out, int ldo, cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  const int outb = cnt <= 64 ? 64 : 128;
  const size_t smem = (size_t)K * outb * sizeof(float);
  const int grid = grid_for(n, 128, num_sms, 8);
  note_launches(1);
  if (outb == 64) {
    cudaFuncSetAttribute(k_tall_mm<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_tall_mm<64><<<grid, 128, smem, st>>>(In, n, K, ldi, M, ldm, cnt, Out, ldo);
  } else {
    cudaFuncSetAttribute(k_tall_mm<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_tall_mm<128><<<grid, 128, smem, st>>>(In, n, K, ldi, M, ldm, cnt, Out, ldo);
  }
  return cudaGetLastError();
}

cudaError_t launch_apply_right_f32(const float* In, int64_t n, int ld, const float* M, float* Out,
                                   cudaStream_t st, int num_sms) {
  return tall_mm(In, n, ld, ld, M, ld, ld, Out, ld, st, num_sms);
}

// ---------------------------------------------------------------------------
// Gene-side FP64 ops.  Block = 256 threads handles 256 / ld rows at a time.
// ---------------------------------------------------------------------------
__global__ void k_center_apply(const double* __restrict__ W, int64_t g, int ld,
                               const double* __restrict__ mu, const double* __restrict__ s,
                               const double* __restrict__ M, double* __restrict__ Z) {
  extern __shared__ double sm[];  // M [ld][ld], rows [256/ld][ld]
  double* Ms = sm;
  double* rows = sm + ld * ld;
  for (int t = threadIdx.x; t < ld * ld; t += blockDim.x) Ms[t] = M[t];
  const int rpb = blockDim.x / ld;
  const int r = threadIdx.x / ld, c = threadIdx.x % ld;
  for (int64_t j0 = (int64_t)blockIdx.x * rpb; j0 < g; j0 += (int64_t)gridDim.x * rpb) {
    __syncthreads();
    const int64_t j = j0 + r;
    if (r < rpb && j < g) {
      double v = W[j * ld + c];
      if (mu) v -= mu[j] * s[c];
      rows[r * ld + c] = v;
    }
    __syncthreads();
    if (r < rpb && j < g) {
      double acc = 0.0;
      for (int l = 0; l < ld; ++l) acc = fma(rows[r * ld + l], Ms[l * ld + c], acc);
      Z[j * ld + c] = acc;
    }
  }
}

cudaError_t launch_center_apply(const double* W, int64_t g, int ld, const double* mu,
                                const double* s, const double* M, double* Z, cudaStream_t st) {
  size_t smem = (size_t)(ld * ld + 256) * sizeof(double);
  cudaFuncSetAttribute(k_center_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int rpb = 256 / ld;
  int grid = (int)std::min<int64_t>((g + rpb - 1) / rpb, 1184);
  note_launches(1);
  k_center_apply<<<grid, 256, smem, st>>>(W, g, ld, mu, s, M, Z);
  return cudaGetLastError();
}

cudaError_t launch_apply_right_f64(double* A, int64_t g, int ld, const double* M, cudaStream_t st) {
  return launch_center_apply(A, g, ld, nullptr, nullptr, M, A, st);
}

__global__ void k_round_v(const double* __restrict__ A, int64_t g, int ld, float* __restrict__ Vf) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < g * ld;
       t += (int64_t)gridDim.x * blockDim.x)
    Vf[t] = (float)A[t];
}

// mc[c] = sum_j mu_j Vf[j][c], FP64 accumulation, one block per column.
__global__ void k_mean_prefactor(const float* __restrict__ Vf, int64_t g, int ld,
                                 const double* __restrict__ mu, float* __restrict__ mc) {
  __shared__ double red[256];
  const int c = blockIdx.x;
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
// Parallel cyclic Jacobi (round-robin pairing) for the symmetric k x k block
// of C.  Each round rotates kk/2 disjoint pairs: angles first, then column
// rotations of A and E, then row rotations of A.  Stops when the off-diagonal
// mass falls below (1e-15)^2 of the total or after 40 sweeps.
// ---------------------------------------------------------------------------
__global__ void k_jacobi(const double* __restrict__ C, int k, int ld, double* __restrict__ evals,
                         double* __restrict__ evecs, double* __restrict__ Eglob, int* sweeps_out) {
  extern __shared__ double sm[];
  const int kk = (k + 1) & ~1;  // even number of players; index k (if odd) is a dummy
  double* A = sm;               // [kk][kk]
  double* E = (Eglob != nullptr) ? Eglob : sm + kk * kk;
  __shared__ double cs[kMaxK / 2], sn[kMaxK / 2];
  __shared__ int pp[kMaxK / 2], qq[kMaxK / 2];
  __shared__ double red[256];
  __shared__ int done;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int t = tid; t < kk * kk; t += nt) {
    int r = t / kk, c = t % kk;
    A[t] = (r < k && c < k) ? C[r * ld + c] : 0.0;
    E[t] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int npair = kk / 2;
  int sweep = 0;
  (void)red;
  for (; sweep < 40; ++sweep) {
    // Converged when a whole sweep performs no rotation: every off-diagonal
    // entry is below 1e-15 of the geometric mean of its two diagonal entries.
    if (tid == 0) done = 1;
    __syncthreads();
    for (int round = 0; round < kk - 1; ++round) {
      for (int i = tid; i < npair; i += nt) {
        int a, b;
        if (i == 0) { a = round; b = kk - 1; }
        else { a = (round + i) % (kk - 1); b = (round - i + (kk - 1)) % (kk - 1); }
        int p = min(a, b), q = max(a, b);
        double c = 1.0, s = 0.0;
        if (q < k) {
          double apq = A[p * kk + q];
          double app = A[p * kk + p], aqq = A[q * kk + q];
          if (fabs(apq) > 1e-300 && fabs(apq) > 1e-15 * sqrt(fabs(app * aqq))) {
            double theta = (aqq - app) / (2.0 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            s = t * c;
            done = 0;
          }
        }
        pp[i] = p; qq[i] = q; cs[i] = c; sn[i] = s;
      }
      __syncthreads();
      // columns of A and E: (x_p, x_q) <- (c x_p - s x_q, s x_p + c x_q)
      for (int t = tid; t < npair * kk; t += nt) {
        int i = t / kk, r = t % kk;
        double c = cs[i], s = sn[i];
        if (s == 0.0) continue;
        int p = pp[i], q = qq[i];
        double xp = A[r * kk + p], xq = A[r * kk + q];
        A[r * kk + p] = c * xp - s * xq;
        A[r * kk + q] = s * xp + c * xq;
        double ep = E[r * kk + p], eq = E[r * kk + q];
        E[r * kk + p] = c * ep - s * eq;
        E[r * kk + q] = s * ep + c * eq;
      }
      __syncthreads();
      // rows of A
      for (int t = tid; t < npair * kk; t += nt) {
        int i = t / kk, col = t % kk;
        double c = cs[i], s = sn[i];
        if (s == 0.0) continue;
        int p = pp[i], q = qq[i];
        double xp = A[p * kk + col], xq = A[q * kk + col];
        A[p * kk + col] = c * xp - s * xq;
        A[q * kk + col] = s * xp + c * xq;
      }
      __syncthreads();
    }
    if (done) break;
    __syncthreads();
  }
  // sort eigenvalues descending: rank of each by counting (ties by index)
  for (int i = tid; i < k; i += nt) {
    double v = A[i * kk + i];
    int rank = 0;
    for (int j = 0; j < k; ++j) {
      double w = A[j * kk + j];
      if (w > v || (w == v && j < i)) ++rank;
    }
    evals[rank] = v;
    for (int r = 0; r < ld; ++r) evecs[r * ld + rank] = (r < k) ? E[r * kk + i] : 0.0;
  }
  for (int t = tid; t < ld * ld; t += nt) {
    int c = t % ld;
    if (c >= k) evecs[t] = 0.0;
  }
  if (tid == 0 && sweeps_out) *sweeps_out = sweep;
}

cudaError_t launch_jacobi_eig(const double* C, int k, int ld, double* evals, double* evecs,
                              int* sweeps, cudaStream_t st) {
  int kk = (k + 1) & ~1;
  size_t both = (size_t)2 * kk * kk * sizeof(double);
  size_t one = (size_t)kk * kk * sizeof(double);
  // E lives in shared memory when both matrices fit, else in the tail of evecs'
  // allocation is not available, so use a dedicated global scratch: evecs itself
  // cannot be reused (it is written at the end), so the caller's evecs buffer is
  // followed by kk*kk doubles of scratch (the plan allocates 2 * ld * ld).
  double* eglob = nullptr;
  size_t smem = both;
  if (both > 200 * 1024) {
    eglob = evecs + (size_t)ld * ld;
    smem = one;
  }
  cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  note_launches(1);
  k_jacobi<<<1, 256, smem, st>>>(C, k, ld, evals, evecs, eglob, sweeps);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Rayleigh-Ritz finish (single kernel, one block per gene row for the
// components plus block 0 building M_emb).
// ---------------------------------------------------------------------------
__global__ void k_ritz_finish(const double* __restrict__ B, int64_t g, int ld, int k, int nc,
                              const double* __restrict__ evals, const double* __restrict__ E,
                              const double* __restrict__ Rinv2, double* __restrict__ sigma,
                              float* __restrict__ comps, float* __restrict__ M_emb) {
  extern __shared__ double sm[];
  double* Es = sm;             // [ld][nc]
  double* sg = sm + ld * nc;   // [nc]
  for (int t = threadIdx.x; t < ld * nc; t += blockDim.x) {
    int l = t / nc, c = t % nc;
    Es[t] = E[l * ld + c];
  }
  for (int c = threadIdx.x; c < nc; c += blockDim.x) sg[c] = sqrt(fmax(evals[c], 0.0));
  __syncthreads();
  if (blockIdx.x == 0) {
    for (int c = threadIdx.x; c < k; c += blockDim.x) sigma[c] = sqrt(fmax(evals[c], 0.0));
    for (int t = threadIdx.x; t < ld * nc; t += blockDim.x) {
      int l = t / nc, c = t % nc;
      double acc = 0.0;
      for (int m = 0; m < ld; ++m) acc = fma(Rinv2[l * ld + m], Es[m * nc + c], acc);
      M_emb[t] = (float)(acc * sg[c]);
    }
  }
  for (int64_t j = blockIdx.x; j < g; j += gridDim.x) {
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
      double acc = 0.0;
      for (int l = 0; l < k; ++l) acc = fma(B[j * ld + l], Es[l * nc + c], acc);
      comps[(int64_t)c * g + j] = sg[c] > 0.0 ? (float)(acc / sg[c]) : 0.f;
    }
  }
}

cudaError_t launch_ritz_finish(const double* B, int64_t g, int ld, int k, int nc,
                               const double* evals, const double* evecs, const double* Rinv2,
                               double* sigma, float* components, float* M_emb, cudaStream_t st) {
  size_t smem = (size_t)(ld * nc + nc) * sizeof(double);
  cudaFuncSetAttribute(k_ritz_finish, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int grid = (int)std::min<int64_t>(g, 2048);
  note_launches(1);
  k_ritz_finish<<<grid, 128, smem, st>>>(B, g, ld, k, nc, evals, evecs, Rinv2, sigma, components,
                                         M_emb);
  return cudaGetLastError();
}

// Embeddings U = Q M_emb (n x nc row-major).
cudaError_t launch_embed(const float* Q, int64_t n, int ld, int k, const float* M_emb, int nc,
                         float* U, cudaStream_t st, int num_sms) {
  (void)k;  // rows k..ld-1 of M_emb are zero
  return tall_mm(Q, n, ld, ld, M_emb, nc, nc, U, nc, st, num_sms);
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
