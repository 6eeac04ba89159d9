// Kernels of the truncated-SVD adjoint (the backward pass of the PCA scores).
//
// Scores S = X~ V (n x c), X~ = (X - 1 mu^T) diag(s) the plan's working
// matrix, V its top-c right singular vectors.  Given dL/dS = G, the gradient
// with respect to X~ is the rank-2c matrix
//     D = (G + X~ A) V^T + S A^T,
// where A (n_vars x c) collects, per component i, the solution a_i of
// (lambda_i I - X~^T X~) a_i = (I - v_i v_i^T) X~^T g_i on the complement of
// v_i: the part inside the sketch subspace comes from the Ritz pairs
// (coefficients 1 / (lambda_i - lambda_j)), the part outside it from a few
// conjugate-gradient steps, each one more power-iteration block X~^T X~ P.
// D is never formed: an SDDMM samples it at the stored entries only (the
// gradient of each stored value), and its column sums come from the low-rank
// factors (the gradients of the per-gene centre and scale vectors).
// These kernels hold the gene-side (n_vars x ld, FP64) algebra and the SDDMM;
// the sparse products reuse the plan's forward and transposed SpMM.
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace scx {

namespace {

// Column sums of a tall float matrix (n x ld, first ncols columns): block b
// sums rows [b n / nparts, (b + 1) n / nparts) in FP64 in a fixed order and
// writes part[b * ld + c]; k_reduce_rows finishes the sum in block order.
__global__ void __launch_bounds__(256) k_colsum_f32(const float* __restrict__ A, int64_t n, int ld, int ncols,
                                                   double* __restrict__ part) {
  __shared__ double red[256];
  const int per = 256 / ncols;  // row lanes
  const int c = threadIdx.x % ncols, ro = threadIdx.x / ncols;
  const int64_t r0 = (int64_t)blockIdx.x * n / gridDim.x, r1 = (int64_t)(blockIdx.x + 1) * n / gridDim.x;
  double acc = 0.0;
  if (ro < per)
    for (int64_t r = r0 + ro; r < r1; r += per) acc += (double)A[r * ld + c];
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < ld) {
    double s = 0.0;
    if (threadIdx.x < ncols)
      for (int u = 0; u < per; ++u) s += red[u * ncols + threadIdx.x];
    part[(int64_t)blockIdx.x * ld + threadIdx.x] = s;
  }
}

// T[a][b] = sum_j A[j][a] B[j][b] for a < ka, b < kb (ld x ld output, zero
// elsewhere).  One thread per output, a fixed j order: deterministic.
__global__ void k_atb(const double* __restrict__ A, const double* __restrict__ B, int64_t g, int ld, int ka,
                      int kb, double* __restrict__ T) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ld * ld) return;
  const int a = t / ld, b = t % ld;
  double acc = 0.0;
  if (a < ka && b < kb)
    for (int64_t j = 0; j < g; ++j) acc = fma(A[j * ld + a], B[j * ld + b], acc);
  T[t] = acc;
}

// M = E diag(1 / sigma) over the first k columns (sigma = sqrt(max(lambda, 0));
// a zero sigma gives a zero column), zero elsewhere.
__global__ void k_ritz_scale(const double* __restrict__ E, const double* __restrict__ evals, int k, int ld,
                             double* __restrict__ M) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ld * ld; t += gridDim.x * blockDim.x) {
    const int l = t % ld;
    const double sg = l < k ? sqrt(fmax(evals[l], 0.0)) : 0.0;
    M[t] = sg > 0.0 ? E[t] / sg : 0.0;
  }
}

// Phi[j][i] = T[j][i] / (lambda_i - lambda_j) for j < k, i < c, j != i
// (a tie lambda_i == lambda_j contributes nothing), zero elsewhere.
__global__ void k_phi(const double* __restrict__ T, const double* __restrict__ evals, int k, int c, int ld,
                      double* __restrict__ Phi) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ld * ld; t += gridDim.x * blockDim.x) {
    const int j = t / ld, i = t % ld;
    double v = 0.0;
    if (j < k && i < c && j != i) {
      const double gap = evals[i] - evals[j];
      v = gap != 0.0 ? T[t] / gap : 0.0;
    }
    Phi[t] = v;
  }
}

// Out = X + beta Y elementwise over the first c columns (g x ld; the padding
// columns are zeroed).
__global__ void k_axpy_cols(const double* __restrict__ X, const double* __restrict__ Y, double beta, int64_t g,
                            int ld, int c, double* __restrict__ Out) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < g * ld; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % ld);
    Out[t] = i < c ? X[t] + beta * Y[t] : 0.0;
  }
}

// out[i] = sum_j X[j][i] Y[j][i], one block per column (fixed tree order).
__global__ void __launch_bounds__(256) k_coldot(const double* __restrict__ X, const double* __restrict__ Y, int64_t g,
                                                int ld, double* __restrict__ out) {
  __shared__ double red[256];
  const int i = blockIdx.x;
  double acc = 0.0;
  for (int64_t j = threadIdx.x; j < g; j += blockDim.x) acc = fma(X[j * ld + i], Y[j * ld + i], acc);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[i] = red[0];
}

// Shifted operator on the complement: Ap = lambda_i p - (W - Proj), with
// W = X~^T X~ p and Proj its component inside the sketch subspace.
__global__ void k_cg_ap(const double* __restrict__ P, const double* __restrict__ W, const double* __restrict__ Proj,
                        const double* __restrict__ evals, int64_t g, int ld, int c, double* __restrict__ Ap) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < g * ld; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % ld);
    Ap[t] = i < c ? evals[i] * P[t] - (W[t] - Proj[t]) : 0.0;
  }
}

// CG step per column i: alpha = rr / pAp; x += alpha p; r -= alpha Ap.
// A column whose residual is already zero (rr == 0) or whose curvature is
// not positive stops moving.
__global__ void k_cg_step(double* __restrict__ X, double* __restrict__ R, const double* __restrict__ P,
                          const double* __restrict__ Ap, const double* __restrict__ rr,
                          const double* __restrict__ pAp, int64_t g, int ld, int c) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < g * ld; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % ld);
    if (i >= c) continue;
    const double alpha = (rr[i] > 0.0 && pAp[i] > 0.0) ? rr[i] / pAp[i] : 0.0;
    X[t] += alpha * P[t];
    R[t] -= alpha * Ap[t];
  }
}

// New search direction p = r + (rr_new / rr) p, then rr = rr_new.
__global__ void k_cg_dir(double* __restrict__ P, const double* __restrict__ R, double* __restrict__ rr,
                         const double* __restrict__ rr_new, int64_t g, int ld, int c) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < g * ld; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % ld);
    if (i >= c) continue;
    const double beta = rr[i] > 0.0 ? rr_new[i] / rr[i] : 0.0;
    P[t] = R[t] + beta * P[t];
  }
}

__global__ void k_copy_vec(double* __restrict__ dst, const double* __restrict__ src, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

// colD[j] = sum_i sF[i] V[j][i] + sS[i] A[j][i]: the column sums of D.
__global__ void k_col_d(const double* __restrict__ V, const double* __restrict__ A, const double* __restrict__ sF,
                        const double* __restrict__ sS, int64_t g, int ld, int c, double* __restrict__ colD) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < g; j += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int i = 0; i < c; ++i) acc = fma(sF[i], V[j * ld + i], fma(sS[i], A[j * ld + i], acc));
    colD[j] = acc;
  }
}

// grad_center[j] = -s_j colD_j ; grad_scale[j] = sum_stored(D P)_j / s_j - center_j colD_j.
__global__ void k_grad_vectors(const double* __restrict__ colD, const double* __restrict__ sumDP,
                               const double* __restrict__ center, const double* __restrict__ scale, int64_t g,
                               double* __restrict__ grad_center, double* __restrict__ grad_scale) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < g; j += (int64_t)gridDim.x * blockDim.x) {
    const double s = scale ? scale[j] : 1.0;
    const double m = center ? center[j] : 0.0;
    if (grad_center) grad_center[j] = -s * colD[j];
    if (grad_scale) grad_scale[j] = (s != 0.0 ? sumDP[j] / s : 0.0) - m * colD[j];
  }
}

// ---------------------------------------------------------------------------
// SDDMM: for every stored entry p = (r, j) of the CSR,
//     d = sum_i (G[r][i] + Y[r][i]) V[j][i] + S[r][i] A[j][i]
//     grad_values[p] (+)= d * s_j
// and per gene sum_p d * x~_p (x~ the working value) into part[chunk][j].
// Grid (row chunks) x (gene blocks of GB genes): a block stages its genes'
// rows of [V | A] in shared memory as FP32 (row stride odd in 16-byte units,
// so a warp's 16-byte reads of different genes spread over the banks); a warp
// takes one row at a time, stages [G + Y | S] of that row, and each lane
// computes the dot product of one stored entry.  cs columns at a time: the
// caller loops over column slices with `accumulate`.
// ---------------------------------------------------------------------------
constexpr int kSddmmGB = kTransposeGeneBlock;

template <typename ValT>
__global__ void __launch_bounds__(512) k_sddmm(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                                               const ValT* __restrict__ val, int64_t n_obs, int32_t g,
                                               const int32_t* __restrict__ rbp, int nb, int64_t rows_per_chunk,
                                               const float* __restrict__ G, int ldg, const float* __restrict__ Y,
                                               int ldy, const float* __restrict__ S, int lds,
                                               const double* __restrict__ V, const double* __restrict__ A, int ldv,
                                               int cs, const double* __restrict__ scale, int accumulate,
                                               float* __restrict__ grad, double* __restrict__ part) {
  extern __shared__ __align__(16) float smf[];
  const int stride = ((2 * cs + 3) / 4 | 1) * 4;  // floats per staged row, odd number of float4
  float* VA = smf;                                 // [GB][stride]
  float* rowbuf = VA + kSddmmGB * stride;          // [warps][stride]
  double* acc = reinterpret_cast<double*>(rowbuf + (blockDim.x >> 5) * stride);  // [GB]
  const int b = blockIdx.y, chunk = blockIdx.x;
  const int g0 = b * kSddmmGB;
  const int gb = min(kSddmmGB, g - g0);
  for (int t = threadIdx.x; t < kSddmmGB * stride; t += blockDim.x) {
    const int jj = t / stride, u = t % stride;
    float v = 0.f;
    if (jj < gb) {
      const int64_t j = g0 + jj;
      if (u < cs) v = (float)V[j * ldv + u];
      else if (u < 2 * cs) v = (float)A[j * ldv + (u - cs)];
    }
    VA[t] = v;
  }
  for (int t = threadIdx.x; t < kSddmmGB; t += blockDim.x) acc[t] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float* rb = rowbuf + wid * stride;
  const int nq = stride / 4;
  const int64_t r0 = (int64_t)chunk * rows_per_chunk, r1 = min(n_obs, r0 + rows_per_chunk);
  for (int64_t row = r0 + wid; row < r1; row += nw) {
    const int64_t base = indptr[row];
    const int32_t* rr = rbp + row * (nb + 1);
    const int64_t s0 = base + rr[b], e0 = base + rr[b + 1];
    if (s0 >= e0) continue;
    for (int u = lane; u < stride; u += 32) {
      float v = 0.f;
      if (u < cs) v = G[row * ldg + u] + Y[row * ldy + u];
      else if (u < 2 * cs) v = S[row * lds + (u - cs)];
      rb[u] = v;
    }
    __syncwarp();
    const float4* rb4 = reinterpret_cast<const float4*>(rb);
    for (int64_t p = s0 + lane; p < e0; p += 32) {
      const int32_t j = idx[p];
      const float4* va4 = reinterpret_cast<const float4*>(VA + (j - g0) * stride);
      float d = 0.f;
      for (int u = 0; u < nq; ++u) {
        const float4 x = rb4[u], y = va4[u];
        d = fmaf(x.x, y.x, d);
        d = fmaf(x.y, y.y, d);
        d = fmaf(x.z, y.z, d);
        d = fmaf(x.w, y.w, d);
      }
      const float sj = scale ? (float)scale[j] : 1.f;
      grad[p] = accumulate ? grad[p] + d * sj : d * sj;
      atomicAdd(&acc[j - g0], (double)d * (double)to_f32(val[p]));
    }
    __syncwarp();
  }
  __syncthreads();
  for (int t = threadIdx.x; t < gb; t += blockDim.x) part[(int64_t)chunk * g + g0 + t] = acc[t];
}

}  // namespace

cudaError_t launch_colsum_f32(const float* A, int64_t n, int ld, int ncols, double* part, int nparts,
                              double* out, cudaStream_t st, int num_sms) {
  if (ncols > 256 || ld > 256) return cudaErrorInvalidValue;
  note_launches(1);
  k_colsum_f32<<<nparts, 256, 0, st>>>(A, n, ld, ncols, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_rows_f64(part, nparts, ld, out, 0, st, num_sms);
}

cudaError_t launch_atb(const double* A, const double* B, int64_t g, int ld, int ka, int kb, double* T,
                       cudaStream_t st) {
  note_launches(1);
  k_atb<<<(ld * ld + 127) / 128, 128, 0, st>>>(A, B, g, ld, ka, kb, T);
  return cudaGetLastError();
}

cudaError_t launch_ritz_scale(const double* E, const double* evals, int k, int ld, double* M, cudaStream_t st) {
  note_launches(1);
  k_ritz_scale<<<(ld * ld + 255) / 256, 256, 0, st>>>(E, evals, k, ld, M);
  return cudaGetLastError();
}

cudaError_t launch_phi(const double* T, const double* evals, int k, int c, int ld, double* Phi, cudaStream_t st) {
  note_launches(1);
  k_phi<<<(ld * ld + 255) / 256, 256, 0, st>>>(T, evals, k, c, ld, Phi);
  return cudaGetLastError();
}

static int gene_grid(int64_t g, int ld) { return (int)std::min<int64_t>((g * ld + 255) / 256, 1184); }

cudaError_t launch_axpy_cols(const double* X, const double* Y, double beta, int64_t g, int ld, int c, double* Out,
                             cudaStream_t st) {
  note_launches(1);
  k_axpy_cols<<<gene_grid(g, ld), 256, 0, st>>>(X, Y, beta, g, ld, c, Out);
  return cudaGetLastError();
}

cudaError_t launch_coldot(const double* X, const double* Y, int64_t g, int ld, int c, double* out, cudaStream_t st) {
  note_launches(1);
  k_coldot<<<c, 256, 0, st>>>(X, Y, g, ld, out);
  return cudaGetLastError();
}

cudaError_t launch_cg_ap(const double* P, const double* W, const double* Proj, const double* evals, int64_t g,
                         int ld, int c, double* Ap, cudaStream_t st) {
  note_launches(1);
  k_cg_ap<<<gene_grid(g, ld), 256, 0, st>>>(P, W, Proj, evals, g, ld, c, Ap);
  return cudaGetLastError();
}

cudaError_t launch_cg_step(double* X, double* R, const double* P, const double* Ap, const double* rr,
                           const double* pAp, int64_t g, int ld, int c, cudaStream_t st) {
  note_launches(1);
  k_cg_step<<<gene_grid(g, ld), 256, 0, st>>>(X, R, P, Ap, rr, pAp, g, ld, c);
  return cudaGetLastError();
}

cudaError_t launch_cg_dir(double* P, const double* R, double* rr, const double* rr_new, int64_t g, int ld, int c,
                          cudaStream_t st) {
  note_launches(2);
  k_cg_dir<<<gene_grid(g, ld), 256, 0, st>>>(P, R, rr, rr_new, g, ld, c);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_copy_vec<<<1, 128, 0, st>>>(rr, rr_new, c);
  return cudaGetLastError();
}

cudaError_t launch_col_d(const double* V, const double* A, const double* sF, const double* sS, int64_t g, int ld,
                         int c, double* colD, cudaStream_t st) {
  note_launches(1);
  k_col_d<<<(int)std::min<int64_t>((g + 255) / 256, 1184), 256, 0, st>>>(V, A, sF, sS, g, ld, c, colD);
  return cudaGetLastError();
}

cudaError_t launch_grad_vectors(const double* colD, const double* sumDP, const double* center, const double* scale,
                                int64_t g, double* grad_center, double* grad_scale, cudaStream_t st) {
  note_launches(1);
  k_grad_vectors<<<(int)std::min<int64_t>((g + 255) / 256, 1184), 256, 0, st>>>(colD, sumDP, center, scale, g,
                                                                               grad_center, grad_scale);
  return cudaGetLastError();
}

size_t sddmm_smem_bytes(int cs) {
  const int stride = ((2 * cs + 3) / 4 | 1) * 4;
  return (size_t)(kSddmmGB + 16) * stride * sizeof(float) + kSddmmGB * sizeof(double);
}

template <typename ValT>
static cudaError_t sddmm_t(const int64_t* indptr, const int32_t* idx, const void* val, int64_t n, int32_t g,
                           const int32_t* rbp, int nb, int nchunks, int64_t rows_per_chunk, const float* G, int ldg,
                           const float* Y, int ldy, const float* S, int lds, const double* V, const double* A,
                           int ldv, int cs, const double* scale, int accumulate, float* grad, double* part,
                           cudaStream_t st) {
  const size_t smem = sddmm_smem_bytes(cs);
  if (cudaError_t e = allow_smem(k_sddmm<ValT>, smem); e != cudaSuccess) return e;
  dim3 grid(nchunks, nb);
  note_launches(1);
  k_sddmm<ValT><<<grid, 512, smem, st>>>(indptr, idx, static_cast<const ValT*>(val), n, g, rbp, nb, rows_per_chunk,
                                         G, ldg, Y, ldy, S, lds, V, A, ldv, cs, scale, accumulate, grad, part);
  return cudaGetLastError();
}

cudaError_t launch_sddmm(int dtype, const int64_t* indptr, const int32_t* idx, const void* val, int64_t n, int32_t g,
                         const int32_t* rbp, int nb, int nchunks, int64_t rows_per_chunk, const float* G, int ldg,
                         const float* Y, int ldy, const float* S, int lds, const double* V, const double* A, int ldv,
                         int cs, const double* scale, int accumulate, float* grad, double* part, cudaStream_t st) {
  if (cs <= 0 || cs > 64) return cudaErrorInvalidValue;
  switch (dtype) {
    case 0:
      return sddmm_t<float>(indptr, idx, val, n, g, rbp, nb, nchunks, rows_per_chunk, G, ldg, Y, ldy, S, lds, V, A,
                            ldv, cs, scale, accumulate, grad, part, st);
    case 1:
      return sddmm_t<__nv_bfloat16>(indptr, idx, val, n, g, rbp, nb, nchunks, rows_per_chunk, G, ldg, Y, ldy, S, lds,
                                    V, A, ldv, cs, scale, accumulate, grad, part, st);
    default:
      return sddmm_t<__half>(indptr, idx, val, n, g, rbp, nb, nchunks, rows_per_chunk, G, ldg, Y, ldy, S, lds, V, A,
                             ldv, cs, scale, accumulate, grad, part, st);
  }
}

}  // namespace scx
