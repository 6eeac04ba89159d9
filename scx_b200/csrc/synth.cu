// Device generator of the synthetic negative-binomial cells x genes CSR used
// by the benchmark (no reference counterpart; the reference benchmarks on the
// census_1m atlas, which this stands in for with the same shape and value
// distribution).
//
//   mu_g ~ LogNormal(loc, 1.5)       s_c ~ LogNormal(0, 0.5)
//   x_cg ~ Poisson(Gamma(r, mu_g s_c / r)),  r = 1 / dispersion
//   value = log1p(1e4 * x_cg / rowsum_c)
//
// Every draw comes from Philox4x32-10 keyed by the seed, with the counter
// holding (cell, gene, stream, attempt), so the two passes (count, fill)
// regenerate identical counts without storing them.  Gamma: Marsaglia & Tsang
// (2000); Poisson: multiplication method below 12, PTRS (Hoermann 1993) above.
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "launch.h"

namespace scx {

namespace {

__device__ __forceinline__ void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
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

// Stream of uniforms in (0, 1) for one (a, b) coordinate of one stream.
struct Rng {
  uint32_t k0, k1, a, b, tag, block;
  uint32_t buf[4];
  int pos;
  __device__ Rng(uint64_t seed, uint32_t a_, uint32_t b_, uint32_t stream)
      : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), a(a_), b(b_), tag(stream << 24), block(0), pos(4) {}
  __device__ float uniform() {
    if (pos == 4) {
      buf[0] = a; buf[1] = b; buf[2] = tag | block; buf[3] = 0x5ca1ab1e;
      philox(buf, k0, k1);
      ++block;
      pos = 0;
    }
    uint32_t x = buf[pos++];
    return ((x >> 8) + 0.5f) * (1.0f / 16777216.0f);
  }
  __device__ float normal() {
    float u1 = uniform(), u2 = uniform();
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
  }
};

__device__ float gamma_draw(Rng& rng, float shape) {
  // shape >= 1 (dispersion <= 1)
  const float d = shape - 1.0f / 3.0f;
  const float c = rsqrtf(9.0f * d);
  for (int it = 0; it < 64; ++it) {
    float x = rng.normal();
    float v = 1.0f + c * x;
    if (v <= 0.0f) continue;
    v = v * v * v;
    float u = rng.uniform();
    if (logf(u) < 0.5f * x * x + d - d * v + d * logf(v)) return d * v;
  }
  return d;  // bounded: practically never reached (acceptance > 0.95)
}

__device__ int poisson_draw(Rng& rng, float lam) {
  if (lam <= 0.0f) return 0;
  if (lam < 12.0f) {
    const float L = expf(-lam);
    float p = 1.0f;
    int k = 0;
    for (int it = 0; it < 256; ++it) {
      p *= rng.uniform();
      if (p <= L) return k;
      ++k;
    }
    return k;
  }
  const float slam = sqrtf(lam), loglam = logf(lam);
  const float b = 0.931f + 2.53f * slam;
  const float a = -0.059f + 0.02483f * b;
  const float invalpha = 1.1239f + 1.1328f / (b - 3.4f);
  const float vr = 0.9277f - 3.6224f / (b - 2.0f);
  for (int it = 0; it < 256; ++it) {
    float U = rng.uniform() - 0.5f;
    float V = rng.uniform();
    float us = 0.5f - fabsf(U);
    float kf = floorf((2.0f * a / us + b) * U + lam + 0.43f);
    if (us >= 0.07f && V <= vr) return (int)kf;
    if (kf < 0.0f || (us < 0.013f && V > us)) continue;
    if (logf(V) + logf(invalpha) - logf(a / (us * us) + b) <= -lam + kf * loglam - lgammaf(kf + 1.0f))
      return (int)kf;
  }
  return (int)lam;
}

__device__ __forceinline__ int draw_count(uint64_t seed, int64_t cell, int64_t gene, float m,
                                          float shape) {
  Rng rng(seed, (uint32_t)cell, (uint32_t)((uint64_t)cell >> 32) ^ ((uint32_t)gene << 8), 3u);
  float lam = gamma_draw(rng, shape) * (m / shape);
  return poisson_draw(rng, lam);
}

__device__ __forceinline__ float size_factor(uint64_t seed, int64_t cell) {
  Rng rng(seed, (uint32_t)cell, (uint32_t)((uint64_t)cell >> 32), 2u);
  return expf(0.5f * rng.normal());
}

__global__ void k_gene_means(uint64_t seed, int64_t g, float loc, float* mu) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < g;
       j += (int64_t)gridDim.x * blockDim.x) {
    Rng rng(seed, (uint32_t)j, 0u, 1u);
    mu[j] = expf(loc + 1.5f * rng.normal());
  }
}

__global__ void k_count(uint64_t seed, int64_t n, int64_t g, float shape,
                        const float* __restrict__ mu, int64_t* __restrict__ row_nnz,
                        float* __restrict__ rowsum) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = warp; c < n; c += nwarps) {
    const float s = size_factor(seed, c);
    int cnt = 0;
    float sum = 0.f;
    for (int64_t j = lane; j < g; j += 32) {
      int x = draw_count(seed, c, j, s * __ldg(mu + j), shape);
      cnt += (x > 0);
      sum += (float)x;
    }
    for (int o = 16; o > 0; o >>= 1) {
      cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if (lane == 0) {
      row_nnz[c] = cnt;
      rowsum[c] = sum;
    }
  }
}

__global__ void k_fill(uint64_t seed, int64_t n, int64_t g, float shape,
                       const float* __restrict__ mu, const int64_t* __restrict__ indptr,
                       const float* __restrict__ rowsum, int32_t* __restrict__ idx,
                       float* __restrict__ val) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = warp; c < n; c += nwarps) {
    const float s = size_factor(seed, c);
    const float scale = 1e4f / fmaxf(rowsum[c], 1.0f);
    int64_t pos = indptr[c];
    for (int64_t j0 = 0; j0 < g; j0 += 32) {
      const int64_t j = j0 + lane;
      int x = 0;
      if (j < g) x = draw_count(seed, c, j, s * __ldg(mu + j), shape);
      const unsigned bal = __ballot_sync(0xffffffffu, x > 0);
      if (x > 0) {
        const int off = __popc(bal & ((1u << lane) - 1u));
        idx[pos + off] = (int32_t)j;
        val[pos + off] = log1pf((float)x * scale);
      }
      pos += __popc(bal);
    }
  }
}

}  // namespace

cudaError_t launch_synth_gene_means(uint64_t seed, int64_t g, double loc, float* mu_g,
                                    cudaStream_t st) {
  note_launches(1);
  k_gene_means<<<(int)((g + 255) / 256), 256, 0, st>>>(seed, g, (float)loc, mu_g);
  return cudaGetLastError();
}

cudaError_t launch_synth_count(uint64_t seed, int64_t n, int64_t g, double loc, double disp,
                               const float* mu_g, int64_t* row_nnz, float* rowsum,
                               cudaStream_t st, int num_sms) {
  (void)loc;
  note_launches(1);
  k_count<<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(seed, n, g, (float)(1.0 / disp), mu_g,
                                                            row_nnz, rowsum);
  return cudaGetLastError();
}

cudaError_t launch_synth_fill(uint64_t seed, int64_t n, int64_t g, double loc, double disp,
                              const float* mu_g, const int64_t* indptr, const float* rowsum,
                              int32_t* idx, float* val, cudaStream_t st, int num_sms) {
  (void)loc;
  note_launches(1);
  k_fill<<<grid_for(n * 32, 256, num_sms, 8), 256, 0, st>>>(seed, n, g, (float)(1.0 / disp), mu_g,
                                                           indptr, rowsum, idx, val);
  return cudaGetLastError();
}

// Exclusive prefix sum of n int64 counts into out[0..n] (out[n] = total).
cudaError_t launch_exclusive_scan_i64(const int64_t* in, int64_t n, int64_t* out, cudaStream_t st) {
  cudaError_t err = cudaMemsetAsync(out, 0, sizeof(int64_t), st);
  if (err != cudaSuccess || n == 0) return err;
  size_t temp = 0;
  err = cub::DeviceScan::InclusiveSum(nullptr, temp, in, out + 1, n, st);
  if (err != cudaSuccess) return err;
  void* d_temp = nullptr;
  err = cudaMallocAsync(&d_temp, temp, st);
  if (err != cudaSuccess) return err;
  err = cub::DeviceScan::InclusiveSum(d_temp, temp, in, out + 1, n, st);
  cudaFreeAsync(d_temp, st);
  return err;
}

}  // namespace scx
