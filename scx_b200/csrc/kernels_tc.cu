// Tensor-core SpMM for the mixed-precision path (BF16/FP16 values, FP32
// accumulation in TMEM), sm_100a.
//
// Sparse format ("tile-chunk packed"), built once per plan:
//   rows are grouped in tiles of 128 cells, genes in chunks of 64; the stored
//   entries of tile t and chunk c form one segment, ordered by row then gene,
//   padded with zero words to a multiple of 4 entries (16 bytes), so every
//   segment starts on a 16-byte boundary.  Each entry is one 32-bit word:
//       bits  0..15  value (bf16 or f16 bits)
//       bits 16..29  byte offset of (row within the tile, gene within the
//                    chunk) in the 128 x 64 swizzled tile (sw128_offset)
//   meta[t * n_chunks + c] (16 bytes) = {segment start, q[0..2], q[3]}: q[w] is
//   the number of entries in rows < 32 (w + 1), so densify warp w handles
//   entries [q[w-1], q[w]) and q[3] is the segment's real entry count.
//   4 bytes per stored entry instead of 6 (bf16 value + int32 index).
//
// Both products densify a segment into a 128 x 64 16-bit shared-memory tile
// (128-byte swizzle, see tc.cuh) and run tcgen05.mma on it.  The dense
// operand enters as its 16-bit image: column 2 j holds hi = round(x_j),
// column 2 j + 1 holds lo = round(x_j - hi), so one MMA multiplies both
// halves and the epilogue adds each (hi, lo) pair of accumulator columns:
// about 16 mantissa bits on the dense operand, the matrix values being the
// only operand rounded to 16 bits.
//
// At ld 64 (k_fwd_swap, k_rmat_swap) the image is the MMA's A operand
// (M = 128 image columns, MN-major) and the densified tiles are its B:
//   forward    Y^T(128 x 256 cells) += Vimg_c^T [A_(t0,c) | A_(t1,c)]^T
//   transposed Z^T(128 x 256 genes) += Qimg_t^T [A_(t,4q) | ... | A_(t,4q+3)]
// A tcgen05.mma at M = 128 costs about the same to issue whatever its N, so
// spanning two row tiles (forward) or four gene chunks (transposed) in
// N = 256 halves the instructions per segment against N = 128.  At ld 128
// (k_fwd_tc, k_rmat_tc) the image is the B operand (N = 256) and the tiles
// the A:
//   forward    Y(128 cells x 256) += A(cells x 64 genes, K-major) Vimg_c
//   transposed Z(128 genes x 256) += A^T(genes x cells, MN-major) Qimg_t
//
// Warp roles (23 warps): warps 0-15 densify in four groups of four; warps
// 16-19 drain TMEM (one lane quarter each); warp 20 issues the MMAs from one
// thread; warp 21 loads the dense operand by TMA; warp 22 copies segment
// metadata per tile (or band of two tiles) and prefetches their entries into
// L2.  Each densify warp reads its quarter of a segment straight from global
// memory with 16-byte loads, keeping the loads of its group's next segment
// in flight in registers while the current one is scattered, so many warps
// -- not one issuing thread -- keep the entry stream moving.  All waits are
// bounded (tc.cuh).
#include <algorithm>

#include "common.cuh"
#include "launch.h"
#include "tc.cuh"

namespace scx {

using namespace tc;

namespace {

constexpr int TM = 128;          // cells per tile
constexpr int CW = 64;           // genes per chunk
constexpr int kGroups = 4;       // densify groups of four warps
constexpr int kThreads = 736;    // 23 warps
constexpr int kMaxChunks = 128;  // genes <= 8192
constexpr int W_EPI = 4 * kGroups, W_MMA = W_EPI + 4, W_DENSE = W_MMA + 1, W_META = W_MMA + 2;

struct SegMeta {
  int64_t start;
  uint16_t q[4];
};
static_assert(sizeof(SegMeta) == 16, "segment metadata is one 16-byte record");

// Pipeline shapes of the ld-128 kernels (k_fwd_tc, k_rmat_tc; ld 64 has its
// own, next to k_fwd_swap / k_rmat_swap).  In the forward kernel densify group
// g takes the stages it with it % G == g and owns A stage buffers g and g + G
// (S == 2 G), so it densifies its next segment while the MMAs read the
// previous one.  In the transposed kernel a stage (two 64-gene sub-tiles) is
// filled by a pair of groups, one sub-tile each; pair p takes the stages it
// with it % 2 == p.  Either way each waiter runs at most one barrier phase
// ahead of the phase it waits for, which is what a parity wait can
// distinguish.  The forward kernel's dense operand has its own ring of
// fwd_bslots(LD) chunk buffers, filled ahead of the MMAs.
__host__ __device__ constexpr int fwd_stages(int LD) { return 2 * kGroups; }
__host__ __device__ constexpr int fwd_bslots(int LD) { return 2; }
__host__ __device__ constexpr int rmat_stages(int LD) { return 2; }
// 16-byte entry words a densify lane keeps in flight per segment quarter
// (x 128 entries per warp); a larger quarter loads the rest on demand.
constexpr int kFwdRegs = 4;
constexpr int kRmatRegs = 4;

__host__ __device__ __forceinline__ int padded4(int x) { return (x + 3) & ~3; }

// ---------------------------------------------------------------------------
// format build
// ---------------------------------------------------------------------------
__global__ void k_tile_count(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                             int64_t n, int64_t n_tiles, int nc, int64_t* __restrict__ counts) {
  extern __shared__ int cnt[];
  for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    for (int c = threadIdx.x; c < nc; c += blockDim.x) cnt[c] = 0;
    __syncthreads();
    const int64_t r0 = t * TM, r1 = min(n, r0 + TM);
    for (int64_t p = indptr[r0] + threadIdx.x; p < indptr[r1]; p += blockDim.x)
      atomicAdd(&cnt[__ldg(idx + p) >> 6], 1);
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += blockDim.x) counts[t * nc + c] = padded4(cnt[c]);
    __syncthreads();
  }
}

__global__ void k_tile_fill(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                            const uint16_t* __restrict__ val, int64_t n, int64_t n_tiles, int nc,
                            const int64_t* __restrict__ seg, uint32_t* __restrict__ ent,
                            SegMeta* __restrict__ meta) {
  extern __shared__ int sm[];
  int* colpre = sm;            // [TM][nc]: entries of chunk c in rows before r
  int* rowpre = sm + TM * nc;  // [TM][nc]: entries of row r in chunks before c
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    for (int i = threadIdx.x; i < TM * nc; i += blockDim.x) colpre[i] = 0;
    __syncthreads();
    const int64_t r0 = t * TM;
    const int rows = (int)min((int64_t)TM, n - r0);
    for (int r = warp; r < rows; r += nw)
      for (int64_t p = indptr[r0 + r] + lane; p < indptr[r0 + r + 1]; p += 32)
        atomicAdd(&colpre[r * nc + (__ldg(idx + p) >> 6)], 1);
    __syncthreads();
    for (int r = threadIdx.x; r < TM; r += blockDim.x) {
      int run = 0;
      for (int c = 0; c < nc; ++c) {
        rowpre[r * nc + c] = run;
        run += colpre[r * nc + c];
      }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
      SegMeta m;
      m.start = seg[t * nc + c];
      int run = 0;
      for (int r = 0; r < TM; ++r) {
        const int v = colpre[r * nc + c];
        colpre[r * nc + c] = run;
        run += v;
        if (r == 31 || r == 63 || r == 95) m.q[r >> 5] = (uint16_t)run;
      }
      m.q[3] = (uint16_t)run;
      meta[t * nc + c] = m;
    }
    __syncthreads();
    for (int r = warp; r < rows; r += nw) {
      const int64_t s = indptr[r0 + r];
      for (int64_t p = s + lane; p < indptr[r0 + r + 1]; p += 32) {
        const int32_t j = __ldg(idx + p);
        const int c = j >> 6;
        const int64_t dst = seg[t * nc + c] + colpre[r * nc + c] + ((p - s) - rowpre[r * nc + c]);
        ent[dst] = (uint32_t)val[p] | (sw128_offset((uint32_t)r, (uint32_t)(j & 63)) << 16);
      }
    }
    __syncthreads();
  }
}


// ---------------------------------------------------------------------------
// shared pieces of the two product kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

__device__ __forceinline__ void sts_u16(uint32_t addr, uint32_t v) {
  asm volatile("st.shared.u16 [%0], %1;" ::"r"(addr), "h"((unsigned short)v) : "memory");
}
__device__ __forceinline__ void sts_zero16(uint32_t addr) {
  asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(addr), "r"(0u) : "memory");
}
// 16 bytes of entries, read-only path (the packed matrix never changes during a launch).
__device__ __forceinline__ uint4 ldg_entries(const uint32_t* p) {
  uint4 v;
  asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// Two floats as a pair of 16-bit values (fmt 1 = bf16, 0 = f16), low word first.
__device__ __forceinline__ uint32_t pack16x2(float a, float b, int fmt) {
  if (fmt) {
    __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&p);
  }
  __half2 p = __floats2half2_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&p);
}
__device__ __forceinline__ float unpack16(uint32_t bits, int fmt) {
  if (fmt) return __bfloat162float(__ushort_as_bfloat16((unsigned short)bits));
  return __half2float(__ushort_as_half((unsigned short)bits));
}
// The (hi, lo) pair of x as one word, hi in the low half: hi = round16(x),
// lo = round16(x - hi) -- two adjacent columns of the 16-bit image.
__device__ __forceinline__ uint32_t hilo16(float x, int fmt) {
  const uint32_t h = pack16x2(x, 0.f, fmt) & 0xFFFFu;
  const uint32_t l = pack16x2(x - unpack16(h, fmt), 0.f, fmt) & 0xFFFFu;
  return h | (l << 16);
}

// Zero rows 32q .. 32q+31 of a 128 x 64 16-bit swizzled tile, lane = row.
// Iteration i writes physical chunk i ^ (row % 8): the 32 lanes of one store
// cover all eight 16-byte bank groups, so every store is conflict-free.
__device__ __forceinline__ void zero_rows(uint32_t tile, int quarter, int lane) {
  const uint32_t row = 32u * quarter + lane;
  const uint32_t base = tile + (row >> 3) * 1024u + (row & 7u) * 128u;
#pragma unroll
  for (uint32_t i = 0; i < 8; ++i) sts_zero16(base + ((i ^ (row & 7u)) << 4));
}

__device__ __forceinline__ void scatter_one(uint32_t tile, uint32_t w) { sts_u16(tile + (w >> 16), w & 0xFFFFu); }

// Entries [lo, hi) of quarter q of segment m (indices into the entry array).
struct Span {
  int64_t lo, hi;
};
// `m` lives in shared memory (the metadata ring): one 16-byte load, then
// warp-uniform selects (q is the warp's quarter).
__device__ __forceinline__ Span quarter_span(const SegMeta& m, int q) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(smem_u32(&m)));
  const int64_t start = (int64_t)(((uint64_t)v.y << 32) | v.x);
  const uint32_t q0 = v.z & 0xFFFFu, q1 = v.z >> 16, q2 = v.w & 0xFFFFu, q3 = v.w >> 16;
  const uint32_t hi = q == 0 ? q0 : q == 1 ? q1 : q == 2 ? q2 : q3;
  const uint32_t lo = q == 0 ? 0u : q == 1 ? q0 : q == 2 ? q1 : q2;
  return Span{start + (int64_t)lo, start + (int64_t)hi};
}

// Issue the first R 16-byte loads of a span (its start rounded down to a
// 16-byte boundary; segments start on one and are padded to one, so a load
// never leaves its segment).  Lane L holds words 4 (L + 32 r) .. + 3.
template <int R>
__device__ __forceinline__ void span_load(const uint32_t* __restrict__ ent, Span sp, int lane, uint4 (&w)[R]) {
  const int64_t a0 = sp.lo & ~int64_t(3);
  const int phi = (int)(sp.hi - a0);
  const uint32_t* base = ent + a0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int p = 4 * (lane + 32 * r);
    w[r] = p < phi ? ldg_entries(base + p) : make_uint4(0u, 0u, 0u, 0u);
  }
}

// The four words at span positions p .. p + 3 (counted from the span's 16-byte
// aligned start); those outside [plo, phi) belong to the neighbouring spans.
// With d = p - plo and n = phi - plo, word k is in the span iff
// (unsigned)(d + k) < n: one 32-bit compare per word.
__device__ __forceinline__ void scatter4(uint32_t tile, const uint4& w, int d, unsigned n) {
  if ((unsigned)d < n) scatter_one(tile, w.x);
  if ((unsigned)(d + 1) < n) scatter_one(tile, w.y);
  if ((unsigned)(d + 2) < n) scatter_one(tile, w.z);
  if ((unsigned)(d + 3) < n) scatter_one(tile, w.w);
}

// Scatter a span into `tile` (already zeroed): the R words in flight first,
// then whatever lies beyond them, loaded here.
template <int R>
__device__ __forceinline__ void span_scatter(uint32_t tile, const uint32_t* __restrict__ ent, Span sp, int lane,
                                             const uint4 (&w)[R]) {
  const int64_t a0 = sp.lo & ~int64_t(3);
  const int plo = (int)(sp.lo - a0), phi = (int)(sp.hi - a0);  // a quarter holds at most 2,048 entries
  const unsigned n = (unsigned)(phi - plo);
#pragma unroll
  for (int r = 0; r < R; ++r) scatter4(tile, w[r], 4 * (lane + 32 * r) - plo, n);
  for (int p = 4 * (lane + 32 * R); p < phi; p += 128) scatter4(tile, ldg_entries(ent + a0 + p), p - plo, n);
}

// Meta loader: L2 prefetch of the entries of segments [c0, c1) of one tile
// (metadata `mt`), so the densify warps' loads a tile later find them in L2.
__device__ __forceinline__ void prefetch_segments(const uint32_t* __restrict__ ent, const SegMeta* mt, int c0,
                                                  int c1) {
  const int64_t b = mt[c0].start;
  const int64_t e = mt[c1 - 1].start + padded4(mt[c1 - 1].q[3]);
  for (int64_t p = b; p < e; p += 8192) bulk_prefetch_l2(ent + p, (uint32_t)(min((int64_t)8192, e - p) * 4));
}

// Meta loader: `records` metadata records from `src` into slot mi & 1 of a
// two-slot ring of `slot_records` records per slot.
__device__ __forceinline__ bool load_meta(const SegMeta* __restrict__ src, int records, SegMeta* mring,
                                          int slot_records, uint64_t* mfull, uint64_t* mempty, uint32_t mi,
                                          volatile int* abort_flag, int* err, int code) {
  const int ms = mi & 1u;
  if (!mbar_wait(&mempty[ms], ((mi >> 1) & 1u) ^ 1u, abort_flag, err, code)) return false;
  const uint32_t bytes = (uint32_t)records * 16u;
  mbar_arrive_expect_tx(&mfull[ms], bytes);
  bulk_load(mring + (size_t)ms * slot_records, src, bytes, &mfull[ms]);
  return true;
}

// ---------------------------------------------------------------------------
// forward: Y[tile rows, :LD] = A_tile (Vhi + Vlo) - mc   (persistent over tiles)
// ---------------------------------------------------------------------------
template <int LD>
__global__ void __launch_bounds__(kThreads, 1)
    k_fwd_tc(const uint32_t* __restrict__ ent, const SegMeta* __restrict__ meta, int64_t n_tiles, int nc,
             int64_t n, const __grid_constant__ CUtensorMap vmap, const float* __restrict__ mc,
             float* __restrict__ Y, uint16_t* __restrict__ Yimg, int fmt, int* err) {
  constexpr int N2 = 2 * LD;                // [hi | lo] columns
  constexpr int S = fwd_stages(LD);         // A stages, two per densify group
  constexpr int G = kGroups;
  constexpr int NB = fwd_bslots(LD);        // dense-operand ring
  constexpr int A_BYTES = TM * CW * 2;      // 16 KB
  constexpr int B_BYTES = CW * N2 * 2;      // 64 genes x N2 image columns
  static_assert(S == 2 * G, "two A stages per densify group");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* As = smem;
  uint8_t* Bs = As + S * A_BYTES;
  SegMeta* mring = reinterpret_cast<SegMeta*>(Bs + NB * B_BYTES);  // [2][kMaxChunks]
  uint64_t* bars = reinterpret_cast<uint64_t*>(mring + 2 * kMaxChunks);
  uint64_t* full = bars;            // [S]  A stage densified (4 warp arrivals)
  uint64_t* empty = full + S;       // [S]  A stage consumed (MMA commit)
  uint64_t* bfull = empty + S;      // [NB] dense chunk landed (TMA)
  uint64_t* bempty = bfull + NB;    // [NB] dense chunk consumed (MMA commit)
  uint64_t* acc_full = bempty + NB;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* mfull = acc_empty + 2;
  uint64_t* mempty = mfull + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 4);  // one arrival per warp of the stage's densify group
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < NB; ++b) {
      mbar_init(&bfull[b], 1);
      mbar_init(&bempty[b], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 4);  // one arrival per epilogue warp
      mbar_init(&mfull[a], 1);
      mbar_init(&mempty[a], 4 * kGroups);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == W_MMA) {
    tmem_alloc(tmem_slot, 2 * N2);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < W_EPI) {
    // ---- densify: group (warp / 4) takes stages it % G == group ----
    const int group = warp >> 2, q = warp & 3;
    uint32_t it = 0, ti = 0;
    uint4 w[kFwdRegs];
    Span pre{-1, -1};  // span whose loads are in flight in w
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x, ++ti) {
      if (!warp_wait(&mfull[ti & 1u], (ti >> 1) & 1u, abort_flag, err, 11)) goto done;
      const SegMeta* mt = mring + (ti & 1u) * kMaxChunks;
      for (int c = 0; c < nc; ++c, ++it) {
        if ((int)(it % G) != group) continue;
        const Span sp = quarter_span(mt[c], q);
        if (sp.lo != pre.lo || sp.hi != pre.hi) span_load<kFwdRegs>(ent, sp, lane, w);
        const int s = it % S;
        if (!warp_wait(&empty[s], ((it / S) & 1u) ^ 1u, abort_flag, err, 12)) goto done;
        const uint32_t tile = smem_u32(As + s * A_BYTES);
        zero_rows(tile, q, lane);
        __syncwarp();
        span_scatter<kFwdRegs>(tile, ent, sp, lane, w);
        // put the group's next segment in flight: chunk c + G of this tile, or
        // of the next tile once its metadata is in
        pre = Span{-1, -1};
        const int cn = c + G;
        if (cn < nc) {
          pre = quarter_span(mt[cn], q);
        } else if (cn - nc < nc && t + gridDim.x < n_tiles) {
          if (!warp_wait(&mfull[(ti + 1) & 1u], ((ti + 1) >> 1) & 1u, abort_flag, err, 11)) goto done;
          pre = quarter_span(mring[((ti + 1) & 1u) * kMaxChunks + (cn - nc)], q);
        }
        if (pre.lo >= 0) span_load<kFwdRegs>(ent, pre, lane, w);
        // every lane's shared stores -> async proxy, then one arrival per warp
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&full[s]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&mempty[ti & 1u]);
    }
  } else if (warp < W_MMA) {
    // ---- epilogue: TMEM (hi, lo) column pairs -> Y (FP32) and its 16-bit image ----
    const int q = warp & 3;
    const uint32_t row = 32u * q + lane;
    uint32_t k = 0;
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x, ++k) {
      const uint32_t a = k & 1u, ph = (k >> 1) & 1u;
      if (!warp_wait(&acc_full[a], ph, abort_flag, err, 14)) goto done;
      tc_fence_after();
      const uint32_t tbase = tmem + ((32u * q) << 16) + a * N2;
      const int64_t grow = t * TM + row;
#pragma unroll 1
      for (int cb = 0; cb < N2 / 16; ++cb) {  // 16 image columns = 8 output columns
        uint32_t r[16];
        tmem_ld16(tbase + cb * 16, r);
        tmem_wait_ld();
        if (grow < n) {
          float o[8];
          uint32_t w[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            o[i] = __uint_as_float(r[2 * i]) + __uint_as_float(r[2 * i + 1]) - __ldg(mc + cb * 8 + i);
            w[i] = hilo16(o[i], fmt);
          }
          if (Y) {  // the FP32 copy only when the caller reads it
            float4* yr = reinterpret_cast<float4*>(Y + grow * LD + cb * 8);
            yr[0] = make_float4(o[0], o[1], o[2], o[3]);
            yr[1] = make_float4(o[4], o[5], o[6], o[7]);
          }
          uint4* ir = reinterpret_cast<uint4*>(Yimg + grow * N2 + cb * 16);
          ir[0] = make_uint4(w[0], w[1], w[2], w[3]);
          ir[1] = make_uint4(w[4], w[5], w[6], w[7]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[a]);
    }
  } else if (warp == W_MMA) {
    // ---- MMA issuer ----
    if (lane == 0) {
      // The issue loop is the pipeline's critical path: descriptors are
      // formed once and advanced by constant offsets (their address field is
      // in 16-byte units; shared addresses stay below 256 KB, so no carry).
      const uint32_t idesc = idesc_f16(128, N2, fmt, 0, 1);
      const uint64_t adesc0 = sdesc_sw128(smem_u32(As), 16, 1024);
      const uint64_t bdesc0 = sdesc_sw128(smem_u32(Bs), CW * 128, 1024);
      static_assert((S & (S - 1)) == 0 && (NB & (NB - 1)) == 0, "power-of-two rings");
      uint32_t it = 0, k = 0;
      for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x, ++k) {
        const uint32_t a = k & 1u, ph = (k >> 1) & 1u;
        if (!mbar_wait(&acc_empty[a], ph ^ 1u, abort_flag, err, 15)) break;
        tc_fence_after();
        const uint32_t d = tmem + a * N2;
        bool ok = true;
        for (int c = 0; c < nc; ++c, ++it) {
          const int s = it % S, b = it % NB;
          if (!mbar_wait(&bfull[b], (it / NB) & 1u, abort_flag, err, 16) ||
              !mbar_wait(&full[s], (it / S) & 1u, abort_flag, err, 16)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ad = adesc0 + (uint64_t)(s * (A_BYTES >> 4));
          const uint64_t bd = bdesc0 + (uint64_t)(b * (B_BYTES >> 4));
          umma_f16(d, ad, bd, idesc, c != 0);
#pragma unroll
          for (int kk = 1; kk < CW / 16; ++kk)  // K steps: +32 B along A's rows, +2 KB down B
            umma_f16(d, ad + 2 * kk, bd + 128 * kk, idesc, 1u);
          umma_commit(&empty[s]);
          umma_commit(&bempty[b]);
        }
        if (!ok) break;
        umma_commit(&acc_full[a]);
      }
    }
    __syncwarp();
  } else if (warp == W_DENSE) {
    // ---- dense loader: [Vhi | Vlo] chunks into the B ring, up to NB ahead ----
    if (lane == 0) {
      uint32_t it = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        for (int c = 0; c < nc; ++c, ++it) {
          const int b = it % NB;
          if (!mbar_wait(&bempty[b], ((it / NB) & 1u) ^ 1u, abort_flag, err, 19)) {
            ok = false;
            break;
          }
          uint8_t* bb = Bs + b * B_BYTES;
          mbar_arrive_expect_tx(&bfull[b], B_BYTES);
#pragma unroll
          for (int h = 0; h < N2 / 64; ++h) tma_load_2d(bb + h * (CW * 128), &vmap, &bfull[b], 64 * h, CW * c);
        }
      }
    }
    __syncwarp();
  } else if (warp == W_META) {
    // ---- meta loader: tile metadata, and the tile's entries into L2 ----
    if (lane == 0) {
      uint32_t ti = 0;
      for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x, ++ti) {
        if (!load_meta(meta + t * nc, nc, mring, kMaxChunks, mfull, mempty, ti, abort_flag, err, 17)) break;
        if (!mbar_wait(&mfull[ti & 1u], (ti >> 1) & 1u, abort_flag, err, 18)) break;
        prefetch_segments(ent, mring + (ti & 1u) * kMaxChunks, 0, nc);
      }
    }
    __syncwarp();
  }
done:
  // After an abort, give MMAs and copies already issued time to land
  // (microseconds of work) before the block frees TMEM and shared memory.
  if (*abort_flag) __nanosleep(500000);
  tc_fence_before();
  __syncthreads();
  if (warp == W_MMA) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * N2);
  }
}

// ---------------------------------------------------------------------------
// transposed: part[row group][genes of this CTA, :LD] = sum over its tiles of
// A_tile^T (Qhi_tile + Qlo_tile).  grid = G gene groups x R row groups; one
// CTA per SM (the accumulators fill TMEM).
// ---------------------------------------------------------------------------
template <int LD>
__global__ void __launch_bounds__(kThreads, 1)
    k_rmat_tc(const uint32_t* __restrict__ ent, const SegMeta* __restrict__ meta, int64_t n_tiles, int nc,
              int64_t g, int n_gene_groups, const __grid_constant__ CUtensorMap qmap, float* __restrict__ part,
              int fmt, int* err) {
  constexpr int N2 = 2 * LD;
  constexpr int S = rmat_stages(LD);     // A stages, one per pair of densify groups
  constexpr int SUB = TM * CW * 2;       // one 64-gene sub-tile, 16 KB
  constexpr int A_BYTES = 2 * SUB;       // 128 genes
  constexpr int Q_BYTES = TM * N2 * 2;   // 128 cells x N2 image columns
  constexpr int SPG = 512 / N2;          // 128-gene super-chunks per CTA (TMEM columns)
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* As = smem;
  uint8_t* Qs = As + S * A_BYTES;  // [2 buffers][hi, lo]
  SegMeta* mring = reinterpret_cast<SegMeta*>(Qs + 2 * Q_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(mring + 2 * kMaxChunks);
  uint64_t* full = bars;
  uint64_t* empty = full + S;
  uint64_t* qfull = empty + S;
  uint64_t* qempty = qfull + 2;
  uint64_t* mfull = qempty + 2;
  uint64_t* mempty = mfull + 2;
  uint64_t* done_bar = mempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gg = blockIdx.x % n_gene_groups;
  const int rg = blockIdx.x / n_gene_groups;
  const int R = gridDim.x / n_gene_groups;
  const int64_t t0 = (int64_t)rg * n_tiles / R, t1 = (int64_t)(rg + 1) * n_tiles / R;
  const int n_super = (nc + 1) / 2;
  const int sc0 = gg * SPG, sc1 = min(n_super, sc0 + SPG);
  const int nsc = max(0, sc1 - sc0);
  const bool have_work = (t1 > t0) && nsc > 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 8);  // one arrival per warp of the stage's two densify groups
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&qfull[b], 1);
      mbar_init(&qempty[b], 1);
      mbar_init(&mfull[b], 1);
      mbar_init(&mempty[b], 4 * kGroups);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == W_MMA) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < W_EPI) {
    // ---- densify: a stage (128-gene super-chunk) is split over a pair of
    // groups, one 64-gene sub-tile each: group g fills sub-tile g & 1 of the
    // stages it with it % 2 == g >> 1, so each pair owns every other stage
    // buffer and has its next stage in hand while the MMAs read this one ----
    const int group = warp >> 2, q = warp & 3;
    const int h = group & 1, pg = group >> 1;
    uint32_t it = 0, ti = 0;
    uint4 w[kRmatRegs];
    Span pre{-1, -1};  // span whose loads are in flight in w
    if (have_work)
      for (int64_t t = t0; t < t1; ++t, ++ti) {
        if (!warp_wait(&mfull[ti & 1u], (ti >> 1) & 1u, abort_flag, err, 21)) goto done;
        const SegMeta* mt = mring + (ti & 1u) * kMaxChunks;
        for (int sc = sc0; sc < sc1; ++sc, ++it) {
          if ((int)(it & 1u) != pg) continue;
          const int ch = 2 * sc + h;
          const Span sp = ch < nc ? quarter_span(mt[ch], q) : Span{0, 0};
          if (sp.lo != pre.lo || sp.hi != pre.hi) span_load<kRmatRegs>(ent, sp, lane, w);
          const int s = it % S;
          if (!warp_wait(&empty[s], ((it / S) & 1u) ^ 1u, abort_flag, err, 22)) goto done;
          const uint32_t tile = smem_u32(As + s * A_BYTES) + h * SUB;
          zero_rows(tile, q, lane);
          __syncwarp();
          span_scatter<kRmatRegs>(tile, ent, sp, lane, w);
          // the pair's next stage: super-chunk sc + 2 of this tile, or of the next
          pre = Span{-1, -1};
          const int scn = sc + 2;
          const SegMeta* mn = nullptr;
          int scx = 0;
          if (scn < sc1) {
            mn = mt;
            scx = scn;
          } else if (scn - nsc < sc1 && t + 1 < t1) {
            if (!warp_wait(&mfull[(ti + 1) & 1u], ((ti + 1) >> 1) & 1u, abort_flag, err, 21)) goto done;
            mn = mring + ((ti + 1) & 1u) * kMaxChunks;
            scx = scn - nsc;
          }
          if (mn && 2 * scx + h < nc) {
            pre = quarter_span(mn[2 * scx + h], q);
            span_load<kRmatRegs>(ent, pre, lane, w);
          }
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(&full[s]);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&mempty[ti & 1u]);
      }
  } else if (warp < W_MMA) {
    // ---- epilogue: accumulators (hi + lo halves) -> partials ----
    const int q = warp & 3;
    const uint32_t row = 32u * q + lane;
    if (have_work && !warp_wait(done_bar, 0, abort_flag, err, 24)) goto done;
    tc_fence_after();
    for (int j = 0; j < nsc; ++j) {
      const int64_t gene = (int64_t)(sc0 + j) * 128 + row;
      const uint32_t tbase = tmem + ((32u * q) << 16) + j * N2;
#pragma unroll 1
      for (int cb = 0; cb < N2 / 16; ++cb) {  // 16 image columns = 8 output columns
        uint32_t r[16];
        if (have_work) {
          tmem_ld16(tbase + cb * 16, r);
          tmem_wait_ld();
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) r[i] = 0u;
        }
        if (gene < g) {
          float4* out = reinterpret_cast<float4*>(part + ((int64_t)rg * g + gene) * LD + cb * 8);
#pragma unroll
          for (int i = 0; i < 2; ++i)
            out[i] = make_float4(__uint_as_float(r[8 * i]) + __uint_as_float(r[8 * i + 1]),
                                 __uint_as_float(r[8 * i + 2]) + __uint_as_float(r[8 * i + 3]),
                                 __uint_as_float(r[8 * i + 4]) + __uint_as_float(r[8 * i + 5]),
                                 __uint_as_float(r[8 * i + 6]) + __uint_as_float(r[8 * i + 7]));
        }
      }
    }
  } else if (warp == W_MMA) {
    // ---- MMA issuer ----
    if (lane == 0 && have_work) {
      // descriptors formed once and advanced by constant offsets (see k_fwd_tc)
      const uint32_t idesc = idesc_f16(128, N2, fmt, 1, 1);
      const uint64_t adesc0 = sdesc_sw128(smem_u32(As), SUB, 1024);
      const uint64_t qdesc0 = sdesc_sw128(smem_u32(Qs), TM * 128, 1024);
      uint32_t it = 0, ti = 0;
      bool ok = true;
      for (int64_t t = t0; t < t1 && ok; ++t, ++ti) {
        const uint32_t b = ti & 1u;
        if (!mbar_wait(&qfull[b], (ti >> 1) & 1u, abort_flag, err, 25)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t qd = qdesc0 + (uint64_t)(b * (Q_BYTES >> 4));
        for (int sc = sc0; sc < sc1; ++sc, ++it) {
          const int s = it % S;
          if (!mbar_wait(&full[s], (it / S) & 1u, abort_flag, err, 26)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ad = adesc0 + (uint64_t)(s * (A_BYTES >> 4));
          const uint32_t d = tmem + (sc - sc0) * N2;
          umma_f16(d, ad, qd, idesc, ti != 0);
#pragma unroll
          for (int kk = 1; kk < TM / 16; ++kk)  // K steps of 16 cells: +2 KB down both operands
            umma_f16(d, ad + 128 * kk, qd + 128 * kk, idesc, 1u);
          umma_commit(&empty[s]);
        }
        if (!ok) break;
        umma_commit(&qempty[b]);
      }
      if (ok) umma_commit(done_bar);
    }
    __syncwarp();
  } else if (warp == W_DENSE) {
    // ---- dense loader: [Qhi | Qlo] tiles, double-buffered per row tile ----
    if (lane == 0 && have_work) {
      uint32_t ti = 0;
      for (int64_t t = t0; t < t1; ++t, ++ti) {
        const uint32_t b = ti & 1u;
        if (!mbar_wait(&qempty[b], ((ti >> 1) & 1u) ^ 1u, abort_flag, err, 28)) break;
        uint8_t* qb = Qs + b * Q_BYTES;
        mbar_arrive_expect_tx(&qfull[b], Q_BYTES);
#pragma unroll
        for (int h = 0; h < N2 / 64; ++h) tma_load_2d(qb + h * (TM * 128), &qmap, &qfull[b], 64 * h, (int)(t * TM));
      }
    }
    __syncwarp();
  } else if (warp == W_META) {
    // ---- meta loader: tile metadata, and this gene group's entries of the tile into L2 ----
    if (lane == 0 && have_work) {
      uint32_t ti = 0;
      for (int64_t t = t0; t < t1; ++t, ++ti) {
        if (!load_meta(meta + t * nc, nc, mring, kMaxChunks, mfull, mempty, ti, abort_flag, err, 27)) break;
        if (!mbar_wait(&mfull[ti & 1u], (ti >> 1) & 1u, abort_flag, err, 29)) break;
        prefetch_segments(ent, mring + (ti & 1u) * kMaxChunks, 2 * sc0, min(nc, 2 * sc1));
      }
    }
    __syncwarp();
  }
done:
  if (*abort_flag) __nanosleep(500000);
  tc_fence_before();
  __syncthreads();
  if (warp == W_MMA) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------------------
// Tall Gram on tensor cores (ld = 64): for the rows of this CTA, with I the
// 16-bit image of Y (128 columns, (hi, lo) of column j at 2 j and 2 j + 1),
//   D  = I^T I   (128 x 128, FP32 in TMEM)  -> G = hh + hl + lh + ll
//   Ds = I^T 1   (128 x 64)                 -> column sums of h + l
// (TMA, 4-stage ring).  One MMA per 16 rows
// for each; the per-CTA partial is written in FP64 as [G (64 x 64), colsum
// (64)], the layout the fixed-order reduction expects.
// ---------------------------------------------------------------------------
constexpr int kGramStages = 4;

// One CTA's work: the row tiles [t0, t1) of one image, into the partial at `out`.
struct GramJob {
  const CUtensorMap* qmap;
  double* out;
  int* err;
  int64_t t0, t1;
};

template <bool kGlobalMaps>
__device__ __forceinline__ void gram_tc_body(const GramJob& job, int fmt) {
  constexpr int LD = 64;
  constexpr int PLANE = TM * LD * 2;  // 64 image columns of 128 rows, 16 KB
  constexpr int TILE = 2 * PLANE;     // the 128 image columns of a row tile
  constexpr int S = kGramStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* tiles = smem;
  uint8_t* ones = tiles + S * TILE;  // 128 rows x 64 ones, 16 KB
  float* pbuf = reinterpret_cast<float*>(ones + PLANE);  // [128][64] partial sums for the epilogue
  uint64_t* bars = reinterpret_cast<uint64_t*>(pbuf + TM * LD);
  uint64_t* full = bars;
  uint64_t* empty = full + S;
  uint64_t* done_bar = empty + S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t0 = job.t0, t1 = job.t1;
  int* err = job.err;
  const uint16_t one16 = fmt ? (uint16_t)0x3F80u : (uint16_t)0x3C00u;
  {
    const uint32_t w = (uint32_t)one16 | ((uint32_t)one16 << 16);
    uint32_t* o = reinterpret_cast<uint32_t*>(ones);
    for (int i = threadIdx.x; i < PLANE / 4; i += blockDim.x) o[i] = w;  // all ones: swizzle-invariant
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  fence_proxy_async_smem();
  if (warp == 1) {
    tmem_alloc(tmem_slot, 256);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const bool have_work = t1 > t0;

  if (threadIdx.x == 0 && have_work) {
    // loader
    if (kGlobalMaps) tmap_acquire(job.qmap);
    uint32_t it = 0;
    for (int64_t t = t0; t < t1; ++t, ++it) {
      const int s = it % S;
      if (!mbar_wait(&empty[s], ((it / S) & 1u) ^ 1u, abort_flag, err, 41)) break;
      uint8_t* tile = tiles + s * TILE;
      mbar_arrive_expect_tx(&full[s], TILE);
      tma_load_2d(tile, job.qmap, &full[s], 0, (int)(t * TM));
      tma_load_2d(tile + PLANE, job.qmap, &full[s], 64, (int)(t * TM));
    }
  } else if (threadIdx.x == 32 && have_work) {
    // MMA issuer
    const uint32_t idesc_g = idesc_f16(128, 128, fmt, 1, 1);
    const uint32_t idesc_s = idesc_f16(128, 64, fmt, 1, 1);
    const uint32_t ones_base = smem_u32(ones);
    uint32_t it = 0;
    bool ok = true;
    for (int64_t t = t0; t < t1; ++t, ++it) {
      const int s = it % S;
      if (!mbar_wait(&full[s], (it / S) & 1u, abort_flag, err, 42)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t base = smem_u32(tiles + s * TILE);
#pragma unroll
      for (int kk = 0; kk < TM / 16; ++kk) {
        const uint64_t d = sdesc_sw128(base + kk * 2048, PLANE, 1024);
        umma_f16(tmem, d, d, idesc_g, (it | kk) != 0);
        umma_f16(tmem + 128, d, sdesc_sw128(ones_base + kk * 2048, PLANE, 1024), idesc_s, (it | kk) != 0);
      }
      umma_commit(&empty[s]);
    }
    if (ok) umma_commit(done_bar);
  }
  __syncwarp();
  // epilogue: all four warps (TMEM lane quarter = warp)
  const uint32_t row = 32u * warp + lane;
  float srow = 0.f;
  if (have_work) {
    if (!warp_wait(done_bar, 0, abort_flag, err, 43)) goto done;
    tc_fence_after();
    const uint32_t tb = tmem + ((32u * warp) << 16);
#pragma unroll 1
    for (int cb = 0; cb < 8; ++cb) {  // image columns (2 j', 2 j' + 1) -> column j'
      uint32_t a[16];
      tmem_ld16(tb + cb * 16, a);
      tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i)
        pbuf[row * LD + cb * 8 + i] = __uint_as_float(a[2 * i]) + __uint_as_float(a[2 * i + 1]);
    }
    uint32_t c16[16];
    tmem_ld16(tb + 128, c16);
    tmem_wait_ld();
    srow = __uint_as_float(c16[0]);
  } else {
    for (int j = 0; j < LD; ++j) pbuf[row * LD + j] = 0.f;
  }
  __syncthreads();
  {
    double* out = job.out;
    // image rows 2 i (hi) and 2 i + 1 (lo) belong to column i
    for (int t = threadIdx.x; t < LD * LD; t += blockDim.x) {
      const int i = t / LD, j = t % LD;
      out[t] = (double)pbuf[(2 * i) * LD + j] + (double)pbuf[(2 * i + 1) * LD + j];
    }
    pbuf[row * LD] = srow;  // column sums of [h | l], one per row of Ds
  }
  __syncthreads();
  if (threadIdx.x < LD) {
    double* out = job.out;
    out[LD * LD + threadIdx.x] = (double)pbuf[(2 * threadIdx.x) * LD] + (double)pbuf[(2 * threadIdx.x + 1) * LD];
  }
done:
  if (*abort_flag) __nanosleep(500000);
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// CTA b takes the tiles [tc_range_begin(b), tc_range_begin(b + 1)) and writes partial b.
__global__ void __launch_bounds__(128, 1)
    k_gram_tc(int64_t n_tiles, const __grid_constant__ CUtensorMap qmap, double* __restrict__ part, int fmt,
              int* err) {
  const GramJob job{&qmap, part + (int64_t)blockIdx.x * (64 * 64 + 64), err,
                    tc_range_begin(blockIdx.x, gridDim.x, n_tiles), tc_range_begin(blockIdx.x + 1, gridDim.x, n_tiles)};
  gram_tc_body<false>(job, fmt);
}

// One item (segment, tile range, partial) per CTA, over every segment of a batch.
__global__ void __launch_bounds__(128, 1)
    k_gram_tc_batch(const TcSegment* __restrict__ segs, const TcItem* __restrict__ items, int fmt) {
  const TcItem it = items[blockIdx.x];
  const TcSegment& sg = segs[it.seg];
  const GramJob job{sg.qmap, sg.gpart + (int64_t)it.slot * (64 * 64 + 64), sg.err, it.t0, it.t1};
  gram_tc_body<true>(job, fmt);
}

// ---------------------------------------------------------------------------
// Embeddings U = Q M (n x nc, nc <= 64) on tensor cores, from the 16-bit image
// of Q (ld 64: columns 2 j, 2 j + 1 = hi, lo of Q[:, j], TMA-loaded in tiles
// of 128 rows) and the image of M: B[n][2 j] = B[n][2 j + 1] = hi(M[j][n])
// for n < 64 and lo(M[j][n - 64]) for 64 <= n < 128, so one MMA chain
// (M = 128 rows, N = 128, K = 128 image columns) gives Q hi(M) in columns
// 0..63 and Q lo(M) in 64..127, which the epilogue adds: about 16 mantissa
// bits on both operands, FP32 accumulation.  A CTA walks a contiguous range
// of row tiles: warp 4 loads image tiles into a four-stage ring, warp 5
// issues the MMAs into one of two TMEM accumulators, and warps 0-3 (one TMEM
// lane quarter each) drain the other, staging the tile's rows of U in shared
// memory so they leave in whole contiguous rows.  All waits are bounded.
// ---------------------------------------------------------------------------
constexpr int kEmbedStages = 4;
constexpr int kEmbedThreads = 192;

__host__ __device__ constexpr size_t embed_tc_smem() {
  return 1024 + (size_t)kEmbedStages * 2 * TM * 64 * 2 + 2 * 128 * 64 * 2 + (size_t)TM * 64 * 4 + 256;
}

__global__ void __launch_bounds__(kEmbedThreads, 1)
    k_embed_tc(int64_t n, int64_t n_tiles, const __grid_constant__ CUtensorMap qmap, const float* __restrict__ M,
               int nc, float* __restrict__ U, int fmt, int* err) {
  constexpr int PLANE = TM * 64 * 2;  // 64 image columns of 128 rows, 16 KB
  constexpr int TILE = 2 * PLANE;
  constexpr int S = kEmbedStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* tiles = smem;
  uint8_t* Bs = tiles + S * TILE;                           // [2 planes][128 n][64 k], swizzled
  float* Us = reinterpret_cast<float*>(Bs + 2 * PLANE);     // [128 rows][nc]
  uint64_t* bars = reinterpret_cast<uint64_t*>(Us + TM * 64);
  uint64_t* full = bars;
  uint64_t* empty = full + S;
  uint64_t* acc_full = empty + S;
  uint64_t* acc_empty = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t0 = tc_range_begin(blockIdx.x, gridDim.x, n_tiles), t1 = tc_range_begin(blockIdx.x + 1, gridDim.x, n_tiles);

  // B from M (ld 64 rows, nc columns): element (n, k) of plane k / 64
  for (int e = threadIdx.x; e < 128 * 128; e += blockDim.x) {
    const int nn = e >> 7, k = e & 127, j = k >> 1;
    const int col = nn & 63;
    uint16_t v = 0;
    if (col < nc) {
      const uint32_t w = hilo16(M[j * nc + col], fmt);
      v = (uint16_t)(nn < 64 ? (w & 0xFFFFu) : (w >> 16));
    }
    *reinterpret_cast<uint16_t*>(Bs + (k >> 6) * PLANE + sw128_offset((uint32_t)nn, (uint32_t)(k & 63))) = v;
  }
  if (threadIdx.x == 0) {
    for (int st = 0; st < S; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 4);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  fence_proxy_async_smem();  // B, written by threads, is read by the tensor cores
  if (warp == 5) {
    tmem_alloc(tmem_slot, 256);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    if (lane == 0) {
      uint32_t it = 0;
      for (int64_t t = t0; t < t1; ++t, ++it) {
        const int st = it % S;
        if (!mbar_wait(&empty[st], ((it / S) & 1u) ^ 1u, abort_flag, err, 51)) break;
        uint8_t* tile = tiles + st * TILE;
        mbar_arrive_expect_tx(&full[st], TILE);
        tma_load_2d(tile, &qmap, &full[st], 0, (int)(t * TM));
        tma_load_2d(tile + PLANE, &qmap, &full[st], 64, (int)(t * TM));
      }
    }
    __syncwarp();
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(128, 128, fmt, 0, 0);  // both K-major
      const uint32_t bbase = smem_u32(Bs);
      uint32_t it = 0;
      for (int64_t t = t0; t < t1; ++t, ++it) {
        const int st = it % S;
        const uint32_t a = it & 1u, u = it >> 1;
        if (!mbar_wait(&acc_empty[a], (u & 1u) ^ 1u, abort_flag, err, 52) ||
            !mbar_wait(&full[st], (it / S) & 1u, abort_flag, err, 53))
          break;
        tc_fence_after();
        const uint32_t abase = smem_u32(tiles + st * TILE);
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {  // K = 16 image columns per step: +32 B along a row, plane after 4
          const uint32_t off = (uint32_t)(kk >> 2) * PLANE + (uint32_t)(kk & 3) * 32u;
          umma_f16(tmem + a * 128, sdesc_sw128(abase + off, 16, 1024), sdesc_sw128(bbase + off, 16, 1024), idesc,
                   kk != 0);
        }
        umma_commit(&empty[st]);
        umma_commit(&acc_full[a]);
      }
    }
    __syncwarp();
  } else {
    // epilogue: TMEM lane quarter = warp; row 32 warp + lane of the tile
    const int row = 32 * warp + lane;
    uint32_t it = 0;
    for (int64_t t = t0; t < t1; ++t, ++it) {
      const uint32_t a = it & 1u, u = it >> 1;
      if (!warp_wait(&acc_full[a], u & 1u, abort_flag, err, 54)) break;
      tc_fence_after();
      const uint32_t tb = tmem + ((32u * warp) << 16) + a * 128;
#pragma unroll
      for (int h = 0; h < 2; ++h) {  // output columns 32 h .. 32 h + 31
        uint32_t x[32], y[32];
        tmem_ld32(tb + 32 * h, x);
        tmem_ld32(tb + 64 + 32 * h, y);
        tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (32 * h + c < nc) Us[row * nc + 32 * h + c] = __uint_as_float(x[c]) + __uint_as_float(y[c]);
      }
      tc_fence_before();
      __syncwarp();  // the warp's 32 rows of U are staged
      if (lane == 0) mbar_arrive(&acc_empty[a]);
      // the warp's rows are contiguous in U: it copies them out alone (no
      // barrier with the other epilogue warps, which could wait on a warp that
      // gave up on a timed-out wait)
      const int64_t r0 = t * TM + 32 * warp;
      const int64_t cnt = max((int64_t)0, min((int64_t)32, n - r0)) * nc;
      float* dst = U + r0 * nc;
      const float* src = Us + 32 * warp * nc;
      for (int64_t e = lane; e < cnt; e += 32) dst[e] = src[e];
      __syncwarp();  // the warp's rows of Us are free for the next tile
    }
  }
  if (*abort_flag) __nanosleep(500000);
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// 16-bit image of x: words (hi | lo << 16), hi = round16(x), lo = round16(x - hi)
// (fmt 1 = bf16, 0 = f16).
__global__ void k_split16(const float* __restrict__ in, int64_t count, uint32_t* __restrict__ img, int fmt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    img[i] = hilo16(in[i], fmt);
}

// One matrix per grid row y (batched segments).
__global__ void k_split16_batch(const SplitTask* __restrict__ tasks, int64_t count, int fmt) {
  const SplitTask t = tasks[blockIdx.y];
  uint32_t* img = reinterpret_cast<uint32_t*>(t.img);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    img[i] = hilo16(t.in[i], fmt);
}

// ---------------------------------------------------------------------------
// ld 64: the two products with the dense operand's image as the MMA's A and
// the densified tiles as its B, so one instruction spans N = 256 cells (two
// tiles, forward) or 256 genes (four chunks, transposed).  The issue cost of
// a tcgen05.mma at M = 128 does not depend on N, so the wider N halves the
// instructions per segment.  The accumulator is transposed: TMEM lane m is
// image column m = 2 j + p ((hi, lo) of output column j), so lanes 2 j and
// 2 j + 1 hold the two halves of one output column and a lane shuffle adds
// them.
// ---------------------------------------------------------------------------
constexpr int kSwapFwdStages = 4;  // pair stages: the two tiles of a band, one chunk
constexpr int kSwapFwdSlots = 5;   // dense-operand ring (16 KB image chunks)

__host__ __device__ constexpr size_t fwd_swap_smem() {
  return 1024 + (size_t)kSwapFwdStages * 2 * (TM * CW * 2) + (size_t)kSwapFwdSlots * (CW * 128 * 2) +
         2 * 2 * (size_t)kMaxChunks * sizeof(SegMeta) + 64 * sizeof(uint64_t) + 64;
}

// The operands of one band: of the one matrix of k_fwd_swap (FwdOne), or of
// the segment it belongs to in k_fwd_swap_batch (FwdBatch).
struct FwdBand {
  const uint32_t* ent;
  const SegMeta* meta;  // the band's first metadata record
  const CUtensorMap* vmap;
  const float* mc;
  float* Y;             // null: no FP32 copy
  uint16_t* Yimg;
  int* err;
  int64_t row0;         // the band's first row in its matrix
  int64_t n;            // rows of its matrix
  int tiles;            // 1 or 2
};

struct FwdOne {
  const uint32_t* ent;
  const SegMeta* meta;
  const CUtensorMap* vmap;
  const float* mc;
  float* Y;
  uint16_t* Yimg;
  int* err;
  int64_t n_tiles, n;
  int nc;
  static constexpr bool kGlobalMaps = false;
  __device__ int64_t bands() const { return (n_tiles + 1) / 2; }
  __device__ FwdBand band(int64_t b) const {
    return FwdBand{ent, meta + b * 2 * nc, vmap, mc, Y, Yimg, err, b * 2 * TM, n,
                   (int)min((int64_t)2, n_tiles - b * 2)};
  }
};

struct FwdBatch {
  const TcSegment* segs;
  const int32_t* band_seg;
  int64_t n_bands;
  int nc, write_y;
  static constexpr bool kGlobalMaps = true;  // tensor maps in global memory
  __device__ int64_t bands() const { return n_bands; }
  __device__ FwdBand band(int64_t b) const {
    const TcSegment& sg = segs[__ldg(band_seg + b)];
    const int64_t lb = b - sg.band0, n_tiles = (sg.n + TM - 1) / TM;
    return FwdBand{sg.ent, static_cast<const SegMeta*>(sg.meta) + lb * 2 * nc, sg.vmap, sg.mc,
                   write_y ? sg.Y : nullptr, sg.Yimg, sg.err, lb * 2 * TM, sg.n,
                   (int)min((int64_t)2, n_tiles - lb * 2)};
  }
};

// A band is two consecutive row tiles.  Per band:
// Y^T[m, its 256 cells] = sum over chunks c of Vimg_c^T (m x 64 genes) [A_(t0,c) | A_(t1,c)]^T.
template <class Src>
__device__ __forceinline__ void fwd_swap_body(const Src& src, int nc, int fmt) {
  constexpr int LD = 64;
  constexpr int S = kSwapFwdStages;
  constexpr int NB = kSwapFwdSlots;
  constexpr int TILE = TM * CW * 2;      // one 128 x 64 tile, 16 KB
  constexpr int STAGE = 2 * TILE;        // the band's two tiles, 256 cell rows
  constexpr int B_BYTES = CW * 128 * 2;  // 64 genes x 128 image columns
  constexpr int MSLOT = 2 * kMaxChunks;
  static_assert(S == 4, "stage of chunk counter cc is cc % 4; groups (cc & 1, tile) own two stages each");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* As = smem;
  uint8_t* Bs = As + S * STAGE;
  SegMeta* mring = reinterpret_cast<SegMeta*>(Bs + NB * B_BYTES);  // [2][2 * kMaxChunks]
  uint64_t* bars = reinterpret_cast<uint64_t*>(mring + 2 * MSLOT);
  uint64_t* full = bars;            // [S]  stage densified (two groups x 4 warps)
  uint64_t* empty = full + S;       // [S]  stage consumed (MMA commit)
  uint64_t* bfull = empty + S;      // [NB] image chunk landed (TMA)
  uint64_t* bempty = bfull + NB;    // [NB] image chunk consumed (MMA commit)
  uint64_t* acc_full = bempty + NB;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* mfull = acc_empty + 2;
  uint64_t* mempty = mfull + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n_bands = src.bands();
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 8);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < NB; ++b) {
      mbar_init(&bfull[b], 1);
      mbar_init(&bempty[b], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 4);
      mbar_init(&mfull[a], 1);
      mbar_init(&mempty[a], 4 * kGroups);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == W_MMA) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < W_EPI) {
    // ---- densify: group (cc & 1, u) fills tile u of the stage of chunk
    // counter cc; a band with one tile leaves its u = 1 groups idle, but they
    // still take part in the stage handshake ----
    const int group = warp >> 2, q = warp & 3;
    const int par = group >> 1, u = group & 1;
    uint32_t cc = 0, bi = 0;
    uint4 w[kFwdRegs];
    Span pre{-1, -1};             // span whose loads are in flight in w
    const uint32_t* pre_ent = nullptr;  // the entry array pre indexes
    for (int64_t band = blockIdx.x; band < n_bands; band += gridDim.x, ++bi) {
      const FwdBand bd = src.band(band);
      int* err = bd.err;
      const bool has = u < bd.tiles;
      if (!warp_wait(&mfull[bi & 1u], (bi >> 1) & 1u, abort_flag, err, 11)) goto done;
      const SegMeta* mt = mring + (bi & 1u) * MSLOT;
      for (int c = 0; c < nc; ++c, ++cc) {
        if ((int)(cc & 1u) != par) continue;
        // the span loaded ahead (pre) is this segment's whenever one was loaded
        const Span sp = !has ? Span{0, 0} : pre.lo >= 0 ? pre : quarter_span(mt[u * nc + c], q);
        const uint32_t* sp_ent = pre.lo >= 0 ? pre_ent : bd.ent;
        if (has && pre.lo < 0) span_load<kFwdRegs>(sp_ent, sp, lane, w);
        const int s = cc % S;
        if (!warp_wait(&empty[s], ((cc / S) & 1u) ^ 1u, abort_flag, err, 12)) goto done;
        if (has) {
          const uint32_t tile = smem_u32(As + s * STAGE + u * TILE);
          zero_rows(tile, q, lane);
          __syncwarp();
          span_scatter<kFwdRegs>(tile, sp_ent, sp, lane, w);
        }
        // the group's next segment: chunk c + 2 of this band, or of the next
        pre = Span{-1, -1};
        if (c + 2 < nc) {
          if (has) {
            pre = quarter_span(mt[u * nc + c + 2], q);
            pre_ent = bd.ent;
          }
        } else if (band + gridDim.x < n_bands && c + 2 - nc < nc) {
          const FwdBand nx = src.band(band + gridDim.x);
          if (u < nx.tiles) {
            if (!warp_wait(&mfull[(bi + 1) & 1u], ((bi + 1) >> 1) & 1u, abort_flag, err, 11)) goto done;
            pre = quarter_span(mring[((bi + 1) & 1u) * MSLOT + u * nc + (c + 2 - nc)], q);
            pre_ent = nx.ent;
          }
        }
        if (pre.lo >= 0) span_load<kFwdRegs>(pre_ent, pre, lane, w);
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&full[s]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&mempty[bi & 1u]);
    }
  } else if (warp < W_MMA) {
    // ---- epilogue: lane pair (2 j, 2 j + 1) -> column j of Y and its image ----
    const int q = warp & 3;
    const int p = lane & 1, j = 16 * q + (lane >> 1);
    uint32_t k = 0;
    for (int64_t band = blockIdx.x; band < n_bands; band += gridDim.x, ++k) {
      const FwdBand bd = src.band(band);
      int* err = bd.err;
      const int64_t n = bd.n;
      const float mcj = __ldg(bd.mc + j);
      uint16_t* Yimg = bd.Yimg;
      float* Y = bd.Y;
      const uint32_t a = k & 1u, ph = (k >> 1) & 1u;
      if (!warp_wait(&acc_full[a], ph, abort_flag, err, 14)) goto done;
      tc_fence_after();
      for (int u = 0; u < bd.tiles; ++u) {
        const uint32_t tbase = tmem + ((32u * q) << 16) + a * 256 + u * 128;
        const int64_t row0 = bd.row0 + u * TM;
#pragma unroll 1
        for (int cb = 0; cb < TM / 32; ++cb) {  // 32 cells per TMEM load
          uint32_t r[32];
          tmem_ld32(tbase + cb * 32, r);
          tmem_wait_ld();
          const int64_t c0 = row0 + cb * 32;
          const int lim = (int)min((int64_t)32, n - c0);  // cells of this block inside the matrix
          // word j of an image row holds (hi, lo) of column j; lane p handles cell i + p
          uint32_t* dst = reinterpret_cast<uint32_t*>(Yimg) + c0 * 64 + 16 * q + (lane >> 1);
          float* ydst = Y ? Y + c0 * LD + j : nullptr;
#pragma unroll
          for (int i = 0; i < 32; i += 2) {
            const float x0 = __uint_as_float(r[i]), x1 = __uint_as_float(r[i + 1]);
            const float s0 = x0 + __shfl_xor_sync(0xffffffffu, x0, 1) - mcj;
            const float s1 = x1 + __shfl_xor_sync(0xffffffffu, x1, 1) - mcj;
            const float sm = p ? s1 : s0;
            if (i + p < lim) {
              dst[(i + p) * 64] = hilo16(sm, fmt);
              if (ydst) ydst[(i + p) * LD] = sm;
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[a]);
    }
  } else if (warp == W_MMA) {
    // ---- MMA issuer: per chunk, four K = 16 steps over both tiles of the band ----
    if (lane == 0) {
      const uint32_t idesc2 = idesc_f16(128, 256, fmt, 1, 0);
      const uint32_t idesc1 = idesc_f16(128, 128, fmt, 1, 0);
      const uint64_t vdesc0 = sdesc_sw128(smem_u32(Bs), CW * 128, 1024);  // MN-major, two 64-column blocks
      const uint64_t tdesc0 = sdesc_sw128(smem_u32(As), 16, 1024);        // K-major, 256 cell rows
      uint32_t cc = 0, k = 0;
      bool ok = true;
      for (int64_t band = blockIdx.x; band < n_bands && ok; band += gridDim.x, ++k) {
        const FwdBand bd = src.band(band);
        int* err = bd.err;
        const uint32_t idesc = bd.tiles == 2 ? idesc2 : idesc1;
        const uint32_t a = k & 1u, ph = (k >> 1) & 1u;
        if (!mbar_wait(&acc_empty[a], ph ^ 1u, abort_flag, err, 15)) break;
        tc_fence_after();
        const uint32_t d = tmem + a * 256;
        for (int c = 0; c < nc; ++c, ++cc) {
          const int b = cc % NB, s = cc % S;
          if (!mbar_wait(&bfull[b], (cc / NB) & 1u, abort_flag, err, 16) ||
              !mbar_wait(&full[s], (cc / S) & 1u, abort_flag, err, 16)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t vd = vdesc0 + (uint64_t)(b * (B_BYTES >> 4));
          const uint64_t td = tdesc0 + (uint64_t)(s * (STAGE >> 4));
          umma_f16(d, vd, td, idesc, c != 0);
#pragma unroll
          for (int kk = 1; kk < CW / 16; ++kk)  // K steps of 16 genes: +2 KB down the image, +32 B along the tiles
            umma_f16(d, vd + 128 * kk, td + 2 * kk, idesc, 1u);
          umma_commit(&empty[s]);
          umma_commit(&bempty[b]);
        }
        if (ok) umma_commit(&acc_full[a]);
      }
    }
    __syncwarp();
  } else if (warp == W_DENSE) {
    // ---- dense loader: image chunks into the ring, up to NB ahead ----
    if (lane == 0) {
      uint32_t cc = 0;
      bool ok = true;
      for (int64_t band = blockIdx.x; band < n_bands && ok; band += gridDim.x) {
        const FwdBand bd = src.band(band);
        int* err = bd.err;
        if (Src::kGlobalMaps) tmap_acquire(bd.vmap);
        for (int c = 0; c < nc; ++c, ++cc) {
          const int b = cc % NB;
          if (!mbar_wait(&bempty[b], ((cc / NB) & 1u) ^ 1u, abort_flag, err, 19)) {
            ok = false;
            break;
          }
          uint8_t* bb = Bs + b * B_BYTES;
          mbar_arrive_expect_tx(&bfull[b], B_BYTES);
          tma_load_2d(bb, bd.vmap, &bfull[b], 0, CW * c);
          tma_load_2d(bb + CW * 128, bd.vmap, &bfull[b], 64, CW * c);
        }
      }
    }
    __syncwarp();
  } else if (warp == W_META) {
    // ---- meta loader: band metadata, and the band's entries into L2 ----
    if (lane == 0) {
      uint32_t bi = 0;
      for (int64_t band = blockIdx.x; band < n_bands; band += gridDim.x, ++bi) {
        const FwdBand bd = src.band(band);
        int* err = bd.err;
        const int records = bd.tiles * nc;  // the band's tiles are consecutive in `meta`
        if (!load_meta(bd.meta, records, mring, MSLOT, mfull, mempty, bi, abort_flag, err, 17)) break;
        if (!mbar_wait(&mfull[bi & 1u], (bi >> 1) & 1u, abort_flag, err, 18)) break;
        prefetch_segments(bd.ent, mring + (bi & 1u) * MSLOT, 0, records);
      }
    }
    __syncwarp();
  }
done:
  if (*abort_flag) __nanosleep(500000);
  tc_fence_before();
  __syncthreads();
  if (warp == W_MMA) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

__global__ void __launch_bounds__(kThreads, 1)
    k_fwd_swap(const uint32_t* __restrict__ ent, const SegMeta* __restrict__ meta, int64_t n_tiles, int nc,
               int64_t n, const __grid_constant__ CUtensorMap vmap, const float* __restrict__ mc,
               float* __restrict__ Y, uint16_t* __restrict__ Yimg, int fmt, int* err) {
  fwd_swap_body(FwdOne{ent, meta, &vmap, mc, Y, Yimg, err, n_tiles, n, nc}, nc, fmt);
}

// Every band of every segment of a batch in one persistent launch.
__global__ void __launch_bounds__(kThreads, 1)
    k_fwd_swap_batch(const TcSegment* __restrict__ segs, const int32_t* __restrict__ band_seg, int64_t n_bands,
                     int nc, int write_y, int fmt) {
  fwd_swap_body(FwdBatch{segs, band_seg, n_bands, nc, write_y}, nc, fmt);
}

constexpr int kSwapRmatStages = 4;  // stages: one half tile (64 cells) of a quad's four chunks
constexpr int kSwapQuads = 2;       // 256-gene quads per CTA (2 x 256 TMEM columns)

__host__ __device__ constexpr size_t rmat_swap_smem() {
  return 1024 + (size_t)kSwapRmatStages * 4 * (64 * CW * 2) + 2 * (size_t)(TM * 128 * 2) +
         2 * (size_t)kMaxChunks * sizeof(SegMeta) + 64 * sizeof(uint64_t) + 64;
}

// part[row group][genes of this CTA, :64]: per quad of four chunks (256 genes)
// Z^T[m, the quad's genes] = sum over the CTA's row tiles t of
// Qimg_t^T (m x 128 cells) [A_(t,4qd) | ... | A_(t,4qd+3)].  grid = gene groups x row groups.
// A stage holds one half (64 cells) of a tile for the quad's four chunks, so
// K = 64 per stage and the densify warps split into two teams of eight, team
// h filling the cells 64 h .. 64 h + 63 of every tile (warp = chunk x quarter).
// One CTA's work: gene group gg over the row tiles [t0, t1) of one matrix,
// written as partial `rg` of `part`.
struct RmatJob {
  const uint32_t* ent;
  const SegMeta* meta;
  const CUtensorMap* qmap;
  float* part;
  int* err;
  int64_t t0, t1;
  int gg, rg;
};

template <bool kGlobalMaps>
__device__ __forceinline__ void rmat_swap_body(const RmatJob& job, int nc, int64_t g, int fmt) {
  constexpr int LD = 64;
  constexpr int S = kSwapRmatStages;
  constexpr int HSUB = 64 * CW * 2;      // half a chunk tile (64 cells x 64 genes), 8 KB
  constexpr int STAGE = 4 * HSUB;        // 64 cells x 256 genes
  constexpr int Q_BYTES = TM * 128 * 2;  // 128 cells x 128 image columns
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* As = smem;
  uint8_t* Qs = As + S * STAGE;  // [2 buffers]
  SegMeta* mring = reinterpret_cast<SegMeta*>(Qs + 2 * Q_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(mring + 2 * kMaxChunks);
  uint64_t* full = bars;
  uint64_t* empty = full + S;
  uint64_t* qfull = empty + S;
  uint64_t* qempty = qfull + 2;
  uint64_t* mfull = qempty + 2;
  uint64_t* mempty = mfull + 2;
  uint64_t* done_bar = mempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t* ent = job.ent;
  const SegMeta* meta = job.meta;
  float* part = job.part;
  int* err = job.err;
  const int64_t t0 = job.t0, t1 = job.t1;
  const int gg = job.gg, rg = job.rg;
  const int n_quads = (nc + 3) / 4;
  const int qd0 = gg * kSwapQuads, qd1 = min(n_quads, qd0 + kSwapQuads);
  const int nq = max(0, qd1 - qd0);
  const bool have_work = (t1 > t0) && nq > 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 8);  // the eight warps of one team
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&qfull[b], 1);
      mbar_init(&qempty[b], 1);
      mbar_init(&mfull[b], 1);
      mbar_init(&mempty[b], 4 * kGroups);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == W_MMA) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < W_EPI) {
    // ---- densify: team h (warps 8 h .. 8 h + 7) fills the half-tile stages
    // of cells 64 h .. 64 h + 63; warp (c, r) of a team takes chunk 4 qd + c,
    // quarter 2 h + r of the tile ----
    const int h = warp >> 3, cofs = (warp >> 1) & 3, q = 2 * h + (warp & 1);
    uint32_t ti = 0;
    uint4 w[kRmatRegs];
    Span pre{-1, -1};     // span whose loads are in flight in w
    bool zeroed = false;  // this warp's rows of its next stage were zeroed ahead
    if (have_work)
      for (int64_t t = t0; t < t1; ++t, ++ti) {
        if (!warp_wait(&mfull[ti & 1u], (ti >> 1) & 1u, abort_flag, err, 21)) goto done;
        const SegMeta* mt = mring + (ti & 1u) * kMaxChunks;
        for (int jq = 0; jq < nq; ++jq) {
          const uint32_t it = (ti * (uint32_t)nq + jq) * 2u + h;  // this stage in the MMA's order
          const int ch = 4 * (qd0 + jq) + cofs;
          const bool has = ch < nc;
          // the span loaded ahead (pre) is this segment's whenever one was loaded
          const Span sp = !has ? Span{0, 0} : pre.lo >= 0 ? pre : quarter_span(mt[ch], q);
          if (has && pre.lo < 0) span_load<kRmatRegs>(ent, sp, lane, w);
          const int s = it % S;
          if (!warp_wait(&empty[s], ((it / S) & 1u) ^ 1u, abort_flag, err, 22)) goto done;
          if (has) {
            // entry offsets address the whole 128-row tile: rows 64 h.. start 8 KB before the half
            const uint32_t tile = smem_u32(As + s * STAGE + cofs * HSUB) - h * HSUB;
            if (!zeroed) zero_rows(tile, q, lane);
            __syncwarp();
            span_scatter<kRmatRegs>(tile, ent, sp, lane, w);
          }
          // the warp's next segment: the next quad of this tile, or the first of the next tile
          pre = Span{-1, -1};
          bool next = false;
          if (jq + 1 < nq) {
            next = ch + 4 < nc;
            if (next) pre = quarter_span(mt[ch + 4], q);
          } else if (t + 1 < t1 && 4 * qd0 + cofs < nc) {
            next = true;
            if (!warp_wait(&mfull[(ti + 1) & 1u], ((ti + 1) >> 1) & 1u, abort_flag, err, 21)) goto done;
            pre = quarter_span(mring[((ti + 1) & 1u) * kMaxChunks + 4 * qd0 + cofs], q);
          }
          if (pre.lo >= 0) span_load<kRmatRegs>(ent, pre, lane, w);
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(&full[s]);
          // Zero this warp's rows of its next stage now, so the stores drain
          // while the next segment's metadata and entries are fetched and the
          // warp barrier before the next scatter finds them done (measured:
          // -9 % on this kernel; the forward kernel, whose stage holds two
          // tiles of one chunk, gained nothing and zeroes in place).
          zeroed = false;
          if (next) {
            const uint32_t itn = it + 2;  // this team's next stage
            const int sn = itn % S;
            if (!warp_wait(&empty[sn], ((itn / S) & 1u) ^ 1u, abort_flag, err, 22)) goto done;
            zero_rows(smem_u32(As + sn * STAGE + cofs * HSUB) - h * HSUB, q, lane);
            zeroed = true;
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&mempty[ti & 1u]);
      }
  } else if (warp < W_MMA) {
    // ---- epilogue: lane pair (2 j, 2 j + 1) -> column j of the partial ----
    const int q = warp & 3;
    const int p = lane & 1, j = 16 * q + (lane >> 1);
    if (have_work && !warp_wait(done_bar, 0, abort_flag, err, 24)) goto done;
    tc_fence_after();
    for (int jq = 0; jq < nq; ++jq) {
      const uint32_t tbase = tmem + ((32u * q) << 16) + jq * 256;
      const int64_t gene0 = (int64_t)(qd0 + jq) * 256;
#pragma unroll 1
      for (int gb = 0; gb < 16; ++gb) {  // 16 genes per TMEM load
        uint32_t r[16];
        if (have_work) {
          tmem_ld16(tbase + gb * 16, r);
          tmem_wait_ld();
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) r[i] = 0u;
        }
        float v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const float x = __uint_as_float(r[i]);
          v[i] = x + __shfl_xor_sync(0xffffffffu, x, 1);
        }
        // lane p writes genes 2 i + p: 16 consecutive columns per gene row
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
          const int64_t gene = gene0 + gb * 16 + i + p;
          if (gene < g) part[((int64_t)rg * g + gene) * LD + j] = p ? v[i + 1] : v[i];
        }
      }
    }
  } else if (warp == W_MMA) {
    // ---- MMA issuer: per stage, eight K = 16 steps over the quad's 256 genes ----
    if (lane == 0 && have_work) {
      const uint64_t qdesc0 = sdesc_sw128(smem_u32(Qs), TM * 128, 1024);  // MN-major, two 64-column blocks
      const uint64_t tdesc0 = sdesc_sw128(smem_u32(As), HSUB, 1024);      // MN-major, four 64-gene blocks
      uint32_t it = 0, ti = 0;
      bool ok = true;
      for (int64_t t = t0; t < t1 && ok; ++t, ++ti) {
        const uint32_t b = ti & 1u;
        if (!mbar_wait(&qfull[b], (ti >> 1) & 1u, abort_flag, err, 25)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t qd = qdesc0 + (uint64_t)(b * (Q_BYTES >> 4));
        for (int jq = 0; jq < nq && ok; ++jq) {
          const int nch = min(4, nc - 4 * (qd0 + jq));  // chunk tiles in this quad
          const uint32_t idesc = idesc_f16(128, 64 * nch, fmt, 1, 1);
          const uint32_t d = tmem + jq * 256;
          for (int h = 0; h < 2; ++h, ++it) {  // the two half tiles
            const int s = it % S;
            if (!mbar_wait(&full[s], (it / S) & 1u, abort_flag, err, 26)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint64_t td = tdesc0 + (uint64_t)(s * (STAGE >> 4));
            const uint64_t qh = qd + (uint64_t)(h * (64 * 128 >> 4));  // cells 64 h.. of the image tile
            umma_f16(d, qh, td, idesc, (ti | h) != 0);
#pragma unroll
            for (int kk = 1; kk < 64 / 16; ++kk)  // K steps of 16 cells: +2 KB down both operands
              umma_f16(d, qh + 128 * kk, td + 128 * kk, idesc, 1u);
            umma_commit(&empty[s]);
          }
        }
        if (!ok) break;
        umma_commit(&qempty[b]);
      }
      if (ok) umma_commit(done_bar);
    }
    __syncwarp();
  } else if (warp == W_DENSE) {
    // ---- dense loader: image tiles of Q, double-buffered per row tile ----
    if (lane == 0 && have_work) {
      if (kGlobalMaps) tmap_acquire(job.qmap);
      uint32_t ti = 0;
      for (int64_t t = t0; t < t1; ++t, ++ti) {
        const uint32_t b = ti & 1u;
        if (!mbar_wait(&qempty[b], ((ti >> 1) & 1u) ^ 1u, abort_flag, err, 28)) break;
        uint8_t* qb = Qs + b * Q_BYTES;
        mbar_arrive_expect_tx(&qfull[b], Q_BYTES);
        tma_load_2d(qb, job.qmap, &qfull[b], 0, (int)(t * TM));
        tma_load_2d(qb + TM * 128, job.qmap, &qfull[b], 64, (int)(t * TM));
      }
    }
    __syncwarp();
  } else if (warp == W_META) {
    // ---- meta loader: tile metadata, and this gene group's entries of the tile into L2 ----
    if (lane == 0 && have_work) {
      uint32_t ti = 0;
      for (int64_t t = t0; t < t1; ++t, ++ti) {
        if (!load_meta(meta + t * nc, nc, mring, kMaxChunks, mfull, mempty, ti, abort_flag, err, 27)) break;
        if (!mbar_wait(&mfull[ti & 1u], (ti >> 1) & 1u, abort_flag, err, 29)) break;
        prefetch_segments(ent, mring + (ti & 1u) * kMaxChunks, 4 * qd0, min(nc, 4 * qd1));
      }
    }
    __syncwarp();
  }
done:
  if (*abort_flag) __nanosleep(500000);
  tc_fence_before();
  __syncthreads();
  if (warp == W_MMA) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// CTA b = (row group b / gene groups, gene group b % gene groups); the row
// groups split the tiles evenly (tc_range_begin).
__global__ void __launch_bounds__(kThreads, 1)
    k_rmat_swap(const uint32_t* __restrict__ ent, const SegMeta* __restrict__ meta, int64_t n_tiles, int nc,
                int64_t g, int n_gene_groups, const __grid_constant__ CUtensorMap qmap, float* __restrict__ part,
                int fmt, int* err) {
  const int gg = blockIdx.x % n_gene_groups, rg = blockIdx.x / n_gene_groups;
  const int R = gridDim.x / n_gene_groups;
  const RmatJob job{ent, meta, &qmap, part, err, tc_range_begin(rg, R, n_tiles), tc_range_begin(rg + 1, R, n_tiles),
                    gg, rg};
  rmat_swap_body<false>(job, nc, g, fmt);
}

// One item (segment, gene group, row group, tile range) per CTA, over every
// segment of a batch.
__global__ void __launch_bounds__(kThreads, 1)
    k_rmat_swap_batch(const TcSegment* __restrict__ segs, const TcItem* __restrict__ items, int nc, int64_t g,
                      int fmt) {
  const TcItem it = items[blockIdx.x];
  const TcSegment& sg = segs[it.seg];
  const RmatJob job{sg.ent, static_cast<const SegMeta*>(sg.meta), sg.qmap, sg.part, sg.err, it.t0, it.t1, it.gg,
                    it.slot};
  rmat_swap_body<true>(job, nc, g, fmt);
}

size_t smem_tail() { return 2 * kMaxChunks * sizeof(SegMeta) + 64 * sizeof(uint64_t) + 64; }
size_t fwd_smem(int LD) {
  return 1024 + (size_t)fwd_stages(LD) * (TM * CW * 2) + (size_t)fwd_bslots(LD) * (2 * CW * LD * 2) + smem_tail();
}
size_t rmat_smem(int LD) {
  return 1024 + (size_t)rmat_stages(LD) * (2 * TM * CW * 2) + 4 * (size_t)TM * LD * 2 + smem_tail();
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
size_t tile_meta_bytes(int64_t n, int nc) { return (size_t)((n + TM - 1) / TM) * nc * sizeof(SegMeta); }

cudaError_t tile_format_count(const int64_t* indptr, const int32_t* idx, int64_t n, int nc,
                              int64_t* counts, cudaStream_t st, int num_sms) {
  const int64_t n_tiles = (n + TM - 1) / TM;
  note_launches(1);
  k_tile_count<<<grid_for(n_tiles, 1, num_sms, 8), 256, nc * sizeof(int), st>>>(indptr, idx, n, n_tiles,
                                                                               nc, counts);
  return cudaGetLastError();
}

cudaError_t tile_format_fill(const int64_t* indptr, const int32_t* idx, const void* val16, int64_t n,
                             int nc, const int64_t* seg, uint32_t* ent, void* meta, cudaStream_t st,
                             int num_sms) {
  const int64_t n_tiles = (n + TM - 1) / TM;
  size_t smem = (size_t)2 * TM * nc * sizeof(int);
  if (cudaError_t e = allow_smem(k_tile_fill, smem); e != cudaSuccess) return e;
  note_launches(1);
  k_tile_fill<<<grid_for(n_tiles, 1, num_sms, 2), 512, smem, st>>>(
      indptr, idx, static_cast<const uint16_t*>(val16), n, n_tiles, nc, seg, ent,
      static_cast<SegMeta*>(meta));
  return cudaGetLastError();
}

// The driver entry point is resolved through the runtime, so the library
// does not link libcuda directly (it still loads on hosts without a driver).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Row-major 16-bit matrix [rows][cols] (fmt 1 = bf16, 0 = f16) as a TMA map
// with 64 x box_rows boxes, 128-byte swizzle; out-of-range rows read as zero.
int make_tmap16(CUtensorMap* map, const void* base, int64_t rows, int64_t cols, int box_rows, int fmt) {
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1u, 1u};
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return -1;
  CUresult r = enc(map, fmt ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (int)r;
}

cudaError_t launch_fwd_tc(int ld, const uint32_t* ent, const void* meta, int64_t n, int nc, const CUtensorMap* vmap,
                          const float* mc, float* Y, uint16_t* Yimg, int fmt, int* err, cudaStream_t st, int num_sms) {
  const int64_t n_tiles = (n + TM - 1) / TM;
  const SegMeta* m = static_cast<const SegMeta*>(meta);
  note_launches(1);
  if (ld == 64) {
    const int grid = (int)std::min<int64_t>((n_tiles + 1) / 2, (int64_t)num_sms);
    const size_t smem = fwd_swap_smem();
    if (cudaError_t e = allow_smem(k_fwd_swap, smem); e != cudaSuccess) return e;
    k_fwd_swap<<<grid, kThreads, smem, st>>>(ent, m, n_tiles, nc, n, *vmap, mc, Y, Yimg, fmt, err);
  } else {
    const int grid = (int)std::min<int64_t>(n_tiles, (int64_t)num_sms);
    const size_t smem = fwd_smem(128);
    if (cudaError_t e = allow_smem(k_fwd_tc<128>, smem); e != cudaSuccess) return e;
    k_fwd_tc<128><<<grid, kThreads, smem, st>>>(ent, m, n_tiles, nc, n, *vmap, mc, Y, Yimg, fmt, err);
  }
  return cudaGetLastError();
}

int rmat_tc_groups(int ld, int nc, int num_sms, int* gene_groups) {
  int G;
  if (ld == 64) {
    G = ((nc + 3) / 4 + kSwapQuads - 1) / kSwapQuads;  // 512 genes per CTA
  } else {
    const int spg = 256 / ld;  // 512 TMEM columns / (2 ld) per super-chunk
    G = ((nc + 1) / 2 + spg - 1) / spg;
  }
  *gene_groups = G;
  return std::max(1, num_sms / G);  // row groups
}

cudaError_t launch_rmat_tc(int ld, const uint32_t* ent, const void* meta, int64_t n, int nc, int64_t g,
                           int gene_groups, int row_groups, const CUtensorMap* qmap, float* part, int fmt, int* err,
                           cudaStream_t st) {
  const int64_t n_tiles = (n + TM - 1) / TM;
  const int grid = gene_groups * row_groups;
  const SegMeta* m = static_cast<const SegMeta*>(meta);
  note_launches(1);
  if (ld == 64) {
    const size_t smem = rmat_swap_smem();
    if (cudaError_t e = allow_smem(k_rmat_swap, smem); e != cudaSuccess) return e;
    k_rmat_swap<<<grid, kThreads, smem, st>>>(ent, m, n_tiles, nc, g, gene_groups, *qmap, part, fmt, err);
  } else {
    const size_t smem = rmat_smem(128);
    if (cudaError_t e = allow_smem(k_rmat_tc<128>, smem); e != cudaSuccess) return e;
    k_rmat_tc<128><<<grid, kThreads, smem, st>>>(ent, m, n_tiles, nc, g, gene_groups, *qmap, part, fmt, err);
  }
  return cudaGetLastError();
}

cudaError_t launch_split16_batch(const SplitTask* tasks, int ntasks, int64_t count, int fmt, cudaStream_t st) {
  if (ntasks <= 0 || count <= 0) return cudaSuccess;
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, 64));
  note_launches(1);
  k_split16_batch<<<dim3((unsigned)gx, (unsigned)ntasks), 256, 0, st>>>(tasks, count, fmt);
  return cudaGetLastError();
}

cudaError_t launch_split16(const float* in, int64_t count, uint16_t* img, int fmt, cudaStream_t st, int num_sms) {
  note_launches(1);
  k_split16<<<grid_for(count, 256, num_sms), 256, 0, st>>>(in, count, reinterpret_cast<uint32_t*>(img), fmt);
  return cudaGetLastError();
}

int gram_tc_parts(int64_t n, int parts, int num_sms) {
  const int64_t n_tiles = (n + TM - 1) / TM;
  return (int)std::max<int64_t>(1, std::min<int64_t>(n_tiles, parts > 0 ? parts : num_sms));
}

static constexpr size_t gram_tc_smem() {
  return 1024 + (size_t)kGramStages * 2 * TM * 64 * 2 + TM * 64 * 2 + TM * 64 * 4 + 256;
}

int launch_gram_tc(int64_t n, const CUtensorMap* qmap, double* part, int fmt, int* err, cudaStream_t st,
                   int num_sms, int parts) {
  const int64_t n_tiles = (n + TM - 1) / TM;
  const int grid = gram_tc_parts(n, parts, num_sms);
  if (allow_smem(k_gram_tc, gram_tc_smem()) != cudaSuccess) return -1;
  note_launches(1);
  k_gram_tc<<<grid, 128, gram_tc_smem(), st>>>(n_tiles, *qmap, part, fmt, err);
  return cudaGetLastError() == cudaSuccess ? grid : -1;
}

cudaError_t launch_embed_tc(int64_t n, const CUtensorMap* qmap, const float* M, int nc, float* U, int fmt, int* err,
                            cudaStream_t st, int num_sms) {
  if (n <= 0) return cudaSuccess;
  if (nc <= 0 || nc > 64) return cudaErrorInvalidValue;
  const int64_t n_tiles = (n + TM - 1) / TM;
  const int grid = (int)std::min<int64_t>(n_tiles, (int64_t)num_sms);
  if (cudaError_t e = allow_smem(k_embed_tc, embed_tc_smem()); e != cudaSuccess) return e;
  note_launches(1);
  k_embed_tc<<<grid, kEmbedThreads, embed_tc_smem(), st>>>(n, n_tiles, *qmap, M, nc, U, fmt, err);
  return cudaGetLastError();
}

cudaError_t launch_fwd_tc_batch(const TcSegment* segs, const int32_t* band_seg, int64_t n_bands, int nc,
                                int write_y, int fmt, cudaStream_t st, int num_sms) {
  if (n_bands <= 0) return cudaSuccess;
  const int grid = (int)std::min<int64_t>(n_bands, (int64_t)num_sms);
  const size_t smem = fwd_swap_smem();
  if (cudaError_t e = allow_smem(k_fwd_swap_batch, smem); e != cudaSuccess) return e;
  note_launches(1);
  k_fwd_swap_batch<<<grid, kThreads, smem, st>>>(segs, band_seg, n_bands, nc, write_y, fmt);
  return cudaGetLastError();
}

cudaError_t launch_rmat_tc_batch(const TcSegment* segs, const TcItem* items, int n_items, int nc, int64_t g,
                                 int gene_groups, int fmt, cudaStream_t st) {
  (void)gene_groups;  // each item names its gene group
  if (n_items <= 0) return cudaSuccess;
  const size_t smem = rmat_swap_smem();
  if (cudaError_t e = allow_smem(k_rmat_swap_batch, smem); e != cudaSuccess) return e;
  note_launches(1);
  k_rmat_swap_batch<<<n_items, kThreads, smem, st>>>(segs, items, nc, g, fmt);
  return cudaGetLastError();
}

cudaError_t launch_gram_tc_batch(const TcSegment* segs, const TcItem* items, int n_items, int fmt, cudaStream_t st) {
  if (n_items <= 0) return cudaSuccess;
  if (cudaError_t e = allow_smem(k_gram_tc_batch, gram_tc_smem()); e != cudaSuccess) return e;
  note_launches(1);
  k_gram_tc_batch<<<n_items, 128, gram_tc_smem(), st>>>(segs, items, fmt);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The give-up path of the bounded pipeline wait, on its own.  One block; the
// barrier expects one arrival and no thread ever arrives, so thread 0's wait
// (the same mbar_wait the tensor-core kernels use) runs to its limit, raises
// the block's abort flag and records `code` in err.  Every other warp then
// sees the abort flag in its own wait and leaves at once, as the roles of a
// tensor-core kernel do.  No copy or MMA is in flight, so the block ends
// cleanly and the context stays usable.
// ---------------------------------------------------------------------------
__global__ void k_wait_selftest(int* err, int code) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_s;
  volatile int* abort_flag = &abort_s;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
    *abort_flag = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_wait(&bar, 0u, abort_flag, err, code);
  } else if ((threadIdx.x & 31) == 0) {
    // wait for the abort (bounded as well: twice the limit of thread 0)
    const long long t0 = clock64();
    while (!*abort_flag && clock64() - t0 < 2 * kWaitCycles) __nanosleep(20000);
  }
  __syncthreads();
}

cudaError_t launch_wait_selftest(int* err, int code, cudaStream_t st) {
  note_launches(1);
  k_wait_selftest<<<1, 128, 0, st>>>(err, code);
  return cudaGetLastError();
}

size_t fwd_tc_smem_bytes(int ld) { return ld == 64 ? fwd_swap_smem() : fwd_smem(ld); }
size_t rmat_tc_smem_bytes(int ld) { return ld == 64 ? rmat_swap_smem() : rmat_smem(ld); }

}  // namespace scx
