// CUDA-core SpMM pair with FP32 products and a fixed summation order (the
// strict FP32 path, and the CUDA-core path of 16-bit values when the tensor
// cores cannot take a matrix).  Both kernels read their dense operand from
// shared memory and accumulate in registers; neither uses atomics, so every
// result is bit-identical from run to run.
//
//   forward    Y = P V - 1 mc^T   (CSR rows, V staged in gene chunks)
//   transposed W_part = P^T Q     (tile-CSC copy, Q staged one row tile at a time)
//
// Restate spmm_forward_row (scx-accel/src/pca/cpu.rs:1500-1523) with the mean
// correction of forward_mean_prefactor (scx-gpu/src/gpu_pca.rs:218-237), and
// spmm_transpose_block (scx-accel/src/pca/cpu.rs:1282-1328) with the output-
// partitioned reduction of spmm_transpose_into (cpu.rs:1330-1389).
//
// Layouts (device memory):
//   CSR      : int64 indptr[n+1], int32 idx[nnz], values[nnz], rows sorted by gene
//   V        : float [n_vars][ld] gene-major;  Y, Q: float [n_obs][ld] cell-major
//   tile CSC : for row tile t (kStrictTile rows, entries indptr[t T] .. indptr[(t+1) T]),
//              the same entries reordered by (slot, row): cell[p] = row within the
//              tile (uint8), cval[p] = value; tptr[t (S + 1) + s] = offset of slot
//              s's first entry from indptr[t T] (S + 1 offsets per tile).  Genes are
//              relabelled to slots (gene2slot) so that each warp of the transposed
//              product owns GPW consecutive slots of about equal stored-entry count.
//   partial  : float [ranges][n_vars][ld], summed in range order by k_reduce_rows
#include <algorithm>
#include <functional>
#include <queue>
#include <utility>
#include <vector>

#include "common.cuh"
#include "launch.h"

namespace scx {

namespace {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Copy `bytes` (a multiple of 16, both addresses 16-byte aligned) with the
// whole block, as 16-byte asynchronous copies.
__device__ __forceinline__ void block_copy_async(void* smem, const void* gmem, int bytes) {
  for (int o = threadIdx.x * 16; o < bytes; o += blockDim.x * 16)
    cp_async16(static_cast<char*>(smem) + o, static_cast<const char*>(gmem) + o);
}

// Copy `rows` rows of LD floats, row stride `lds` floats in global memory
// (a column panel of a wider matrix), to consecutive rows in shared memory.
// With lds == LD it is the contiguous copy.
template <int LD>
__device__ __forceinline__ void block_copy_rows_async(float* smem, const float* gmem, int rows, int lds) {
  if (lds == LD) {
    block_copy_async(smem, gmem, rows * LD * 4);
    return;
  }
  constexpr int Q = LD / 4;  // 16-byte pieces per row
  for (int o = threadIdx.x; o < rows * Q; o += blockDim.x) {
    const int r = o / Q, q = o - r * Q;
    cp_async16(smem + r * LD + 4 * q, gmem + (int64_t)r * lds + 4 * q);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Tile-CSC build, one warp per row tile (once per plan).  Counting sort of
// the tile's entries by slot (the relabelled gene); rows are visited in
// order, so within a slot the entries keep row order.  Within one 32-entry
// step two lanes can name the same gene only across a duplicate; the step is
// cut into runs of strictly increasing gene, applied in lane order, which
// keeps the placement (and so the later summation order) deterministic.
// k_gene_counts gives the stored entries per gene that the slot assignment
// balances.
// ---------------------------------------------------------------------------
__global__ void k_gene_counts(const int32_t* __restrict__ idx, int64_t nnz, int32_t* __restrict__ counts) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(counts + __ldg(idx + p), 1);
}

template <typename ValT>
__global__ void k_tile_csc(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                           const ValT* __restrict__ val, int64_t n, const int32_t* __restrict__ gene2slot,
                           int32_t nslots, int64_t n_tiles, int32_t* __restrict__ tptr, uint8_t* __restrict__ cell,
                           ValT* __restrict__ cval) {
  extern __shared__ int32_t cur_all[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  int32_t* cur = cur_all + (int64_t)wib * (nslots + 1);
  const unsigned lanemask_le = 0xffffffffu >> (31 - lane);
  for (int64_t t = (int64_t)blockIdx.x * warps + wib; t < n_tiles; t += (int64_t)gridDim.x * warps) {
    const int64_t r0 = t * kStrictTile;
    const int64_t r1 = min(n, r0 + kStrictTile);
    const int64_t base = indptr[r0];
    const int64_t end = indptr[r1];
    for (int j = lane; j <= nslots; j += 32) cur[j] = 0;
    __syncwarp();
    // counts (integer atomics: the counts do not depend on the order)
    for (int64_t p = base + lane; p < end; p += 32) atomicAdd(&cur[__ldg(gene2slot + __ldg(idx + p))], 1);
    __syncwarp();
    // exclusive scan of cur[0..nslots] -> offsets; lane owns a contiguous segment
    const int per = (nslots + 1 + 31) / 32;
    const int j0 = min(nslots + 1, lane * per), j1 = min(nslots + 1, j0 + per);
    int32_t sum = 0;
    for (int j = j0; j < j1; ++j) sum += cur[j];
    int32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    int32_t run = incl - sum;
    for (int j = j0; j < j1; ++j) {
      const int32_t c = cur[j];
      cur[j] = run;
      tptr[t * (nslots + 1) + j] = run;
      run += c;
    }
    __syncwarp();
    // fill, rows in order
    for (int64_t r = r0; r < r1; ++r) {
      const int64_t s = indptr[r], e = indptr[r + 1];
      const uint8_t rl = (uint8_t)(r - r0);
      for (int64_t b = s; b < e; b += 32) {
        const int64_t p = b + lane;
        const bool ok = p < e;
        const int32_t j = ok ? __ldg(idx + p) : -1;
        const ValT x = ok ? val[p] : ValT();
        const int32_t jl = __shfl_up_sync(0xffffffffu, j, 1);
        const unsigned starts = __ballot_sync(0xffffffffu, lane > 0 && ok && j <= jl);
        const int my_run = __popc(starts & lanemask_le);
        const int runs = __popc(starts) + 1;
        const int32_t slot = ok ? __ldg(gene2slot + j) : 0;
        for (int rr = 0; rr < runs; ++rr) {
          if (ok && my_run == rr) {
            const int32_t q = cur[slot]++;
            cell[base + q] = rl;
            cval[base + q] = x;
          }
          __syncwarp();
        }
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Forward product, quarter-warp layout.  A quarter (8 lanes) owns RPQ rows and
// lane l8 of it the columns 4 l8 + 32 s + e (s < LD / 32, e < 4) of each:
// an entry's V row is read as LD / 32 16-byte loads per lane, the quarter's
// eight lanes covering 128 consecutive bytes, so the four quarters of a warp
// read four V rows in four shared-memory wavefronts, conflict-free.  Each
// entry is broadcast to the 8 lanes of its quarter only (the four quarters
// take four entries with one shuffle), and every lane does 4 LD / 32 FMAs per
// entry, against 2 shuffles for LD / 32 FMAs when a whole warp owns a row
// (measured at 250,000 cells, LD 64: 1.51 ms against 1.85 ms per launch).
//
// Per gene chunk and row, each quarter keeps an 8-entry window of the row
// (one entry per lane; consumed entries marked -1, entries past the row's
// end INT32_MAX), takes the entries whose gene falls in the chunk (the next
// unconsumed ones: rows are sorted), and reloads the window once all 8 are
// consumed.  The four quarters step together: a step runs the largest take
// count of the four, and a quarter past its own count adds 0 x (a staged row
// of V), so every shuffle is warp-uniform.  Entries are added in row order.
// ---------------------------------------------------------------------------
template <int LD, int RPQ, int GC, typename ValT>
__global__ void __launch_bounds__(256, 2) k_fwd_strict_q(const int64_t* __restrict__ indptr,
                                                         const int32_t* __restrict__ idx,
                                                         const ValT* __restrict__ val, int64_t n, int32_t g,
                                                         const float* __restrict__ V, const float* __restrict__ mc,
                                                         float* __restrict__ Y, int lds) {
  constexpr int S4 = LD / 32;  // 16-byte column groups per lane
  constexpr int32_t kDone = -1;
  constexpr unsigned FULL = 0xffffffffu;
  static_assert(RPQ <= 8, "a quarter holds the window bounds of its rows in its 8 lanes");
  extern __shared__ __align__(16) float vs[];  // [2][GC][LD]
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int qw = lane >> 3, l8 = lane & 7;
  const int64_t row0 = (int64_t)blockIdx.x * (32 * RPQ) + (int64_t)wib * (4 * RPQ) + qw * RPQ;
  // lane l8 < RPQ of a quarter: window start and end of its row row0 + l8
  int64_t my_base = 0, my_end = 0;
  if (l8 < RPQ && row0 + l8 < n) {
    my_base = indptr[row0 + l8];
    my_end = indptr[row0 + l8 + 1];
  }
  float acc[RPQ][4 * S4];
  int32_t wi[RPQ], ni[RPQ];  // the window, and the next 8 entries of the row already loaded
  float wv[RPQ], nv[RPQ];
#pragma unroll
  for (int r = 0; r < RPQ; ++r) {
#pragma unroll
    for (int c = 0; c < 4 * S4; ++c) acc[r][c] = 0.f;
    const int64_t base = __shfl_sync(FULL, my_base, r, 8);
    const int64_t end = __shfl_sync(FULL, my_end, r, 8);
    const int64_t p = base + l8;
    wi[r] = p < end ? __ldg(idx + p) : INT32_MAX;
    wv[r] = p < end ? to_f32(val[p]) : 0.f;
    ni[r] = p + 8 < end ? __ldg(idx + p + 8) : INT32_MAX;
    nv[r] = p + 8 < end ? to_f32(val[p + 8]) : 0.f;
  }
  const int nchunk = (g + GC - 1) / GC;
  block_copy_rows_async<LD>(vs, V, min(GC, (int)g), lds);
  cp_async_commit();
  for (int ch = 0; ch < nchunk; ++ch) {
    const int g0 = ch * GC;
    const int g1 = min((int)g, g0 + GC);
    if (ch + 1 < nchunk) {
      const int n1 = min(GC, (int)g - g1);
      block_copy_rows_async<LD>(vs + ((ch + 1) & 1) * GC * LD, V + (int64_t)g1 * lds, n1, lds);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const float* vc = vs + (ch & 1) * GC * LD + 4 * l8;
#pragma unroll
    for (int r = 0; r < RPQ; ++r) {
      while (true) {
        const bool take = (unsigned)wi[r] < (unsigned)g1;
        const unsigned mq = (__ballot_sync(FULL, take) >> (8 * qw)) & 0xffu;
        const int cnt = __popc(mq);
        const int t0 = cnt ? __ffs(mq) - 1 : 0;
        const int steps = (int)__reduce_max_sync(FULL, (unsigned)cnt);
        for (int t = 0; t < steps; ++t) {
          const int src = min(t0 + t, 7);
          const int32_t j = __shfl_sync(FULL, wi[r], src, 8);
          const float x = __shfl_sync(FULL, wv[r], src, 8);
          const bool in = t < cnt;
          const float xs = in ? x : 0.f;
          // a taken gene is in [g0, g1); a step past the quarter's count
          // reads row 0 of the chunk (always staged) and adds zero
          const unsigned jl = in ? min((unsigned)(j - g0), (unsigned)(GC - 1)) : 0u;
          const float* vr = vc + jl * LD;
#pragma unroll
          for (int s4 = 0; s4 < S4; ++s4) {
            const float4 v = *reinterpret_cast<const float4*>(vr + 32 * s4);
            acc[r][4 * s4 + 0] = fmaf(xs, v.x, acc[r][4 * s4 + 0]);
            acc[r][4 * s4 + 1] = fmaf(xs, v.y, acc[r][4 * s4 + 1]);
            acc[r][4 * s4 + 2] = fmaf(xs, v.z, acc[r][4 * s4 + 2]);
            acc[r][4 * s4 + 3] = fmaf(xs, v.w, acc[r][4 * s4 + 3]);
          }
        }
        if (take) wi[r] = kDone;
        // a quarter whose 8 window entries are all consumed loads the next 8
        const unsigned dq = (__ballot_sync(FULL, wi[r] == kDone) >> (8 * qw)) & 0xffu;
        const bool reload = dq == 0xffu;
        if (!__any_sync(FULL, reload)) break;
        if (reload && l8 == r) my_base += 8;
        const int64_t base = __shfl_sync(FULL, my_base, r, 8);
        const int64_t end = __shfl_sync(FULL, my_end, r, 8);
        if (reload) {
          // the next window was loaded a window ahead; fetch the one after it
          wi[r] = ni[r];
          wv[r] = nv[r];
          const int64_t p = base + 8 + l8;
          ni[r] = p < end ? __ldg(idx + p) : INT32_MAX;
          nv[r] = p < end ? to_f32(val[p]) : 0.f;
        }
      }
    }
    __syncthreads();  // everyone is done with this buffer before it is refilled
  }
  cp_async_wait<0>();
  float m[4 * S4];
#pragma unroll
  for (int s4 = 0; s4 < S4; ++s4)
#pragma unroll
    for (int e = 0; e < 4; ++e) m[4 * s4 + e] = mc ? mc[4 * l8 + 32 * s4 + e] : 0.f;
#pragma unroll
  for (int r = 0; r < RPQ; ++r) {
    const int64_t row = row0 + r;
    if (row < n) {
#pragma unroll
      for (int s4 = 0; s4 < S4; ++s4)
        *reinterpret_cast<float4*>(Y + row * lds + 4 * l8 + 32 * s4) =
            make_float4(acc[r][4 * s4 + 0] - m[4 * s4 + 0], acc[r][4 * s4 + 1] - m[4 * s4 + 1],
                        acc[r][4 * s4 + 2] - m[4 * s4 + 2], acc[r][4 * s4 + 3] - m[4 * s4 + 3]);
    }
  }
}

// ---------------------------------------------------------------------------
// Transposed product, quarter-warp layout.  Block (range, b) owns the slots
// [b 32 GPQ, (b + 1) 32 GPQ) and the row tiles of one contiguous range; warp
// w owns the GPW = 4 GPQ slots of one group of the slot assignment
// (strict_genes_per_warp), and its quarter qw the slots slot0 + 4 i + qw
// (i < GPQ), so the group's heaviest genes, which fill its first slots,
// spread over the four quarters.  For each tile, Q's rows (kStrictTile x LD
// floats) are staged in shared memory (double-buffered, asynchronous
// copies).  The block writes one partial row per gene it owns.  Lane l8 owns
// the columns 4 l8 + 32 s + e: a cell's Q row is read as LD / 32 16-byte
// loads per lane, the quarter covering 128 consecutive bytes, and each entry
// is broadcast within its quarter only.  For each slot the four quarters walk
// their entry lists 8 at a time in step (the longest list sets the count; a
// lane past its list holds x = 0 and cell 0, a staged row).  Entries are added
// in tile-CSC order, so the partials do not depend on the schedule.
// ---------------------------------------------------------------------------
template <int LD, int GPQ, typename ValT>
__global__ void __launch_bounds__(256, 2) k_rmat_strict_q(const int64_t* __restrict__ indptr,
                                                          const int32_t* __restrict__ tptr,
                                                          const uint8_t* __restrict__ cell,
                                                          const ValT* __restrict__ cval, int64_t n, int32_t g,
                                                          int32_t nslots, const int32_t* __restrict__ slot2gene,
                                                          int64_t tiles_per_range, const float* __restrict__ Q,
                                                          int lds, float* __restrict__ part) {
  constexpr int S4 = LD / 32;
  constexpr int T = kStrictTile;
  constexpr unsigned FULL = 0xffffffffu;
  static_assert(GPQ <= 8, "a quarter holds the list bounds of its slots in its 8 lanes");
  extern __shared__ __align__(16) float qs[];  // [2][T][LD]
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int qw = lane >> 3, l8 = lane & 7;
  const int64_t n_tiles = (n + T - 1) / T;
  const int64_t t0 = (int64_t)blockIdx.x * tiles_per_range;
  const int64_t t1 = min(n_tiles, t0 + tiles_per_range);
  const int slot0 = (blockIdx.y * 8 + wib) * (4 * GPQ);
  // lane l8 < GPQ of a quarter reads the list bounds of its slot i = l8
  const int my_slot = slot0 + 4 * (l8 % GPQ) + qw;
  float acc[GPQ][4 * S4];
#pragma unroll
  for (int i = 0; i < GPQ; ++i)
#pragma unroll
    for (int c = 0; c < 4 * S4; ++c) acc[i][c] = 0.f;
  if (t0 < t1) {
    auto stage = [&](int64_t t, int buf) {
      const int64_t r0 = t * T;
      const int rows = (int)min((int64_t)T, n - r0);
      block_copy_rows_async<LD>(qs + buf * T * LD, Q + r0 * lds, rows, lds);
    };
    stage(t0, 0);
    cp_async_commit();
    for (int64_t t = t0; t < t1; ++t) {
      const int buf = (int)((t - t0) & 1);
      if (t + 1 < t1) stage(t + 1, buf ^ 1);
      cp_async_commit();
      const int64_t tb = indptr[t * T];
      int32_t p0 = 0, p1 = 0;
      if (my_slot < nslots) {
        p0 = __ldg(tptr + t * (nslots + 1) + my_slot);
        p1 = __ldg(tptr + t * (nslots + 1) + my_slot + 1);
      }
      cp_async_wait<1>();
      __syncthreads();
      const float* qt = qs + buf * T * LD + 4 * l8;
#pragma unroll
      for (int i = 0; i < GPQ; ++i) {
        const int32_t s = __shfl_sync(FULL, p0, i, 8);
        const int32_t len = __shfl_sync(FULL, p1, i, 8) - s;
        const int32_t longest = (int32_t)__reduce_max_sync(FULL, (unsigned)max(len, 0));
        for (int32_t b = 0; b < longest; b += 8) {
          const int32_t q = b + l8;
          int cl = 0;
          float x = 0.f;
          if (q < len) {
            cl = __ldg(cell + tb + s + q);
            x = to_f32(cval[tb + s + q]);
          }
          const int steps = min(8, longest - b);
          for (int u = 0; u < steps; ++u) {
            const int cu = __shfl_sync(FULL, cl, u, 8) & (T - 1);
            const float xu = __shfl_sync(FULL, x, u, 8);
            const float* qr = qt + cu * LD;
#pragma unroll
            for (int s4 = 0; s4 < S4; ++s4) {
              const float4 v = *reinterpret_cast<const float4*>(qr + 32 * s4);
              acc[i][4 * s4 + 0] = fmaf(xu, v.x, acc[i][4 * s4 + 0]);
              acc[i][4 * s4 + 1] = fmaf(xu, v.y, acc[i][4 * s4 + 1]);
              acc[i][4 * s4 + 2] = fmaf(xu, v.z, acc[i][4 * s4 + 2]);
              acc[i][4 * s4 + 3] = fmaf(xu, v.w, acc[i][4 * s4 + 3]);
            }
          }
        }
      }
      __syncthreads();  // this buffer is read before it is refilled
    }
    cp_async_wait<0>();
  }
  float* out = part + (int64_t)blockIdx.x * g * LD;
#pragma unroll
  for (int i = 0; i < GPQ; ++i) {
    const int slot = slot0 + 4 * i + qw;
    const int j = slot < nslots ? __ldg(slot2gene + slot) : -1;
    if (j >= 0) {
#pragma unroll
      for (int s4 = 0; s4 < S4; ++s4)
        *reinterpret_cast<float4*>(out + (int64_t)j * LD + 4 * l8 + 32 * s4) =
            make_float4(acc[i][4 * s4 + 0], acc[i][4 * s4 + 1], acc[i][4 * s4 + 2], acc[i][4 * s4 + 3]);
    }
  }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
int strict_genes_per_warp(int ld) { return ld <= 64 ? 32 : 16; }

int strict_slot_count(int64_t g, int ld) {
  const int per_block = 8 * strict_genes_per_warp(ld);
  return (int)((g + per_block - 1) / per_block) * per_block;
}

// Longest-processing-time assignment of genes to the warps of the
// transposed product: genes in decreasing stored-entry count (ties by gene
// index) each go to the warp group with the smallest count so far that still
// has a free slot (ties by group index).  slot2gene[s] = -1 marks an empty
// slot.  Deterministic for given counts.
void strict_assign_slots(const std::vector<int32_t>& counts, int ld, std::vector<int32_t>& gene2slot,
                         std::vector<int32_t>& slot2gene) {
  const int64_t g = (int64_t)counts.size();
  const int gpw = strict_genes_per_warp(ld);
  const int nslots = strict_slot_count(g, ld);
  const int groups = nslots / gpw;
  std::vector<int32_t> order(g);
  for (int64_t j = 0; j < g; ++j) order[j] = (int32_t)j;
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return counts[a] > counts[b]; });
  // min-heap of (load, group) over groups with a free slot
  using Item = std::pair<int64_t, int32_t>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
  for (int32_t q = 0; q < groups; ++q) heap.push({0, q});
  std::vector<int32_t> fill(groups, 0);
  gene2slot.assign(g, 0);
  slot2gene.assign(nslots, -1);
  for (int32_t j : order) {
    Item it = heap.top();
    heap.pop();
    const int32_t q = it.second;
    const int32_t slot = q * gpw + fill[q]++;
    gene2slot[j] = slot;
    slot2gene[slot] = j;
    if (fill[q] < gpw) heap.push({it.first + counts[j], q});
  }
}

cudaError_t launch_gene_counts(const int32_t* idx, int64_t nnz, int32_t* counts, cudaStream_t st, int num_sms) {
  if (nnz == 0) return cudaSuccess;
  k_gene_counts<<<grid_for(nnz, 256, num_sms), 256, 0, st>>>(idx, nnz, counts);
  note_launches(1);
  return cudaGetLastError();
}

size_t strict_tile_smem_bytes(int nslots) { return sizeof(int32_t) * (size_t)(nslots + 1); }

template <typename ValT>
static cudaError_t tile_csc_t(const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                              const int32_t* gene2slot, int32_t nslots, int32_t* tptr, uint8_t* cell, void* cval,
                              cudaStream_t st, int num_sms) {
  const int64_t n_tiles = (n + kStrictTile - 1) / kStrictTile;
  const size_t per_warp = strict_tile_smem_bytes(nslots);
  if (per_warp > kStatsSmemMax) return cudaErrorInvalidValue;
  const int warps = (int)std::min<size_t>(8, kStatsSmemMax / per_warp);
  const size_t smem = per_warp * warps;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_tile_csc<ValT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n_tiles + warps - 1) / warps, (int64_t)num_sms * 4));
  k_tile_csc<ValT><<<grid, warps * 32, smem, st>>>(indptr, idx, static_cast<const ValT*>(val), n, gene2slot, nslots,
                                                   n_tiles, tptr, cell, static_cast<ValT*>(cval));
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_tile_csc(int dtype, const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                            const int32_t* gene2slot, int32_t nslots, int32_t* tptr, uint8_t* cell, void* cval,
                            cudaStream_t st, int num_sms) {
  if (n == 0) return cudaSuccess;
  switch (dtype) {
    case 0: return tile_csc_t<float>(indptr, idx, val, n, gene2slot, nslots, tptr, cell, cval, st, num_sms);
    case 1: return tile_csc_t<__nv_bfloat16>(indptr, idx, val, n, gene2slot, nslots, tptr, cell, cval, st, num_sms);
    default: return tile_csc_t<__half>(indptr, idx, val, n, gene2slot, nslots, tptr, cell, cval, st, num_sms);
  }
}

template <int LD, typename ValT>
static cudaError_t fwd_strict_t(const int64_t* indptr, const int32_t* idx, const void* val, int64_t n, int32_t g,
                                const float* V, const float* mc, float* Y, int lds, cudaStream_t st) {
  constexpr int RPQ = LD <= 32 ? 8 : 4;  // rows per quarter-warp: RPQ x LD / 8 accumulators per lane
  constexpr int GC = (8192 / LD) & ~7;
  const size_t smem = (size_t)2 * GC * LD * sizeof(float);
  auto kern = k_fwd_strict_q<LD, RPQ, GC, ValT>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int64_t rows_per_block = 32 * RPQ;
  const int64_t grid = (n + rows_per_block - 1) / rows_per_block;
  kern<<<(unsigned)grid, 256, smem, st>>>(indptr, idx, static_cast<const ValT*>(val), n, g, V, mc, Y, lds);
  note_launches(1);
  return cudaGetLastError();
}

template <typename ValT>
static cudaError_t fwd_strict_v(int ld, const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                                int32_t g, const float* V, const float* mc, float* Y, int lds, cudaStream_t st) {
  switch (ld) {
    case 32: return fwd_strict_t<32, ValT>(indptr, idx, val, n, g, V, mc, Y, lds, st);
    case 64: return fwd_strict_t<64, ValT>(indptr, idx, val, n, g, V, mc, Y, lds, st);
    case 96: return fwd_strict_t<96, ValT>(indptr, idx, val, n, g, V, mc, Y, lds, st);
    case 128: return fwd_strict_t<128, ValT>(indptr, idx, val, n, g, V, mc, Y, lds, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fwd_strict(int dtype, int ld, const int64_t* indptr, const int32_t* idx, const void* val,
                              int64_t n, int32_t g, const float* V, const float* mc, float* Y, cudaStream_t st,
                              int lds) {
  if (n == 0) return cudaSuccess;
  if (lds == 0) lds = ld;
  if (lds < ld || (lds & 3)) return cudaErrorInvalidValue;
  switch (dtype) {
    case 0: return fwd_strict_v<float>(ld, indptr, idx, val, n, g, V, mc, Y, lds, st);
    case 1: return fwd_strict_v<__nv_bfloat16>(ld, indptr, idx, val, n, g, V, mc, Y, lds, st);
    default: return fwd_strict_v<__half>(ld, indptr, idx, val, n, g, V, mc, Y, lds, st);
  }
}

template <int LD, typename ValT>
static cudaError_t rmat_strict_t(const int64_t* indptr, const int32_t* tptr, const uint8_t* cell, const void* cval,
                                 int64_t n, int32_t g, int32_t nslots, const int32_t* slot2gene, int ranges,
                                 const float* Q, int lds, float* part, cudaStream_t st) {
  constexpr int GPW = LD <= 64 ? 32 : 16;  // slots per warp (strict_genes_per_warp)
  const size_t smem = (size_t)2 * kStrictTile * LD * sizeof(float);
  auto kern = k_rmat_strict_q<LD, GPW / 4, ValT>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (nslots % (8 * GPW) != 0) return cudaErrorInvalidValue;
  const int64_t n_tiles = (n + kStrictTile - 1) / kStrictTile;
  const int64_t per = (n_tiles + ranges - 1) / ranges;
  dim3 grid((unsigned)ranges, (unsigned)(nslots / (8 * GPW)));
  kern<<<grid, 256, smem, st>>>(indptr, tptr, cell, static_cast<const ValT*>(cval), n, g, nslots, slot2gene, per, Q,
                                lds, part);
  note_launches(1);
  return cudaGetLastError();
}

template <typename ValT>
static cudaError_t rmat_strict_v(int ld, const int64_t* indptr, const int32_t* tptr, const uint8_t* cell,
                                 const void* cval, int64_t n, int32_t g, int32_t nslots, const int32_t* slot2gene,
                                 int ranges, const float* Q, int lds, float* part, cudaStream_t st) {
  switch (ld) {
    case 32: return rmat_strict_t<32, ValT>(indptr, tptr, cell, cval, n, g, nslots, slot2gene, ranges, Q, lds, part, st);
    case 64: return rmat_strict_t<64, ValT>(indptr, tptr, cell, cval, n, g, nslots, slot2gene, ranges, Q, lds, part, st);
    case 96: return rmat_strict_t<96, ValT>(indptr, tptr, cell, cval, n, g, nslots, slot2gene, ranges, Q, lds, part, st);
    case 128:
      return rmat_strict_t<128, ValT>(indptr, tptr, cell, cval, n, g, nslots, slot2gene, ranges, Q, lds, part, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_rmat_strict(int dtype, int ld, const int64_t* indptr, const int32_t* tptr, const uint8_t* cell,
                               const void* cval, int64_t n, int32_t g, int32_t nslots, const int32_t* slot2gene,
                               int ranges, const float* Q, float* part, cudaStream_t st, int lds) {
  if (lds == 0) lds = ld;
  if (lds < ld || (lds & 3)) return cudaErrorInvalidValue;
  switch (dtype) {
    case 0:
      return rmat_strict_v<float>(ld, indptr, tptr, cell, cval, n, g, nslots, slot2gene, ranges, Q, lds, part, st);
    case 1:
      return rmat_strict_v<__nv_bfloat16>(ld, indptr, tptr, cell, cval, n, g, nslots, slot2gene, ranges, Q, lds,
                                          part, st);
    default:
      return rmat_strict_v<__half>(ld, indptr, tptr, cell, cval, n, g, nslots, slot2gene, ranges, Q, lds, part, st);
  }
}

}  // namespace scx
