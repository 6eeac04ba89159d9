// Host orchestration and C ABI of the randomized PCA (libscxpca.so).
//
// A plan owns (or borrows) the device CSR, its per-gene statistics and every
// work buffer; running it enqueues the whole power loop and Rayleigh-Ritz
// step on one stream with no host synchronisation until the end.
//
// Power loop (same step order as run_power_loop,
// scx-gpu/src/pca_operator.rs:100-119):
//   Y = (X - mu) Omega ; qr(Y) ; [ Z = (X - mu)^T Q ; qr(Z) ; Y = (X - mu) Z ;
//   qr(Y) ] x q ; B = (X - mu)^T Q
// qr(Y) is a Cholesky QR whose Gram Y^T Y is accumulated in FP64 from the
// stored FP32 Y; inside the loop Q = Y R^{-1} stays implicit
// (Z = (X^T Y - mu (1^T Y)^T) R^{-1}), and the last Q is formed explicitly
// and re-orthonormalised (second Cholesky pass folded into B and the
// embeddings) before the final projection.  qr(Z) is one CholeskyQR pass in
// FP64.
// The SVD of B is an FP64 Jacobi eigendecomposition of B^T B on the device.
#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/scxpca.h"
#include "common.cuh"
#include "launch.h"
#include "power_loop.h"

using namespace scx;

namespace scx {
static std::atomic<int64_t> g_launches{0};
void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace scx

namespace {

struct Failure {
  int32_t code;
  std::string msg;
};

[[noreturn]] void fail(int32_t code, const std::string& msg) { throw Failure{code, msg}; }

void ck(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  int32_t code = (e == cudaErrorMemoryAllocation) ? SCXPCA_OUT_OF_MEMORY : SCXPCA_CUDA_ERROR;
  fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(expr) ck((expr), #expr)

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  size_t n = std::min(len - 1, msg.size());
  memcpy(err, msg.data(), n);
  err[n] = '\0';
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
      fail(SCXPCA_CUDA_ERROR, "no CUDA device is available");
    if (dev < 0 || dev >= count)
      fail(SCXPCA_INVALID_ARGUMENT, "device_ordinal " + std::to_string(dev) + " out of range (" +
                                        std::to_string(count) + " devices)");
    CK(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Device memory of the plans comes from one stream-ordered pool per device
// that keeps what is freed (release threshold: unlimited), so a plan built
// after another one reuses its memory without mapping pages again, and
// freeing costs a stream operation instead of a device-wide cudaFree.  Every
// pooled allocation and free is ordered on one allocation stream per device
// (so freed blocks are always reusable by the next allocation), fenced
// against the stream that uses the memory by events.  The pool's memory
// stays reserved by the process until it exits.
struct DevicePool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t st = nullptr;  // allocation stream
};

DevicePool& pool_for(int dev) {
  static std::mutex mu;
  static DevicePool pools[256];
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 256) fail(SCXPCA_INVALID_ARGUMENT, "device ordinal out of range");
  DevicePool& dp = pools[dev];
  if (!dp.pool) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    CK(cudaMemPoolCreate(&dp.pool, &props));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(dp.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    CK(cudaStreamCreateWithFlags(&dp.st, cudaStreamNonBlocking));
  }
  return dp;
}

// Order `to` after the work enqueued so far on `from`.
void stream_fence(cudaStream_t from, cudaStream_t to) {
  cudaEvent_t e;
  CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CK(cudaEventRecord(e, from));
  CK(cudaStreamWaitEvent(to, e, 0));
  cudaEventDestroy(e);
}

// Phase timing of the calling thread's one-shot call (scxpca_randomized):
// when on, each phase boundary records an event on the plan's stream, and
// the intervals between consecutive boundaries (device clock, idle gaps
// while the host prepares the next phase included) become the phases.
struct PhaseRec {
  bool on = false;
  cudaStream_t st = nullptr;
  int next = 0;
  cudaEvent_t ev[SCXPCA_NUM_PHASES + 1] = {};
  double ms[SCXPCA_NUM_PHASES] = {};
  double wall_ms = 0.0;
};
thread_local PhaseRec t_phase;

// Mark the end of phase `ph` (and of every phase before it not yet marked).
void phase_mark(int ph, cudaStream_t st) {
  PhaseRec& r = t_phase;
  if (!r.on) return;
  if (r.next == 0) {  // the first mark opens the clock
    if (cudaEventCreate(&r.ev[0]) != cudaSuccess || cudaEventRecord(r.ev[0], st) != cudaSuccess) {
      cudaGetLastError();
      r.on = false;
      return;
    }
    r.st = st;
    r.next = 1;
  }
  while (r.next <= ph + 1 && r.next <= SCXPCA_NUM_PHASES) {
    if (cudaEventCreate(&r.ev[r.next]) != cudaSuccess || cudaEventRecord(r.ev[r.next], st) != cudaSuccess) {
      cudaGetLastError();
      r.on = false;
      return;
    }
    ++r.next;
  }
}

// Allocation context of the calling thread: DevBufs allocated inside a
// PoolScope come from the device's pool and are used on the scope's stream.
struct AllocCtx {
  DevicePool* dp = nullptr;
  cudaStream_t use = nullptr;
};
thread_local AllocCtx t_alloc;

struct PoolScope {
  AllocCtx prev;
  PoolScope(int dev, cudaStream_t use) : prev(t_alloc) { t_alloc = AllocCtx{&pool_for(dev), use}; }
  ~PoolScope() { t_alloc = prev; }
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevicePool* dp = nullptr;   // pool of a pooled allocation
  cudaStream_t st = nullptr;  // stream the pooled memory is used on
  bool pooled = false;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) {
      if (pooled) {  // after the work already enqueued on the using stream
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
          cudaEventRecord(e, st);
          cudaStreamWaitEvent(dp->st, e, 0);
          cudaEventDestroy(e);
        }
        cudaFreeAsync(p, dp->st);
      } else {
        cudaFree(p);
      }
    }
    p = nullptr;
    bytes = 0;
    pooled = false;
  }
  void alloc(size_t b) {
    if (b <= bytes && p) return;
    release();
    if (b == 0) b = 16;
    cudaError_t e;
    if (t_alloc.dp) {
      e = cudaMallocFromPoolAsync(&p, b, t_alloc.dp->pool, t_alloc.dp->st);
      if (e == cudaSuccess) {
        dp = t_alloc.dp;
        st = t_alloc.use;
        pooled = true;
        stream_fence(dp->st, st);  // the using stream starts after the allocation
      }
    } else {
      e = cudaMalloc(&p, b);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      pooled = false;
      fail(SCXPCA_OUT_OF_MEMORY, "device allocation of " + std::to_string(b) + " bytes failed: " +
                                     cudaGetErrorString(e));
    }
    bytes = b;
  }
  // take over another buffer's memory
  void adopt(DevBuf& o) {
    release();
    p = o.p;
    bytes = o.bytes;
    dp = o.dp;
    st = o.st;
    pooled = o.pooled;
    o.p = nullptr;
    o.bytes = 0;
    o.pooled = false;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

size_t dtype_size(int dt) { return dt == SCXPCA_F32 ? 4 : 2; }

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

struct scxpca_plan {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  scxpca_params params{};
  int64_t n = 0, g = 0, nnz = 0, k = 0, ld = 0, nc = 0;
  int in_dtype = 0, dtype = 0;  // input and compute value types
  bool centered = true;
  bool scaled = false;
  double clip = 0.0;

  const int64_t* indptr = nullptr;
  const int32_t* idx = nullptr;
  const void* val = nullptr;
  DevBuf b_indptr, b_idx, b_val, b_stage;

  // statistics
  int stats_parts = 0;
  DevBuf stats_part, stats_out, d_mu, d_inv_std, d_cshift;
  std::vector<double> mean_x, std_x, col_sum, col_sq;  // working-matrix sums
  double total_var = 0.0;
  bool total_var_recomputed = false;

  // CUDA-core transposed product: the tile-CSC copy (slots balanced by
  // stored-entry count) and its per-range partials; the row-block pointer
  // table of the gradient's SDDMM (and of the atomic fallback for matrices
  // too wide for the tile-CSC copy) is built on first use
  bool strict_csc = false;
  int nslots = 0, strict_ranges = 0;
  DevBuf csc_tptr, csc_cell, csc_val, d_slot2gene;
  int nb = 0, nchunks = 0;
  int64_t rows_per_chunk = 0;
  bool rbp_built = false;
  DevBuf rbp, wpart;

  // dense work
  int gram_parts = 0, gram_parts_small = 0;
  DevBuf Y, W, Z, V, mc, gpart, G, R, Rinv, Rinv_f, R2inv, eye, evals, evecs, sigma, comps,
      M_emb, U, status, omega_stage;
  size_t device_bytes = 0;

  double tau = 1e-8;

  // tensor-core path (16-bit values): tile-chunk packed matrix, 16-bit dense
  // operands and their TMA maps
  bool use_tc = false;
  int fmt16 = 1;  // 1 = bf16, 0 = f16
  int n_chunks = 0, tc_gene_groups = 0, tc_row_groups = 0;
  int tc_gram_parts = 0;  // partials of the tensor-core Gram (0: one per SM)
  // embeddings on tensor cores from Q's 16-bit image (ld 64); a batch's plans
  // keep the CUDA-core product, which its batched embedding launch shares, and
  // SCXPCA_EMBED_TC=0 keeps it for any plan
  bool embed_tc = !(getenv("SCXPCA_EMBED_TC") && getenv("SCXPCA_EMBED_TC")[0] == '0');
  // 16-bit images (column 2 j = hi, 2 j + 1 = lo of column j) of the dense
  // operands of the tensor-core products: V (g x 2 ld) and the tall Y/Q (n x 2 ld)
  DevBuf tf_meta, tf_ent, Vimg, Yimg, tc_part, tc_err;
  CUtensorMap vmap{}, qmap{};

  // differentiation: raw per-gene centre c and scale s of X~ = (X - 1 c^T) diag(s)
  // (device, n_vars each), whether the last run's Ritz state (B in Z, E, evals)
  // is intact, and the backward pass's work buffers
  DevBuf d_center_raw, d_scale_raw;
  bool affine = false;
  bool rows_resorted = false;
  bool run_valid = false;
  DevBuf bw_Vk, bw_H, bw_A, bw_X, bw_R, bw_P, bw_Ap, bw_Proj, bw_T, bw_M, bw_vec, bw_colD, bw_sumDP, bw_part,
      bw_cpart;

  // streamed plan: the matrix stays in the caller's host memory and every
  // product uploads it again in row shards of whole 128-row tiles, two device
  // slots deep (the copy of shard s + 1 overlaps the work on shard s)
  struct Shard {
    int64_t r0, r1, p0, p1;  // rows [r0, r1), stored entries [p0, p1)
    CUtensorMap qmap;        // TMA map of the shard's rows of the tall image
    int row_groups;          // partials of its tensor-core transposed product
    int ranges;              // partials of its CUDA-core transposed product
  };
  struct Slot {
    DevBuf ip, idx, vin, vwork, counts, seg, ent, meta, tptr, cell, cval;
  };
  bool streaming = false;
  bool stream_sort = false;       // re-sort every shard after its upload
  bool stream_transform = false;  // working values differ from the input's
  int stream_mode = 0;            // value transform mode (k_transform_values)
  const int64_t* h_indptr = nullptr;
  const int32_t* h_idx = nullptr;
  const void* h_val = nullptr;
  std::vector<Shard> shards;
  int64_t shard_rows_max = 0, shard_nnz_max = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
  Slot slot[2];
  DevBuf t_mu, t_inv_std, t_cshift, d_gene2slot;

  // baseline-aware (PFlog) plan: the working matrix is [delta | b] with the
  // baseline as its last column; g_user = the caller's gene count (g - 1 for
  // PFlog, g otherwise)
  bool pflog = false;
  int64_t g_user = 0;

  // opt-in stage timing
  bool profiling = false;

  // A plan run replayed as a CUDA graph: recorded on the second run with the
  // same (power iterations, seed, omega, embeddings buffer), replayed while
  // they stay the same (one launch instead of ~375).
  struct RunGraph {
    cudaGraphExec_t exec = nullptr;
    int64_t q = -1;
    uint64_t seed = 0;
    const float* omega = nullptr;
    float* U = nullptr;
    int64_t launches = 0;  // kernels in the graph
    bool seen = false;     // the key was run once without a graph
  } rg;
  std::vector<cudaEvent_t> events;
  std::vector<std::pair<int, int>> marks;  // (stage, index of the begin event)
  int events_used = 0;
  scxpca_profile prof{};

  ~scxpca_plan() {
    if (rg.exec) cudaGraphExecDestroy(rg.exec);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    if (copy_stream) {
      cudaStreamSynchronize(copy_stream);
      cudaStreamDestroy(copy_stream);
    }
    for (int i = 0; i < 2; ++i) {
      if (ev_copied[i]) cudaEventDestroy(ev_copied[i]);
      if (ev_free[i]) cudaEventDestroy(ev_free[i]);
    }
  }
};

namespace {

// ---------------------------------------------------------------------------
// validation of arguments (scx-accel/src/pca/cpu.rs:979-997; gpu_pca.rs:433-446)
// ---------------------------------------------------------------------------
void validate_params(const scxpca_csr* x, const scxpca_params* p) {
  if (!x || !p) fail(SCXPCA_INVALID_ARGUMENT, "null csr or params");
  if (x->n_obs < 0 || x->n_vars < 0 || x->nnz < 0)
    fail(SCXPCA_INVALID_ARGUMENT, "negative matrix dimension");
  if (p->n_components <= 0) fail(SCXPCA_INVALID_ARGUMENT, "n_components must be > 0");
  if (x->n_obs == 0 || x->n_vars == 0) fail(SCXPCA_INVALID_ARGUMENT, "matrix must be non-empty");
  int64_t mn = std::min(x->n_obs, x->n_vars);
  if (p->n_components > mn)
    fail(SCXPCA_INVALID_ARGUMENT, "n_components (" + std::to_string(p->n_components) +
                                      ") exceeds matrix rank bound min(n_obs, n_vars) = " +
                                      std::to_string(mn));
  if (p->n_oversamples < 0 || p->n_power_iterations < 0)
    fail(SCXPCA_INVALID_ARGUMENT, "n_oversamples and n_power_iterations must be >= 0");
  if (x->n_vars > INT32_MAX) fail(SCXPCA_INVALID_ARGUMENT, "n_vars exceeds int32 index range");
  if (x->values_dtype < 0 || x->values_dtype > 2) fail(SCXPCA_INVALID_ARGUMENT, "bad values_dtype");
  if (p->math_mode < 0 || p->math_mode > 2) fail(SCXPCA_INVALID_ARGUMENT, "bad math_mode");
  if (p->qr_method < 0 || p->qr_method > 1) fail(SCXPCA_INVALID_ARGUMENT, "bad qr_method");
  if (x->nnz > 0 && (!x->indices || !x->values)) fail(SCXPCA_INVALID_ARGUMENT, "null CSR arrays");
  if (!x->indptr) fail(SCXPCA_INVALID_ARGUMENT, "null indptr");
  if (!std::isfinite(p->clip_max)) fail(SCXPCA_INVALID_ARGUMENT, "clip_max must be finite");
  int64_t k = std::min({p->n_components + p->n_oversamples, x->n_vars, x->n_obs});
  if (k > kMaxKWide)
    fail(SCXPCA_UNSUPPORTED, "sketch width k = min(n_components + n_oversamples, n_vars, n_obs) = " +
                                 std::to_string(k) + " exceeds the supported maximum " +
                                 std::to_string(kMaxKWide));
}

// Pieces a host matrix's entries are copied in (statistics overlap the copy).
constexpr int kUploadPieces = 8;

// Reduce the statistics partials already written to stats_part and bring
// the column sums and sums of squares to the host.
void stats_finish(scxpca_plan* pl, std::vector<double>& sums, std::vector<double>& sq) {
  CK(launch_col_stats_reduce(pl->stats_part.as<double>(), pl->stats_parts, (int32_t)pl->g,
                             pl->stats_out.as<double>(), pl->stream, pl->num_sms));
  std::vector<double> host(2 * pl->g);
  CK(cudaMemcpyAsync(host.data(), pl->stats_out.p, sizeof(double) * 2 * pl->g,
                     cudaMemcpyDeviceToHost, pl->stream));
  CK(cudaStreamSynchronize(pl->stream));
  sums.assign(host.begin(), host.begin() + pl->g);
  sq.assign(host.begin() + pl->g, host.end());
}

void stats_pass(scxpca_plan* pl, const void* val, int dtype, std::vector<double>& sums,
                std::vector<double>& sq) {
  CK(launch_col_stats(dtype, pl->idx, val, pl->nnz, (int32_t)pl->g, pl->stats_part.as<double>(),
                      pl->stats_parts, pl->stats_out.as<double>(), pl->stream, pl->num_sms));
  std::vector<double> host(2 * pl->g);
  CK(cudaMemcpyAsync(host.data(), pl->stats_out.p, sizeof(double) * 2 * pl->g,
                     cudaMemcpyDeviceToHost, pl->stream));
  CK(cudaStreamSynchronize(pl->stream));
  sums.assign(host.begin(), host.begin() + pl->g);
  sq.assign(host.begin() + pl->g, host.end());
}

void upload(DevBuf& buf, const std::vector<double>& v, cudaStream_t st) {
  buf.alloc(sizeof(double) * v.size());
  CK(cudaMemcpyAsync(buf.p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, st));
}

// Closed-form total variance with the cancellation guard
// (scx-sparse/src/csr.rs:868-880, moments.rs:288-308, scx-accel cpu.rs:1066-1171).
void compute_total_variance(scxpca_plan* pl) {
  const double n = (double)pl->n;
  const double denom = std::max(n - 1.0, 1.0);
  double sumsq = 0.0, meansq = 0.0;
  for (int64_t j = 0; j < pl->g; ++j) sumsq += pl->col_sq[j];
  if (!pl->centered) {
    pl->total_var = sumsq / denom;
    return;
  }
  double total = 0.0;
  std::vector<double> mu(pl->g);
  for (int64_t j = 0; j < pl->g; ++j) {
    mu[j] = pl->col_sum[j] / n;
    total += pl->col_sq[j] - n * mu[j] * mu[j];
    meansq += mu[j] * mu[j];
  }
  pl->total_var = total / denom;
  if (sumsq <= 0.0) return;                          // degenerate: exact zero
  if (!(sumsq - meansq * n <= 1e-7 * sumsq)) return;  // usable
  // Cancelled: stable recompute sum (x - mu)^2 over stored entries plus
  // implicit zeros (n - nnz_j) mu_j^2, on the device.
  DevBuf dmu, shifted;
  upload(dmu, mu, pl->stream);
  shifted.alloc(sizeof(float) * std::max<int64_t>(pl->nnz, 1));
  // (x - mu) in FP32 is exact enough for a variance that the FP64 closed form lost.
  std::vector<double> zero(pl->g, 0.0), one(pl->g, 1.0);
  DevBuf dz, d1;
  upload(dz, zero, pl->stream);
  upload(d1, one, pl->stream);
  CK(launch_transform_values(pl->dtype, 0, pl->idx, pl->val, shifted.p, pl->nnz, 1, dmu.as<double>(),
                             d1.as<double>(), dz.as<double>(), 0.0, pl->stream, pl->num_sms));
  std::vector<double> s1, s2;
  stats_pass(pl, shifted.p, 0, s1, s2);
  // nnz per gene from sum x and sum (x - mu): nnz_j = (sum x - sum(x - mu)) / mu_j
  double t = 0.0;
  for (int64_t j = 0; j < pl->g; ++j) {
    double nnz_j = (mu[j] != 0.0) ? std::round((pl->col_sum[j] - s1[j]) / mu[j]) : 0.0;
    double zeros = std::max(n - nnz_j, 0.0);
    t += s2[j] + zeros * mu[j] * mu[j];
  }
  pl->total_var = t / denom;
  pl->total_var_recomputed = true;
}

// Explicit centre / scale vectors of an affine plan (either may be null).
struct AffineSpec {
  const double* center;
  const double* scale;
  int32_t memory;  // scxpca_memory of both vectors
};

std::vector<double> read_vec(const double* src, int64_t n, int32_t memory, double fill, cudaStream_t st) {
  std::vector<double> v(n, fill);
  if (!src) return v;
  if (memory == SCXPCA_MEM_DEVICE) {
    CK(cudaMemcpyAsync(v.data(), src, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  } else {
    memcpy(v.data(), src, sizeof(double) * n);
  }
  return v;
}

// Row-block pointer table (the SDDMM of the gradient, and the transposed
// product of matrices too wide for the tile-CSC copy), built on first use.
void ensure_rbp(scxpca_plan* pl) {
  if (pl->rbp_built) return;
  PoolScope pool_scope(pl->device, pl->stream);
  pl->rbp.alloc(sizeof(int32_t) * pl->n * (pl->nb + 1));
  CK(launch_row_block_ptr(pl->indptr, pl->idx, pl->n, pl->nb, kTransposeGeneBlock, pl->rbp.as<int32_t>(),
                          pl->stream, pl->num_sms));
  if (!pl->strict_csc && !pl->use_tc)
    pl->wpart.alloc(sizeof(float) * (size_t)pl->nchunks * pl->g * pl->ld);
  pl->rbp_built = true;
}

// Tile-CSC copy of the working matrix for the CUDA-core transposed product:
// per-gene stored-entry counts -> balanced slot assignment (host) -> the
// copy, and the per-range partial buffer.
// Column panel the CUDA-core SpMM pair takes per launch: the whole sketch up
// to 128 columns, else 128-column panels of it.
int panel_width(const scxpca_plan* pl) { return (int)std::min<int64_t>(pl->ld, kPanel); }

void build_tile_csc(scxpca_plan* pl) {
  cudaStream_t st = pl->stream;
  const int64_t n = pl->n, g = pl->g, nnz = pl->nnz;
  DevBuf counts;
  counts.alloc(sizeof(int32_t) * g);
  CK(cudaMemsetAsync(counts.p, 0, sizeof(int32_t) * g, st));
  CK(launch_gene_counts(pl->idx, nnz, counts.as<int32_t>(), st, pl->num_sms));
  std::vector<int32_t> hc(g);
  CK(cudaMemcpyAsync(hc.data(), counts.p, sizeof(int32_t) * g, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::vector<int32_t> gene2slot, slot2gene;
  const int pw = panel_width(pl);
  strict_assign_slots(hc, pw, gene2slot, slot2gene);
  DevBuf d_g2s;
  d_g2s.alloc(sizeof(int32_t) * g);
  CK(cudaMemcpyAsync(d_g2s.p, gene2slot.data(), sizeof(int32_t) * g, cudaMemcpyHostToDevice, st));
  pl->d_slot2gene.alloc(sizeof(int32_t) * pl->nslots);
  CK(cudaMemcpyAsync(pl->d_slot2gene.p, slot2gene.data(), sizeof(int32_t) * pl->nslots, cudaMemcpyHostToDevice,
                     st));
  const int64_t n_tiles = (n + kStrictTile - 1) / kStrictTile;
  pl->csc_tptr.alloc(sizeof(int32_t) * (size_t)n_tiles * (pl->nslots + 1));
  pl->csc_cell.alloc(std::max<int64_t>(nnz, 1));
  pl->csc_val.alloc(dtype_size(pl->dtype) * std::max<int64_t>(nnz, 1));
  CK(launch_tile_csc(pl->dtype, pl->indptr, pl->idx, pl->val, n, d_g2s.as<int32_t>(), pl->nslots,
                     pl->csc_tptr.as<int32_t>(), pl->csc_cell.as<uint8_t>(), pl->csc_val.p, st, pl->num_sms));
  // ranges: about four blocks per SM over all gene blocks, for balance
  const int gblocks = pl->nslots / (8 * strict_genes_per_warp(pw));
  pl->strict_ranges = (int)std::max<int64_t>(1, std::min<int64_t>(n_tiles, (4 * pl->num_sms + gblocks - 1) / gblocks));
  pl->wpart.alloc(sizeof(float) * (size_t)pl->strict_ranges * g * pw);
  CK(cudaStreamSynchronize(st));  // the host vectors above go out of scope
}

// ---------------------------------------------------------------------------
// Streamed plan: the matrix stays in host memory, products take it in row
// shards (the counterpart of StreamingPcaOperator and drive_row_segments,
// scx-gpu/src/linear_operator.rs:61-288).  Each shard is uploaded on a copy
// stream into one of two device slots and prepared on the plan's stream
// (indptr rebased, rows sorted when the input needs it, values transformed,
// and the shard packed into the tile format of the product that reads it),
// so the upload of shard s + 1 overlaps the work on shard s.  Everything
// tall (Y, its 16-bit image) stays resident; a shard's rows are whole
// 128-row tiles of it.
// ---------------------------------------------------------------------------
constexpr int64_t kShardEntriesMax = int64_t(1) << 26;  // stored entries per shard at most

void alloc_work_buffers(scxpca_plan* pl);

// Bytes one device slot needs per stored entry and per row.
double slot_bytes_per_entry(const scxpca_plan* pl, bool tc) {
  double b = 4.0 + (double)dtype_size(pl->in_dtype) + (double)dtype_size(pl->dtype);
  b += tc ? 4.0 * 1.2 : 1.0 + (double)dtype_size(pl->dtype);
  return b;
}

void shard_upload(scxpca_plan* pl, size_t s, int k) {
  const scxpca_plan::Shard& sh = pl->shards[s];
  scxpca_plan::Slot& sl = pl->slot[k];
  cudaStream_t cs = pl->copy_stream;
  const int64_t rows = sh.r1 - sh.r0, cnt = sh.p1 - sh.p0;
  CK(cudaStreamWaitEvent(cs, pl->ev_free[k], 0));
  CK(cudaMemcpyAsync(sl.ip.p, pl->h_indptr + sh.r0, sizeof(int64_t) * (rows + 1), cudaMemcpyHostToDevice, cs));
  if (cnt) {
    CK(cudaMemcpyAsync(sl.idx.p, pl->h_idx + sh.p0, sizeof(int32_t) * cnt, cudaMemcpyHostToDevice, cs));
    const size_t vs = dtype_size(pl->in_dtype);
    CK(cudaMemcpyAsync(sl.vin.p, static_cast<const char*>(pl->h_val) + vs * sh.p0, vs * cnt, cudaMemcpyHostToDevice,
                       cs));
  }
  CK(cudaEventRecord(pl->ev_copied[k], cs));
}

// Bring an uploaded shard to the working form on the plan's stream: the
// rebased indptr, sorted rows when needed, working values (`work`), and, per
// `pack` (0 none, 1 tensor-core tiles, 2 tile-CSC), the packed copy.
const void* shard_prepare(scxpca_plan* pl, size_t s, int k, bool work, int pack) {
  const scxpca_plan::Shard& sh = pl->shards[s];
  scxpca_plan::Slot& sl = pl->slot[k];
  cudaStream_t st = pl->stream;
  const int64_t rows = sh.r1 - sh.r0, cnt = sh.p1 - sh.p0;
  CK(cudaStreamWaitEvent(st, pl->ev_copied[k], 0));
  CK(launch_rebase_indptr(sl.ip.as<int64_t>(), rows, sh.p0, st, pl->num_sms));
  if (pl->stream_sort) CK(launch_sort_rows(pl->in_dtype, sl.ip.as<int64_t>(), sl.idx.as<int32_t>(), sl.vin.p, rows, st,
                                           pl->num_sms));
  const void* vals = sl.vin.p;
  if (work && pl->stream_transform) {
    CK(launch_transform_values(pl->in_dtype, pl->dtype, sl.idx.as<int32_t>(), sl.vin.p, sl.vwork.p, cnt,
                               pl->stream_mode, pl->t_mu.as<double>(), pl->t_inv_std.as<double>(),
                               pl->t_cshift.as<double>(), pl->clip, st, pl->num_sms));
    vals = sl.vwork.p;
  }
  if (pack == 1) {
    const int64_t nseg = (rows + 127) / 128 * pl->n_chunks;
    CK(tile_format_count(sl.ip.as<int64_t>(), sl.idx.as<int32_t>(), rows, pl->n_chunks, sl.counts.as<int64_t>(), st,
                         pl->num_sms));
    CK(launch_exclusive_scan_i64(sl.counts.as<int64_t>(), nseg, sl.seg.as<int64_t>(), st));
    CK(cudaMemsetAsync(sl.ent.p, 0, sizeof(uint32_t) * (size_t)(cnt + 3 * nseg + 4), st));
    CK(tile_format_fill(sl.ip.as<int64_t>(), sl.idx.as<int32_t>(), vals, rows, pl->n_chunks, sl.seg.as<int64_t>(),
                        sl.ent.as<uint32_t>(), sl.meta.p, st, pl->num_sms));
  } else if (pack == 2) {
    CK(launch_tile_csc(pl->dtype, sl.ip.as<int64_t>(), sl.idx.as<int32_t>(), vals, rows, pl->d_gene2slot.as<int32_t>(),
                       pl->nslots, sl.tptr.as<int32_t>(), sl.cell.as<uint8_t>(), sl.cval.p, st, pl->num_sms));
  }
  return vals;
}

void shard_release(scxpca_plan* pl, int k) { CK(cudaEventRecord(pl->ev_free[k], pl->stream)); }

// Run `body(s, slot)` over every shard in order, each after its upload, with
// the upload of the next shard issued ahead.
template <typename F>
void for_each_shard(scxpca_plan* pl, F&& body) {
  const size_t ns = pl->shards.size();
  for (size_t s = 0; s < ns; ++s) {
    shard_upload(pl, s, (int)(s & 1));
    if (s >= 1) {
      body(s - 1, (int)((s - 1) & 1));
      shard_release(pl, (int)((s - 1) & 1));
    }
  }
  if (ns) {
    body(ns - 1, (int)((ns - 1) & 1));
    shard_release(pl, (int)((ns - 1) & 1));
  }
}

// Per-gene statistics over the shards, of the input (work = false) or the
// working values (work = true); optional validation flags and gene counts.
void stream_stats(scxpca_plan* pl, bool work, std::vector<double>& sums, std::vector<double>& sq, int32_t* flags,
                  int32_t* gene_counts) {
  cudaStream_t st = pl->stream;
  const int64_t g = pl->g;
  for_each_shard(pl, [&](size_t s, int k) {
    const scxpca_plan::Shard& sh = pl->shards[s];
    scxpca_plan::Slot& sl = pl->slot[k];
    const int64_t rows = sh.r1 - sh.r0, cnt = sh.p1 - sh.p0;
    const void* vals = shard_prepare(pl, s, k, work, 0);
    if (flags)
      CK(launch_validate_csr(pl->in_dtype, sl.ip.as<int64_t>(), sl.idx.as<int32_t>(), sl.vin.p, rows, g, cnt, flags,
                             st, pl->num_sms));
    if (gene_counts) CK(launch_gene_counts(sl.idx.as<int32_t>(), cnt, gene_counts, st, pl->num_sms));
    CK(launch_col_stats(work ? pl->dtype : pl->in_dtype, sl.idx.as<int32_t>(), vals, cnt, (int32_t)g,
                        pl->stats_part.as<double>(), pl->stats_parts, pl->stats_out.as<double>(), st, pl->num_sms,
                        s > 0 ? 1 : 0));
  });
  std::vector<double> host(2 * g);
  CK(cudaMemcpyAsync(host.data(), pl->stats_out.p, sizeof(double) * 2 * g, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  sums.assign(host.begin(), host.begin() + g);
  sq.assign(host.begin() + g, host.end());
}

// Streamed products (the tall operands and outputs stay resident).
void stream_forward(scxpca_plan* pl, bool f32) {
  cudaStream_t st = pl->stream;
  const int64_t ld = pl->ld;
  for_each_shard(pl, [&](size_t s, int k) {
    const scxpca_plan::Shard& sh = pl->shards[s];
    scxpca_plan::Slot& sl = pl->slot[k];
    const int64_t rows = sh.r1 - sh.r0;
    const void* vals = shard_prepare(pl, s, k, true, pl->use_tc ? 1 : 0);
    if (pl->use_tc) {
      CK(launch_fwd_tc((int)ld, sl.ent.as<uint32_t>(), sl.meta.p, rows, pl->n_chunks, &pl->vmap, pl->mc.as<float>(),
                       f32 ? pl->Y.as<float>() + sh.r0 * ld : nullptr, pl->Yimg.as<uint16_t>() + sh.r0 * 2 * ld,
                       pl->fmt16, pl->tc_err.as<int>(), st, pl->num_sms));
    } else {
      CK(launch_fwd_strict(pl->dtype, (int)ld, sl.ip.as<int64_t>(), sl.idx.as<int32_t>(), vals, rows, (int32_t)pl->g,
                           pl->V.as<float>(), pl->centered ? pl->mc.as<float>() : nullptr,
                           pl->Y.as<float>() + sh.r0 * ld, st));
    }
  });
}

void stream_rmat(scxpca_plan* pl, const float* A) {
  cudaStream_t st = pl->stream;
  const int64_t ld = pl->ld, g = pl->g;
  for_each_shard(pl, [&](size_t s, int k) {
    const scxpca_plan::Shard& sh = pl->shards[s];
    scxpca_plan::Slot& sl = pl->slot[k];
    const int64_t rows = sh.r1 - sh.r0;
    shard_prepare(pl, s, k, true, pl->use_tc ? 1 : 2);
    if (pl->use_tc) {
      CK(launch_rmat_tc((int)ld, sl.ent.as<uint32_t>(), sl.meta.p, rows, pl->n_chunks, g, pl->tc_gene_groups,
                        sh.row_groups, &sh.qmap, pl->tc_part.as<float>(), pl->fmt16, pl->tc_err.as<int>(), st));
      CK(launch_reduce_rows_f32(pl->tc_part.as<float>(), sh.row_groups, g * ld, pl->W.as<double>(), s > 0 ? 1 : 0,
                                st, pl->num_sms));
    } else {
      CK(launch_rmat_strict(pl->dtype, (int)ld, sl.ip.as<int64_t>(), sl.tptr.as<int32_t>(), sl.cell.as<uint8_t>(),
                            sl.cval.p, rows, (int32_t)g, pl->nslots, pl->d_slot2gene.as<int32_t>(), sh.ranges,
                            A + sh.r0 * ld, pl->wpart.as<float>(), st));
      CK(launch_reduce_rows_f32(pl->wpart.as<float>(), sh.ranges, g * ld, pl->W.as<double>(), s > 0 ? 1 : 0, st,
                                pl->num_sms));
    }
  });
}

// The transform of the input values into the working values (scaling with
// clipping; or a plain conversion to the compute type) from the input
// statistics: fills mode/mu/inv_std/cshift like the resident path and
// returns whether the working values differ from the input's.
bool value_transform(scxpca_plan* pl, const std::vector<double>& sx, const std::vector<double>& sxx, int& mode,
                     std::vector<double>& mu, std::vector<double>& inv_std, std::vector<double>& cshift) {
  const int64_t g = pl->g, n = pl->n;
  mu.assign(g, 0.0);
  inv_std.assign(g, 1.0);
  cshift.assign(g, 0.0);
  mode = 0;
  if (pl->scaled) {
    pl->std_x.resize(g);
    for (int64_t j = 0; j < g; ++j) {
      const double m = pl->mean_x[j];
      const double var = (sxx[j] - (double)n * m * m) / std::max<double>((double)n - 1.0, 1.0);
      double sd = std::sqrt(std::max(var, 0.0));
      if (sd == 0.0) sd = 1.0;
      pl->std_x[j] = sd;
      mu[j] = m;
      inv_std[j] = 1.0 / sd;
      if (pl->centered) {
        double c = -m / sd;
        if (pl->clip > 0) c = std::min(std::max(c, -pl->clip), pl->clip);
        cshift[j] = c;
      }
    }
    mode = pl->centered ? 1 : 2;
  }
  (void)sx;
  return pl->scaled || pl->in_dtype != pl->dtype;
}

// Streamed plan set-up (called by create_plan for a host matrix that does not
// fit the device budget).  `limit` = the device bytes the plan may hold.
void setup_streaming(scxpca_plan* pl, const scxpca_csr* x, size_t limit) {
  cudaStream_t st = pl->stream;
  const int64_t n = pl->n, g = pl->g, nnz = pl->nnz;
  pl->streaming = true;
  pl->h_indptr = x->indptr;
  pl->h_idx = x->indices;
  pl->h_val = x->values;
  // the row pointers are in host memory: check them there
  if (x->indptr[0] != 0 || x->indptr[n] != nnz)
    fail(SCXPCA_INVALID_CSR, "invalid CSR: indptr is not monotone within [0, nnz]");
  for (int64_t i = 0; i < n; ++i)
    if (x->indptr[i + 1] < x->indptr[i]) fail(SCXPCA_INVALID_CSR, "invalid CSR: indptr is not monotone within [0, nnz]");
  const bool tc_allowed = !(getenv("SCXPCA_TC") && getenv("SCXPCA_TC")[0] == '0');
  pl->use_tc = tc_allowed && pl->dtype != SCXPCA_F32 && g <= 64 * 128;
  if (pl->use_tc) pl->ld = (pl->k + 63) / 64 * 64;
  pl->fmt16 = pl->dtype == SCXPCA_BF16 ? 1 : 0;
  const int64_t ld = pl->ld;
  // what stays resident: the tall buffers (Y; the 16-bit image), the gene-side
  // and statistics buffers; the rest of `limit` is the two shard slots
  const double resident = (double)n * ld * 4 * (pl->use_tc ? 2 : 1) + (double)n * pl->nc * 4 +
                          (double)g * ld * 8 * 8 + (double)2 * g * 8 * (2 * pl->num_sms + 1) + (64 << 20);
  const double per_entry = slot_bytes_per_entry(pl, pl->use_tc) + (pl->use_tc ? 0.0 : 1.0);
  const double room = ((double)limit / 1.1 - resident) / 2.0;
  int64_t cap = (int64_t)std::min<double>((double)kShardEntriesMax, room / per_entry);
  // shards: whole 128-row tiles, at most `cap` stored entries (or one tile)
  pl->shards.clear();
  for (int64_t r0 = 0; r0 < n;) {
    int64_t r1 = std::min(n, r0 + 128);
    while (r1 < n) {
      const int64_t nr = std::min(n, r1 + 128);
      if (x->indptr[nr] - x->indptr[r0] > cap) break;
      r1 = nr;
    }
    scxpca_plan::Shard sh{};
    sh.r0 = r0;
    sh.r1 = r1;
    sh.p0 = x->indptr[r0];
    sh.p1 = x->indptr[r1];
    pl->shards.push_back(sh);
    pl->shard_rows_max = std::max(pl->shard_rows_max, r1 - r0);
    pl->shard_nnz_max = std::max(pl->shard_nnz_max, sh.p1 - sh.p0);
    r0 = r1;
  }
  if (room <= 0.0 || (double)pl->shard_nnz_max * per_entry > room * 1.5)
    fail(SCXPCA_OUT_OF_MEMORY, "streamed GPU PCA: the device budget of " + std::to_string(limit >> 20) +
                                   " MB does not hold the resident buffers and two shard slots");
  CK(cudaStreamCreateWithFlags(&pl->copy_stream, cudaStreamNonBlocking));
  for (int i = 0; i < 2; ++i) {
    CK(cudaEventCreateWithFlags(&pl->ev_copied[i], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&pl->ev_free[i], cudaEventDisableTiming));
  }
  const int64_t rmax = pl->shard_rows_max, emax = std::max<int64_t>(pl->shard_nnz_max, 1);
  for (auto& sl : pl->slot) {
    sl.ip.alloc(sizeof(int64_t) * (rmax + 1));
    sl.idx.alloc(sizeof(int32_t) * emax);
    sl.vin.alloc(dtype_size(pl->in_dtype) * emax);
  }
  phase_mark(SCXPCA_PHASE_UPLOAD, st);

  // ---- validation, input statistics (and gene counts) over the shards ----
  pl->stats_parts = 4 * pl->num_sms;
  pl->stats_part.alloc(sizeof(double) * 2 * g * pl->stats_parts);
  pl->stats_out.alloc(sizeof(double) * 2 * g);
  DevBuf flags, counts;
  flags.alloc(16);
  CK(cudaMemsetAsync(flags.p, 0, 16, st));
  counts.alloc(sizeof(int32_t) * g);
  CK(cudaMemsetAsync(counts.p, 0, sizeof(int32_t) * g, st));
  std::vector<double> sx, sxx;
  stream_stats(pl, false, sx, sxx, flags.as<int32_t>(), counts.as<int32_t>());
  int32_t hf[4];
  CK(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (hf[1]) fail(SCXPCA_INVALID_CSR, "invalid CSR: column index out of range [0, n_vars)");
  if (hf[3]) fail(SCXPCA_INVALID_CSR, "invalid CSR: non-finite value");
  if (hf[2]) {
    // unsorted or duplicated rows: every upload sorts its shard; duplicates
    // (found after sorting) take the CUDA-core path
    pl->stream_sort = true;
    pl->rows_resorted = true;
    CK(cudaMemsetAsync(flags.p, 0, 16, st));
    for_each_shard(pl, [&](size_t s, int k) {
      const scxpca_plan::Shard& sh = pl->shards[s];
      scxpca_plan::Slot& sl = pl->slot[k];
      shard_prepare(pl, s, k, false, 0);
      CK(launch_validate_csr(pl->in_dtype, sl.ip.as<int64_t>(), sl.idx.as<int32_t>(), sl.vin.p, sh.r1 - sh.r0, g,
                             sh.p1 - sh.p0, flags.as<int32_t>(), st, pl->num_sms));
    });
    CK(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hf[2] && pl->use_tc) {
      pl->use_tc = false;
      pl->ld = padded_k(pl->k);
    }
  }
  pl->mean_x.resize(g);
  for (int64_t j = 0; j < g; ++j) pl->mean_x[j] = sx[j] / (double)n;
  phase_mark(SCXPCA_PHASE_VALIDATE, st);
  phase_mark(SCXPCA_PHASE_STATS, st);

  // ---- working values and their statistics ----
  std::vector<double> mu, inv_std, cshift;
  pl->stream_transform = value_transform(pl, sx, sxx, pl->stream_mode, mu, inv_std, cshift);
  if (pl->stream_transform) {
    upload(pl->t_mu, mu, st);
    upload(pl->t_inv_std, inv_std, st);
    upload(pl->t_cshift, cshift, st);
    for (auto& sl : pl->slot) sl.vwork.alloc(dtype_size(pl->dtype) * emax);
    stream_stats(pl, true, pl->col_sum, pl->col_sq, nullptr, nullptr);
  } else {
    pl->col_sum = sx;
    pl->col_sq = sxx;
  }
  {
    std::vector<double> mu_w(g, 0.0);
    if (pl->centered)
      for (int64_t j = 0; j < g; ++j) mu_w[j] = pl->col_sum[j] / (double)n;
    upload(pl->d_mu, mu_w, st);
    // closed-form total variance with the cancellation guard; the recompute
    // takes one more pass over the shards (the working values minus mu)
    const double denom = std::max<double>((double)n - 1.0, 1.0);
    double sumsq = 0.0, meansq = 0.0, total = 0.0;
    for (int64_t j = 0; j < g; ++j) {
      sumsq += pl->col_sq[j];
      meansq += mu_w[j] * mu_w[j];
      total += pl->col_sq[j] - (double)n * mu_w[j] * mu_w[j];
    }
    pl->total_var = (pl->centered ? total : sumsq) / denom;
    if (pl->centered && sumsq > 0.0 && sumsq - meansq * (double)n <= 1e-7 * sumsq) {
      DevBuf d_shift, d_one, d_zero, shifted;
      std::vector<double> one(g, 1.0), zero(g, 0.0);
      upload(d_shift, mu_w, st);
      upload(d_one, one, st);
      upload(d_zero, zero, st);
      shifted.alloc(sizeof(float) * emax);
      for_each_shard(pl, [&](size_t s, int k) {
        const scxpca_plan::Shard& sh = pl->shards[s];
        scxpca_plan::Slot& sl = pl->slot[k];
        const int64_t cnt = sh.p1 - sh.p0;
        const void* vals = shard_prepare(pl, s, k, true, 0);
        CK(launch_transform_values(pl->stream_transform ? pl->dtype : pl->in_dtype, 0, sl.idx.as<int32_t>(), vals,
                                   shifted.p, cnt, 1, d_shift.as<double>(), d_one.as<double>(), d_zero.as<double>(),
                                   0.0, st, pl->num_sms));
        CK(launch_col_stats(0, sl.idx.as<int32_t>(), shifted.p, cnt, (int32_t)g, pl->stats_part.as<double>(),
                            pl->stats_parts, pl->stats_out.as<double>(), st, pl->num_sms, s > 0 ? 1 : 0));
      });
      std::vector<double> host(2 * g);
      CK(cudaMemcpyAsync(host.data(), pl->stats_out.p, sizeof(double) * 2 * g, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      double t = 0.0;
      for (int64_t j = 0; j < g; ++j) {
        const double nnz_j = mu_w[j] != 0.0 ? std::round((pl->col_sum[j] - host[j]) / mu_w[j]) : 0.0;
        t += host[g + j] + std::max((double)n - nnz_j, 0.0) * mu_w[j] * mu_w[j];
      }
      pl->total_var = t / denom;
      pl->total_var_recomputed = true;
    }
  }
  {
    std::vector<double> c(g), sc(g);
    for (int64_t j = 0; j < g; ++j) {
      c[j] = pl->centered ? pl->mean_x[j] : 0.0;
      sc[j] = pl->scaled ? 1.0 / pl->std_x[j] : 1.0;
    }
    upload(pl->d_center_raw, c, st);
    upload(pl->d_scale_raw, sc, st);
    CK(cudaStreamSynchronize(st));
  }
  phase_mark(SCXPCA_PHASE_TRANSFORM, st);

  // ---- the packed per-shard copies and the resident image ----
  const int64_t tiles_max = (rmax + 127) / 128;
  if (pl->use_tc) {
    pl->n_chunks = (int)((g + 63) / 64);
    const int64_t nseg_max = tiles_max * pl->n_chunks;
    for (auto& sl : pl->slot) {
      sl.counts.alloc(sizeof(int64_t) * nseg_max);
      sl.seg.alloc(sizeof(int64_t) * (nseg_max + 1));
      sl.ent.alloc(sizeof(uint32_t) * (size_t)(emax + 3 * nseg_max + 4));
      sl.meta.alloc(tile_meta_bytes(rmax, pl->n_chunks));
    }
    pl->Vimg.alloc(sizeof(uint16_t) * g * 2 * ld);
    pl->Yimg.alloc(sizeof(uint16_t) * n * 2 * ld);
    pl->tc_err.alloc(sizeof(int) * 4);
    CK(cudaMemsetAsync(pl->tc_err.p, 0, sizeof(int) * 4, st));
    const int rg = rmat_tc_groups((int)ld, pl->n_chunks, pl->num_sms, &pl->tc_gene_groups);
    int rg_max = 1;
    for (auto& sh : pl->shards) {
      sh.row_groups = (int)std::min<int64_t>(rg, (sh.r1 - sh.r0 + 127) / 128);
      rg_max = std::max(rg_max, sh.row_groups);
      const int r = make_tmap16(&sh.qmap, pl->Yimg.as<uint16_t>() + sh.r0 * 2 * ld, sh.r1 - sh.r0, 2 * ld, 128,
                                pl->fmt16);
      if (r) fail(SCXPCA_CUDA_ERROR, "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")");
    }
    pl->tc_row_groups = rg_max;
    pl->tc_part.alloc(sizeof(float) * (size_t)rg_max * g * ld);
    const int r1 = make_tmap16(&pl->vmap, pl->Vimg.p, g, 2 * ld, 64, pl->fmt16);
    const int r2 = make_tmap16(&pl->qmap, pl->Yimg.p, n, 2 * ld, 128, pl->fmt16);
    if (r1 || r2)
      fail(SCXPCA_CUDA_ERROR, "cuTensorMapEncodeTiled failed (" + std::to_string(r1) + ", " + std::to_string(r2) + ")");
  } else {
    pl->nslots = strict_slot_count(g, (int)ld);
    if (strict_tile_smem_bytes(pl->nslots) > kStatsSmemMax)
      fail(SCXPCA_UNSUPPORTED, "a streamed CUDA-core PCA takes at most " +
                                   std::to_string(kStatsSmemMax / sizeof(int32_t) - 1) + " genes");
    std::vector<int32_t> hc(g), gene2slot, slot2gene;
    CK(cudaMemcpyAsync(hc.data(), counts.p, sizeof(int32_t) * g, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    strict_assign_slots(hc, (int)ld, gene2slot, slot2gene);
    pl->d_gene2slot.alloc(sizeof(int32_t) * g);
    pl->d_slot2gene.alloc(sizeof(int32_t) * pl->nslots);
    CK(cudaMemcpyAsync(pl->d_gene2slot.p, gene2slot.data(), sizeof(int32_t) * g, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(pl->d_slot2gene.p, slot2gene.data(), sizeof(int32_t) * pl->nslots, cudaMemcpyHostToDevice,
                       st));
    for (auto& sl : pl->slot) {
      sl.tptr.alloc(sizeof(int32_t) * (size_t)tiles_max * (pl->nslots + 1));
      sl.cell.alloc(emax);
      sl.cval.alloc(dtype_size(pl->dtype) * emax);
    }
    const int gblocks = pl->nslots / (8 * strict_genes_per_warp((int)ld));
    int ranges_max = 1;
    for (auto& sh : pl->shards) {
      const int64_t nt = (sh.r1 - sh.r0 + kStrictTile - 1) / kStrictTile;
      sh.ranges = (int)std::max<int64_t>(1, std::min<int64_t>(nt, (4 * pl->num_sms + gblocks - 1) / gblocks));
      ranges_max = std::max(ranges_max, sh.ranges);
    }
    pl->strict_csc = true;
    pl->wpart.alloc(sizeof(float) * (size_t)ranges_max * g * ld);
    CK(cudaStreamSynchronize(st));  // the host vectors above go out of scope
  }
  phase_mark(SCXPCA_PHASE_PACK, st);
  alloc_work_buffers(pl);
}

// The dense work buffers of a run (tall Y, gene-side factors, k x k FP64).
void alloc_work_buffers(scxpca_plan* pl) {
  const int64_t n = pl->n, g = pl->g, ld = pl->ld;
  pl->gram_parts = 2 * pl->num_sms;
  pl->gram_parts_small = (int)std::max<int64_t>(1, std::min<int64_t>(2 * pl->num_sms, (g + 31) / 32));
  pl->Y.alloc(sizeof(float) * n * ld);
  pl->W.alloc(sizeof(double) * g * ld);
  pl->Z.alloc(sizeof(double) * g * ld);
  pl->V.alloc(sizeof(float) * g * ld);
  pl->mc.alloc(sizeof(float) * ld);
  pl->gpart.alloc(sizeof(double) * pl->gram_parts * (ld * ld + ld));
  pl->G.alloc(sizeof(double) * (ld * ld + ld));
  pl->R.alloc(sizeof(double) * ld * ld);
  pl->Rinv.alloc(sizeof(double) * ld * ld);
  pl->Rinv_f.alloc(sizeof(float) * ld * ld);
  pl->R2inv.alloc(sizeof(double) * ld * ld);
  pl->evals.alloc(sizeof(double) * ld);
  pl->evecs.alloc(sizeof(double) * (ld * ld + 2 * ld * (ld + 1)));  // + eigensolver scratch
  pl->sigma.alloc(sizeof(double) * ld);
  pl->comps.alloc(sizeof(float) * pl->nc * g);
  pl->M_emb.alloc(sizeof(float) * ld * pl->nc);
  pl->status.alloc(sizeof(int) * 4);
  std::vector<double> eye(ld * ld, 0.0);
  for (int64_t i = 0; i < ld; ++i) eye[i * ld + i] = 1.0;
  upload(pl->eye, eye, pl->stream);
  CK(cudaStreamSynchronize(pl->stream));  // `eye` goes out of scope
}

// The baseline of a PFlog plan: the working matrix's last column holds b.
struct PflogSpec {
  double b_mean;  // mean of the FP64 baseline (total variance)
  double b2;      // sum_i b_i^2
  double cross;   // sum_i b_i * (row sum of delta_i)
};

scxpca_plan* create_plan(const scxpca_csr* x, const scxpca_params* p, const AffineSpec* aff = nullptr,
                         const PflogSpec* pf = nullptr) {
  if (!pf) validate_params(x, p);
  auto pl = new scxpca_plan();
  try {
    pl->device = p->device_ordinal;
    CK(cudaDeviceGetAttribute(&pl->num_sms, cudaDevAttrMultiProcessorCount, pl->device));
    pl->params = *p;
    pl->n = x->n_obs;
    pl->g = x->n_vars;
    pl->pflog = pf != nullptr;
    pl->g_user = pf ? x->n_vars - 1 : x->n_vars;
    pl->nnz = x->nnz;
    pl->k = std::min({p->n_components + p->n_oversamples, pl->g_user, x->n_obs});
    pl->ld = padded_k(pl->k);
    pl->nc = p->n_components;
    pl->in_dtype = x->values_dtype;
    pl->dtype = p->math_mode == SCXPCA_MATH_STRICT_FP32 ? SCXPCA_F32
                : p->math_mode == SCXPCA_MATH_MIXED_BF16 ? SCXPCA_BF16
                                                         : SCXPCA_F16;
    pl->affine = aff != nullptr;
    pl->centered = aff ? aff->center != nullptr : p->zero_center != 0;
    pl->scaled = aff ? false : p->scale != 0;
    pl->clip = (!aff && p->clip_max > 0) ? p->clip_max : 0.0;
    if (p->stream) {
      pl->stream = static_cast<cudaStream_t>(p->stream);
    } else {
      CK(cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking));
      pl->own_stream = true;
    }
    cudaStream_t st = pl->stream;
    PoolScope pool_scope(pl->device, st);
    const int64_t n = pl->n, g = pl->g, nnz = pl->nnz;
    phase_mark(-1, st);  // opens the phase clock of a one-shot call

    // ---- pre-flight (gpu_pca.rs:450-462): resident CSR + work buffers ----
    {
      const int64_t ldp = (pl->k + 63) / 64 * 64;
      size_t need = (size_t)(n + 1) * 8 + (size_t)nnz * 4 + (size_t)nnz * dtype_size(pl->dtype) * 2 +
                    (size_t)nnz * 4 + (size_t)n * ldp * 8 + (size_t)n * pl->nc * 4 + (size_t)n * 36 +
                    (size_t)g * ldp * 4 * 400;
      size_t fr = 0, tot = 0;
      CK(cudaMemGetInfo(&fr, &tot));
      {  // memory our pool holds but does not use is free for this plan
        uint64_t reserved = 0, used = 0;
        cudaMemPool_t pool = pool_for(pl->device).pool;
        CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
        CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
        if (reserved > used) fr += (size_t)(reserved - used);
      }
      double with_headroom = (double)need * 1.1;
      // A host matrix that does not fit (the free memory, or the caller's
      // device budget) is streamed from host memory instead of held resident
      // (gpu_pca.rs:520-590); SCXPCA_RESIDENT=0 forces it.
      size_t limit = fr;
      if (p->device_budget > 0) limit = std::min(limit, (size_t)p->device_budget);
      const char* res_env = getenv("SCXPCA_RESIDENT");
      const bool force_stream = res_env && res_env[0] == '0';
      if (x->memory != SCXPCA_MEM_DEVICE && !aff && !pf && (force_stream || with_headroom > (double)limit)) {
        if (pl->k > kMaxK)
          fail(SCXPCA_UNSUPPORTED, "a sketch wider than " + std::to_string(kMaxK) +
                                       " columns needs the matrix resident on the device (it is not streamed)");
        setup_streaming(pl, x, limit);
        phase_mark(SCXPCA_PHASE_BUFFERS, st);
        CK(cudaStreamSynchronize(st));
        pl->device_bytes = pl->stats_part.bytes + pl->Y.bytes + pl->Yimg.bytes + pl->tc_part.bytes +
                           pl->wpart.bytes + pl->gpart.bytes + pl->W.bytes + pl->Z.bytes + pl->V.bytes;
        for (auto& sl : pl->slot)
          pl->device_bytes += sl.ip.bytes + sl.idx.bytes + sl.vin.bytes + sl.vwork.bytes + sl.counts.bytes +
                              sl.seg.bytes + sl.ent.bytes + sl.meta.bytes + sl.tptr.bytes + sl.cell.bytes +
                              sl.cval.bytes;
        return pl;
      }
      if (with_headroom > (double)fr)
        fail(SCXPCA_OUT_OF_MEMORY, "GPU PCA requires ~" + std::to_string((size_t)with_headroom >> 20) +
                                       " MB but only " + std::to_string(fr >> 20) +
                                       " MB free on device");
    }

    // ---- resident CSR ----
    const bool dev_in = x->memory == SCXPCA_MEM_DEVICE;
    pl->stats_parts = 4 * pl->num_sms;
    pl->stats_part.alloc(sizeof(double) * 2 * g * pl->stats_parts);
    pl->stats_out.alloc(sizeof(double) * 2 * g);
    const void* vin = x->values;
    bool stats_queued = false;  // the statistics blocks already ran under the copy
    if (dev_in) {
      pl->indptr = x->indptr;
      pl->idx = x->indices;
    } else {
      pl->b_indptr.alloc(sizeof(int64_t) * (n + 1));
      pl->b_idx.alloc(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
      CK(cudaMemcpyAsync(pl->b_indptr.p, x->indptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
      pl->indptr = pl->b_indptr.as<int64_t>();
      pl->idx = pl->b_idx.as<int32_t>();
      if (nnz) {
        // The entries cross in pieces on a copy stream, each piece a run of
        // whole blocks of the statistics partition; the plan's stream runs a
        // piece's statistics blocks as soon as it has landed, so the column
        // sums are computed under the copy and equal (bit for bit) those of
        // one launch over the whole matrix.  The statistics kernel checks
        // every index it reads; validation follows the copy.
        const size_t vs = dtype_size(pl->in_dtype);
        pl->b_stage.alloc(vs * nnz);
        vin = pl->b_stage.p;
        if (!pl->copy_stream) CK(cudaStreamCreateWithFlags(&pl->copy_stream, cudaStreamNonBlocking));
        cudaStream_t cs = pl->copy_stream;
        const int parts = pl->stats_parts;
        const int pieces = std::min(kUploadPieces, parts);
        std::vector<cudaEvent_t> landed(pieces + 1, nullptr);
        for (auto& e : landed) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaEventRecord(landed[pieces], st));  // the buffers exist before the copies start
        CK(cudaStreamWaitEvent(cs, landed[pieces], 0));
        for (int c = 0; c < pieces; ++c) {
          const int b0 = (int)((int64_t)c * parts / pieces), b1 = (int)((int64_t)(c + 1) * parts / pieces);
          const int64_t e0 = col_stats_block_begin(nnz, parts, b0), e1 = col_stats_block_begin(nnz, parts, b1);
          if (e1 > e0) {
            CK(cudaMemcpyAsync(pl->b_idx.as<int32_t>() + e0, x->indices + e0, sizeof(int32_t) * (e1 - e0),
                               cudaMemcpyHostToDevice, cs));
            CK(cudaMemcpyAsync(static_cast<char*>(pl->b_stage.p) + vs * e0,
                               static_cast<const char*>(x->values) + vs * e0, vs * (e1 - e0),
                               cudaMemcpyHostToDevice, cs));
          }
          CK(cudaEventRecord(landed[c], cs));
          CK(cudaStreamWaitEvent(st, landed[c], 0));
          CK(launch_col_stats_blocks(pl->in_dtype, pl->idx, vin, nnz, (int32_t)g, pl->stats_part.as<double>(),
                                     parts, b0, b1 - b0, st));
        }
        for (auto& e : landed) CK(cudaEventDestroy(e));  // released once the pending work completes
        stats_queued = true;
      }
    }
    phase_mark(SCXPCA_PHASE_UPLOAD, st);

    // ---- validation ----
    {
      DevBuf flags;
      flags.alloc(16);
      CK(cudaMemsetAsync(flags.p, 0, 16, st));
      CK(launch_validate_csr(pl->in_dtype, pl->indptr, pl->idx, vin, n, g, nnz, flags.as<int32_t>(),
                             st, pl->num_sms));
      int32_t hf[4];
      CK(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (hf[0]) fail(SCXPCA_INVALID_CSR, "invalid CSR: indptr is not monotone within [0, nnz]");
      if (hf[1]) fail(SCXPCA_INVALID_CSR, "invalid CSR: column index out of range [0, n_vars)");
      if (hf[3]) fail(SCXPCA_INVALID_CSR, "invalid CSR: non-finite value");
      bool duplicates = false;
      if (hf[2]) {
        // unsorted (or duplicated) rows: sort an owned copy by gene
        if (dev_in) {
          pl->b_idx.alloc(sizeof(int32_t) * nnz);
          CK(cudaMemcpyAsync(pl->b_idx.p, pl->idx, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, st));
          pl->idx = pl->b_idx.as<int32_t>();
          pl->b_stage.alloc(dtype_size(pl->in_dtype) * nnz);
          CK(cudaMemcpyAsync(pl->b_stage.p, vin, dtype_size(pl->in_dtype) * nnz, cudaMemcpyDeviceToDevice, st));
          vin = pl->b_stage.p;
        }
        CK(launch_sort_rows(pl->in_dtype, pl->indptr, pl->b_idx.as<int32_t>(), pl->b_stage.p, n, st,
                            pl->num_sms));
        pl->rows_resorted = true;
        // after sorting, any remaining "not strictly ascending" pair is a duplicate
        CK(cudaMemsetAsync(flags.p, 0, 16, st));
        CK(launch_validate_csr(pl->in_dtype, pl->indptr, pl->idx, vin, n, g, nnz, flags.as<int32_t>(),
                               st, pl->num_sms));
        CK(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        duplicates = hf[2] != 0;
      }
      // Tensor cores for 16-bit values on sorted, duplicate-free rows with at
      // most 128 gene chunks (8,192 genes); SCXPCA_TC=0 forces the CUDA cores.
      const char* env = getenv("SCXPCA_TC");
      const bool tc_allowed = !(env && env[0] == '0');
      pl->use_tc = tc_allowed && pl->dtype != SCXPCA_F32 && !duplicates && g <= 64 * 128 && pl->k <= kMaxK;
      if (pl->use_tc) pl->ld = (pl->k + 63) / 64 * 64;
      pl->fmt16 = pl->dtype == SCXPCA_BF16 ? 1 : 0;
    }
    const int64_t ld = pl->ld;
    phase_mark(SCXPCA_PHASE_VALIDATE, st);

    // ---- statistics of the input ----
    std::vector<double> sx, sxx;
    if (stats_queued && !pl->rows_resorted)
      stats_finish(pl, sx, sxx);
    else
      stats_pass(pl, vin, pl->in_dtype, sx, sxx);
    pl->mean_x.resize(g);
    for (int64_t j = 0; j < g; ++j) pl->mean_x[j] = sx[j] / (double)n;
    phase_mark(SCXPCA_PHASE_STATS, st);

    // ---- working values ----
    std::vector<double> center_raw(g, 0.0), scale_raw(g, 1.0);
    const bool affine_scaled = aff && aff->scale;
    const bool borrow = !pl->scaled && !affine_scaled && pl->in_dtype == pl->dtype;
    if (aff) {
      center_raw = read_vec(aff->center, g, aff->memory, 0.0, st);
      scale_raw = read_vec(aff->scale, g, aff->memory, 1.0, st);
      for (int64_t j = 0; j < g; ++j) {
        if (!std::isfinite(center_raw[j]) || !std::isfinite(scale_raw[j]) || scale_raw[j] == 0.0)
          fail(SCXPCA_INVALID_ARGUMENT, "center and scale must be finite and scale non-zero (gene " +
                                            std::to_string(j) + ")");
      }
    }
    if (borrow) {
      pl->val = vin;
      if (!dev_in || vin != x->values) {
        // vin is our staging buffer: keep it
        pl->b_val.adopt(pl->b_stage);
        pl->val = pl->b_val.p;
      }
      pl->col_sum = sx;
      pl->col_sq = sxx;
    } else {
      pl->b_val.alloc(dtype_size(pl->dtype) * std::max<int64_t>(nnz, 1));
      int mode = 0;
      std::vector<double> mu(g, 0.0), inv_std(g, 1.0), cshift(g, 0.0);
      if (affine_scaled) {
        inv_std = scale_raw;  // x -> x s, no clip; the centring stays implicit
        mode = 2;
      } else if (pl->scaled) {
        pl->std_x.resize(g);
        for (int64_t j = 0; j < g; ++j) {
          double m = pl->mean_x[j];
          double var = (sxx[j] - (double)n * m * m) / std::max<double>((double)n - 1.0, 1.0);
          double sd = std::sqrt(std::max(var, 0.0));
          if (sd == 0.0) sd = 1.0;
          pl->std_x[j] = sd;
          mu[j] = m;
          inv_std[j] = 1.0 / sd;
          if (pl->centered) {
            double c = -m / sd;
            if (pl->clip > 0) c = std::min(std::max(c, -pl->clip), pl->clip);
            cshift[j] = c;
          }
        }
        mode = pl->centered ? 1 : 2;
      }
      upload(pl->d_mu, mu, st);
      upload(pl->d_inv_std, inv_std, st);
      upload(pl->d_cshift, cshift, st);
      CK(launch_transform_values(pl->in_dtype, pl->dtype, pl->idx, vin, pl->b_val.p, nnz, mode,
                                 pl->d_mu.as<double>(), pl->d_inv_std.as<double>(),
                                 pl->d_cshift.as<double>(), pl->clip, st, pl->num_sms));
      pl->val = pl->b_val.p;
      stats_pass(pl, pl->val, pl->dtype, pl->col_sum, pl->col_sq);
      pl->b_stage.release();
    }
    if (aff) {
      // X~ = P - 1 (c s)^T: the centre is the given vector, not the column mean
      std::vector<double> mu_w(g, 0.0);
      double t = 0.0;
      for (int64_t j = 0; j < g; ++j) {
        if (pl->centered) mu_w[j] = center_raw[j] * scale_raw[j];
        t += pl->col_sq[j] - 2.0 * mu_w[j] * pl->col_sum[j] + (double)n * mu_w[j] * mu_w[j];
      }
      upload(pl->d_mu, mu_w, st);
      pl->total_var = t / std::max<double>((double)n - 1.0, 1.0);
    } else if (pf) {
      // Z = delta + b 1^T: column means colmean(delta)_j + mean(b) (cpu.rs:836-842);
      // the baseline column itself is not centred.  Total variance in closed
      // form: sum_ij (delta_ij + b_i)^2 = S_dd + 2 sum_i b_i r_i + D sum_i b_i^2
      // (r_i the row sums of delta), minus n sum_j mu_j^2 when centred; with
      // the PFlog baseline b_i = -r_i / D this is pflog_total_variance's
      // S_dd - D B2 - n sum mu^2 (cpu.rs:689-786).
      // The centring takes the mean baseline from the stored baseline column
      // (the values the products see, in the compute type), so it is
      // consistent with the products; the total variance uses the FP64
      // baseline.
      const int64_t gu = pl->g_user;
      const double b_mean = pl->col_sum[gu] / (double)n;
      std::vector<double> mu_w(g, 0.0);
      double s_dd = 0.0, m2 = 0.0;
      for (int64_t j = 0; j < gu; ++j) {
        s_dd += pl->col_sq[j];
        if (pl->centered) {
          mu_w[j] = pl->col_sum[j] / (double)n + b_mean;
          const double mu64 = pl->col_sum[j] / (double)n + pf->b_mean;
          m2 += mu64 * mu64;
        }
      }
      for (int64_t j = 0; j < gu; ++j) pl->mean_x[j] = pl->col_sum[j] / (double)n + b_mean;
      pl->mean_x.resize(gu);
      upload(pl->d_mu, mu_w, st);
      const double tss = s_dd + 2.0 * pf->cross + (double)gu * pf->b2 - (double)n * m2;
      pl->total_var = std::max(tss, 0.0) / std::max<double>((double)n - 1.0, 1.0);
    } else {
      std::vector<double> mu_w(g, 0.0);
      if (pl->centered)
        for (int64_t j = 0; j < g; ++j) mu_w[j] = pl->col_sum[j] / (double)n;
      upload(pl->d_mu, mu_w, st);
      compute_total_variance(pl);
      // the same matrix as an affine map of the input, for the backward pass
      for (int64_t j = 0; j < g; ++j) {
        center_raw[j] = pl->centered ? pl->mean_x[j] : 0.0;
        scale_raw[j] = pl->scaled ? 1.0 / pl->std_x[j] : 1.0;
      }
    }
    upload(pl->d_center_raw, center_raw, st);
    upload(pl->d_scale_raw, scale_raw, st);
    if (aff && aff->scale) {
      pl->std_x.resize(g);
      for (int64_t j = 0; j < g; ++j) pl->std_x[j] = 1.0 / scale_raw[j];
    }
    phase_mark(SCXPCA_PHASE_TRANSFORM, st);

    // ---- tensor-core path: tile-chunk packed matrix, 16-bit operands, TMA maps ----
    if (pl->use_tc) {
      const int64_t n_tiles = (n + 127) / 128;
      pl->n_chunks = (int)((g + 63) / 64);
      const int64_t nseg = n_tiles * pl->n_chunks;
      DevBuf counts, seg;
      counts.alloc(sizeof(int64_t) * nseg);
      seg.alloc(sizeof(int64_t) * (nseg + 1));
      CK(tile_format_count(pl->indptr, pl->idx, n, pl->n_chunks, counts.as<int64_t>(), st, pl->num_sms));
      CK(launch_exclusive_scan_i64(counts.as<int64_t>(), nseg, seg.as<int64_t>(), st));
      int64_t padded_nnz = 0;
      CK(cudaMemcpyAsync(&padded_nnz, seg.as<int64_t>() + nseg, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      pl->tf_ent.alloc(sizeof(uint32_t) * std::max<int64_t>(padded_nnz, 4));
      CK(cudaMemsetAsync(pl->tf_ent.p, 0, sizeof(uint32_t) * std::max<int64_t>(padded_nnz, 4), st));
      pl->tf_meta.alloc(tile_meta_bytes(n, pl->n_chunks));
      CK(tile_format_fill(pl->indptr, pl->idx, pl->val, n, pl->n_chunks, seg.as<int64_t>(),
                          pl->tf_ent.as<uint32_t>(), pl->tf_meta.p, st, pl->num_sms));
      pl->Vimg.alloc(sizeof(uint16_t) * g * 2 * ld);
      pl->Yimg.alloc(sizeof(uint16_t) * n * 2 * ld);
      pl->tc_err.alloc(sizeof(int) * 4);
      CK(cudaMemsetAsync(pl->tc_err.p, 0, sizeof(int) * 4, st));
      pl->tc_row_groups = rmat_tc_groups((int)ld, pl->n_chunks, pl->num_sms, &pl->tc_gene_groups);
      pl->tc_row_groups = (int)std::min<int64_t>(pl->tc_row_groups, n_tiles);  // no idle row groups
      pl->tc_part.alloc(sizeof(float) * (size_t)pl->tc_row_groups * g * ld);
      int r1 = make_tmap16(&pl->vmap, pl->Vimg.p, g, 2 * ld, 64, pl->fmt16);
      int r2 = make_tmap16(&pl->qmap, pl->Yimg.p, n, 2 * ld, 128, pl->fmt16);
      if (r1 || r2)
        fail(SCXPCA_CUDA_ERROR,
             "cuTensorMapEncodeTiled failed (" + std::to_string(r1) + ", " + std::to_string(r2) + ")");
    }

    // ---- CUDA-core products: tile-CSC copy for the transposed product ----
    pl->nb = (int)((g + kTransposeGeneBlock - 1) / kTransposeGeneBlock);
    pl->nchunks = std::max(1, (2 * pl->num_sms + pl->nb - 1) / pl->nb);
    pl->nchunks = (int)std::min<int64_t>(pl->nchunks, n);
    pl->rows_per_chunk = (n + pl->nchunks - 1) / pl->nchunks;
    if (!pl->use_tc) {
      pl->nslots = strict_slot_count(g, panel_width(pl));
      pl->strict_csc = strict_tile_smem_bytes(pl->nslots) <= kStatsSmemMax;
    }
    if (pl->ld > kMaxK && !pl->strict_csc)
      fail(SCXPCA_UNSUPPORTED, "a sketch wider than " + std::to_string(kMaxK) + " columns needs the tile-CSC "
                               "copy, whose per-gene offsets exceed shared memory at n_vars = " + std::to_string(g));
    if (pl->strict_csc) build_tile_csc(pl);
    else if (!pl->use_tc) ensure_rbp(pl);
    phase_mark(SCXPCA_PHASE_PACK, st);

    // ---- dense work buffers ----
    alloc_work_buffers(pl);
    phase_mark(SCXPCA_PHASE_BUFFERS, st);
    CK(cudaStreamSynchronize(st));
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    pl->device_bytes = pl->b_indptr.bytes + pl->b_idx.bytes + pl->b_val.bytes + pl->stats_part.bytes +
                       pl->rbp.bytes + pl->wpart.bytes + pl->Y.bytes + pl->gpart.bytes +
                       pl->W.bytes + pl->Z.bytes + pl->V.bytes + pl->csc_tptr.bytes + pl->csc_cell.bytes +
                       pl->csc_val.bytes + pl->tf_ent.bytes + pl->Yimg.bytes + pl->tc_part.bytes;
    return pl;
  } catch (...) {
    // the buffers are freed in the stream's order: delete the plan first
    const bool own = pl->own_stream;
    cudaStream_t st = pl->stream;
    delete pl;
    if (own && st) cudaStreamDestroy(st);
    throw;
  }
}

// ---- stage timing: events bracket each stage on the plan's stream ----
int stage_begin(scxpca_plan* pl) {
  if (!pl->profiling) return -1;
  if (pl->events_used + 2 > (int)pl->events.size()) {
    for (int i = 0; i < 64; ++i) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      pl->events.push_back(e);
    }
  }
  int i = pl->events_used;
  pl->events_used += 2;
  CK(cudaEventRecord(pl->events[i], pl->stream));
  return i;
}

void stage_end(scxpca_plan* pl, int stage, int i) {
  if (i < 0) return;
  CK(cudaEventRecord(pl->events[i + 1], pl->stream));
  pl->marks.emplace_back(stage, i);
}

// Fold the recorded stage intervals into the profile (stream already synced).
void collect_stages(scxpca_plan* pl) {
  for (auto& m : pl->marks) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, pl->events[m.second], pl->events[m.second + 1]));
    pl->prof.device_ms[m.first] += ms;
    pl->prof.launches[m.first] += 1;
  }
  pl->marks.clear();
  pl->events_used = 0;
}

// The Gram (FP64, with column sums after it) of a tall A into G.  With
// `from_image` (tensor-core path, ld 64) it is taken on tensor cores from the
// 16-bit image of A held in Yimg; otherwise from the FP32 A with FP64 FMAs.
void tall_gram(scxpca_plan* pl, const float* A, int64_t rows, bool from_image) {
  cudaStream_t st = pl->stream;
  const int ld = (int)pl->ld;
  int parts = (int)std::max<int64_t>(1, std::min<int64_t>(pl->gram_parts, (rows + 31) / 32));
  int s = stage_begin(pl);
  if (from_image && pl->use_tc && ld == 64) {
    parts = launch_gram_tc(rows, &pl->qmap, pl->gpart.as<double>(), pl->fmt16,
                           pl->tc_err.as<int>(), st, pl->num_sms, pl->tc_gram_parts);
    if (parts < 0) CK(cudaGetLastError());
  } else
  CK(launch_gram_f32(A, rows, ld, pl->gpart.as<double>(), parts, st));
  CK(launch_reduce_rows_f64(pl->gpart.as<double>(), parts, (int64_t)ld * ld + ld, pl->G.as<double>(), 0,
                            st, pl->num_sms));
  stage_end(pl, SCXPCA_STAGE_GRAM, s);
}

// The k x k Cholesky of G: R, and R^{-1} into Rinv / Rinv_f.
void gram_chol(scxpca_plan* pl, double* Rinv, float* Rinv_f, int shift) {
  int s = stage_begin(pl);
  CK(launch_cholesky(pl->G.as<double>(), (int)pl->k, (int)pl->ld, pl->tau, shift, pl->R.as<double>(), Rinv,
                     Rinv_f, pl->status.as<int>(), pl->stream));
  stage_end(pl, SCXPCA_STAGE_SMALL, s);
}

// The same factorisation as one task of a batched launch.
CholTask gram_chol_task(scxpca_plan* pl, double* Rinv, float* Rinv_f) {
  return CholTask{pl->G.as<double>(), pl->R.as<double>(), Rinv, Rinv_f, pl->status.as<int>()};
}

// Tall Gram + Cholesky (FP64) of a tall matrix A.
void tall_chol(scxpca_plan* pl, const float* A, int64_t rows, double* Rinv, float* Rinv_f,
               int shift, bool from_image = false) {
  tall_gram(pl, A, rows, from_image);
  gram_chol(pl, Rinv, Rinv_f, shift);
}

// One CholeskyQR pass of a gene-side FP64 matrix in place.  The Gram and the
// triangular apply are both FP64, so the loss of orthogonality is about
// cond(A)^2 * 1e-16: the second pass of CholeskyQR2, which repairs a Gram
// formed in working precision, is not needed on this FP64 gene-side matrix
// (the tall FP32 Q keeps its second pass).  In halves: small_gram, the
// Cholesky, small_apply.
void small_gram(scxpca_plan* pl, const double* A) {
  cudaStream_t st = pl->stream;
  const int ld = (int)pl->ld;
  CK(launch_gram_f64(A, pl->g, ld, pl->gpart.as<double>(), pl->gram_parts_small, st));
  CK(launch_reduce_rows_f64(pl->gpart.as<double>(), pl->gram_parts_small, (int64_t)ld * ld + ld,
                            pl->G.as<double>(), 0, st, pl->num_sms));
}

void small_apply(scxpca_plan* pl, double* A) {
  CK(launch_apply_right_f64(A, pl->g, (int)pl->ld, pl->Rinv.as<double>(), pl->stream));
}

void small_qr(scxpca_plan* pl, double* A, int shift) {
  small_gram(pl, A);
  CK(launch_cholesky(pl->G.as<double>(), (int)pl->k, (int)pl->ld, pl->tau, shift, pl->R.as<double>(),
                     pl->Rinv.as<double>(), pl->Rinv_f.as<float>(), pl->status.as<int>(), pl->stream));
  small_apply(pl, A);
}

// W = X^T A (raw, uncentred), FP64, for a tall float A (n x ld).
// W = X^T A (raw, uncentred) into pl->W (FP64).  On the tensor-core path the
// tall operand enters as its 16-bit image Yimg: `split` != 0 first writes
// the image of the FP32 A; otherwise it already holds the image of A (the
// forward product's, or the explicit Q's).
void rmatmat_raw(scxpca_plan* pl, float* A, int split) {
  cudaStream_t st = pl->stream;
  if (pl->streaming) {
    int s = stage_begin(pl);
    if (pl->use_tc && split)
      CK(launch_split16(A, pl->n * pl->ld, pl->Yimg.as<uint16_t>(), pl->fmt16, st, pl->num_sms));
    stage_end(pl, SCXPCA_STAGE_APPLY, s);
    s = stage_begin(pl);
    stream_rmat(pl, A);
    stage_end(pl, SCXPCA_STAGE_TRANSPOSE, s);
    return;
  }
  if (pl->use_tc) {
    int s = stage_begin(pl);
    if (split)
      CK(launch_split16(A, pl->n * pl->ld, pl->Yimg.as<uint16_t>(), pl->fmt16, st, pl->num_sms));
    stage_end(pl, SCXPCA_STAGE_APPLY, s);
    s = stage_begin(pl);
    CK(launch_rmat_tc((int)pl->ld, pl->tf_ent.as<uint32_t>(), pl->tf_meta.p, pl->n, pl->n_chunks, pl->g,
                      pl->tc_gene_groups, pl->tc_row_groups, &pl->qmap, pl->tc_part.as<float>(), pl->fmt16,
                      pl->tc_err.as<int>(), st));
    stage_end(pl, SCXPCA_STAGE_TRANSPOSE, s);
    s = stage_begin(pl);
    CK(launch_reduce_rows_f32(pl->tc_part.as<float>(), pl->tc_row_groups, pl->g * pl->ld,
                              pl->W.as<double>(), 0, st, pl->num_sms));
    stage_end(pl, SCXPCA_STAGE_REDUCE, s);
    return;
  }
  if (pl->strict_csc && pl->ld > kMaxK) {
    // one 128-column panel of A per launch, each panel's partials reduced
    // into its columns of W
    const int ld = (int)pl->ld, pw = panel_width(pl);
    for (int c0 = 0; c0 < ld; c0 += pw) {
      int s = stage_begin(pl);
      CK(launch_rmat_strict(pl->dtype, pw, pl->indptr, pl->csc_tptr.as<int32_t>(), pl->csc_cell.as<uint8_t>(),
                            pl->csc_val.p, pl->n, (int32_t)pl->g, pl->nslots, pl->d_slot2gene.as<int32_t>(),
                            pl->strict_ranges, A + c0, pl->wpart.as<float>(), st, ld));
      stage_end(pl, SCXPCA_STAGE_TRANSPOSE, s);
      s = stage_begin(pl);
      CK(launch_reduce_panel_f32(pl->wpart.as<float>(), pl->strict_ranges, pl->g, pw, pl->W.as<double>() + c0, ld,
                                 st, pl->num_sms));
      stage_end(pl, SCXPCA_STAGE_REDUCE, s);
    }
    return;
  }
  int s = stage_begin(pl);
  int parts = pl->nchunks;
  if (pl->strict_csc) {
    CK(launch_rmat_strict(pl->dtype, (int)pl->ld, pl->indptr, pl->csc_tptr.as<int32_t>(), pl->csc_cell.as<uint8_t>(),
                          pl->csc_val.p, pl->n, (int32_t)pl->g, pl->nslots, pl->d_slot2gene.as<int32_t>(),
                          pl->strict_ranges, A, pl->wpart.as<float>(), st));
    parts = pl->strict_ranges;
  } else {
    CK(launch_spmm_t(pl->dtype, (int)pl->ld, pl->indptr, pl->idx, pl->val, pl->n, (int32_t)pl->g,
                     pl->rbp.as<int32_t>(), pl->nb, pl->nchunks, pl->rows_per_chunk, A,
                     pl->wpart.as<float>(), st));
  }
  stage_end(pl, SCXPCA_STAGE_TRANSPOSE, s);
  s = stage_begin(pl);
  CK(launch_reduce_rows_f32(pl->wpart.as<float>(), parts, pl->g * pl->ld, pl->W.as<double>(), 0,
                            st, pl->num_sms));
  stage_end(pl, SCXPCA_STAGE_REDUCE, s);
}

// Y = (X - mu) V.  On the tensor-core path V enters as its 16-bit image and
// the product also leaves the image of Y for the Gram and the transposed
// product; `f32` = false skips the FP32 copy of Y when nothing reads it
// (inside the power loop at ld 64, whose Gram uses the image).
// `split_v` = false: V's 16-bit image is already written (a batch writes all
// segments' images in one launch).
void forward(scxpca_plan* pl, bool f32 = true, bool split_v = true) {
  cudaStream_t st = pl->stream;
  if (pl->streaming) {
    int s = stage_begin(pl);
    if (pl->use_tc)
      CK(launch_split16(pl->V.as<float>(), pl->g * pl->ld, pl->Vimg.as<uint16_t>(), pl->fmt16, st, pl->num_sms));
    stage_end(pl, SCXPCA_STAGE_SMALL, s);
    s = stage_begin(pl);
    stream_forward(pl, f32);
    stage_end(pl, SCXPCA_STAGE_FORWARD, s);
    return;
  }
  if (pl->use_tc) {
    int s = stage_begin(pl);
    if (split_v)
      CK(launch_split16(pl->V.as<float>(), pl->g * pl->ld, pl->Vimg.as<uint16_t>(), pl->fmt16, st, pl->num_sms));
    stage_end(pl, SCXPCA_STAGE_SMALL, s);
    s = stage_begin(pl);
    CK(launch_fwd_tc((int)pl->ld, pl->tf_ent.as<uint32_t>(), pl->tf_meta.p, pl->n, pl->n_chunks, &pl->vmap,
                     pl->mc.as<float>(), f32 ? pl->Y.as<float>() : nullptr, pl->Yimg.as<uint16_t>(), pl->fmt16,
                     pl->tc_err.as<int>(), st, pl->num_sms));
    stage_end(pl, SCXPCA_STAGE_FORWARD, s);
    return;
  }
  int s = stage_begin(pl);
  const int ld = (int)pl->ld, pw = panel_width(pl);
  for (int c0 = 0; c0 < ld; c0 += pw)
    CK(launch_fwd_strict(pl->dtype, pw, pl->indptr, pl->idx, pl->val, pl->n, (int32_t)pl->g, pl->V.as<float>() + c0,
                         pl->centered ? pl->mc.as<float>() + c0 : nullptr, pl->Y.as<float>() + c0, st, ld));
  stage_end(pl, SCXPCA_STAGE_FORWARD, s);
}

// Raise the error a tensor-core kernel recorded (a bounded wait that ran out).
void check_tc_error(scxpca_plan* pl) {
  if (!pl->use_tc) return;
  int e = 0;
  CK(cudaMemcpyAsync(&e, pl->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, pl->stream));
  CK(cudaStreamSynchronize(pl->stream));
  if (e != 0) {
    CK(cudaMemsetAsync(pl->tc_err.p, 0, sizeof(int), pl->stream));
    fail(SCXPCA_TIMEOUT, "tensor-core pipeline wait timed out (site " + std::to_string(e) + ")");
  }
}

// V = Omega (seeded, or the caller's), zero-padded to g x ld; V's mean
// prefactor is load_omega's.
void load_omega_v(scxpca_plan* pl, const scxpca_params* p) {
  cudaStream_t st = pl->stream;
  const int64_t g = pl->g, gu = pl->g_user, k = pl->k, ld = pl->ld;
  CK(cudaMemsetAsync(pl->V.p, 0, sizeof(float) * g * ld, st));
  if (p->omega) {
    const float* src = p->omega;
    if (p->omega_memory != SCXPCA_MEM_DEVICE) {
      pl->omega_stage.alloc(sizeof(float) * gu * k);
      CK(cudaMemcpyAsync(pl->omega_stage.p, p->omega, sizeof(float) * gu * k, cudaMemcpyHostToDevice, st));
      src = pl->omega_stage.as<float>();
    }
    CK(launch_colmajor_to_padded(src, gu, k, (int)ld, pl->V.as<float>(), st, pl->num_sms));
  } else {
    CK(launch_gaussian(p->seed, gu, k, pl->V.as<float>(), (int)ld, st, pl->num_sms));
  }
  if (pl->pflog) CK(launch_aug_colsum(pl->V.as<float>(), (int32_t)gu, (int)ld, st));
}

void load_omega(scxpca_plan* pl, const scxpca_params* p) {
  load_omega_v(pl, p);
  CK(launch_mean_prefactor(pl->V.as<float>(), pl->g, (int)pl->ld, pl->centered ? pl->d_mu.as<double>() : nullptr,
                           pl->mc.as<float>(), pl->stream));
}

// Parameters of one run: the plan's, with the per-run overrides of `over`.
scxpca_params run_params(const scxpca_plan* pl, const scxpca_params* over) {
  scxpca_params p = pl->params;
  if (over) {
    p.seed = over->seed;
    p.omega = over->omega;
    p.omega_memory = over->omega_memory;
    p.n_power_iterations = over->n_power_iterations;
    if (p.n_power_iterations < 0) fail(SCXPCA_INVALID_ARGUMENT, "n_power_iterations must be >= 0");
  }
  return p;
}

// The plan's power-loop operator (the steps run_power_loop drives).  The Y
// factor stays implicit inside the loop: qr(Y) is the FP64 Cholesky R of
// Y^T Y, and the next transposed product applies R^{-1}
// (Z = (X^T Y - mu (1^T Y)) R^{-1}).  qr(Z) is one FP64 CholeskyQR pass and
// rounds Z into V, the next forward product's operand.  finalize_q forms
// Q = Y R^{-1} and factors it again (R2; a third pass under the Householder
// contract), so the closing product gives B = (X - mu)^T Q R2^{-1}.
struct DeviceOperator {
  scxpca_plan* pl;
  const scxpca_params& p;
  int shift;           // Householder contract: shifted factorisations allowed
  bool image_only;     // tensor-core Gram at ld 64: the loop needs only Y's image
  const double* mu;    // working-matrix centre (null without centring)
  double* sY;          // column sums of Y, written after its Gram
  bool closing = false;

  void matmat(Operand src, bool last) {
    if (src == Operand::kOmega) {
      int s = stage_begin(pl);
      load_omega(pl, &p);
      stage_end(pl, SCXPCA_STAGE_SMALL, s);
    }
    // Only the last forward product's FP32 Y is read (by finalize_q); the
    // tensor-core Gram at ld 64 reads the 16-bit image.
    forward(pl, !image_only || last);
  }
  // The size-proportional halves of matmat and rmatmat, for a batch that runs
  // the gene-side halves (V's image; the centring and R^{-1} apply) of all
  // segments in one launch each.
  void matmat_products(bool last) { forward(pl, !image_only || last, false); }
  void rmatmat_products() {
    rmatmat_raw(pl, pl->Y.as<float>(), 0);
    if (pl->pflog) CK(launch_aug_fold(pl->W.as<double>(), (int32_t)pl->g_user, (int)pl->ld, pl->stream, pl->num_sms));
  }
  ApplyTask rmatmat_task() const {
    return ApplyTask{pl->W.as<double>(), mu, sY, closing ? pl->R2inv.as<double>() : pl->Rinv.as<double>(),
                     pl->Z.as<double>()};
  }
  void qr(Buf b) {
    if (b == Buf::kY) {
      tall_chol(pl, pl->Y.as<float>(), pl->n, pl->Rinv.as<double>(), pl->Rinv_f.as<float>(), shift, true);
      return;
    }
    const int ld = (int)pl->ld;
    int s = stage_begin(pl);
    small_qr(pl, pl->Z.as<double>(), shift);
    CK(launch_round_v(pl->Z.as<double>(), pl->g, ld, mu, pl->V.as<float>(), pl->mc.as<float>(), pl->stream));
    if (pl->pflog) CK(launch_aug_colsum(pl->V.as<float>(), (int32_t)pl->g_user, ld, pl->stream));
    stage_end(pl, SCXPCA_STAGE_SMALL, s);
  }
  void rmatmat() {
    const int ld = (int)pl->ld;
    rmatmat_raw(pl, pl->Y.as<float>(), 0);
    int s = stage_begin(pl);
    if (pl->pflog) CK(launch_aug_fold(pl->W.as<double>(), (int32_t)pl->g_user, ld, pl->stream, pl->num_sms));
    CK(launch_center_apply(pl->W.as<double>(), pl->g, ld, mu, sY,
                           closing ? pl->R2inv.as<double>() : pl->Rinv.as<double>(), pl->Z.as<double>(), pl->stream));
    stage_end(pl, SCXPCA_STAGE_SMALL, s);
  }
  void apply_q() {  // Y <- Y Rinv_f, with the 16-bit image on the tensor-core path
    const int ld = (int)pl->ld;
    int s = stage_begin(pl);
    if (pl->use_tc)
      CK(launch_apply_right_split(pl->Y.as<float>(), pl->n, ld, pl->Rinv_f.as<float>(), pl->Y.as<float>(),
                                  pl->Yimg.as<uint16_t>(), pl->fmt16, pl->stream, pl->num_sms));
    else
      CK(launch_apply_right_f32(pl->Y.as<float>(), pl->n, ld, pl->Rinv_f.as<float>(), pl->Y.as<float>(), pl->stream,
                                pl->num_sms));
    stage_end(pl, SCXPCA_STAGE_APPLY, s);
  }
  // qr(b) around its k x k Cholesky, for a batch that factors every
  // segment's Gram in one launch: qr_gram, then the factorisation of
  // qr_task(), then qr_after.
  void qr_gram(Buf b) {
    if (b == Buf::kY) {
      tall_gram(pl, pl->Y.as<float>(), pl->n, true);
      return;
    }
    int s = stage_begin(pl);
    small_gram(pl, pl->Z.as<double>());
    stage_end(pl, SCXPCA_STAGE_SMALL, s);
  }
  CholTask qr_task() { return gram_chol_task(pl, pl->Rinv.as<double>(), pl->Rinv_f.as<float>()); }
  void qr_after(Buf b) {
    if (b == Buf::kY) return;
    const int ld = (int)pl->ld;
    int s = stage_begin(pl);
    small_apply(pl, pl->Z.as<double>());
    CK(launch_round_v(pl->Z.as<double>(), pl->g, ld, mu, pl->V.as<float>(), pl->mc.as<float>(), pl->stream));
    if (pl->pflog) CK(launch_aug_colsum(pl->V.as<float>(), (int32_t)pl->g_user, ld, pl->stream));
    stage_end(pl, SCXPCA_STAGE_SMALL, s);
  }
  // finalize_q in the same way: each pass is finalize_gram, then the
  // factorisation of finalize_task(); then the operator is closing.
  void finalize_gram() {
    apply_q();
    tall_gram(pl, pl->Y.as<float>(), pl->n, true);
  }
  CholTask finalize_task() { return gram_chol_task(pl, pl->R2inv.as<double>(), pl->Rinv_f.as<float>()); }
  void finalize_q() {
    // Explicit Q = Y R^{-1}, re-orthonormalised by a second FP64 Cholesky pass.
    apply_q();
    tall_chol(pl, pl->Y.as<float>(), pl->n, pl->R2inv.as<double>(), pl->Rinv_f.as<float>(), shift, true);
    if (shift) {
      // Householder contract (an orthonormal Q whatever the conditioning):
      // when the first factorisation had to be shifted, CholeskyQR2 leaves Q
      // with an orthogonality error of about u cond(Q1); a third pass (shifted
      // CholeskyQR3) brings it to working precision.  Applied unconditionally
      // in this mode, so the enqueued sequence does not depend on device results.
      apply_q();
      tall_chol(pl, pl->Y.as<float>(), pl->n, pl->R2inv.as<double>(), pl->Rinv_f.as<float>(), shift, true);
    }
    closing = true;
  }
};

// Enqueue one run on the plan's stream: power loop, Rayleigh-Ritz step and
// embeddings into the device buffer U (n_obs x n_components).  No host
// synchronisation and, when omega is NULL or device memory, no allocation:
// the sequence can be captured into a CUDA graph.
DeviceOperator device_operator(scxpca_plan* pl, const scxpca_params& p) {
  const int ld = (int)pl->ld;
  return DeviceOperator{pl, p, p.qr_method == SCXPCA_QR_HOUSEHOLDER ? 1 : 0, pl->use_tc && ld == 64,
                        pl->centered ? pl->d_mu.as<double>() : nullptr,
                        pl->G.as<double>() + (size_t)ld * ld};  // column sums follow the Gram
}

void enqueue_finish(scxpca_plan* pl, float* U);

void enqueue_run(scxpca_plan* pl, const scxpca_params& p, float* U) {
  CK(cudaMemsetAsync(pl->status.p, 0, sizeof(int) * 4, pl->stream));
  DeviceOperator op = device_operator(pl, p);
  run_power_loop(op, p.n_power_iterations);
  enqueue_finish(pl, U);
}

// After the loop: the SVD of B (in Z) through the FP64 eigendecomposition of
// B^T B, the components, and the embeddings U = Q R2^{-1} E Sigma.  In parts
// (finish_gram, the eigensolve of finish_task, finish_after) for a batch that
// solves every segment's eigenproblem in one launch.
void finish_gram(scxpca_plan* pl) {
  int s = stage_begin(pl);
  small_gram(pl, pl->Z.as<double>());
  stage_end(pl, SCXPCA_STAGE_SMALL, s);
}

JacobiTask finish_task(scxpca_plan* pl) {
  return JacobiTask{pl->G.as<double>(), pl->evals.as<double>(), pl->evecs.as<double>(), pl->status.as<int>() + 2};
}

// The Rayleigh-Ritz finish's arguments, as one task of a batched launch.
RitzTask ritz_task(scxpca_plan* pl) {
  return RitzTask{pl->Z.as<double>(), pl->evals.as<double>(), pl->evecs.as<double>(), pl->R2inv.as<double>(),
                  pl->sigma.as<double>(), pl->comps.as<float>(), pl->M_emb.as<float>()};
}

// Embeddings U = Q R2^{-1} E Sigma (first n_components).
void finish_embed(scxpca_plan* pl, float* U) {
  int s = stage_begin(pl);
  if (pl->use_tc && pl->ld == 64 && pl->embed_tc && !pl->streaming)
    CK(launch_embed_tc(pl->n, &pl->qmap, pl->M_emb.as<float>(), (int)pl->nc, U, pl->fmt16, pl->tc_err.as<int>(),
                       pl->stream, pl->num_sms));
  else
    CK(launch_embed(pl->Y.as<float>(), pl->n, (int)pl->ld, (int)pl->k, pl->M_emb.as<float>(), (int)pl->nc, U,
                    pl->stream, pl->num_sms));
  stage_end(pl, SCXPCA_STAGE_EMBED, s);
}

void finish_after(scxpca_plan* pl, float* U) {
  const RitzTask t = ritz_task(pl);
  int s = stage_begin(pl);
  CK(launch_ritz_finish(t.B, pl->g, (int)pl->ld, (int)pl->k, (int)pl->nc, t.evals, t.evecs, t.Rinv2, t.sigma,
                        t.comps, t.M_emb, pl->stream));
  stage_end(pl, SCXPCA_STAGE_SMALL, s);
  finish_embed(pl, U);
}

void enqueue_finish(scxpca_plan* pl, float* U) {
  finish_gram(pl);
  int s = stage_begin(pl);
  CK(launch_jacobi_eig(pl->G.as<double>(), (int)pl->k, (int)pl->ld, pl->evals.as<double>(), pl->evecs.as<double>(),
                       pl->status.as<int>() + 2, pl->stream));
  stage_end(pl, SCXPCA_STAGE_SMALL, s);
  finish_after(pl, U);
}

// Host side of a finished run: the status words and singular values copied
// back from the device -> the result record.
void finish_result(scxpca_plan* pl, const int* hstatus, const double* sigma, scxpca_result* out) {
  if (hstatus[0] < 0)
    fail(SCXPCA_NOT_SPD, "CholeskyQR2 failed: non-SPD; retry with qr_method='householder'");
  const double denom = std::max<double>((double)pl->n - 1.0, 1.0);
  for (int64_t c = 0; c < pl->nc; ++c) {
    double ve = sigma[c] * sigma[c] / denom;
    if (out->variance_explained) out->variance_explained[c] = ve;
    if (out->variance_ratio) out->variance_ratio[c] = pl->total_var > 0.0 ? ve / pl->total_var : 0.0;
    if (out->singular_values) out->singular_values[c] = sigma[c];
  }
  if (out->mean) {
    for (int64_t j = 0; j < pl->g_user; ++j) out->mean[j] = pl->mean_x[j];
  }
  if (out->std) {
    for (int64_t j = 0; j < pl->g_user; ++j) out->std[j] = pl->std_x.empty() ? 1.0 : pl->std_x[j];
  }
  out->resident_csr = pl->streaming ? 0 : 1;
  out->n_shards = pl->streaming ? (int32_t)pl->shards.size() : 0;
  out->total_var_recomputed = pl->total_var_recomputed ? 1 : 0;
  out->shifted_cholesky = hstatus[0] > 0 ? hstatus[0] : 0;
  out->eig_sweeps = hstatus[2];
  out->total_var = pl->total_var;
  pl->run_valid = true;
}

// One run on the plan's stream.  A plan run again with the same power
// iterations, seed, omega and embeddings buffer replays the graph of that run
// (recorded on its second occurrence); stage profiling, a host omega (staged
// by an allocation) and SCXPCA_GRAPH=0 keep the plain launches.
void enqueue_run_replayed(scxpca_plan* pl, const scxpca_params& p, float* U) {
  const char* env = getenv("SCXPCA_GRAPH");
  const bool allowed = !(env && env[0] == '0') && !pl->profiling && !pl->streaming &&
                       (!p.omega || p.omega_memory == SCXPCA_MEM_DEVICE);
  scxpca_plan::RunGraph& g = pl->rg;
  const bool same = g.q == p.n_power_iterations && g.seed == p.seed && g.omega == p.omega && g.U == U;
  if (allowed && same && g.exec) {
    CK(cudaGraphLaunch(g.exec, pl->stream));
    pl->prof.kernel_launches += g.launches;
    return;
  }
  if (!allowed || !same || !g.seen) {
    if (!same) {
      if (g.exec) CK(cudaGraphExecDestroy(g.exec));
      g = scxpca_plan::RunGraph{};
      g.q = p.n_power_iterations;
      g.seed = p.seed;
      g.omega = p.omega;
      g.U = U;
    }
    g.seen = true;
    const int64_t launches0 = launches_total();
    enqueue_run(pl, p, U);
    pl->prof.kernel_launches += launches_total() - launches0;
    return;
  }
  // second run with this key: record it, then replay
  cudaGraph_t graph = nullptr;
  const int64_t launches0 = launches_total();
  CK(cudaStreamBeginCapture(pl->stream, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_run(pl, p, U);
  } catch (...) {
    cudaStreamEndCapture(pl->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    throw;
  }
  g.launches = launches_total() - launches0;
  CK(cudaStreamEndCapture(pl->stream, &graph));
  cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    g.exec = nullptr;
    CK(e);
  }
  CK(cudaGraphLaunch(g.exec, pl->stream));
  pl->prof.kernel_launches += g.launches;
}

void run_plan(scxpca_plan* pl, const scxpca_params* over, scxpca_result* out) {
  if (!out) fail(SCXPCA_INVALID_ARGUMENT, "null result");
  if (!out->embeddings) fail(SCXPCA_INVALID_ARGUMENT, "null embeddings output");
  const scxpca_params p = run_params(pl, over);
  cudaStream_t st = pl->stream;
  float* U = out->embeddings;
  const bool host_out = out->embeddings_memory != SCXPCA_MEM_DEVICE;
  if (host_out) {
    pl->U.alloc(sizeof(float) * pl->n * pl->nc);
    U = pl->U.as<float>();
  }
  enqueue_run_replayed(pl, p, U);
  pl->prof.runs += 1;
  phase_mark(SCXPCA_PHASE_PCA, st);
  if (host_out)
    CK(cudaMemcpyAsync(out->embeddings, U, sizeof(float) * pl->n * pl->nc, cudaMemcpyDeviceToHost, st));

  int hstatus[4];
  std::vector<double> sigma(pl->k);
  CK(cudaMemcpyAsync(hstatus, pl->status.p, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(sigma.data(), pl->sigma.p, sizeof(double) * pl->k, cudaMemcpyDeviceToHost, st));
  if (out->components)  // the first g_user loadings of every component row
    CK(cudaMemcpy2DAsync(out->components, sizeof(float) * pl->g_user, pl->comps.p, sizeof(float) * pl->g,
                         sizeof(float) * pl->g_user, pl->nc, cudaMemcpyDeviceToHost, st));
  phase_mark(SCXPCA_PHASE_DOWNLOAD, st);
  CK(cudaStreamSynchronize(st));
  collect_stages(pl);
  check_tc_error(pl);
  finish_result(pl, hstatus, sigma.data(), out);
}

// ---------------------------------------------------------------------------
// Backward pass of the scores S = X~ V_c (truncated-SVD adjoint; the
// derivation is in kernels_adjoint.cu).  Uses the last run's Ritz state: B in
// Z, the eigenvectors E and eigenvalues lambda = sigma^2 of B^T B.
// ---------------------------------------------------------------------------
void backward(scxpca_plan* pl, const float* S, const float* GS, int iters, float* gvals, double* gcenter,
              double* gscale) {
  if (!pl->run_valid)
    fail(SCXPCA_INVALID_ARGUMENT, "backward needs the state of a completed run: call scxpca_plan_run first, "
                                  "with no other call on the plan in between");
  if (pl->clip > 0) fail(SCXPCA_UNSUPPORTED, "the backward pass does not support clipped values (clip_max > 0)");
  if (pl->rows_resorted)
    fail(SCXPCA_UNSUPPORTED, "the plan re-sorted unsorted CSR rows, so gradients would not follow the caller's "
                             "entry order; sort each row by gene before creating the plan");
  if (pl->streaming)
    fail(SCXPCA_UNSUPPORTED, "the backward pass needs the matrix resident on the device; this plan streams it "
                             "from host memory");
  if (pl->ld > kMaxK)
    fail(SCXPCA_UNSUPPORTED, "the backward pass takes sketches of at most " + std::to_string(kMaxK) + " columns");
  if (iters < 0 || iters > 1000) fail(SCXPCA_INVALID_ARGUMENT, "solve_iterations must be in [0, 1000]");
  if (!S || !GS || !gvals) fail(SCXPCA_INVALID_ARGUMENT, "null scores, grad_scores or grad_values");
  pl->run_valid = false;
  cudaStream_t st = pl->stream;
  const int64_t n = pl->n, g = pl->g;
  const int ld = (int)pl->ld, k = (int)pl->k, c = (int)pl->nc;
  const double* mu = pl->centered ? pl->d_mu.as<double>() : nullptr;
  const size_t gl = sizeof(double) * g * ld;
  for (DevBuf* b : {&pl->bw_Vk, &pl->bw_H, &pl->bw_A, &pl->bw_X, &pl->bw_R, &pl->bw_P, &pl->bw_Ap, &pl->bw_Proj})
    b->alloc(gl);
  pl->bw_T.alloc(sizeof(double) * ld * ld);
  pl->bw_M.alloc(sizeof(double) * ld * ld);
  pl->bw_vec.alloc(sizeof(double) * ld * 8);
  pl->bw_colD.alloc(sizeof(double) * g);
  pl->bw_sumDP.alloc(sizeof(double) * g);
  pl->bw_part.alloc(sizeof(double) * (size_t)pl->nchunks * g);
  ensure_rbp(pl);
  const int cparts = (int)std::max<int64_t>(1, std::min<int64_t>(2 * pl->num_sms, (n + 255) / 256));
  pl->bw_cpart.alloc(sizeof(double) * (size_t)cparts * 256);
  double* vec = pl->bw_vec.as<double>();
  double *sG = vec, *sY = vec + ld, *sS = vec + 2 * ld, *sF = vec + 3 * ld, *rr = vec + 4 * ld,
         *rr_new = vec + 5 * ld, *pAp = vec + 6 * ld;
  double *Vk = pl->bw_Vk.as<double>(), *H = pl->bw_H.as<double>(), *A = pl->bw_A.as<double>(),
         *X = pl->bw_X.as<double>(), *R = pl->bw_R.as<double>(), *P = pl->bw_P.as<double>(),
         *Ap = pl->bw_Ap.as<double>(), *Proj = pl->bw_Proj.as<double>(), *T = pl->bw_T.as<double>(),
         *M = pl->bw_M.as<double>();
  const double* evals = pl->evals.as<double>();
  const double* eye = pl->eye.as<double>();
  float* Y = pl->Y.as<float>();
  auto colsum = [&](const float* src, int ldsrc, int ncols, double* out) {
    CK(launch_colsum_f32(src, n, ldsrc, ncols, pl->bw_cpart.as<double>(), cparts, out, st, pl->num_sms));
  };
  // X~^T (tall float in Y) -> (g x ld) FP64 in `out`, centring folded in
  auto apply_t = [&](int split, double* out) {
    colsum(Y, ld, ld, sY);
    rmatmat_raw(pl, Y, split);
    CK(launch_center_apply(pl->W.as<double>(), g, ld, mu, sY, eye, out, st));
  };
  // Y = X~ Vg for a gene-side FP64 block Vg
  auto apply_f = [&](const double* Vg) {
    CK(launch_round_v(Vg, g, ld, mu, pl->V.as<float>(), pl->mc.as<float>(), st));
    forward(pl);
  };

  // Ritz vectors of the gene side: Vk = B E diag(1 / sigma)
  CK(launch_ritz_scale(pl->evecs.as<double>(), evals, k, ld, M, st));
  CK(launch_center_apply(pl->Z.as<double>(), g, ld, nullptr, nullptr, M, Vk, st));
  // H = X~^T G
  CK(cudaMemsetAsync(Y, 0, sizeof(float) * n * ld, st));
  CK(cudaMemcpy2DAsync(Y, sizeof(float) * ld, GS, sizeof(float) * c, sizeof(float) * c, n, cudaMemcpyDeviceToDevice,
                       st));
  colsum(Y, ld, ld, sG);
  apply_t(1, H);
  // inside the sketch subspace: A_in = Vk Phi, Phi_ji = (Vk^T H)_ji / (lambda_i - lambda_j)
  CK(launch_atb(Vk, H, g, ld, k, c, T, st));
  CK(launch_phi(T, evals, k, c, ld, M, st));
  CK(launch_center_apply(Vk, g, ld, nullptr, nullptr, M, A, st));
  // outside it: (lambda_i I - X~^T X~) x_i = r_i on the complement, r = H - Vk (Vk^T H), by CG
  CK(launch_center_apply(Vk, g, ld, nullptr, nullptr, T, Proj, st));
  CK(launch_axpy_cols(H, Proj, -1.0, g, ld, c, R, st));
  CK(cudaMemsetAsync(X, 0, gl, st));
  CK(cudaMemcpyAsync(P, R, gl, cudaMemcpyDeviceToDevice, st));
  CK(launch_coldot(R, R, g, ld, c, rr, st));
  for (int m = 0; m < iters; ++m) {
    apply_f(P);
    apply_t(0, H);  // H <- X~^T X~ P
    CK(launch_atb(Vk, H, g, ld, k, c, T, st));
    CK(launch_center_apply(Vk, g, ld, nullptr, nullptr, T, Proj, st));
    CK(launch_cg_ap(P, H, Proj, evals, g, ld, c, Ap, st));
    CK(launch_coldot(P, Ap, g, ld, c, pAp, st));
    CK(launch_cg_step(X, R, P, Ap, rr, pAp, g, ld, c, st));
    CK(launch_coldot(R, R, g, ld, c, rr_new, st));
    CK(launch_cg_dir(P, R, rr, rr_new, g, ld, c, st));
  }
  CK(launch_axpy_cols(A, X, 1.0, g, ld, c, A, st));
  // F = G + X~ A ; column sums of F and S ; column sums of D
  apply_f(A);
  colsum(Y, ld, ld, sY);
  colsum(S, c, c, sS);
  CK(launch_axpy_cols(sG, sY, 1.0, 1, ld, c, sF, st));
  CK(launch_col_d(Vk, A, sF, sS, g, ld, c, pl->bw_colD.as<double>(), st));
  // SDDMM at the stored entries, 64 columns at a time
  for (int c0 = 0; c0 < c; c0 += 64) {
    const int cs = std::min(64, c - c0);
    CK(launch_sddmm(pl->dtype, pl->indptr, pl->idx, pl->val, n, (int32_t)g, pl->rbp.as<int32_t>(), pl->nb,
                    pl->nchunks, pl->rows_per_chunk, GS + c0, c, Y + c0, ld, S + c0, c, Vk + c0, A + c0, ld, cs,
                    pl->d_scale_raw.as<double>(), c0 > 0, gvals, pl->bw_part.as<double>(), st));
    CK(launch_reduce_rows_f64(pl->bw_part.as<double>(), pl->nchunks, g, pl->bw_sumDP.as<double>(), c0 > 0, st,
                              pl->num_sms));
  }
  if (gcenter || gscale)
    CK(launch_grad_vectors(pl->bw_colD.as<double>(), pl->bw_sumDP.as<double>(), pl->d_center_raw.as<double>(),
                           pl->d_scale_raw.as<double>(), g, gcenter, gscale, st));
  CK(cudaStreamSynchronize(st));
  check_tc_error(pl);
}

template <typename F>
int32_t guarded(char* err, size_t err_len, F&& f) {
  try {
    f();
    write_err(err, err_len, "");
    return SCXPCA_OK;
  } catch (const Failure& e) {
    write_err(err, err_len, e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    write_err(err, err_len, "host allocation failed");
    return SCXPCA_OUT_OF_MEMORY;
  } catch (...) {
    write_err(err, err_len, "unexpected internal error");
    return SCXPCA_CUDA_ERROR;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Batched sub-PCAs: one resident plan per row segment of one CSR, all runs
// recorded into one CUDA graph whose parallel branches each take a list of
// segments, launched as a single graph; or, for comparison, one plain
// (synchronising) plan run per segment.
// ---------------------------------------------------------------------------
struct scxpca_batch {
  int device = 0;
  cudaStream_t main = nullptr;
  bool own_main = false;
  std::vector<cudaStream_t> branch;   // fork streams of the capture
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  std::vector<scxpca_plan*> plans;     // one per segment
  std::vector<int64_t> offsets;        // segment row offsets (n_segments + 1)
  std::vector<DevBuf*> indptrs;        // rebased device indptr of each segment (owned)
  std::vector<double> seg_ms;          // measured plain-run time of each segment (schedule weights)
  int64_t n_obs = 0, n_vars = 0, nc = 0, k = 0;
  DevBuf emb;                          // n_obs x n_components, written by the graph
  int32_t* h_status = nullptr;         // pinned: [seg][4]
  double* h_sigma = nullptr;           // pinned: [seg][k]
  float* h_comps = nullptr;            // pinned: [seg][nc][n_vars]
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int branches = 0;
  bool lockstep = false;               // schedule of the recorded graph (see batch_capture)
  size_t graph_nodes = 0;
  // graph time per tried schedule: [0..5] segment-per-branch with 1, 2, 4, 8,
  // 16, 32 branches; [6..11] lockstep over as many streams
  double tuned_ms[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  scxpca_params params{};
  // the lockstep schedule's batched launches: one task per segment for the
  // loop's Cholesky (R^{-1}), the closing one (R2^{-1}) and the eigensolve;
  // and for the gene-side work (V's image, the centring + R^{-1} apply of the
  // transposed product in the loop and at the close, Z's Gram, Z R^{-1},
  // the rounding of Z into V)
  DevBuf task_qr, task_fin, task_eig;
  DevBuf task_split, task_apply_loop, task_apply_close, task_small_apply, task_gram_z, task_round, task_ritz;
  // the lockstep schedule's tensor-core products at ld 64: every segment's
  // forward product, transposed product and Gram in one launch each, with
  // the per-segment sums of their partials in one launch
  DevBuf tc_segs, tc_maps, band_seg, rmat_items, gram_items, rmat_sums, gram_sums;
  int64_t n_bands = 0;
  int n_rmat_items = 0, n_gram_items = 0;
  // and the tall right-multiplications (Y R^{-1} with its image, the
  // embeddings) over the row tiles of every segment, one launch each
  DevBuf task_tall_q, task_tall_emb;
  int64_t tall_tiles = 0;
  // and the results: every segment's status words zeroed by one launch at the
  // start, its status, sigma and components gathered into the d_* buffers by
  // one launch at the end and copied to the pinned host buffers in three
  DevBuf task_out, d_status, d_sigma, d_comps;

  ~scxpca_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    // buffers are freed in the order of the main stream: before it goes
    for (scxpca_plan* pl : plans) delete pl;
    for (DevBuf* b : indptrs) delete b;
    emb.release();
    for (DevBuf* t : {&task_qr, &task_fin, &task_eig, &task_split, &task_apply_loop, &task_apply_close,
                      &task_small_apply, &task_gram_z, &task_round, &task_ritz, &tc_segs, &tc_maps, &band_seg,
                      &rmat_items, &gram_items, &rmat_sums, &gram_sums, &task_tall_q, &task_tall_emb, &task_out,
                      &d_status, &d_sigma, &d_comps})
      t->release();
    for (cudaStream_t st : branch) cudaStreamDestroy(st);
    for (cudaEvent_t e : join) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (h_status) cudaFreeHost(h_status);
    if (h_sigma) cudaFreeHost(h_sigma);
    if (h_comps) cudaFreeHost(h_comps);
    if (own_main && main) cudaStreamDestroy(main);
  }
};

namespace {

constexpr int kMaxBranches = 32;

void batch_free_graph(scxpca_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_nodes = 0;
}

// Longest-processing-time schedule of the segments over `nb` branches, by
// their measured plain-run times; each branch runs its list in order.
std::vector<std::vector<int>> batch_schedule(const scxpca_batch* b, int nb) {
  const int ns = (int)b->plans.size();
  std::vector<int> order(ns);
  for (int i = 0; i < ns; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int x, int y) { return b->seg_ms[x] > b->seg_ms[y]; });
  std::vector<std::vector<int>> lists(nb);
  std::vector<double> load(nb, 0.0);
  for (int i : order) {
    const int t = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lists[t].push_back(i);
    load[t] += b->seg_ms[i];
  }
  return lists;
}

// The copies of a segment's status, singular values and components to the
// batch's pinned host buffers, on the segment's current stream.
void batch_copy_out(scxpca_batch* b, int q) {
  scxpca_plan* pl = b->plans[q];
  cudaStream_t st = pl->stream;
  CK(cudaMemcpyAsync(b->h_status + 4 * q, pl->status.p, sizeof(int) * 3, cudaMemcpyDeviceToHost, st));
  if (pl->use_tc)
    CK(cudaMemcpyAsync(b->h_status + 4 * q + 3, pl->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(b->h_sigma + b->k * q, pl->sigma.p, sizeof(double) * pl->k, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(b->h_comps + (size_t)b->nc * b->n_vars * q, pl->comps.p, sizeof(float) * pl->nc * pl->g,
                     cudaMemcpyDeviceToHost, st));
}

// The lockstep schedule's operator: every step of run_power_loop is taken by
// all segments at once, each segment on its branch stream (the branches fork
// from the main stream before the step and join it after), so the segments'
// products run together and then their small factorisations run together.
struct BatchOperator {
  scxpca_batch* b;
  std::vector<DeviceOperator> ops;  // one per segment
  std::vector<int> branch_of;       // segment -> branch
  int nb;
  // every segment's k x k Cholesky of a step in ONE launch on the main
  // stream (one block per segment) between the step's two forked halves,
  // instead of one single-block launch per segment on its branch
  bool small_batched = false;
  // the gene-side work of every segment (n_vars x k, the same size for all)
  // in one launch per kernel on the main stream as well
  bool gene_batched = false;
  // the tensor-core products (ld 64) of every segment in one launch each
  bool tc_batched = false;

  template <class F>
  void each(F&& f) {
    CK(cudaEventRecord(b->fork, b->main));
    for (int t = 0; t < nb; ++t) CK(cudaStreamWaitEvent(b->branch[t], b->fork, 0));
    for (size_t q = 0; q < ops.size(); ++q) {
      ops[q].pl->stream = b->branch[branch_of[q]];
      f((int)q, ops[q]);
    }
    for (int t = 0; t < nb; ++t) {
      CK(cudaEventRecord(b->join[t], b->branch[t]));
      CK(cudaStreamWaitEvent(b->main, b->join[t], 0));
    }
  }
  const scxpca_plan* p0() const { return ops[0].pl; }
  int ns() const { return (int)ops.size(); }
  // Y = (X - mu) V for every segment: V's images, then one launch over all
  // bands; the FP32 Y only for the loop's last product (finalize_q reads it)
  void fwd_all(bool last) {
    const scxpca_plan* p = p0();
    CK(launch_split16_batch(b->task_split.as<SplitTask>(), ns(), p->g * p->ld, p->fmt16, b->main));
    CK(launch_fwd_tc_batch(b->tc_segs.as<TcSegment>(), b->band_seg.as<int32_t>(), b->n_bands, p->n_chunks,
                           last ? 1 : 0, p->fmt16, b->main, p->num_sms));
  }
  // W = X^T Q (raw) for every segment: the partials, then their sums
  void rmat_all() {
    const scxpca_plan* p = p0();
    CK(launch_rmat_tc_batch(b->tc_segs.as<TcSegment>(), b->rmat_items.as<TcItem>(), b->n_rmat_items, p->n_chunks,
                            p->g, p->tc_gene_groups, p->fmt16, b->main));
    CK(launch_reduce_rows_batch(1, b->rmat_sums.as<SumTask>(), ns(), p->g * p->ld, b->main));
  }
  // Y's Gram and column sums (from its image) for every segment
  void gram_all() {
    const scxpca_plan* p = p0();
    CK(launch_gram_tc_batch(b->tc_segs.as<TcSegment>(), b->gram_items.as<TcItem>(), b->n_gram_items, p->fmt16,
                            b->main));
    CK(launch_reduce_rows_batch(0, b->gram_sums.as<SumTask>(), ns(), p->ld * p->ld + p->ld, b->main));
  }
  // Omega for every segment: one batch has one (n_vars, k, seed or explicit
  // Omega), so segment 0 fills its V as a lone plan would and the others copy
  // it; then every segment's mean prefactor in one launch
  void load_omega_all() {
    scxpca_plan* p = ops[0].pl;
    p->stream = b->main;
    load_omega_v(p, &ops[0].p);
    CK(launch_broadcast_v(p->V.as<float>(), p->g * p->ld, b->task_round.as<RoundTask>(), ns(), b->main));
    CK(launch_mean_prefactor_batch(b->task_round.as<RoundTask>(), ns(), p->g, (int)p->ld, b->main));
  }
  void matmat(Operand src, bool last) {
    if (tc_batched) {
      if (src == Operand::kOmega) load_omega_all();
      fwd_all(last);
      return;
    }
    if (!gene_batched || src == Operand::kOmega) {
      each([&](int, DeviceOperator& o) { o.matmat(src, last); });
      return;
    }
    if (p0()->use_tc)
      CK(launch_split16_batch(b->task_split.as<SplitTask>(), ns(), p0()->g * p0()->ld, p0()->fmt16, b->main));
    each([&](int, DeviceOperator& o) { o.matmat_products(last); });
  }
  void rmatmat() {
    if (!gene_batched) {
      each([&](int, DeviceOperator& o) { o.rmatmat(); });
      return;
    }
    if (tc_batched)
      rmat_all();
    else
      each([&](int, DeviceOperator& o) { o.rmatmat_products(); });
    const DevBuf& t = ops[0].closing ? b->task_apply_close : b->task_apply_loop;
    CK(launch_center_apply_batch(t.as<ApplyTask>(), ns(), p0()->g, (int)p0()->ld, b->main));
  }
  // Z's Gram for every segment (the closing one, or qr(Z)'s), on the main stream
  void gram_z_all() {
    CK(launch_gram_f64_batch(b->task_gram_z.as<GramTask>(), ns(), p0()->g, (int)p0()->ld, p0()->gram_parts_small,
                             b->main, p0()->num_sms));
  }
  void chol_all(const DevBuf& tasks) {
    const scxpca_plan* p0 = ops[0].pl;
    CK(launch_cholesky_batch(tasks.as<CholTask>(), (int)ops.size(), (int)p0->k, (int)p0->ld, p0->tau,
                             ops[0].shift, b->main));
  }
  void qr(Buf x) {
    if (!small_batched) {
      each([&](int, DeviceOperator& o) { o.qr(x); });
      return;
    }
    if (x == Buf::kZ && gene_batched) {
      // all on the main stream: Gram, factor, Z R^{-1}, rounding into V
      gram_z_all();
      chol_all(b->task_qr);
      CK(launch_center_apply_batch(b->task_small_apply.as<ApplyTask>(), ns(), p0()->g, (int)p0()->ld, b->main));
      CK(launch_round_v_batch(b->task_round.as<RoundTask>(), ns(), p0()->g, (int)p0()->ld, b->main));
      return;
    }
    if (x == Buf::kY && tc_batched)
      gram_all();
    else
      each([&](int, DeviceOperator& o) { o.qr_gram(x); });
    chol_all(b->task_qr);
    if (x == Buf::kZ) each([&](int, DeviceOperator& o) { o.qr_after(x); });
  }
  void finalize_q() {
    if (!small_batched) {
      each([&](int, DeviceOperator& o) { o.finalize_q(); });
      return;
    }
    const int passes = ops[0].shift ? 2 : 1;  // the Householder contract's third pass (DeviceOperator::finalize_q)
    for (int pass = 0; pass < passes; ++pass) {
      if (tc_batched) {
        CK(launch_apply_upper64_batch(b->task_tall_q.as<TallTask>(), ns(), b->tall_tiles, p0()->fmt16, b->main,
                                      p0()->num_sms));
        gram_all();
      } else {
        each([&](int, DeviceOperator& o) { o.finalize_gram(); });
      }
      chol_all(b->task_fin);
    }
    for (DeviceOperator& o : ops) o.closing = true;
  }
};

// Upload the batched launches' task tables (before a capture).  The batched
// kernels take k, ld <= 128 and one (k, ld) for all segments; otherwise the
// lockstep schedule keeps one launch per segment.
bool batch_prepare_tasks(scxpca_batch* b, BatchOperator& bop) {
  const scxpca_plan* p0 = b->plans[0];
  for (const scxpca_plan* pl : b->plans)
    if (pl->k != p0->k || pl->ld != p0->ld) return false;
  if (p0->ld > kMaxK) return false;
  const size_t ns = b->plans.size();
  std::vector<CholTask> tq(ns), tf(ns);
  std::vector<JacobiTask> te(ns);
  for (size_t q = 0; q < ns; ++q) {
    tq[q] = bop.ops[q].qr_task();
    tf[q] = bop.ops[q].finalize_task();
    te[q] = finish_task(b->plans[q]);
  }
  auto put = [&](DevBuf& buf, const void* src, size_t bytes) {
    buf.alloc(bytes);
    CK(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, b->main));
  };
  put(b->task_qr, tq.data(), sizeof(CholTask) * ns);
  put(b->task_fin, tf.data(), sizeof(CholTask) * ns);
  put(b->task_eig, te.data(), sizeof(JacobiTask) * ns);
  // the gene-side tables: every segment has n_vars rows of the same k columns
  bool gene = true;
  for (const scxpca_plan* pl : b->plans)
    gene = gene && pl->use_tc == p0->use_tc && pl->fmt16 == p0->fmt16 && !pl->pflog && !pl->streaming &&
           pl->gram_parts_small == p0->gram_parts_small;
  if (gene) {
    std::vector<SplitTask> tsp(ns);
    std::vector<ApplyTask> tal(ns), tac(ns), tsa(ns);
    std::vector<GramTask> tg(ns);
    std::vector<RoundTask> tr(ns);
    std::vector<RitzTask> tz(ns);
    for (size_t q = 0; q < ns; ++q) {
      scxpca_plan* pl = b->plans[q];
      const DeviceOperator& o = bop.ops[q];
      tsp[q] = SplitTask{pl->V.as<float>(), pl->Vimg.as<uint16_t>()};
      tal[q] = ApplyTask{pl->W.as<double>(), o.mu, o.sY, pl->Rinv.as<double>(), pl->Z.as<double>()};
      tac[q] = ApplyTask{pl->W.as<double>(), o.mu, o.sY, pl->R2inv.as<double>(), pl->Z.as<double>()};
      tsa[q] = ApplyTask{pl->Z.as<double>(), nullptr, nullptr, pl->Rinv.as<double>(), pl->Z.as<double>()};
      tg[q] = GramTask{pl->Z.as<double>(), pl->gpart.as<double>(), pl->G.as<double>()};
      tr[q] = RoundTask{pl->Z.as<double>(), o.mu, pl->V.as<float>(), pl->mc.as<float>()};
      tz[q] = ritz_task(pl);
    }
    if (p0->use_tc) put(b->task_split, tsp.data(), sizeof(SplitTask) * ns);
    put(b->task_apply_loop, tal.data(), sizeof(ApplyTask) * ns);
    put(b->task_apply_close, tac.data(), sizeof(ApplyTask) * ns);
    put(b->task_small_apply, tsa.data(), sizeof(ApplyTask) * ns);
    put(b->task_gram_z, tg.data(), sizeof(GramTask) * ns);
    put(b->task_round, tr.data(), sizeof(RoundTask) * ns);
    put(b->task_ritz, tz.data(), sizeof(RitzTask) * ns);
  }
  bop.gene_batched = gene;
  // the tensor-core products: one segment table, the band numbering of the
  // forward product, and one item per CTA of each segment's transposed
  // product and Gram, partitioned exactly as the segment's own launches
  bool tc = gene && p0->use_tc && p0->ld == 64;
  for (const scxpca_plan* pl : b->plans)
    tc = tc && pl->use_tc && pl->ld == 64 && pl->n_chunks == p0->n_chunks && pl->tc_gene_groups == p0->tc_gene_groups;
  if (tc) {
    b->tc_maps.alloc(sizeof(CUtensorMap) * 2 * ns);
    const CUtensorMap* dmaps = b->tc_maps.as<CUtensorMap>();
    std::vector<CUtensorMap> maps(2 * ns);
    std::vector<TcSegment> segs(ns);
    std::vector<int32_t> bseg;
    std::vector<TcItem> ritems, gitems;
    std::vector<SumTask> rs(ns), gs(ns);
    std::vector<TallTask> tq_tall(ns), te_tall(ns);
    int64_t tile0 = 0;
    for (size_t q = 0; q < ns; ++q) {
      scxpca_plan* pl = b->plans[q];
      tq_tall[q] = TallTask{pl->Y.as<float>(), pl->Y.as<float>(), pl->Yimg.as<uint16_t>(), pl->Rinv_f.as<float>(),
                            pl->n, tile0};
      te_tall[q] = TallTask{pl->Y.as<float>(), b->emb.as<float>() + b->offsets[q] * b->nc, nullptr,
                            pl->M_emb.as<float>(), pl->n, tile0};
      tile0 += (pl->n + 127) / 128;
    }
    put(b->task_tall_q, tq_tall.data(), sizeof(TallTask) * ns);
    put(b->task_tall_emb, te_tall.data(), sizeof(TallTask) * ns);
    b->tall_tiles = tile0;
    std::vector<OutTask> to(ns);
    for (size_t q = 0; q < ns; ++q) {
      scxpca_plan* pl = b->plans[q];
      to[q] = OutTask{pl->status.as<int>(), pl->tc_err.as<int>(), pl->sigma.as<double>(), pl->comps.as<float>()};
      tc = tc && pl->g == b->n_vars;  // the component slots of the host buffer are n_vars long
    }
    put(b->task_out, to.data(), sizeof(OutTask) * ns);
    b->d_status.alloc(sizeof(int) * 4 * ns);
    b->d_sigma.alloc(sizeof(double) * b->k * ns);
    b->d_comps.alloc(sizeof(float) * (size_t)b->nc * b->n_vars * ns);
    int64_t band0 = 0;
    for (size_t q = 0; q < ns; ++q) {
      scxpca_plan* pl = b->plans[q];
      maps[2 * q] = pl->vmap;
      maps[2 * q + 1] = pl->qmap;
      const int64_t n_tiles = (pl->n + 127) / 128, bands = (n_tiles + 1) / 2;
      segs[q] = TcSegment{pl->tf_ent.as<uint32_t>(), pl->tf_meta.p, dmaps + 2 * q, dmaps + 2 * q + 1,
                          pl->mc.as<float>(), pl->Y.as<float>(), pl->Yimg.as<uint16_t>(), pl->tc_part.as<float>(),
                          pl->gpart.as<double>(), pl->tc_err.as<int>(), pl->n, band0};
      bseg.insert(bseg.end(), (size_t)bands, (int32_t)q);
      band0 += bands;
      const int R = pl->tc_row_groups, G = pl->tc_gene_groups;
      for (int rg = 0; rg < R; ++rg)
        for (int gg = 0; gg < G; ++gg)
          ritems.push_back(TcItem{(int32_t)q, gg, rg, 0, tc_range_begin(rg, R, n_tiles),
                                  tc_range_begin(rg + 1, R, n_tiles)});
      const int parts = gram_tc_parts(pl->n, pl->tc_gram_parts, pl->num_sms);
      for (int part = 0; part < parts; ++part)
        gitems.push_back(TcItem{(int32_t)q, 0, part, 0, tc_range_begin(part, parts, n_tiles),
                                tc_range_begin(part + 1, parts, n_tiles)});
      rs[q] = SumTask{pl->tc_part.p, pl->W.as<double>(), R, 0};
      gs[q] = SumTask{pl->gpart.p, pl->G.as<double>(), parts, 0};
    }
    // the longest items first, so the short ones fill the tail
    auto longer = [](const TcItem& x, const TcItem& y) { return x.t1 - x.t0 > y.t1 - y.t0; };
    std::stable_sort(ritems.begin(), ritems.end(), longer);
    std::stable_sort(gitems.begin(), gitems.end(), longer);
    put(b->tc_maps, maps.data(), sizeof(CUtensorMap) * 2 * ns);
    put(b->tc_segs, segs.data(), sizeof(TcSegment) * ns);
    put(b->band_seg, bseg.data(), sizeof(int32_t) * bseg.size());
    put(b->rmat_items, ritems.data(), sizeof(TcItem) * ritems.size());
    put(b->gram_items, gitems.data(), sizeof(TcItem) * gitems.size());
    put(b->rmat_sums, rs.data(), sizeof(SumTask) * ns);
    put(b->gram_sums, gs.data(), sizeof(SumTask) * ns);
    b->n_bands = band0;
    b->n_rmat_items = (int)ritems.size();
    b->n_gram_items = (int)gitems.size();
  }
  bop.tc_batched = tc;
  CK(cudaStreamSynchronize(b->main));
  return true;
}

// Record every segment's run (and the copies of its status, singular values
// and components to pinned host memory) into one graph over `nb` branches.
// Two schedules: segment per branch (a branch runs whole segments one after
// another, the longest first) or lockstep (all segments take each power-loop
// step together; BatchOperator).  Segments go to branches by a
// longest-processing-time schedule of their measured times either way.
void batch_capture(scxpca_batch* b, int nb, bool lockstep) {
  batch_free_graph(b);
  while ((int)b->branch.size() < nb) {
    cudaStream_t st;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->branch.push_back(st);
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->join.push_back(e);
  }
  const auto lists = batch_schedule(b, nb);
  const scxpca_params& p = b->params;
  BatchOperator bop{b, {}, std::vector<int>(b->plans.size(), 0), nb};
  if (lockstep) {
    for (int t = 0; t < nb; ++t)
      for (int q : lists[t]) bop.branch_of[q] = t;
    for (scxpca_plan* pl : b->plans) bop.ops.push_back(device_operator(pl, p));
    bop.small_batched = batch_prepare_tasks(b, bop);
  }
  CK(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeRelaxed));
  try {
    if (lockstep) {
      if (bop.tc_batched)
        CK(launch_zero_status(b->task_out.as<OutTask>(), (int)b->plans.size(), b->main));
      else
        bop.each([&](int, DeviceOperator& o) {
          CK(cudaMemsetAsync(o.pl->status.p, 0, sizeof(int) * 4, o.pl->stream));
        });
      run_power_loop(bop, p.n_power_iterations);
      if (bop.small_batched) {
        if (bop.gene_batched)
          bop.gram_z_all();
        else
          bop.each([&](int, DeviceOperator& o) { finish_gram(o.pl); });
        const scxpca_plan* p0 = b->plans[0];
        CK(launch_jacobi_eig_batch(b->task_eig.as<JacobiTask>(), (int)b->plans.size(), (int)p0->k, (int)p0->ld,
                                   b->main));
        if (bop.gene_batched) {
          CK(launch_ritz_finish_batch(b->task_ritz.as<RitzTask>(), (int)b->plans.size(), p0->g, (int)p0->ld,
                                      (int)p0->k, (int)p0->nc, b->main));
          if (bop.tc_batched) {
            const int ns = (int)b->plans.size();
            CK(launch_embed_batch(b->task_tall_emb.as<TallTask>(), ns, b->tall_tiles, (int)p0->ld, (int)p0->nc,
                                  b->main, p0->num_sms));
            CK(launch_gather_out(b->task_out.as<OutTask>(), ns, (int)b->k, b->nc * b->n_vars, b->d_status.as<int>(),
                                 b->d_sigma.as<double>(), b->d_comps.as<float>(), b->main));
            CK(cudaMemcpyAsync(b->h_status, b->d_status.p, sizeof(int) * 4 * ns, cudaMemcpyDeviceToHost, b->main));
            CK(cudaMemcpyAsync(b->h_sigma, b->d_sigma.p, sizeof(double) * b->k * ns, cudaMemcpyDeviceToHost,
                               b->main));
            CK(cudaMemcpyAsync(b->h_comps, b->d_comps.p, sizeof(float) * (size_t)b->nc * b->n_vars * ns,
                               cudaMemcpyDeviceToHost, b->main));
          } else {
            bop.each([&](int q, DeviceOperator& o) {
              finish_embed(o.pl, b->emb.as<float>() + b->offsets[q] * b->nc);
              batch_copy_out(b, q);
            });
          }
        } else {
          bop.each([&](int q, DeviceOperator& o) {
            finish_after(o.pl, b->emb.as<float>() + b->offsets[q] * b->nc);
            batch_copy_out(b, q);
          });
        }
      } else {
        bop.each([&](int q, DeviceOperator& o) {
          enqueue_finish(o.pl, b->emb.as<float>() + b->offsets[q] * b->nc);
          batch_copy_out(b, q);
        });
      }
    } else {
      CK(cudaEventRecord(b->fork, b->main));
      for (int t = 0; t < nb; ++t) {
        cudaStream_t st = b->branch[t];
        CK(cudaStreamWaitEvent(st, b->fork, 0));
        for (int q : lists[t]) {
          scxpca_plan* pl = b->plans[q];
          pl->stream = st;
          enqueue_run(pl, p, b->emb.as<float>() + b->offsets[q] * b->nc);
          batch_copy_out(b, q);
        }
        CK(cudaEventRecord(b->join[t], st));
        CK(cudaStreamWaitEvent(b->main, b->join[t], 0));
      }
    }
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(b->main, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    for (scxpca_plan* pl : b->plans) pl->stream = b->main;
    throw;
  }
  CK(cudaStreamEndCapture(b->main, &b->graph));
  for (scxpca_plan* pl : b->plans) pl->stream = b->main;
  CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  size_t nodes = 0;
  CK(cudaGraphGetNodes(b->graph, nullptr, &nodes));
  b->graph_nodes = nodes;
  b->branches = nb;
  b->lockstep = lockstep;
}

// One graph launch; returns its device time in ms.
double batch_launch_timed(scxpca_batch* b) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, b->main));
  CK(cudaGraphLaunch(b->exec, b->main));
  CK(cudaEventRecord(e1, b->main));
  CK(cudaStreamSynchronize(b->main));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

// Host results of every segment after a graph launch (pinned buffers).
void batch_collect(scxpca_batch* b, float* components, double* singular_values, double* variance_ratio,
                   double* variance_explained) {
  const int ns = (int)b->plans.size();
  std::vector<double> ve(b->nc), vr(b->nc), sv(b->nc);
  for (int q = 0; q < ns; ++q) {
    scxpca_plan* pl = b->plans[q];
    if (pl->use_tc && b->h_status[4 * q + 3] != 0)
      fail(SCXPCA_TIMEOUT, "segment " + std::to_string(q) + ": tensor-core pipeline wait timed out (site " +
                               std::to_string(b->h_status[4 * q + 3]) + ")");
    scxpca_result r{};
    r.variance_explained = ve.data();
    r.variance_ratio = vr.data();
    r.singular_values = sv.data();
    try {
      finish_result(pl, b->h_status + 4 * q, b->h_sigma + b->k * q, &r);
    } catch (const Failure& f) {
      fail(f.code, "segment " + std::to_string(q) + ": " + f.msg);
    }
    for (int64_t c = 0; c < b->nc; ++c) {
      if (singular_values) singular_values[q * b->nc + c] = sv[c];
      if (variance_ratio) variance_ratio[q * b->nc + c] = vr[c];
      if (variance_explained) variance_explained[q * b->nc + c] = ve[c];
    }
  }
  if (components) memcpy(components, b->h_comps, sizeof(float) * (size_t)ns * b->nc * b->n_vars);
}

// Plain reference execution: one synchronising plan run per segment.
void batch_run_plain(scxpca_batch* b, float* emb_dev, float* components, double* singular_values,
                     double* variance_ratio, double* variance_explained, bool record_times) {
  const int ns = (int)b->plans.size();
  std::vector<double> ve(b->nc), vr(b->nc), sv(b->nc);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (record_times) {
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
  }
  for (int q = 0; q < ns; ++q) {
    scxpca_plan* pl = b->plans[q];
    scxpca_result r{};
    r.embeddings = emb_dev + b->offsets[q] * b->nc;
    r.embeddings_memory = SCXPCA_MEM_DEVICE;
    r.components = components ? components + (size_t)q * b->nc * b->n_vars : nullptr;
    r.variance_explained = ve.data();
    r.variance_ratio = vr.data();
    r.singular_values = sv.data();
    if (record_times) CK(cudaEventRecord(e0, pl->stream));
    try {
      run_plan(pl, &b->params, &r);
    } catch (const Failure& f) {
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      fail(f.code, "segment " + std::to_string(q) + ": " + f.msg);
    }
    if (record_times) {
      CK(cudaEventRecord(e1, pl->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      b->seg_ms[q] = ms;
    }
    for (int64_t c = 0; c < b->nc; ++c) {
      if (singular_values) singular_values[q * b->nc + c] = sv[c];
      if (variance_ratio) variance_ratio[q * b->nc + c] = vr[c];
      if (variance_explained) variance_explained[q * b->nc + c] = ve[c];
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
}

scxpca_batch* create_batch(const scxpca_csr* x, const int64_t* offsets, int64_t n_segments,
                           const scxpca_params* p, int32_t branches) {
  if (!x || !offsets || !p) fail(SCXPCA_INVALID_ARGUMENT, "null csr, offsets or params");
  if (n_segments <= 0) fail(SCXPCA_INVALID_ARGUMENT, "n_segments must be > 0");
  if (branches < -kMaxBranches || branches > kMaxBranches)
    fail(SCXPCA_INVALID_ARGUMENT, "branches must be in [-" + std::to_string(kMaxBranches) + ", " +
                                      std::to_string(kMaxBranches) + "] (0 = autotune, negative = lockstep)");
  if (p->omega && p->omega_memory != SCXPCA_MEM_DEVICE)
    fail(SCXPCA_INVALID_ARGUMENT, "a batch takes a device omega (or NULL for the seeded test matrix)");
  if (p->stream) fail(SCXPCA_INVALID_ARGUMENT, "a batch owns its streams: params.stream must be NULL");
  if (offsets[0] != 0 || offsets[n_segments] != x->n_obs)
    fail(SCXPCA_INVALID_ARGUMENT, "segment offsets must start at 0 and end at n_obs");
  for (int64_t q = 0; q < n_segments; ++q)
    if (offsets[q + 1] <= offsets[q]) fail(SCXPCA_INVALID_ARGUMENT, "segment offsets must increase strictly");
  auto b = new scxpca_batch();
  try {
    b->device = p->device_ordinal;
    b->params = *p;
    b->n_obs = x->n_obs;
    b->n_vars = x->n_vars;
    b->nc = p->n_components;
    CK(cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking));
    b->own_main = true;
    CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    b->offsets.assign(offsets, offsets + n_segments + 1);
    PoolScope pool_scope(b->device, b->main);
    // indptr on the host, to cut and rebase per segment
    std::vector<int64_t> ip(x->n_obs + 1);
    if (x->memory == SCXPCA_MEM_DEVICE)
      CK(cudaMemcpy(ip.data(), x->indptr, sizeof(int64_t) * (x->n_obs + 1), cudaMemcpyDeviceToHost));
    else
      memcpy(ip.data(), x->indptr, sizeof(int64_t) * (x->n_obs + 1));
    const size_t vsz = dtype_size(x->values_dtype);
    int64_t kmax = 0;
    for (int64_t q = 0; q < n_segments; ++q) {
      const int64_t r0 = offsets[q], r1 = offsets[q + 1], nq = r1 - r0;
      const int64_t e0 = ip[r0], nnz_q = ip[r1] - ip[r0];
      std::vector<int64_t> seg(nq + 1);
      for (int64_t i = 0; i <= nq; ++i) seg[i] = ip[r0 + i] - e0;
      scxpca_csr xs = *x;
      xs.n_obs = nq;
      xs.nnz = nnz_q;
      if (x->memory == SCXPCA_MEM_DEVICE) {
        auto* d = new DevBuf();
        b->indptrs.push_back(d);
        d->alloc(sizeof(int64_t) * (nq + 1));
        CK(cudaMemcpy(d->p, seg.data(), sizeof(int64_t) * (nq + 1), cudaMemcpyHostToDevice));
        xs.indptr = d->as<int64_t>();
      } else {
        xs.indptr = seg.data();
      }
      xs.indices = x->indices + e0;
      xs.values = static_cast<const char*>(x->values) + vsz * e0;
      scxpca_params ps = *p;
      ps.stream = b->main;
      if (p->n_components > std::min(nq, x->n_vars))
        fail(SCXPCA_INVALID_ARGUMENT, "segment " + std::to_string(q) + " has " + std::to_string(nq) +
                                          " rows, fewer than n_components");
      b->plans.push_back(create_plan(&xs, &ps));
      kmax = std::max<int64_t>(kmax, b->plans.back()->k);
    }
    b->k = kmax;
    // The gene-side Grams (n_vars x k, FP64) of all segments run together in
    // the batched launches: split each into fewer row ranges than a lone plan
    // does, so the partials written and summed stay small.  Every path of the
    // batch (graph or plain launches) then sums in the same order.
    // Likewise the transposed product's row groups: at least sixteen row
    // tiles each.  Every row group writes (and the sum reads) one n_vars x k
    // FP32 partial: at four tiles per group, 256 segments of 1.66M cells moved
    // 1.8 GB of partials per product, more than the packed matrix itself.
    for (scxpca_plan* pl : b->plans) {
      pl->embed_tc = false;
      pl->gram_parts_small = (int)std::max<int64_t>(
          1, std::min<int64_t>(pl->gram_parts_small, (2 * pl->num_sms + n_segments - 1) / n_segments));
      if (pl->use_tc && !pl->streaming) {
        pl->tc_row_groups = (int)std::max<int64_t>(1, std::min<int64_t>(pl->tc_row_groups, (pl->n + 2047) / 2048));
        pl->tc_gram_parts = (int)std::max<int64_t>(1, (pl->n + 1023) / 1024);  // eight row tiles each
      }
    }
    b->seg_ms.assign(n_segments, 1.0);
    b->emb.alloc(sizeof(float) * b->n_obs * b->nc);
    CK(cudaMallocHost(&b->h_status, sizeof(int32_t) * 4 * n_segments));
    memset(b->h_status, 0, sizeof(int32_t) * 4 * n_segments);
    CK(cudaMallocHost(&b->h_sigma, sizeof(double) * b->k * n_segments));
    CK(cudaMallocHost(&b->h_comps, sizeof(float) * (size_t)b->nc * b->n_vars * n_segments));
    // measured per-segment times: one plain pass (warms every plan up too)
    batch_run_plain(b, b->emb.as<float>(), nullptr, nullptr, nullptr, nullptr, true);
    if (branches != 0) {
      batch_capture(b, std::abs(branches), branches < 0);
    } else {
      // autotune the schedule and the branch count: time one launch of each
      // candidate graph, keep the fastest
      double best = 0.0;
      int best_nb = 1;
      bool best_lock = false, first = true;
      const int cands[6] = {1, 2, 4, 8, 16, 32};
      for (int lock = 0; lock < 2; ++lock) {
        for (int i = 0; i < 6; ++i) {
          const int nb = cands[i];
          if (nb > n_segments) break;
          batch_capture(b, nb, lock != 0);
          batch_launch_timed(b);  // warm
          const double ms = batch_launch_timed(b);
          b->tuned_ms[6 * lock + i] = ms;
          if (first || ms < best) {
            best = ms;
            best_nb = nb;
            best_lock = lock != 0;
            first = false;
          }
        }
      }
      if (b->branches != best_nb || b->lockstep != best_lock) batch_capture(b, best_nb, best_lock);
    }
    return b;
  } catch (...) {
    delete b;
    throw;
  }
}

}  // namespace

extern "C" {

int32_t scxpca_batch_create(const scxpca_csr* x, const int64_t* segment_offsets, int64_t n_segments,
                            const scxpca_params* params, int32_t branches, scxpca_batch** batch, char* err,
                            size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!batch) fail(SCXPCA_INVALID_ARGUMENT, "null batch output");
    *batch = nullptr;
    if (!params) fail(SCXPCA_INVALID_ARGUMENT, "null params");
    validate_params(x, params);
    DeviceGuard dg(params->device_ordinal);
    *batch = create_batch(x, segment_offsets, n_segments, params, branches);
  });
}

int32_t scxpca_batch_run(scxpca_batch* batch, int32_t use_graph, float* embeddings, int32_t embeddings_memory,
                         float* components, double* singular_values, double* variance_ratio,
                         double* variance_explained, double* device_ms, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!batch) fail(SCXPCA_INVALID_ARGUMENT, "null batch");
    if (!embeddings) fail(SCXPCA_INVALID_ARGUMENT, "null embeddings output");
    DeviceGuard dg(batch->device);
    scxpca_batch* b = batch;
    const size_t bytes = sizeof(float) * b->n_obs * b->nc;
    const cudaMemcpyKind kind =
        embeddings_memory == SCXPCA_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, b->main));
    if (use_graph) {
      CK(cudaGraphLaunch(b->exec, b->main));
      CK(cudaEventRecord(e1, b->main));
      CK(cudaMemcpyAsync(embeddings, b->emb.p, bytes, kind, b->main));
      CK(cudaStreamSynchronize(b->main));
      batch_collect(b, components, singular_values, variance_ratio, variance_explained);
    } else {
      batch_run_plain(b, b->emb.as<float>(), components, singular_values, variance_ratio, variance_explained,
                      false);
      CK(cudaEventRecord(e1, b->main));
      CK(cudaMemcpyAsync(embeddings, b->emb.p, bytes, kind, b->main));
      CK(cudaStreamSynchronize(b->main));
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (device_ms) *device_ms = ms;
  });
}

int32_t scxpca_batch_info(const scxpca_batch* batch, int32_t* branches, int64_t* graph_nodes,
                          double* tuned_ms) {
  if (!batch) return SCXPCA_INVALID_ARGUMENT;
  if (branches) *branches = batch->lockstep ? -batch->branches : batch->branches;
  if (graph_nodes) *graph_nodes = (int64_t)batch->graph_nodes;
  if (tuned_ms)
    for (int i = 0; i < 12; ++i) tuned_ms[i] = batch->tuned_ms[i];
  return SCXPCA_OK;
}

void scxpca_batch_destroy(scxpca_batch* batch) {
  if (!batch) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(batch->device);
  cudaStreamSynchronize(batch->main);
  delete batch;
  if (prev >= 0) cudaSetDevice(prev);
}

const char* scxpca_status_string(int32_t s) {
  switch (s) {
    case SCXPCA_OK: return "ok";
    case SCXPCA_INVALID_ARGUMENT: return "invalid argument";
    case SCXPCA_OUT_OF_MEMORY: return "out of memory";
    case SCXPCA_NOT_SPD: return "not SPD";
    case SCXPCA_INVALID_CSR: return "invalid CSR";
    case SCXPCA_CUDA_ERROR: return "CUDA error";
    case SCXPCA_TIMEOUT: return "timeout";
    case SCXPCA_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

int32_t scxpca_abi_version(void) { return SCXPCA_ABI_VERSION; }

int32_t scxpca_plan_create(const scxpca_csr* x, const scxpca_params* params, scxpca_plan** plan,
                           char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan) fail(SCXPCA_INVALID_ARGUMENT, "null plan output");
    *plan = nullptr;
    if (!params) fail(SCXPCA_INVALID_ARGUMENT, "null params");
    validate_params(x, params);
    DeviceGuard dg(params->device_ordinal);
    *plan = create_plan(x, params);
  });
}

int32_t scxpca_plan_create_affine(const scxpca_csr* x, const scxpca_params* params, const double* center,
                                  const double* scale, int32_t vectors_memory, scxpca_plan** plan, char* err,
                                  size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan) fail(SCXPCA_INVALID_ARGUMENT, "null plan output");
    *plan = nullptr;
    if (!params) fail(SCXPCA_INVALID_ARGUMENT, "null params");
    if (params->scale != 0 || params->clip_max > 0)
      fail(SCXPCA_INVALID_ARGUMENT, "explicit center/scale vectors replace params.scale and params.clip_max "
                                    "(set scale = 0 and clip_max <= 0)");
    if (vectors_memory != SCXPCA_MEM_HOST && vectors_memory != SCXPCA_MEM_DEVICE)
      fail(SCXPCA_INVALID_ARGUMENT, "bad vectors_memory");
    validate_params(x, params);
    DeviceGuard dg(params->device_ordinal);
    AffineSpec aff{center, scale, vectors_memory};
    *plan = create_plan(x, params, &aff);
  });
}

int32_t scxpca_plan_backward(scxpca_plan* plan, const float* scores, const float* grad_scores,
                             int32_t solve_iterations, float* grad_values, double* grad_center, double* grad_scale,
                             char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan) fail(SCXPCA_INVALID_ARGUMENT, "null plan");
    DeviceGuard dg(plan->device);
    PoolScope pool_scope(plan->device, plan->stream);
    backward(plan, scores, grad_scores, solve_iterations, grad_values, grad_center, grad_scale);
  });
}

void scxpca_plan_destroy(scxpca_plan* plan) {
  if (!plan) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(plan->device);
  cudaStreamSynchronize(plan->stream);
  bool own = plan->own_stream;
  cudaStream_t st = plan->stream;
  delete plan;
  if (own) cudaStreamDestroy(st);
  if (prev >= 0) cudaSetDevice(prev);
}

int32_t scxpca_plan_run(scxpca_plan* plan, const scxpca_params* params, scxpca_result* out,
                        char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan) fail(SCXPCA_INVALID_ARGUMENT, "null plan");
    DeviceGuard dg(plan->device);
    PoolScope pool_scope(plan->device, plan->stream);
    run_plan(plan, params, out);
  });
}

int32_t scxpca_plan_set_profiling(scxpca_plan* plan, int32_t enable) {
  if (!plan) return SCXPCA_INVALID_ARGUMENT;
  plan->profiling = enable != 0;
  plan->prof = scxpca_profile{};
  plan->marks.clear();
  plan->events_used = 0;
  return SCXPCA_OK;
}

int32_t scxpca_plan_get_profile(const scxpca_plan* plan, scxpca_profile* out) {
  if (!plan || !out) return SCXPCA_INVALID_ARGUMENT;
  *out = plan->prof;
  return SCXPCA_OK;
}

int32_t scxpca_plan_info(const scxpca_plan* plan, int64_t* k, int64_t* ld, int64_t* device_bytes) {
  if (!plan) return SCXPCA_INVALID_ARGUMENT;
  if (k) *k = plan->k;
  if (ld) *ld = plan->ld;
  if (device_bytes) *device_bytes = (int64_t)plan->device_bytes;
  return SCXPCA_OK;
}

int32_t scxpca_randomized(const scxpca_csr* x, const scxpca_params* params, scxpca_result* out,
                          char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!params) fail(SCXPCA_INVALID_ARGUMENT, "null params");
    if (!out || !out->embeddings) fail(SCXPCA_INVALID_ARGUMENT, "null embeddings output");
    validate_params(x, params);
    DeviceGuard dg(params->device_ordinal);
    // phase timing of this call (scxpca_last_call_phases)
    struct PhaseScope {
      std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
      PhaseScope() {
        for (cudaEvent_t& e : t_phase.ev)
          if (e) cudaEventDestroy(e);
        t_phase = PhaseRec{};
        t_phase.on = true;
      }
      ~PhaseScope() {
        PhaseRec& r = t_phase;
        if (r.on && r.next == SCXPCA_NUM_PHASES) {  // every device phase marked (destroy is host-timed)
          for (int i = 0; i + 1 < SCXPCA_NUM_PHASES; ++i) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, r.ev[i], r.ev[i + 1]) == cudaSuccess) r.ms[i] = ms;
          }
        } else {
          for (double& m : r.ms) m = -1.0;
        }
        cudaGetLastError();
        r.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        r.on = false;
      }
    } phases;
    scxpca_plan* pl = create_plan(x, params);
    PoolScope pool_scope(pl->device, pl->stream);
    try {
      run_plan(pl, nullptr, out);
    } catch (...) {
      scxpca_plan_destroy(pl);
      throw;
    }
    const auto t_destroy = std::chrono::steady_clock::now();
    scxpca_plan_destroy(pl);
    if (t_phase.on && t_phase.next == SCXPCA_NUM_PHASES)
      t_phase.ms[SCXPCA_PHASE_DESTROY] =
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_destroy).count();
  });
}

int32_t scxpca_last_call_phases(double* ms, int32_t capacity, double* wall_ms) {
  const int n = std::min<int32_t>(std::max<int32_t>(capacity, 0), SCXPCA_NUM_PHASES);
  for (int i = 0; i < n; ++i) ms[i] = t_phase.ms[i];
  if (wall_ms) *wall_ms = t_phase.wall_ms;
  return SCXPCA_NUM_PHASES;
}

int32_t scxpca_plan_col_stats(scxpca_plan* plan, double* col_sums, double* col_sum_sq, char* err,
                              size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan) fail(SCXPCA_INVALID_ARGUMENT, "null plan");
    DeviceGuard dg(plan->device);
    PoolScope pool_scope(plan->device, plan->stream);
    std::vector<double> s, q;
    if (plan->streaming) stream_stats(plan, true, s, q, nullptr, nullptr);
    else stats_pass(plan, plan->val, plan->dtype, s, q);
    if (col_sums) memcpy(col_sums, s.data(), sizeof(double) * plan->g);
    if (col_sum_sq) memcpy(col_sum_sq, q.data(), sizeof(double) * plan->g);
  });
}

int32_t scxpca_plan_matmat(scxpca_plan* plan, const float* v, int64_t ld_v, float* y, int64_t ld_y,
                           char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan || !v || !y) fail(SCXPCA_INVALID_ARGUMENT, "null argument");
    if (ld_v < plan->k || ld_y < plan->k) fail(SCXPCA_INVALID_ARGUMENT, "leading dimension < k");
    DeviceGuard dg(plan->device);
    PoolScope pool_scope(plan->device, plan->stream);
    plan->run_valid = false;
    cudaStream_t st = plan->stream;
    const int64_t ld = plan->ld;
    CK(cudaMemsetAsync(plan->V.p, 0, sizeof(float) * plan->g * ld, st));
    CK(cudaMemcpy2DAsync(plan->V.p, sizeof(float) * ld, v, sizeof(float) * ld_v, sizeof(float) * plan->k,
                         plan->g, cudaMemcpyDeviceToDevice, st));
    CK(launch_mean_prefactor(plan->V.as<float>(), plan->g, (int)ld,
                             plan->centered ? plan->d_mu.as<double>() : nullptr, plan->mc.as<float>(), st));
    forward(plan);
    CK(cudaMemcpy2DAsync(y, sizeof(float) * ld_y, plan->Y.p, sizeof(float) * ld, sizeof(float) * plan->k,
                         plan->n, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    check_tc_error(plan);
  });
}

int32_t scxpca_plan_rmatmat(scxpca_plan* plan, const float* q, int64_t ld_q, double* z, int64_t ld_z,
                            char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan || !q || !z) fail(SCXPCA_INVALID_ARGUMENT, "null argument");
    if (ld_q < plan->k || ld_z < plan->k) fail(SCXPCA_INVALID_ARGUMENT, "leading dimension < k");
    DeviceGuard dg(plan->device);
    PoolScope pool_scope(plan->device, plan->stream);
    plan->run_valid = false;
    cudaStream_t st = plan->stream;
    const int64_t ld = plan->ld;
    CK(cudaMemsetAsync(plan->Y.p, 0, sizeof(float) * plan->n * ld, st));
    CK(cudaMemcpy2DAsync(plan->Y.p, sizeof(float) * ld, q, sizeof(float) * ld_q, sizeof(float) * plan->k,
                         plan->n, cudaMemcpyDeviceToDevice, st));
    const int parts = (int)std::max<int64_t>(1, std::min<int64_t>(plan->gram_parts, (plan->n + 31) / 32));
    CK(launch_gram_f32(plan->Y.as<float>(), plan->n, (int)ld, plan->gpart.as<double>(), parts, st));
    CK(launch_reduce_rows_f64(plan->gpart.as<double>(), parts, ld * ld + ld, plan->G.as<double>(), 0, st,
                              plan->num_sms));
    rmatmat_raw(plan, plan->Y.as<float>(), 1);
    CK(launch_center_apply(plan->W.as<double>(), plan->g, (int)ld,
                           plan->centered ? plan->d_mu.as<double>() : nullptr,
                           plan->G.as<double>() + ld * ld, plan->eye.as<double>(), plan->Z.as<double>(), st));
    CK(cudaMemcpy2DAsync(z, sizeof(double) * ld_z, plan->Z.p, sizeof(double) * ld, sizeof(double) * plan->k,
                         plan->g, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    check_tc_error(plan);
  });
}

int32_t scxpca_plan_qr(scxpca_plan* plan, float* a, int64_t m, int64_t ld_a, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!plan || !a) fail(SCXPCA_INVALID_ARGUMENT, "null argument");
    if (ld_a < plan->k) fail(SCXPCA_INVALID_ARGUMENT, "leading dimension < k");
    if (m < plan->k) fail(SCXPCA_INVALID_ARGUMENT, "CholeskyQR2 requires m >= k");
    DeviceGuard dg(plan->device);
    PoolScope pool_scope(plan->device, plan->stream);
    plan->run_valid = false;
    cudaStream_t st = plan->stream;
    const int64_t ld = plan->ld;
    const int shift = plan->params.qr_method == SCXPCA_QR_HOUSEHOLDER ? 1 : 0;
    DevBuf tmp;
    tmp.alloc(sizeof(float) * m * ld);
    CK(cudaMemsetAsync(tmp.p, 0, sizeof(float) * m * ld, st));
    CK(cudaMemcpy2DAsync(tmp.p, sizeof(float) * ld, a, sizeof(float) * ld_a, sizeof(float) * plan->k, m,
                         cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(plan->status.p, 0, sizeof(int) * 4, st));
    // CholeskyQR2; with the Householder contract a third pass (shifted
    // CholeskyQR3), which restores orthogonality after a shifted first pass.
    for (int pass = 0; pass < (shift ? 3 : 2); ++pass) {
      tall_chol(plan, tmp.as<float>(), m, plan->Rinv.as<double>(), plan->Rinv_f.as<float>(), shift);
      CK(launch_apply_right_f32(tmp.as<float>(), m, (int)ld, plan->Rinv_f.as<float>(), tmp.as<float>(), st,
                                plan->num_sms));
    }
    int hs[4];
    CK(cudaMemcpyAsync(hs, plan->status.p, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpy2DAsync(a, sizeof(float) * ld_a, tmp.p, sizeof(float) * ld, sizeof(float) * plan->k, m,
                         cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    if (hs[0] < 0) fail(SCXPCA_NOT_SPD, "CholeskyQR2 failed: non-SPD; retry with qr_method='householder'");
  });
}

int32_t scxpca_gaussian(int32_t device_ordinal, uint64_t seed, int64_t n_rows, int64_t n_cols,
                        float* out, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!out || n_rows < 0 || n_cols < 0) fail(SCXPCA_INVALID_ARGUMENT, "bad gaussian arguments");
    DeviceGuard dg(device_ordinal);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ordinal));
    CK(launch_gaussian(seed, n_rows, n_cols, out, 0, nullptr, sms));
    CK(cudaStreamSynchronize(nullptr));
  });
}

int32_t scxpca_wait_selftest(int32_t device_ordinal, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    DeviceGuard dg(device_ordinal);
    constexpr int kSelftestSite = 99;
    DevBuf code;
    code.alloc(sizeof(int));
    CK(cudaMemsetAsync(code.p, 0, sizeof(int), nullptr));
    CK(launch_wait_selftest(code.as<int>(), kSelftestSite, nullptr));
    int e = 0;
    CK(cudaMemcpyAsync(&e, code.p, sizeof(int), cudaMemcpyDeviceToHost, nullptr));
    CK(cudaStreamSynchronize(nullptr));
    if (e != 0) fail(SCXPCA_TIMEOUT, "pipeline wait timed out (site " + std::to_string(e) + ")");
  });
}

// Shared argument checks of the device-CSR producers: a device CSR with FP32
// values whose indptr is monotone within [0, nnz] and whose column indices
// lie in [0, n_vars) (validated on the device before any kernel indexes with
// them).
void check_device_csr_f32(const scxpca_csr* x, cudaStream_t st, int sms) {
  if (!x) fail(SCXPCA_INVALID_ARGUMENT, "null csr");
  if (x->memory != SCXPCA_MEM_DEVICE) fail(SCXPCA_INVALID_ARGUMENT, "a device CSR (memory = DEVICE) is required");
  if (x->values_dtype != SCXPCA_F32) fail(SCXPCA_INVALID_ARGUMENT, "values must be float32");
  if (x->n_obs < 0 || x->n_vars <= 0 || x->nnz < 0) fail(SCXPCA_INVALID_ARGUMENT, "bad matrix dimensions");
  if (x->n_vars > INT32_MAX) fail(SCXPCA_INVALID_ARGUMENT, "n_vars exceeds int32 index range");
  if (!x->indptr || (x->nnz > 0 && (!x->indices || !x->values))) fail(SCXPCA_INVALID_ARGUMENT, "null CSR arrays");
  DevBuf flags;
  flags.alloc(16);
  CK(cudaMemsetAsync(flags.p, 0, 16, st));
  CK(launch_validate_csr(SCXPCA_F32, x->indptr, x->indices, x->values, x->n_obs, x->n_vars, x->nnz,
                         flags.as<int32_t>(), st, sms));
  int32_t hf[4];
  CK(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (hf[0]) fail(SCXPCA_INVALID_CSR, "invalid CSR: indptr is not monotone within [0, nnz]");
  if (hf[1]) fail(SCXPCA_INVALID_CSR, "invalid CSR: column index out of range [0, n_vars)");
}

int32_t scxpca_preprocess(int32_t device_ordinal, const scxpca_csr* x, float* values_out, double target_sum,
                          int32_t log1p, const float* row_factors, void* stream, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!values_out) fail(SCXPCA_INVALID_ARGUMENT, "null values_out");
    if (!std::isfinite(target_sum)) fail(SCXPCA_INVALID_ARGUMENT, "target_sum must be finite");
    DeviceGuard dg(device_ordinal);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ordinal));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PoolScope pool_scope(device_ordinal, st);
    check_device_csr_f32(x, st, sms);
    CK(launch_normalize_log1p(x->indptr, static_cast<const float*>(x->values), values_out, x->n_obs, target_sum,
                              log1p ? 1 : 0, row_factors, st, sms));
    CK(cudaStreamSynchronize(st));
  });
}

int32_t scxpca_project_columns(int32_t device_ordinal, const scxpca_csr* x, const int32_t* cols, int64_t n_cols,
                               int64_t* out_indptr, int32_t* out_indices, float* out_values, int64_t* nnz_out,
                               void* stream, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!cols || n_cols <= 0 || !out_indptr || !nnz_out) fail(SCXPCA_INVALID_ARGUMENT, "bad projection arguments");
    if ((out_indices == nullptr) != (out_values == nullptr))
      fail(SCXPCA_INVALID_ARGUMENT, "out_indices and out_values must both be given or both be NULL");
    if (!x) fail(SCXPCA_INVALID_ARGUMENT, "null csr");
    // the kept columns: sorted, unique, in range (ProjectedShardSource's contract)
    std::vector<int32_t> col_map(x->n_vars > 0 ? x->n_vars : 0, -1);
    for (int64_t i = 0; i < n_cols; ++i) {
      if (cols[i] < 0 || cols[i] >= x->n_vars) fail(SCXPCA_INVALID_ARGUMENT, "column index out of range");
      if (i > 0 && cols[i] <= cols[i - 1]) fail(SCXPCA_INVALID_ARGUMENT, "cols must be sorted and unique");
      col_map[cols[i]] = (int32_t)i;
    }
    DeviceGuard dg(device_ordinal);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ordinal));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PoolScope pool_scope(device_ordinal, st);
    check_device_csr_f32(x, st, sms);
    const int64_t n = x->n_obs;
    DevBuf d_map, counts;
    d_map.alloc(sizeof(int32_t) * col_map.size());
    CK(cudaMemcpyAsync(d_map.p, col_map.data(), sizeof(int32_t) * col_map.size(), cudaMemcpyHostToDevice, st));
    counts.alloc(sizeof(int64_t) * std::max<int64_t>(n, 1));
    CK(launch_project_count(x->indptr, x->indices, n, d_map.as<int32_t>(), counts.as<int64_t>(), st, sms));
    CK(launch_exclusive_scan_i64(counts.as<int64_t>(), n, out_indptr, st));
    CK(cudaMemcpyAsync(nnz_out, out_indptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (out_indices)
      CK(launch_project_fill(x->indptr, x->indices, static_cast<const float*>(x->values), n, d_map.as<int32_t>(),
                             out_indptr, out_indices, out_values, st, sms));
    CK(cudaStreamSynchronize(st));
  });
}

int32_t scxpca_pflog_prepare(int32_t device_ordinal, const scxpca_csr* x, double four_alpha, float* delta_out,
                             double* baseline_out, void* stream, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!delta_out || !baseline_out) fail(SCXPCA_INVALID_ARGUMENT, "null delta or baseline output");
    if (!(four_alpha > 0.0) || !std::isfinite(four_alpha))
      fail(SCXPCA_INVALID_ARGUMENT, "PFlog four_alpha (= 4 alpha) must be positive and finite, got " +
                                        std::to_string(four_alpha));
    DeviceGuard dg(device_ordinal);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ordinal));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PoolScope pool_scope(device_ordinal, st);
    check_device_csr_f32(x, st, sms);
    DevBuf flags;
    flags.alloc(16);
    CK(cudaMemsetAsync(flags.p, 0, 16, st));
    CK(launch_pflog_prepare(x->indptr, static_cast<const float*>(x->values), x->n_obs, x->n_vars, four_alpha,
                            delta_out, baseline_out, flags.as<int32_t>(), st, sms));
    int32_t hf[4];
    CK(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hf[1])
      fail(SCXPCA_INVALID_ARGUMENT, "PFlog input contains a non-finite value; PFlog requires finite raw counts");
    if (hf[0]) fail(SCXPCA_INVALID_ARGUMENT, "PFlog: negative count; counts must be non-negative");
  });
}

int32_t scxpca_pflog_pca(const scxpca_csr* delta, const double* baseline, int32_t baseline_memory,
                         const scxpca_params* params, scxpca_result* out, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!params) fail(SCXPCA_INVALID_ARGUMENT, "null params");
    if (!out || !out->embeddings) fail(SCXPCA_INVALID_ARGUMENT, "null embeddings output");
    if (!baseline) fail(SCXPCA_INVALID_ARGUMENT, "null baseline");
    validate_params(delta, params);
    if (params->scale) fail(SCXPCA_UNSUPPORTED, "PFlog PCA does not take per-gene scaling");
    if (delta->n_vars + 1 > INT32_MAX) fail(SCXPCA_INVALID_ARGUMENT, "n_vars exceeds int32 index range");
    DeviceGuard dg(params->device_ordinal);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, params->device_ordinal));
    scxpca_params p = *params;
    p.clip_max = 0.0;
    cudaStream_t own = nullptr;
    if (!p.stream) {
      CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
      p.stream = own;
    }
    struct StreamGuard {
      cudaStream_t s;
      ~StreamGuard() {
        if (s) {
          cudaStreamSynchronize(s);
          cudaStreamDestroy(s);
        }
      }
    } own_guard{own};
    cudaStream_t st = static_cast<cudaStream_t>(p.stream);
    PoolScope pool_scope(params->device_ordinal, st);
    const int64_t n = delta->n_obs, g = delta->n_vars, nnz = delta->nnz;
    const size_t vs = dtype_size(delta->values_dtype);
    // the delta CSR and the baseline on the device
    DevBuf d_ip, d_ix, d_vv, d_b, a_ip, a_ix, a_vv, d_cross;
    const int64_t* ip = delta->indptr;
    const int32_t* ix = delta->indices;
    const void* vv = delta->values;
    if (delta->memory != SCXPCA_MEM_DEVICE) {
      d_ip.alloc(sizeof(int64_t) * (n + 1));
      d_ix.alloc(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
      d_vv.alloc(vs * std::max<int64_t>(nnz, 1));
      CK(cudaMemcpyAsync(d_ip.p, ip, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
      if (nnz) {
        CK(cudaMemcpyAsync(d_ix.p, ix, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_vv.p, vv, vs * nnz, cudaMemcpyHostToDevice, st));
      }
      ip = d_ip.as<int64_t>();
      ix = d_ix.as<int32_t>();
      vv = d_vv.p;
    }
    const double* b = baseline;
    std::vector<double> hb(n);
    if (baseline_memory == SCXPCA_MEM_DEVICE) {
      CK(cudaMemcpyAsync(hb.data(), baseline, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    } else {
      memcpy(hb.data(), baseline, sizeof(double) * n);
      d_b.alloc(sizeof(double) * n);
      CK(cudaMemcpyAsync(d_b.p, baseline, sizeof(double) * n, cudaMemcpyHostToDevice, st));
      b = d_b.as<double>();
    }
    // validate the delta CSR before the augmentation kernel indexes with it
    {
      DevBuf flags;
      flags.alloc(16);
      CK(cudaMemsetAsync(flags.p, 0, 16, st));
      CK(launch_validate_csr(delta->values_dtype, ip, ix, vv, n, g, nnz, flags.as<int32_t>(), st, sms));
      int32_t hf[4];
      CK(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (hf[0]) fail(SCXPCA_INVALID_CSR, "invalid CSR: indptr is not monotone within [0, nnz]");
      if (hf[1]) fail(SCXPCA_INVALID_CSR, "invalid CSR: column index out of range [0, n_vars)");
      if (hf[3]) fail(SCXPCA_INVALID_CSR, "invalid CSR: non-finite value");
    }
    for (int64_t i = 0; i < n; ++i)
      if (!std::isfinite(hb[i])) fail(SCXPCA_INVALID_ARGUMENT, "baseline must be finite (cell " + std::to_string(i) + ")");
    // the augmented matrix [delta | b]
    a_ip.alloc(sizeof(int64_t) * (n + 1));
    a_ix.alloc(sizeof(int32_t) * (nnz + n));
    a_vv.alloc(vs * (nnz + n));
    d_cross.alloc(sizeof(double) * n);
    CK(launch_pflog_augment(delta->values_dtype, ip, ix, vv, n, (int32_t)g, b, a_ip.as<int64_t>(),
                            a_ix.as<int32_t>(), a_vv.p, d_cross.as<double>(), st, sms));
    std::vector<double> hc(n);
    CK(cudaMemcpyAsync(hc.data(), d_cross.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    PflogSpec spec{0.0, 0.0, 0.0};
    for (int64_t i = 0; i < n; ++i) {
      spec.b_mean += hb[i];
      spec.b2 += hb[i] * hb[i];
      spec.cross += hc[i];
    }
    spec.b_mean /= (double)std::max<int64_t>(n, 1);
    scxpca_csr xa{n, g + 1, nnz + n, a_ip.as<int64_t>(), a_ix.as<int32_t>(), a_vv.p, delta->values_dtype,
                  SCXPCA_MEM_DEVICE};
    scxpca_plan* pl = create_plan(&xa, &p, nullptr, &spec);
    try {
      run_plan(pl, nullptr, out);
    } catch (...) {
      scxpca_plan_destroy(pl);
      throw;
    }
    scxpca_plan_destroy(pl);
  });
}

int32_t scxpca_synth_nb_csr(int32_t device_ordinal, uint64_t seed, int64_t n_obs, int64_t n_vars,
                            double loc, double dispersion, int64_t* indptr, int32_t* indices,
                            float* values, int64_t* nnz_out, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_obs <= 0 || n_vars <= 0 || !indptr || !nnz_out)
      fail(SCXPCA_INVALID_ARGUMENT, "bad synth arguments");
    if (!(dispersion > 0.0 && dispersion <= 1.0))
      fail(SCXPCA_INVALID_ARGUMENT, "dispersion must be in (0, 1]");
    DeviceGuard dg(device_ordinal);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_ordinal));
    cudaStream_t st = nullptr;
    DevBuf mu, row_nnz, rowsum;
    mu.alloc(sizeof(float) * n_vars);
    row_nnz.alloc(sizeof(int64_t) * n_obs);
    rowsum.alloc(sizeof(float) * n_obs);
    CK(launch_synth_gene_means(seed, n_vars, loc, mu.as<float>(), st));
    CK(launch_synth_count(seed, n_obs, n_vars, loc, dispersion, mu.as<float>(), row_nnz.as<int64_t>(),
                          rowsum.as<float>(), st, sms));
    CK(launch_exclusive_scan_i64(row_nnz.as<int64_t>(), n_obs, indptr, st));
    CK(cudaMemcpyAsync(nnz_out, indptr + n_obs, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (indices && values) {
      CK(launch_synth_fill(seed, n_obs, n_vars, loc, dispersion, mu.as<float>(), indptr,
                           rowsum.as<float>(), indices, values, st, sms));
      CK(cudaStreamSynchronize(st));
    }
  });
}

}  // extern "C"
