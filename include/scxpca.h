/*
 * scxpca.h -- C ABI of the B200 randomized-PCA library (libscxpca.so).
 *
 * Randomized PCA of a sparse cells x genes CSR matrix with implicit per-gene
 * centring (and optional unit-variance scaling with clipping), computed by
 * hand-written sm_100a kernels.  The ABI is plain C: pointers, sizes, status
 * codes; no exceptions cross it and no call aborts the process.
 *
 * Every entry point below replaces one interface of ArcInstitute/scx (paths
 * inside that tree); the citation is in the comment above each declaration.
 *
 * Threading: a plan is used by one host thread at a time.  Separate plans may
 * be used concurrently from different threads.
 */
#ifndef SCXPCA_H
#define SCXPCA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCXPCA_ABI_VERSION 2

/* Status codes.  They mirror the GpuError classes of scx-gpu/src/error.rs:
 * ShapeMismatch -> INVALID_ARGUMENT, OutOfMemory -> OUT_OF_MEMORY,
 * CuSolverError("...non-SPD...") -> NOT_SPD, InvalidShard -> INVALID_CSR,
 * CudaError/KernelLaunchFailed -> CUDA_ERROR. */
typedef enum {
  SCXPCA_OK = 0,
  SCXPCA_INVALID_ARGUMENT = 1,
  SCXPCA_OUT_OF_MEMORY = 2,
  SCXPCA_NOT_SPD = 3,
  SCXPCA_INVALID_CSR = 4,
  SCXPCA_CUDA_ERROR = 5,
  SCXPCA_TIMEOUT = 6,
  SCXPCA_UNSUPPORTED = 7
} scxpca_status;

/* Element type of stored nonzero values. */
typedef enum { SCXPCA_F32 = 0, SCXPCA_BF16 = 1, SCXPCA_F16 = 2 } scxpca_dtype;

/* Where a buffer lives. */
typedef enum { SCXPCA_MEM_HOST = 0, SCXPCA_MEM_DEVICE = 1 } scxpca_memory;

/* Orthonormalisation failure contract (scx-gpu/src/cusolver.rs:256-262).
 * CHOLESKY reports SCXPCA_NOT_SPD when a Gram pivot breaks down (the message
 * contains "non-SPD"); HOUSEHOLDER never fails on finite input: its
 * Cholesky is shifted when a pivot breaks down. */
typedef enum { SCXPCA_QR_HOUSEHOLDER = 0, SCXPCA_QR_CHOLESKY = 1 } scxpca_qr_method;

/* Arithmetic (scx-gpu/src/math_policy.rs:45-84, GpuMathMode).
 * STRICT_FP32: FP32 values, FP32 CUDA-core SpMM, FP64 Gram/Cholesky/SVD.
 * MIXED_BF16 / MIXED_F16: values stream as 16-bit, SpMM products on tensor
 * cores with FP32 accumulation, final projection and small factorisations
 * in FP32/FP64. */
typedef enum {
  SCXPCA_MATH_STRICT_FP32 = 0,
  SCXPCA_MATH_MIXED_BF16 = 1,
  SCXPCA_MATH_MIXED_F16 = 2
} scxpca_math_mode;

/* SpMM reduction order (scx-gpu/src/math_policy.rs:86-136, SpmmAlgPolicy).
 * DETERMINISTIC gives bit-identical results across runs on one device. */
typedef enum { SCXPCA_SPMM_DEFAULT = 0, SCXPCA_SPMM_DETERMINISTIC = 1 } scxpca_spmm_policy;

/* A CSR matrix: rows are cells, columns are genes.  Replaces the ShardSource /
 * ScxCsr input (scx-format-io/src/shard_source.rs:86-140,
 * scx-sparse/src/csr.rs:183-192): int64 indptr (n_obs + 1), int32 indices
 * (nnz), values (nnz) of `values_dtype`.  Column indices must be in
 * [0, n_vars); rows need not be sorted for correctness.  `memory` says whether
 * the three arrays are host or device pointers (device: on `device_ordinal`). */
typedef struct {
  int64_t n_obs;
  int64_t n_vars;
  int64_t nnz;
  const int64_t* indptr;
  const int32_t* indices;
  const void* values;
  int32_t values_dtype; /* scxpca_dtype */
  int32_t memory;       /* scxpca_memory */
} scxpca_csr;

/* Arguments of scx_gpu::gpu_randomized_pca (scx-gpu/src/gpu_pca.rs:706-716)
 * and pyscx.accel.pca (pyscx/src/accel/pca.rs:573-605), plus the explicit
 * test matrix and per-gene scaling, which have no reference counterpart. */
typedef struct {
  int64_t n_components;   /* the sketch k = min(n_components + n_oversamples,
                             n_vars, n_obs) may be up to 256; wider returns
                             SCXPCA_UNSUPPORTED.  128 < k <= 256 runs on the
                             CUDA cores, resident plans only, no backward. */
  int64_t n_oversamples;
  int64_t n_power_iterations;
  int32_t zero_center;    /* subtract per-gene means implicitly */
  int32_t scale;          /* per-gene unit variance (ddof=1), scanpy pp.scale */
  double clip_max;        /* > 0: clip scaled values to +-clip_max (upper only
                             without centring); <= 0: no clip */
  uint64_t seed;          /* used when omega == NULL */
  const float* omega;     /* optional explicit test matrix, n_vars x k,
                             column-major (ld = n_vars), k = min(n_components +
                             n_oversamples, n_vars, n_obs) */
  int32_t omega_memory;   /* scxpca_memory of omega */
  int32_t qr_method;      /* scxpca_qr_method */
  int32_t math_mode;      /* scxpca_math_mode */
  int32_t spmm_policy;    /* scxpca_spmm_policy */
  int32_t device_ordinal;
  int32_t reserved0;
  void* stream;           /* cudaStream_t; NULL = a stream owned by the plan */
  int64_t device_budget;  /* bytes of device memory a plan of a HOST matrix may
                             hold (0 = all free memory).  When the resident plan
                             would not fit, the matrix stays in host memory and
                             every product streams it in row shards
                             (result.resident_csr = 0), as the reference's
                             StreamingPcaOperator does
                             (scx-gpu/src/linear_operator.rs:61-288).  The
                             environment variable SCXPCA_RESIDENT=0 forces
                             streaming (SCX_GPU_PCA_RESIDENT=0 in the
                             reference, gpu_pca_resident.rs:56-73). */
} scxpca_params;

/* Outputs, caller-allocated.  Replaces GpuPcaResult (gpu_pca.rs:76-98) and
 * GpuPcaDeviceResult (gpu_pca.rs:108-128).  `embeddings` is n_obs x
 * n_components row-major float32 in `embeddings_memory` (device: on the plan's
 * device, written asynchronously before the call returns synchronised).  All
 * other arrays are host memory; any of them except `embeddings` may be NULL.
 *
 * Device hand-off (gpu_randomized_pca_device -> CAGRA kNN,
 * scx-gpu/src/gpu_pca.rs:775-838, scx-accel/src/fused/gpu.rs:36-60): with
 * embeddings_memory = DEVICE the caller owns the buffer (n_obs * n_components
 * floats, contiguous rows, the layout of the reference's DeviceEmbedding); the
 * library writes it in place on the plan's stream and returns only after that
 * write completed, so a consumer on any stream of the device may read it at
 * once, and the embedding never crosses to the host. */
typedef struct {
  float* embeddings;            /* n_obs x n_components, row-major */
  float* components;            /* n_components x n_vars, row-major */
  double* variance_explained;   /* n_components: sigma^2 / (n_obs - 1) */
  double* variance_ratio;       /* n_components */
  double* singular_values;      /* n_components */
  double* mean;                 /* n_vars: column means of the input matrix */
  double* std;                  /* n_vars: per-gene std used for scaling */
  int32_t embeddings_memory;    /* scxpca_memory */
  int32_t resident_csr;         /* out: 1 when the matrix was resident on the device,
                                   0 when it was streamed from host memory */
  int32_t total_var_recomputed; /* out: 1 when the cancellation guard fired */
  int32_t shifted_cholesky;     /* out: number of shifted Gram factorisations */
  double total_var;             /* out: total variance used for the ratios */
  int32_t eig_sweeps;           /* out: Jacobi sweeps of the k x k eigensolver */
  int32_t n_shards;             /* out: row shards a streamed matrix was taken in
                                   (0 when resident) */
} scxpca_result;

typedef struct scxpca_plan scxpca_plan;

/* Human-readable name of a status code (static storage). */
const char* scxpca_status_string(int32_t status);

/* ABI version of the loaded library (SCXPCA_ABI_VERSION). */
int32_t scxpca_abi_version(void);

/* One-shot randomized PCA.  Replaces scx_gpu::gpu_randomized_pca
 * (scx-gpu/src/gpu_pca.rs:706-763) and gpu_randomized_pca_device
 * (gpu_pca.rs:775-838) -- device embeddings when embeddings_memory is DEVICE --
 * as wrapped by scx_accel::randomized_pca_gpu (scx-accel/src/pca/gpu.rs:51-95).
 * Builds a plan, runs it, destroys it; all device memory is released on
 * return.  `err` (may be NULL) receives a NUL-terminated message. */
int32_t scxpca_randomized(const scxpca_csr* x, const scxpca_params* params,
                          scxpca_result* out, char* err, size_t err_len);

/* Resident plan: validates the CSR, uploads or borrows it (a device CSR whose
 * values already have the compute type is borrowed, never copied), applies the
 * per-gene statistics and value transform once, and allocates every buffer a
 * run needs.  Replaces try_build_resident_csr + ResidentPcaOperator +
 * GpuPcaScratch (scx-gpu/src/gpu_pca_resident.rs:87-283,
 * gpu_pca.rs:57-73).  A borrowed device CSR must outlive the plan. */
int32_t scxpca_plan_create(const scxpca_csr* x, const scxpca_params* params,
                           scxpca_plan** plan, char* err, size_t err_len);

/* Run the power loop and the Rayleigh-Ritz step on a resident plan
 * (run_resident_power_loop, gpu_pca_resident.rs:295-347, then
 * randomized_pca_core steps 7-8, gpu_pca.rs:590-697).  Only `seed`, `omega`,
 * `omega_memory` and `n_power_iterations` of `params` may differ from the
 * values the plan was created with; NULL reuses the creation parameters.
 * A plan run again with the same n_power_iterations, seed, omega pointer and
 * embeddings buffer records that run as a CUDA graph on its second
 * occurrence and replays it afterwards (same results, one launch); stage
 * profiling, a host omega or the environment variable SCXPCA_GRAPH=0 keep
 * plain kernel launches.  The graph reads omega and writes the embeddings
 * at the pointers given, so their contents may change between runs. */
int32_t scxpca_plan_run(scxpca_plan* plan, const scxpca_params* params,
                        scxpca_result* out, char* err, size_t err_len);

void scxpca_plan_destroy(scxpca_plan* plan);

/* Resident plan of the affine map X~ = (X - 1 center^T) diag(scale) with
 * explicit per-gene vectors (n_vars doubles each, host or device per
 * `vectors_memory`; NULL center = no centring, NULL scale = 1).  The PCA is
 * of X~ itself: no column means are re-subtracted.  With center = column
 * means and scale = 1 / std this is the matrix that zero_center + scale
 * (without clipping) describe.  params->scale must be 0 and clip_max <= 0;
 * params->zero_center is ignored.  Scale entries must be non-zero.  Extends
 * try_build_resident_csr (scx-gpu/src/gpu_pca_resident.rs:87-179) with the
 * differentiable inputs of scxpca_plan_backward; the reference has no
 * gradient path. */
int32_t scxpca_plan_create_affine(const scxpca_csr* x, const scxpca_params* params,
                                  const double* center, const double* scale, int32_t vectors_memory,
                                  scxpca_plan** plan, char* err, size_t err_len);

/* Backward pass of the scores S = X~ V (the embeddings of the plan's last
 * run, V the top n_components right singular vectors) for a loss L(S):
 * given dL/dS, writes dL/dx for every stored value x of the CSR (in the
 * CSR's entry order), dL/dcenter and dL/dscale (n_vars each; either may be
 * NULL).  The gradient is the adjoint of the truncated SVD: the part of each
 * singular-vector derivative inside the sketch subspace comes from the
 * run's Ritz pairs, the part outside it from `solve_iterations` conjugate-
 * gradient steps (each one product with X~^T X~, recomputed rather than
 * stored).  All pointers are device memory on the plan's device: scores and
 * grad_scores n_obs x n_components row-major float32, grad_values nnz float32.
 * Must follow scxpca_plan_run with no other call on the plan in between; not
 * available with clip_max > 0 or when the plan had to re-sort the CSR rows.
 * No reference counterpart (the reference PCA is not differentiable). */
int32_t scxpca_plan_backward(scxpca_plan* plan, const float* scores, const float* grad_scores,
                             int32_t solve_iterations, float* grad_values, double* grad_center,
                             double* grad_scale, char* err, size_t err_len);

/* Plan geometry: k (sketch width), ld (padded row stride of the tall
 * buffers), bytes of device memory the plan holds. */
int32_t scxpca_plan_info(const scxpca_plan* plan, int64_t* k, int64_t* ld,
                         int64_t* device_bytes);

/* Operator seam (scx-gpu/src/pca_operator.rs:69-79, PcaOperator), on device
 * buffers of the plan's device, ordered on the plan's stream:
 *   matmat : Y = (X - 1 mu^T) V      V: n_vars x k row-major (ld_v >= k),
 *                                    Y: n_obs x k row-major (ld_y >= k)
 *            (spmm_forward_segment + forward_mean_prefactor +
 *             mean_correct kernel, gpu_pca.rs:218-289, colmajor_ops.cu:41-57)
 *   rmatmat: Z = (X - 1 mu^T)^T Q    Q: n_obs x k row-major (ld_q >= k),
 *                                    Z: n_vars x k row-major double (ld_z >= k)
 *            (spmm_transpose_segment + transpose_centering_correction,
 *             gpu_pca.rs:302-346, colmajor_ops.cu:78-134, 248-263)
 *   qr     : A (m x k row-major float, ld_a >= k) <- Q factor of A, in place
 *            (gpu_qr_q / gpu_cholesky_qr2, scx-gpu/src/cusolver.rs:87-409)
 * X here is the plan's working matrix (after scaling, in the compute type).
 * The calls synchronise the plan's stream before returning. */
int32_t scxpca_plan_matmat(scxpca_plan* plan, const float* v, int64_t ld_v, float* y,
                           int64_t ld_y, char* err, size_t err_len);
int32_t scxpca_plan_rmatmat(scxpca_plan* plan, const float* q, int64_t ld_q, double* z,
                            int64_t ld_z, char* err, size_t err_len);
int32_t scxpca_plan_qr(scxpca_plan* plan, float* a, int64_t m, int64_t ld_a,
                       char* err, size_t err_len);

/* Batched sub-PCAs: an independent randomized PCA of every row segment
 * [segment_offsets[q], segment_offsets[q + 1]) of one CSR (cell clusters of
 * uneven sizes), each centred on its own column means, with the same
 * parameters.  Creation builds one resident plan per segment (device CSR
 * slices are borrowed, not copied), runs every segment once with plain
 * launches to measure it, and records all runs into ONE CUDA graph whose
 * parallel branches take the segments in a longest-first schedule of the
 * measured times.  Two schedules: segment per branch (each branch runs whole
 * segments one after another) or lockstep (all segments take each step of
 * the power loop together, so their products run together and then their
 * small factorisations run together).  When every segment has the same
 * sketch width at ld 64 on the tensor-core path, each lockstep step is ONE
 * launch over all segments (products, Grams, factorisations, eigensolves,
 * the tall right-multiplications, Omega and the result gathers: a graph of a
 * few dozen nodes whatever the segment count); otherwise the branches launch
 * per segment.  Both schedules give the bits of use_graph = 0.
 * `branches` = b in 1..32 fixes the
 * segment-per-branch schedule over b branches, -b the lockstep schedule over
 * b streams; 0 lets an autotuner time both schedules for 1, 2, 4, ... 32 and
 * keep the fastest.  params->omega must be NULL (seeded) or device memory, and
 * params->stream NULL (the batch owns its streams).  The reference runs one
 * PCA per call (scx-gpu/src/gpu_pca.rs:706-763); a caller with clusters
 * loops over it, which scxpca_batch_run with use_graph = 0 reproduces. */
typedef struct scxpca_batch scxpca_batch;

int32_t scxpca_batch_create(const scxpca_csr* x, const int64_t* segment_offsets, int64_t n_segments,
                            const scxpca_params* params, int32_t branches, scxpca_batch** batch,
                            char* err, size_t err_len);

/* Run every segment: use_graph = 1 launches the recorded graph once;
 * use_graph = 0 runs one plain, synchronising plan run per segment.
 * embeddings: n_obs x n_components float32 row-major (each segment's rows in
 * place), host or device per embeddings_memory.  Host outputs (any may be
 * NULL): components [segment][n_components][n_vars] float32, singular_values
 * / variance_ratio / variance_explained [segment][n_components] double.
 * device_ms (may be NULL) receives the device time of the runs. */
int32_t scxpca_batch_run(scxpca_batch* batch, int32_t use_graph, float* embeddings,
                         int32_t embeddings_memory, float* components, double* singular_values,
                         double* variance_ratio, double* variance_explained, double* device_ms,
                         char* err, size_t err_len);

/* Chosen schedule (branch count; negative = lockstep over that many
 * streams), graph node count, and the autotuner's timings in ms (0 where not
 * tried; 12 entries): [0..5] segment-per-branch schedules with 1, 2, 4, 8,
 * 16, 32 branches, [6..11] lockstep schedules over as many streams. */
int32_t scxpca_batch_info(const scxpca_batch* batch, int32_t* branches, int64_t* graph_nodes,
                          double* tuned_ms);

void scxpca_batch_destroy(scxpca_batch* batch);

/* Opt-in per-stage device timing (the counterpart of SCX_GPU_PROFILE,
 * scx-gpu/src/profile.rs:1-60, and the SpMM timing hook of
 * cusparse.rs:501-528).  When enabled, plan_run brackets each stage's kernels
 * with CUDA events on the plan's stream and accumulates per-stage launch
 * counts and device milliseconds.  kernel_launches counts every kernel the
 * library launched on the plan since the last reset, profiling on or off. */
enum {
  SCXPCA_STAGE_PREPARE = 0,   /* validation, statistics, value transform */
  SCXPCA_STAGE_FORWARD = 1,   /* Y = (X - mu) V */
  SCXPCA_STAGE_TRANSPOSE = 2, /* partial X^T Q */
  SCXPCA_STAGE_REDUCE = 3,    /* fixed-order reduction of the partials */
  SCXPCA_STAGE_GRAM = 4,      /* tall Gram Y^T Y (FP64) */
  SCXPCA_STAGE_APPLY = 5,     /* tall Q = Y R^{-1} */
  SCXPCA_STAGE_SMALL = 6,     /* Cholesky, gene-side QR, Jacobi, Ritz */
  SCXPCA_STAGE_EMBED = 7,     /* embeddings */
  SCXPCA_NUM_STAGES = 8
};

typedef struct {
  int64_t launches[SCXPCA_NUM_STAGES]; /* bracketed stage executions */
  double device_ms[SCXPCA_NUM_STAGES];
  int64_t kernel_launches;             /* all kernels launched since reset */
  int64_t runs;                        /* plan_run calls since reset */
} scxpca_profile;

/* Phases of the calling thread's last scxpca_randomized call, in device
 * milliseconds between consecutive phase boundaries recorded on the call's
 * stream (host gaps between phases included), except DESTROY, which is host
 * time.  The counterpart of the reference's per-call timing log
 * (scx-gpu/src/profile.rs:1-60, gpu_pca.rs:465-697). */
enum {
  SCXPCA_PHASE_UPLOAD = 0,    /* pre-flight, allocations, host-to-device copy */
  SCXPCA_PHASE_VALIDATE = 1,  /* CSR validation (and row sort) */
  SCXPCA_PHASE_STATS = 2,     /* per-gene statistics of the input */
  SCXPCA_PHASE_TRANSFORM = 3, /* value transform, working statistics, total variance */
  SCXPCA_PHASE_PACK = 4,      /* packed tile copy for the products */
  SCXPCA_PHASE_BUFFERS = 5,   /* work buffers */
  SCXPCA_PHASE_PCA = 6,       /* power loop, Rayleigh-Ritz step, embeddings */
  SCXPCA_PHASE_DOWNLOAD = 7,  /* device-to-host copy of the results */
  SCXPCA_PHASE_DESTROY = 8,   /* plan teardown (host time) */
  SCXPCA_NUM_PHASES = 9
};

/* Writes min(capacity, SCXPCA_NUM_PHASES) phase times (-1 when the call failed
 * before its phases completed) and the call's host wall time; returns
 * SCXPCA_NUM_PHASES. */
int32_t scxpca_last_call_phases(double* ms, int32_t capacity, double* wall_ms);

/* Enable (1) or disable (0) stage timing; any call resets the counters. */
int32_t scxpca_plan_set_profiling(scxpca_plan* plan, int32_t enable);
int32_t scxpca_plan_get_profile(const scxpca_plan* plan, scxpca_profile* out);

/* Per-gene statistics of the plan's working matrix: column sums and sums of
 * squares in FP64, host outputs (n_vars each).  Replaces
 * col_means_and_sum_sq_prefetched (scx-format-io/src/prefetch.rs:616-650) and
 * ScxCsr::col_sums_and_sum_sq (scx-sparse/src/csr.rs:570-580). */
int32_t scxpca_plan_col_stats(scxpca_plan* plan, double* col_sums, double* col_sum_sq,
                              char* err, size_t err_len);

/* Per-gene column statistics that allocate no device memory.  This entry point
 * has no counterpart in the reference.  It is for callers that cannot let a
 * library call cudaMalloc: processes whose device memory is owned by a caching
 * pool (a PyTorch or RMM allocator that has reserved the device or enforces a
 * budget), and pipelines where cudaMalloc/cudaFree would add device-wide
 * synchronisation between their streams.
 *
 * `x` must be a device CSR (memory = DEVICE) on `device_ordinal`;
 * `out_stats` is caller-allocated device memory of 2 * n_vars doubles,
 * written as [sum x (n_vars) | sum x^2 (n_vars)] in FP64 (the same sums as
 * scxpca_plan_col_stats on an unscaled plan of the same matrix).  The CSR is
 * validated first (SCXPCA_INVALID_CSR as for plan creation; unsorted rows are
 * accepted).  `stream` may be NULL (the legacy default stream); the call waits
 * for it before returning.
 *
 * Scratch: one static device array of SCXPCA_NOALLOC_SCRATCH_BYTES (8 MiB)
 * that every GPU which loads the library holds until the process exits, so
 * n_vars is limited to SCXPCA_NOALLOC_MAX_VARS; larger matrices get
 * SCXPCA_INVALID_ARGUMENT.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress).  No call can be recorded into a CUDA
 * graph: each one copies the validation flags to the host and synchronises
 * the stream, so a call on a stream that is being captured returns
 * SCXPCA_INVALID_ARGUMENT without touching the capture.  All calls share the
 * array and it keeps the last call's contents: two calls whose kernels
 * overlapped on the GPU would race on it, so the library takes a process-wide
 * lock around each call and synchronises the stream before releasing it. */
#define SCXPCA_NOALLOC_SCRATCH_BYTES (8u << 20)
#define SCXPCA_NOALLOC_MAX_VARS 12800
int32_t scxpca_col_stats_noalloc(int32_t device_ordinal, const scxpca_csr* x, double* out_stats,
                                 void* stream, char* err, size_t err_len);

/* Per-row normalize_total + log1p of a device CSR with float32 values,
 * producing the PCA's input without leaving the device.  For every row with a
 * non-zero sum: v <- v * target_sum / rowsum (FP64 row sum and factor; skipped
 * when target_sum <= 0), then v <- log1p(v) when log1p != 0, then v <- v *
 * row_factors[row] when row_factors (device, n_obs floats) is not NULL.  Rows
 * that sum to zero are only multiplied by their factor.  Writes values_out
 * (device, nnz floats; may be x->values itself for an in-place transform);
 * indptr and indices are unchanged.  The CSR's indptr and indices are validated
 * first (SCXPCA_INVALID_CSR).  `stream` may be NULL; the call synchronises it.
 * Replaces gpu_apply_fused_ops and its wrappers gpu_normalize_log1p /
 * gpu_normalize / gpu_log1p / gpu_row_scale (scx-gpu/src/gpu_preprocess.rs:
 * 252-391, kernels in scx-gpu/kernels/normalize_log1p.cu:17-140). */
int32_t scxpca_preprocess(int32_t device_ordinal, const scxpca_csr* x, float* values_out, double target_sum,
                          int32_t log1p, const float* row_factors, void* stream, char* err, size_t err_len);

/* Column projection of a device CSR with float32 values to the kept columns
 * `cols` (host array of n_cols sorted, unique indices into [0, n_vars)); kept
 * column cols[i] becomes column i, entries keep their row order.  The mask_var
 * / highly_variable selection in front of the PCA, on the device.  Call with
 * out_indices == out_values == NULL first: fills out_indptr (device, n_obs + 1)
 * and *nnz_out; then again with device buffers of *nnz_out entries.  Replaces
 * ProjectedShardSource (scx-accel/src/projected_source.rs:28-80) over
 * scx_engine::project_csr. */
int32_t scxpca_project_columns(int32_t device_ordinal, const scxpca_csr* x, const int32_t* cols, int64_t n_cols,
                               int64_t* out_indptr, int32_t* out_indices, float* out_values, int64_t* nnz_out,
                               void* stream, char* err, size_t err_len);

/* PFlog (v4) representation of a raw-count device CSR (float32 values): the
 * sparse delta = log1p(four_alpha * x) at the stored entries (delta_out,
 * device, nnz floats; may be x->values for in place) and the per-cell
 * baseline b_i = -(1 / n_vars) sum_j delta_ij in FP64 (baseline_out, device,
 * n_obs doubles).  Negative or non-finite counts are rejected
 * (SCXPCA_INVALID_ARGUMENT), as the reference's raw-count guard does.
 * Replaces pflog_baseline_from_raw (scx-accel/src/pflog.rs:122-193) together
 * with the lazy Scale{4 alpha} -> Log1p source it pairs with. */
int32_t scxpca_pflog_prepare(int32_t device_ordinal, const scxpca_csr* x, double four_alpha, float* delta_out,
                             double* baseline_out, void* stream, char* err, size_t err_len);

/* Baseline-aware randomized PCA of Z = delta + baseline 1^T (the exact PFlog
 * matrix, never densified): centring subtracts colmean(delta)_j +
 * mean(baseline); `baseline` holds n_obs doubles in `baseline_memory`.  The
 * baseline enters as one extra column of the working matrix, so both rank-1
 * terms ride on the ordinary products.  params->scale must be 0 (clip_max is
 * ignored); every other parameter and every output field means what it means
 * for scxpca_randomized (mean = the column means of Z).  Total variance in
 * closed form from the column statistics of delta, sum b_i^2 and
 * sum b_i rowsum(delta_i).  Replaces pflog_pca / pflog_pca_with_depth
 * (scx-accel/src/pca/cpu.rs:791-882, with the offset products of :618-687 and
 * pflog_total_variance :689-786); the reference runs it on the CPU only. */
int32_t scxpca_pflog_pca(const scxpca_csr* delta, const double* baseline, int32_t baseline_memory,
                         const scxpca_params* params, scxpca_result* out, char* err, size_t err_len);

/* Seeded N(0,1) test matrix, n_rows x n_cols column-major float32, into device
 * memory `out` on `device_ordinal`.  Replaces random_gaussian_gpu
 * (scx-gpu/src/curand.rs:76-157); the stream is Philox4x32-10 + Box-Muller,
 * not cuRAND XORWOW, so values differ from the reference's at equal seeds. */
int32_t scxpca_gaussian(int32_t device_ordinal, uint64_t seed, int64_t n_rows, int64_t n_cols,
                        float* out, char* err, size_t err_len);

/* Seeded synthetic negative-binomial CSR generated on the device (benchmark
 * input; no reference counterpart).  mu_g ~ LogNormal(loc, 1.5), s_c ~
 * LogNormal(0, 0.5), counts ~ NB(mu_g s_c, dispersion), values =
 * log1p(1e4 * count / rowsum) as float32, rows sorted by gene.  Call with
 * indices == NULL and values == NULL first to obtain *nnz_out and fill
 * `indptr` (device, n_obs + 1); then again with device buffers of *nnz_out
 * entries. */
int32_t scxpca_synth_nb_csr(int32_t device_ordinal, uint64_t seed, int64_t n_obs,
                            int64_t n_vars, double loc, double dispersion, int64_t* indptr,
                            int32_t* indices, float* values, int64_t* nnz_out, char* err,
                            size_t err_len);

/* Self-test of the bounded pipeline wait (diagnostics; no reference
 * counterpart).  Runs one block on `device_ordinal` whose mbarrier wait can
 * never complete (no thread arrives), under the same bounded wait the
 * tensor-core kernels use.  Returns SCXPCA_TIMEOUT, with the site in the
 * message, once the wait's limit (about 1 s) has passed; the context stays
 * usable and the next call runs normally.  Any other status means the
 * give-up path is broken. */
int32_t scxpca_wait_selftest(int32_t device_ordinal, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* SCXPCA_H */
