// Host-side launcher declarations shared by the kernel translation units and
// the plan orchestration (scxpca.cu).  All launchers enqueue on `st` and
// return the launch status; none synchronises.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace scx {

// Process-wide count of kernels launched by this library (every launcher
// adds the number of kernels it enqueued).
void note_launches(int n);
int64_t launches_total();

constexpr size_t kStatsSmemMax = 200 * 1024;  // per-block FP64 gene accumulators
constexpr int kTransposeGeneBlock = 256;       // genes per block, CUDA-core transposed product

// ---- sparse side (kernels_sparse.cu) ----
// out = [sum x (g) | sum x^2 (g)] in FP64, fixed order; accumulate != 0 adds
// to out instead of overwriting it (a matrix taken in row shards).
cudaError_t launch_col_stats(int dtype, const int32_t* idx, const void* val, int64_t nnz,
                             int32_t g, double* partial, int nparts, double* out,
                             cudaStream_t st, int num_sms, int accumulate = 0);
// The same statistics in two halves: blocks [block0, block0 + nblocks) of the
// nparts-block partition write their partials (block b reads entries
// [col_stats_block_begin(b), col_stats_block_begin(b + 1))), then one reduce.
// Launching the partition in pieces gives the bits of one launch.
int64_t col_stats_block_begin(int64_t nnz, int nparts, int b);
cudaError_t launch_col_stats_blocks(int dtype, const int32_t* idx, const void* val, int64_t nnz, int32_t g,
                                    double* partial, int nparts, int block0, int nblocks, cudaStream_t st);
cudaError_t launch_col_stats_reduce(const double* partial, int nparts, int32_t g, double* out, cudaStream_t st,
                                    int num_sms, int accumulate = 0);
cudaError_t launch_transform_values(int in_dtype, int out_dtype, const int32_t* idx,
                                    const void* in, void* out, int64_t nnz, int mode,
                                    const double* mu, const double* inv_std,
                                    const double* cshift, double clip, cudaStream_t st,
                                    int num_sms);
cudaError_t launch_spmm_fwd(int dtype, int ld, const int64_t* indptr, const int32_t* idx,
                            const void* val, int64_t n, const float* V, const float* mc,
                            float* Y, cudaStream_t st, int num_sms);
cudaError_t launch_row_block_ptr(const int64_t* indptr, const int32_t* idx, int64_t n, int nb,
                                 int gb, int32_t* rbp, cudaStream_t st, int num_sms);
cudaError_t launch_spmm_t(int dtype, int ld, const int64_t* indptr, const int32_t* idx,
                          const void* val, int64_t n, int32_t g, const int32_t* rbp, int nb,
                          int nchunks, int64_t rows_per_chunk, const float* Q, float* part,
                          cudaStream_t st);
cudaError_t launch_reduce_rows_f32(const float* part, int nparts, int64_t len, double* out,
                                   int accumulate, cudaStream_t st, int num_sms);
// The same over partials of a column panel: part[b] is rows x width; row r
// of the sum goes to out + r * ldo (a panel of a wider matrix).
cudaError_t launch_reduce_panel_f32(const float* part, int nparts, int64_t rows, int width, double* out, int ldo,
                                    cudaStream_t st, int num_sms);

// ---- CUDA-core SpMM pair in a fixed summation order (kernels_strict.cu) ----
constexpr int kStrictTile = 128;  // rows per tile of the tile-CSC copy (a power of two <= 256)
int strict_genes_per_warp(int ld);
// Slots of the tile-CSC copy: n_vars rounded up to whole blocks of the transposed product.
int strict_slot_count(int64_t g, int ld);
// Balanced gene -> slot assignment from per-gene stored-entry counts.
void strict_assign_slots(const std::vector<int32_t>& counts, int ld, std::vector<int32_t>& gene2slot,
                         std::vector<int32_t>& slot2gene);
size_t strict_tile_smem_bytes(int nslots);
cudaError_t launch_gene_counts(const int32_t* idx, int64_t nnz, int32_t* counts, cudaStream_t st, int num_sms);
// Tile-CSC copy of a row-sorted CSR: tptr [n_tiles][nslots + 1], cell/cval [nnz].
cudaError_t launch_tile_csc(int dtype, const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                            const int32_t* gene2slot, int32_t nslots, int32_t* tptr, uint8_t* cell, void* cval,
                            cudaStream_t st, int num_sms);
// Y (n x ld) = P V - 1 mc^T (mc may be null) from a row-sorted CSR.  `ld` is
// the width of the column panel taken (32, 64, 96 or 128); V, mc and Y point
// at its first column and `lds` is the row stride of V and Y in floats
// (0: lds = ld, the whole matrix).
cudaError_t launch_fwd_strict(int dtype, int ld, const int64_t* indptr, const int32_t* idx, const void* val,
                              int64_t n, int32_t g, const float* V, const float* mc, float* Y, cudaStream_t st,
                              int lds = 0);
// part[range][g][ld] = partial P^T Q over the row tiles of each of `ranges`
// contiguous ranges; Q is a column panel of width ld and row stride lds (0: ld).
cudaError_t launch_rmat_strict(int dtype, int ld, const int64_t* indptr, const int32_t* tptr, const uint8_t* cell,
                               const void* cval, int64_t n, int32_t g, int32_t nslots, const int32_t* slot2gene,
                               int ranges, const float* Q, float* part, cudaStream_t st, int lds = 0);
cudaError_t launch_reduce_rows_f64(const double* part, int nparts, int64_t len, double* out,
                                   int accumulate, cudaStream_t st, int num_sms);

// ---- CSR validation (kernels_csr.cu) ----
// flags[0]: bad indptr (non-monotone / out of range), flags[1]: column index
// out of range, flags[2]: a row not sorted strictly ascending (duplicates or
// disorder), flags[3]: non-finite value.
cudaError_t launch_validate_csr(int dtype, const int64_t* indptr, const int32_t* idx,
                                const void* val, int64_t n, int64_t g, int64_t nnz,
                                int32_t* flags, cudaStream_t st, int num_sms);
// Sort every row by gene in place (values follow), one warp per row.
cudaError_t launch_sort_rows(int dtype, const int64_t* indptr, int32_t* idx, void* val,
                             int64_t n, cudaStream_t st, int num_sms);

// ---- sketches wider than one 128-column panel (kernels_wide.cu; ld = 256) ----
cudaError_t launch_gram_wide_f32(const float* A, int64_t n, int ld, double* part, int nparts, cudaStream_t st);
cudaError_t launch_gram_wide_f64(const double* A, int64_t n, int ld, double* part, int nparts, cudaStream_t st);
cudaError_t launch_cholesky_wide(const double* G, int k, int ld, double tau, int shift_on_fail, double* R,
                                 double* Rinv, float* Rinv_f, int* status, cudaStream_t st);
// Out[:, c0 .. c0 + cnt) = In[:, :K] M[:K, c0 .. c0 + cnt), cnt <= 128.
cudaError_t launch_tall_mm_wide(const float* In, int64_t n, int K, int ldi, const float* M, int ldm, int c0,
                                int cnt, float* Out, int ldo, cudaStream_t st, int num_sms);
// A <- A M in place for an upper-triangular M (ld x ld).
cudaError_t launch_apply_upper_wide(float* A, int64_t n, int ld, const float* M, cudaStream_t st, int num_sms);
cudaError_t launch_center_apply_wide(const double* W, int64_t g, int ld, const double* mu, const double* s,
                                     const double* M, double* Z, cudaStream_t st);

// ---- dense side (kernels_dense.cu) ----
// One k x k factorisation (Cholesky) or eigensolve (Jacobi) of a segment of a
// batch: its arguments, read by one block of a batched launch.
struct CholTask {
  const double* G;
  double* R;
  double* Rinv;
  float* Rinv_f;
  int* status;
};
struct JacobiTask {
  const double* C;
  double* evals;
  double* evecs;
  int* sweeps;
};
// Per-segment arguments of the batched gene-side launches (one grid row per segment).
struct ApplyTask {  // Z = (W - mu s^T) M (mu may be null)
  const double* W;
  const double* mu;
  const double* s;
  const double* M;
  double* Z;
};
struct GramTask {  // Gram partials of A into part, then their sum into G
  const double* A;
  double* part;
  double* G;
};
struct RoundTask {  // Vf = (float) A, mc = mu^T Vf
  const double* A;
  const double* mu;
  float* Vf;
  float* mc;
};
struct SplitTask {  // 16-bit image of a float matrix
  const float* in;
  uint16_t* img;
};
struct RitzTask {  // the Rayleigh-Ritz finish of one segment (launch_ritz_finish's arguments)
  const double* B;
  const double* evals;
  const double* evecs;
  const double* Rinv2;
  double* sigma;
  float* comps;
  float* M_emb;
};
cudaError_t launch_ritz_finish_batch(const RitzTask* tasks, int ntasks, int64_t g, int ld, int k, int nc,
                                     cudaStream_t st);
// One matrix of a batched tall right-multiplication: Out = In M (In n x ld,
// rows in tiles of 128; the 16-bit image of Out too when img is set).  tile0
// is the matrix's first tile in the launch's numbering (the tiles of all
// tasks, task after task).  Each output element gets the FMAs, in the same
// order, of the matrix's own launch_apply_right_split / launch_embed call.
struct TallTask {
  const float* In;
  float* Out;
  uint16_t* img;
  const float* M;
  int64_t n;
  int64_t tile0;
};
// Y <- Y M for an upper-triangular 64 x 64 M (Cholesky inverse), per task.
cudaError_t launch_apply_upper64_batch(const TallTask* tasks, int ntasks, int64_t total_tiles, int fmt,
                                       cudaStream_t st, int num_sms);
// Embeddings U = Q M_emb per task (ld <= 64 and nc <= 64; M_emb ld x nc, U n x nc).
cudaError_t launch_embed_batch(const TallTask* tasks, int ntasks, int64_t total_tiles, int ld, int nc,
                               cudaStream_t st, int num_sms);
cudaError_t launch_center_apply_batch(const ApplyTask* tasks, int ntasks, int64_t g, int ld, cudaStream_t st);
cudaError_t launch_gram_f64_batch(const GramTask* tasks, int ntasks, int64_t n, int ld, int nparts,
                                  cudaStream_t st, int num_sms);
cudaError_t launch_reduce_rows_f64_batch(const GramTask* tasks, int ntasks, int nparts, int64_t len, cudaStream_t st,
                                         int num_sms);
cudaError_t launch_round_v_batch(const RoundTask* tasks, int ntasks, int64_t g, int ld, cudaStream_t st);
// mc = mu^T Vf for every task; and the copy of one test matrix (count floats)
// into the Vf of tasks 1 .. ntasks - 1.
// Where one segment of a batch keeps its results: its status words (4), its
// tensor-core error word (null without one), sigma (k) and components.
struct OutTask {
  int* status;
  const int* tc_err;
  const double* sigma;
  const float* comps;
};
cudaError_t launch_gather_out(const OutTask* tasks, int ntasks, int k, int64_t count, int* status, double* sigma,
                              float* comps, cudaStream_t st);
cudaError_t launch_zero_status(const OutTask* tasks, int ntasks, cudaStream_t st);
cudaError_t launch_mean_prefactor_batch(const RoundTask* tasks, int ntasks, int64_t g, int ld, cudaStream_t st);
cudaError_t launch_broadcast_v(const float* src, int64_t count, const RoundTask* tasks, int ntasks, cudaStream_t st);
cudaError_t launch_split16_batch(const SplitTask* tasks, int ntasks, int64_t count, int fmt, cudaStream_t st);
// ntasks factorisations of one launch, one block each (k, ld <= 128).
cudaError_t launch_cholesky_batch(const CholTask* tasks, int ntasks, int k, int ld, double tau, int shift_on_fail,
                                  cudaStream_t st);
cudaError_t launch_jacobi_eig_batch(const JacobiTask* tasks, int ntasks, int k, int ld, cudaStream_t st);
// Gram partials of a tall row-major matrix A (n x ld, first k columns used):
// part[b] = [A_b^T A_b (ld x ld), colsum(A_b) (ld)] in FP64.
cudaError_t launch_gram_f32(const float* A, int64_t n, int ld, double* part, int nparts,
                            cudaStream_t st);
cudaError_t launch_gram_f64(const double* A, int64_t n, int ld, double* part, int nparts,
                            cudaStream_t st);
// Cholesky G = R^T R of the leading k x k block (single block).  Writes R and
// R^{-1} (ld x ld, zero outside the leading upper triangle; R^{-1} pad
// diagonal = 0), plus R^{-1} as float.  status[0] += 1 on a shifted
// factorisation (shift_on_fail) or is set to -(j+1) on a failed pivot j.
cudaError_t launch_cholesky(const double* G, int k, int ld, double tau, int shift_on_fail,
                            double* R, double* Rinv, float* Rinv_f, int* status, cudaStream_t st);
// Tall apply: Out[i, :] = In[i, :] * M (ld x ld float, upper-triangular: the Cholesky inverse).
cudaError_t launch_apply_right_f32(const float* In, int64_t n, int ld, const float* M,
                                   float* Out, cudaStream_t st, int num_sms);
// Same, also writing the 16-bit image of Out (n x 2 ld; fmt 1 = bf16, 0 = f16).
cudaError_t launch_apply_right_split(const float* In, int64_t n, int ld, const float* M, float* Out,
                                     uint16_t* img, int fmt, cudaStream_t st, int num_sms);
// Gene-side ops (n_vars x ld, FP64):
//   Z = (W - mu s^T) M        (mu may be null)
cudaError_t launch_center_apply(const double* W, int64_t g, int ld, const double* mu,
                                const double* s, const double* M, double* Z, cudaStream_t st);
//   A = A * M  in place (FP64)
cudaError_t launch_apply_right_f64(double* A, int64_t g, int ld, const double* M,
                                   cudaStream_t st);
//   Vf = (float)A ; mc = A^T mu (float, from the rounded Vf) ; mu may be null
cudaError_t launch_round_v(const double* A, int64_t g, int ld, const double* mu, float* Vf,
                           float* mc, cudaStream_t st);
//   mc = Vf^T mu for a float V (mu may be null -> zeros)
cudaError_t launch_mean_prefactor(const float* Vf, int64_t g, int ld, const double* mu,
                                  float* mc, cudaStream_t st);
// Symmetric eigendecomposition (parallel cyclic Jacobi, single block) of the
// leading k x k block of C (ld x ld FP64).  evals descending, evecs columns.
cudaError_t launch_jacobi_eig(const double* C, int k, int ld, double* evals, double* evecs,
                              int* sweeps, cudaStream_t st);
// Rayleigh-Ritz finish: sigma = sqrt(max(evals,0)); components[c][j] =
// (B E)[j][c] / sigma_c (c < nc); M_emb = Rinv2 * E[:, :nc] * diag(sigma)
// (ld x nc, float).
cudaError_t launch_ritz_finish(const double* B, int64_t g, int ld, int k, int nc,
                               const double* evals, const double* evecs, const double* Rinv2,
                               double* sigma, float* components, float* M_emb,
                               cudaStream_t st);
// Embeddings U (n x nc row-major) = Q (n x ld) * M_emb (ld x nc).
cudaError_t launch_embed(const float* Q, int64_t n, int ld, int k, const float* M_emb, int nc,
                         float* U, cudaStream_t st, int num_sms);
// Seeded Gaussian n_rows x n_cols column-major into out (ld_out = n_rows) or,
// when ld_pad > 0, into a gene-major padded buffer out[i * ld_pad + j].
cudaError_t launch_gaussian(uint64_t seed, int64_t n_rows, int64_t n_cols, float* out,
                            int ld_pad, cudaStream_t st, int num_sms);
// Copy a column-major n_rows x n_cols float matrix into a row-major padded one.
cudaError_t launch_colmajor_to_padded(const float* in, int64_t n_rows, int64_t n_cols, int ld,
                                      float* out, cudaStream_t st, int num_sms);

// ---- tensor-core path (kernels_tc.cu) ----
// Tile-chunk packed format: counts[t * nc + c] entries per (128-row tile,
// 64-gene chunk); seg = exclusive scan of counts; ent/qoff filled from a
// sorted, duplicate-free CSR whose values are 16-bit (bf16/f16 bits).
// counts are padded to multiples of 4 entries; meta holds one 16-byte record
// per segment (tile_meta_bytes).
size_t tile_meta_bytes(int64_t n, int nc);
cudaError_t tile_format_count(const int64_t* indptr, const int32_t* idx, int64_t n, int nc,
                              int64_t* counts, cudaStream_t st, int num_sms);
cudaError_t tile_format_fill(const int64_t* indptr, const int32_t* idx, const void* val16, int64_t n,
                             int nc, const int64_t* seg, uint32_t* ent, void* meta, cudaStream_t st,
                             int num_sms);
// TMA map of a row-major [rows][cols] 16-bit matrix (fmt 1 = bf16, 0 = f16);
// returns the CUresult.
int make_tmap16(CUtensorMap* map, const void* base, int64_t rows, int64_t cols, int box_rows, int fmt);
// 16-bit image of a float matrix M (rows x ld): rows x 2 ld values, column
// 2 j = hi(M[:, j]) = round16(M[:, j]), column 2 j + 1 = round16(M[:, j] - hi).
// Y (n x ld, FP32; may be null) = A V - mc with V given by its image (map
// vmap), plus the image of Y.
cudaError_t launch_fwd_tc(int ld, const uint32_t* ent, const void* meta, int64_t n, int nc, const CUtensorMap* vmap,
                          const float* mc, float* Y, uint16_t* Yimg, int fmt, int* err, cudaStream_t st, int num_sms);
// Partials part[row_group][g][ld] of A^T Q, Q given by its image (map qmap);
// returns row groups.
int rmat_tc_groups(int ld, int nc, int num_sms, int* gene_groups);
cudaError_t launch_rmat_tc(int ld, const uint32_t* ent, const void* meta, int64_t n, int nc, int64_t g,
                           int gene_groups, int row_groups, const CUtensorMap* qmap, float* part, int fmt, int* err,
                           cudaStream_t st);
// Gram partials [G (64 x 64), colsum (64)] of hi + lo from the image (ld 64)
// on tensor cores; returns the number of partials written, or -1 on a launch
// error.
// `parts` > 0 asks for that many partials (at most one per row tile), 0 for
// one per SM; gram_tc_parts gives the count a call writes.
int gram_tc_parts(int64_t n, int parts, int num_sms);
int launch_gram_tc(int64_t n, const CUtensorMap* qmap, double* part, int fmt, int* err, cudaStream_t st, int num_sms,
                   int parts = 0);
size_t fwd_tc_smem_bytes(int ld);
size_t rmat_tc_smem_bytes(int ld);
// The products and the Gram above over every segment of a batch in one
// launch (ld 64).  A segment is one plan's packed matrix and buffers; its
// tensor maps are device copies.  The forward kernel walks the bands (pairs
// of row tiles) of all segments, numbered segment after segment
// (band_seg[b] = the segment of band b, TcSegment::band0 its first band); the
// transposed product and the Gram take one item (a tile range of one
// segment, and the partial it writes) per CTA.  Each segment's results have
// the bits of its own launch_*_tc call with the same partition.
struct TcSegment {
  const uint32_t* ent;
  const void* meta;
  const CUtensorMap* vmap;
  const CUtensorMap* qmap;
  const float* mc;
  float* Y;        // FP32 copy of the forward product (written when asked)
  uint16_t* Yimg;
  float* part;     // transposed-product partials [row group][n_vars][64]
  double* gpart;   // Gram partials [part][64 * 64 + 64]
  int* err;
  int64_t n;       // rows
  int64_t band0;
};
struct TcItem {
  int32_t seg;
  int32_t gg;      // gene group (transposed product)
  int32_t slot;    // partial written: row group (transposed) or part (Gram)
  int32_t pad;
  int64_t t0, t1;  // row tiles [t0, t1) of the segment
};
// Embeddings U = Q M (n x nc row-major, nc <= 64; M ld 64 x nc) on tensor
// cores from the 16-bit image of Q (ld 64) behind qmap.
cudaError_t launch_embed_tc(int64_t n, const CUtensorMap* qmap, const float* M, int nc, float* U, int fmt, int* err,
                            cudaStream_t st, int num_sms);
cudaError_t launch_fwd_tc_batch(const TcSegment* segs, const int32_t* band_seg, int64_t n_bands, int nc,
                                int write_y, int fmt, cudaStream_t st, int num_sms);
cudaError_t launch_rmat_tc_batch(const TcSegment* segs, const TcItem* items, int n_items, int nc, int64_t g,
                                 int gene_groups, int fmt, cudaStream_t st);
cudaError_t launch_gram_tc_batch(const TcSegment* segs, const TcItem* items, int n_items, int fmt, cudaStream_t st);
// Tile range [t0, t1) of CTA b of nb over n_tiles row tiles: the split every
// launcher above uses.
__host__ __device__ inline int64_t tc_range_begin(int64_t b, int64_t nb, int64_t n_tiles) { return b * n_tiles / nb; }
// Sums of per-segment partials: out = sum over nparts of part[p][len] (FP64,
// fixed order), one task per segment, one launch.
struct SumTask {
  const void* part;
  double* out;
  int nparts;
  int pad;
};
cudaError_t launch_reduce_rows_batch(int part_dtype_f32, const SumTask* tasks, int ntasks, int64_t len,
                                     cudaStream_t st);
// One block whose pipeline wait never completes: the bounded wait gives up
// after its limit (about 1 s) and writes `code` to err.
cudaError_t launch_wait_selftest(int* err, int code, cudaStream_t st);
// Image of count floats: img[2 i] = round16(x_i), img[2 i + 1] = round16(x_i - img[2 i]).
cudaError_t launch_split16(const float* in, int64_t count, uint16_t* img, int fmt, cudaStream_t st, int num_sms);

// ---- truncated-SVD adjoint (kernels_adjoint.cu) ----
// Column sums (FP64) of a tall float matrix A (n x ld, first ncols columns)
// into out[ld]; part holds nparts x ld partials.
cudaError_t launch_colsum_f32(const float* A, int64_t n, int ld, int ncols, double* part, int nparts,
                              double* out, cudaStream_t st, int num_sms);
// T (ld x ld) = A^T B over g rows, first ka x kb block (FP64).
cudaError_t launch_atb(const double* A, const double* B, int64_t g, int ld, int ka, int kb, double* T,
                       cudaStream_t st);
// M = E diag(1 / sqrt(evals)) over the first k columns.
cudaError_t launch_ritz_scale(const double* E, const double* evals, int k, int ld, double* M, cudaStream_t st);
// Phi[j][i] = T[j][i] / (evals[i] - evals[j]), j < k, i < c, j != i.
cudaError_t launch_phi(const double* T, const double* evals, int k, int c, int ld, double* Phi, cudaStream_t st);
// Out = X + beta Y on the first c columns (g x ld).
cudaError_t launch_axpy_cols(const double* X, const double* Y, double beta, int64_t g, int ld, int c, double* Out,
                             cudaStream_t st);
// out[i] = column i of X . column i of Y, i < c.
cudaError_t launch_coldot(const double* X, const double* Y, int64_t g, int ld, int c, double* out, cudaStream_t st);
// Conjugate-gradient pieces for (lambda_i I - X~^T X~) on the complement of the sketch subspace.
cudaError_t launch_cg_ap(const double* P, const double* W, const double* Proj, const double* evals, int64_t g,
                         int ld, int c, double* Ap, cudaStream_t st);
cudaError_t launch_cg_step(double* X, double* R, const double* P, const double* Ap, const double* rr,
                           const double* pAp, int64_t g, int ld, int c, cudaStream_t st);
cudaError_t launch_cg_dir(double* P, const double* R, double* rr, const double* rr_new, int64_t g, int ld, int c,
                          cudaStream_t st);
// colD[j] = sum_i sF[i] V[j][i] + sS[i] A[j][i].
cudaError_t launch_col_d(const double* V, const double* A, const double* sF, const double* sS, int64_t g, int ld,
                         int c, double* colD, cudaStream_t st);
// Gradients of the per-gene centre and scale (either output may be null).
cudaError_t launch_grad_vectors(const double* colD, const double* sumDP, const double* center, const double* scale,
                                int64_t g, double* grad_center, double* grad_scale, cudaStream_t st);
// SDDMM of the gradient at the stored entries (column slice of cs <= 64
// columns); part[nchunks][g] receives per-gene sums of d * x~.
cudaError_t launch_sddmm(int dtype, const int64_t* indptr, const int32_t* idx, const void* val, int64_t n, int32_t g,
                         const int32_t* rbp, int nb, int nchunks, int64_t rows_per_chunk, const float* G, int ldg,
                         const float* Y, int ldy, const float* S, int lds, const double* V, const double* A, int ldv,
                         int cs, const double* scale, int accumulate, float* grad, double* part, cudaStream_t st);

// ---- upstream producers (kernels_preprocess.cu) ----
// out = [log1p](x * target_sum / rowsum) [* row_factor[row]] per row; target_sum <= 0 skips the
// normalisation; in may equal out.
cudaError_t launch_normalize_log1p(const int64_t* indptr, const float* in, float* out, int64_t n,
                                   double target_sum, int do_log1p, const float* row_factor, cudaStream_t st,
                                   int num_sms);
// Kept entries per row under col_map (new index or -1), then the compacted CSR.
cudaError_t launch_project_count(const int64_t* indptr, const int32_t* idx, int64_t n, const int32_t* col_map,
                                 int64_t* counts, cudaStream_t st, int num_sms);
cudaError_t launch_project_fill(const int64_t* indptr, const int32_t* idx, const float* val, int64_t n,
                                const int32_t* col_map, const int64_t* out_ptr, int32_t* out_idx, float* out_val,
                                cudaStream_t st, int num_sms);

// PFlog: delta = log1p(four_alpha x), baseline b_i = -sum_j delta_ij / d (FP64);
// flags[0] negative count, flags[1] non-finite count.
cudaError_t launch_pflog_prepare(const int64_t* indptr, const float* x, int64_t n, int64_t d, double four_alpha,
                                 float* delta, double* baseline, int32_t* flags, cudaStream_t st, int num_sms);
// Augmented CSR [delta | b] (column g = b_i, one extra entry per row) and
// cross[i] = b_i * rowsum(delta_i).
cudaError_t launch_pflog_augment(int dtype, const int64_t* indptr, const int32_t* idx, const void* val, int64_t n,
                                 int32_t g, const double* baseline, int64_t* aptr, int32_t* aidx, void* aval,
                                 double* cross, cudaStream_t st, int num_sms);
// V[g] = sum_{j<g} V[j] (gene-major float, rows of ld).
cudaError_t launch_aug_colsum(float* V, int32_t g, int ld, cudaStream_t st);
// W[j] += W[g] (j < g), W[g] = 0 (gene-major FP64, rows of ld).
cudaError_t launch_aug_fold(double* W, int32_t g, int ld, cudaStream_t st, int num_sms);

// indptr[i] -= base for i <= n (a row shard's pointers made relative to its first entry).
cudaError_t launch_rebase_indptr(int64_t* indptr, int64_t n, int64_t base, cudaStream_t st, int num_sms);

// ---- synthetic generator (synth.cu) ----
cudaError_t launch_synth_count(uint64_t seed, int64_t n, int64_t g, double loc, double disp,
                               const float* mu_g, int64_t* row_nnz, float* rowsum,
                               cudaStream_t st, int num_sms);
cudaError_t launch_synth_fill(uint64_t seed, int64_t n, int64_t g, double loc, double disp,
                              const float* mu_g, const int64_t* indptr, const float* rowsum,
                              int32_t* idx, float* val, cudaStream_t st, int num_sms);
cudaError_t launch_synth_gene_means(uint64_t seed, int64_t g, double loc, float* mu_g,
                                    cudaStream_t st);
cudaError_t launch_exclusive_scan_i64(const int64_t* in, int64_t n, int64_t* out,
                                      cudaStream_t st);

}  // namespace scx
