// Per-gene column statistics with no device allocation.
//
// Some callers cannot let a library call cudaMalloc: a process whose device
// memory is owned by a caching pool (a PyTorch or RAPIDS/RMM allocator that
// has already reserved the device, or enforces a budget that out-of-band
// allocations would break), and latency-sensitive pipelines where
// cudaMalloc/cudaFree would add implicit device-wide synchronisation between
// their streams.  scxpca_col_stats_noalloc serves them: the caller passes the
// device CSR and the device output, and the only scratch the computation
// needs -- the per-block partial sums of k_col_stats and four validation
// flags -- lives in the file-scope array below, which every GPU that loads
// the library holds (kNoAllocScratchBytes, 8 MiB) until the process exits.
//
// In host code `g_noalloc_scratch` names a host-side stand-in, not a device
// address; a kernel given it would fault or, where the GPU can reach host
// memory, silently use the wrong memory.  The device address is taken once
// per device with cudaGetSymbolAddress (with that device current) on the
// first call there.  No call can be recorded into a CUDA graph: every call
// reads the validation flags back to the host and waits for its stream, so a
// call on a stream that is being captured is refused with
// SCXPCA_INVALID_ARGUMENT instead of breaking the caller's capture.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/scxpca.h"
#include "common.cuh"
#include "launch.h"

namespace scx {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)SCXPCA_NOALLOC_SCRATCH_BYTES;
constexpr size_t kFlagBytes = 256;  // four int32 flags, padded to keep the partials 256-byte aligned
constexpr int64_t kPartialDoubles = (int64_t)((kNoAllocScratchBytes - kFlagBytes) / sizeof(double));
constexpr int kMaxDevices = 256;
static_assert(kPartialDoubles / (2 * SCXPCA_NOALLOC_MAX_VARS) >= 32,
              "the scratch must hold at least 32 per-block partials at the widest matrix");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;               // serialises calls: they share the one array
void* g_scratch_addr[kMaxDevices] = {};  // device address of the array, per device

struct NoAllocError {
  int32_t code;
  std::string msg;
};

void na_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  throw NoAllocError{SCXPCA_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e)};
}

// Device address of the scratch array on the current device `dev`.
unsigned char* scratch_on(int dev) {
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    na_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_addr[dev] = p;
  }
  return static_cast<unsigned char*>(g_scratch_addr[dev]);
}

void col_stats_noalloc(int32_t dev, const scxpca_csr* x, double* out, cudaStream_t st) {
  if (!x || !out) throw NoAllocError{SCXPCA_INVALID_ARGUMENT, "null csr or output"};
  if (x->memory != SCXPCA_MEM_DEVICE)
    throw NoAllocError{SCXPCA_INVALID_ARGUMENT, "scxpca_col_stats_noalloc needs a device CSR (memory = DEVICE)"};
  if (x->n_obs < 0 || x->n_vars <= 0 || x->nnz < 0)
    throw NoAllocError{SCXPCA_INVALID_ARGUMENT, "matrix must have n_vars > 0 and non-negative sizes"};
  if (x->n_vars > SCXPCA_NOALLOC_MAX_VARS)
    throw NoAllocError{SCXPCA_INVALID_ARGUMENT,
                       "n_vars = " + std::to_string(x->n_vars) + " exceeds the no-allocation maximum of " +
                           std::to_string(SCXPCA_NOALLOC_MAX_VARS) + " genes (" +
                           std::to_string(SCXPCA_NOALLOC_SCRATCH_BYTES) +
                           "-byte static scratch); use scxpca_plan_col_stats"};
  if (x->values_dtype < 0 || x->values_dtype > 2) throw NoAllocError{SCXPCA_INVALID_ARGUMENT, "bad values_dtype"};
  if (!x->indptr || (x->nnz > 0 && (!x->indices || !x->values)))
    throw NoAllocError{SCXPCA_INVALID_ARGUMENT, "null CSR arrays"};

  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw NoAllocError{SCXPCA_CUDA_ERROR, "no CUDA device is available"};
  }
  if (dev < 0 || dev >= count || dev >= kMaxDevices)
    throw NoAllocError{SCXPCA_INVALID_ARGUMENT, "device_ordinal " + std::to_string(dev) + " out of range"};
  int prev = -1;
  cudaGetDevice(&prev);
  struct Restore {
    int d;
    ~Restore() {
      if (d >= 0) cudaSetDevice(d);
    }
  } restore{prev};
  na_check(cudaSetDevice(dev), "cudaSetDevice");
  // A non-sticky error left by the caller's earlier work is not this call's
  // failure: clear it so the launch checks below report only our own.
  cudaGetLastError();
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  na_check(cudaStreamIsCapturing(st, &capture), "cudaStreamIsCapturing");
  if (capture != cudaStreamCaptureStatusNone)
    throw NoAllocError{SCXPCA_INVALID_ARGUMENT,
                       "scxpca_col_stats_noalloc cannot run on a stream that is being captured: it reads "
                       "the validation flags back to the host and waits for the stream"};
  int sms = 148;
  na_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");

  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  unsigned char* base = scratch_on(dev);
  int32_t* flags = reinterpret_cast<int32_t*>(base);
  double* partial = reinterpret_cast<double*>(base + kFlagBytes);
  const int64_t g = x->n_vars;
  const int nparts = (int)std::min<int64_t>(2 * (int64_t)sms, kPartialDoubles / (2 * g));

  // Once work is queued, an error must not release the lock while our
  // kernels may still touch the shared array: wait for the stream first
  // (its own status is already being reported) and then throw.
  auto check_queued = [st](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    cudaStreamSynchronize(st);
    na_check(e, what);
  };
  // The flags accumulate with atomicOr: they must start at zero.  The
  // partials are overwritten whole by every call and need no clearing.
  check_queued(cudaMemsetAsync(flags, 0, 4 * sizeof(int32_t), st), "cudaMemsetAsync(flags)");
  check_queued(launch_validate_csr(x->values_dtype, x->indptr, x->indices, x->values, x->n_obs, g, x->nnz, flags,
                                   st, sms),
               "launch_validate_csr");
  int32_t hf[4] = {0, 0, 0, 0};
  check_queued(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(flags)");
  check_queued(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (hf[0]) throw NoAllocError{SCXPCA_INVALID_CSR, "invalid CSR: indptr is not monotone within [0, nnz]"};
  if (hf[1]) throw NoAllocError{SCXPCA_INVALID_CSR, "invalid CSR: column index out of range [0, n_vars)"};
  if (hf[3]) throw NoAllocError{SCXPCA_INVALID_CSR, "invalid CSR: non-finite value"};
  check_queued(launch_col_stats(x->values_dtype, x->indices, x->values, x->nnz, (int32_t)g, partial, nparts, out,
                                st, sms),
               "launch_col_stats");
  // Wait before releasing the lock, so the next call cannot touch the
  // partials while this call's kernels still read them.
  na_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

}  // namespace
}  // namespace scx

extern "C" int32_t scxpca_col_stats_noalloc(int32_t device_ordinal, const scxpca_csr* x, double* out_stats,
                                            void* stream, char* err, size_t err_len) {
  auto write = [&](const std::string& m) {
    if (!err || err_len == 0) return;
    size_t n = std::min(err_len - 1, m.size());
    memcpy(err, m.data(), n);
    err[n] = '\0';
  };
  try {
    scx::col_stats_noalloc(device_ordinal, x, out_stats, static_cast<cudaStream_t>(stream));
    write("");
    return SCXPCA_OK;
  } catch (const scx::NoAllocError& e) {
    write(e.msg);
    return e.code;
  } catch (...) {
    write("unexpected internal error");
    return SCXPCA_CUDA_ERROR;
  }
}
