"""ctypes binding of libscxpca.so (the C ABI declared in include/scxpca.h).

The library is built in-tree (``python -m scx_b200.csrc.build``) and loaded
from the package directory.  Loading never falls back to anything: a missing
or unloadable library raises ``ScxLibraryError``.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libscxpca.so"

OK = 0
INVALID_ARGUMENT = 1
OUT_OF_MEMORY = 2
NOT_SPD = 3
INVALID_CSR = 4
CUDA_ERROR = 5
TIMEOUT = 6
UNSUPPORTED = 7

F32, BF16, F16 = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
QR_HOUSEHOLDER, QR_CHOLESKY = 0, 1
MATH_STRICT_FP32, MATH_MIXED_BF16, MATH_MIXED_F16 = 0, 1, 2
SPMM_DEFAULT, SPMM_DETERMINISTIC = 0, 1

# Static scratch of scxpca_col_stats_noalloc and the widest matrix it takes.
NOALLOC_SCRATCH_BYTES = 8 << 20
NOALLOC_MAX_VARS = 12800

# Every symbol include/scxpca.h declares.
EXPORTED = (
    "scxpca_status_string",
    "scxpca_abi_version",
    "scxpca_randomized",
    "scxpca_plan_create",
    "scxpca_plan_run",
    "scxpca_plan_destroy",
    "scxpca_plan_create_affine",
    "scxpca_plan_backward",
    "scxpca_batch_create",
    "scxpca_batch_run",
    "scxpca_batch_info",
    "scxpca_batch_destroy",
    "scxpca_plan_info",
    "scxpca_plan_matmat",
    "scxpca_plan_rmatmat",
    "scxpca_plan_qr",
    "scxpca_plan_col_stats",
    "scxpca_col_stats_noalloc",
    "scxpca_plan_set_profiling",
    "scxpca_plan_get_profile",
    "scxpca_gaussian",
    "scxpca_synth_nb_csr",
    "scxpca_wait_selftest",
    "scxpca_last_call_phases",
    "scxpca_preprocess",
    "scxpca_project_columns",
    "scxpca_pflog_prepare",
    "scxpca_pflog_pca",
)

STAGES = ("prepare", "forward", "transpose", "reduce", "gram", "apply", "small", "embed")
# Phases of a one-shot call (scxpca_last_call_phases).
PHASES = ("upload", "validate", "stats", "transform", "pack", "buffers", "pca", "download", "destroy")


class ScxLibraryError(RuntimeError):
    pass


class Csr(C.Structure):
    _fields_ = [
        ("n_obs", C.c_int64),
        ("n_vars", C.c_int64),
        ("nnz", C.c_int64),
        ("indptr", C.c_void_p),
        ("indices", C.c_void_p),
        ("values", C.c_void_p),
        ("values_dtype", C.c_int32),
        ("memory", C.c_int32),
    ]


class Params(C.Structure):
    _fields_ = [
        ("n_components", C.c_int64),
        ("n_oversamples", C.c_int64),
        ("n_power_iterations", C.c_int64),
        ("zero_center", C.c_int32),
        ("scale", C.c_int32),
        ("clip_max", C.c_double),
        ("seed", C.c_uint64),
        ("omega", C.c_void_p),
        ("omega_memory", C.c_int32),
        ("qr_method", C.c_int32),
        ("math_mode", C.c_int32),
        ("spmm_policy", C.c_int32),
        ("device_ordinal", C.c_int32),
        ("reserved0", C.c_int32),
        ("stream", C.c_void_p),
        ("device_budget", C.c_int64),
    ]


class Result(C.Structure):
    _fields_ = [
        ("embeddings", C.c_void_p),
        ("components", C.c_void_p),
        ("variance_explained", C.c_void_p),
        ("variance_ratio", C.c_void_p),
        ("singular_values", C.c_void_p),
        ("mean", C.c_void_p),
        ("std", C.c_void_p),
        ("embeddings_memory", C.c_int32),
        ("resident_csr", C.c_int32),
        ("total_var_recomputed", C.c_int32),
        ("shifted_cholesky", C.c_int32),
        ("total_var", C.c_double),
        ("eig_sweeps", C.c_int32),
        ("n_shards", C.c_int32),
    ]


class Profile(C.Structure):
    _fields_ = [
        ("launches", C.c_int64 * len(STAGES)),
        ("device_ms", C.c_double * len(STAGES)),
        ("kernel_launches", C.c_int64),
        ("runs", C.c_int64),
    ]


_lib = None


def load() -> C.CDLL:
    """Load libscxpca.so once; raise ScxLibraryError if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ScxLibraryError(
            f"{LIB_PATH} is missing: build it with `python -m scx_b200.csrc.build` "
            "(the CUDA path has no fallback)")
    try:
        lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    except OSError as e:  # pragma: no cover - depends on the host
        raise ScxLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    P = C.c_void_p
    E = [C.c_char_p, C.c_size_t]
    sigs = {
        "scxpca_status_string": (C.c_char_p, [C.c_int32]),
        "scxpca_abi_version": (C.c_int32, []),
        "scxpca_randomized": (C.c_int32, [C.POINTER(Csr), C.POINTER(Params), C.POINTER(Result), *E]),
        "scxpca_plan_create": (C.c_int32, [C.POINTER(Csr), C.POINTER(Params), C.POINTER(P), *E]),
        "scxpca_plan_run": (C.c_int32, [P, C.POINTER(Params), C.POINTER(Result), *E]),
        "scxpca_plan_destroy": (None, [P]),
        "scxpca_plan_create_affine": (C.c_int32, [C.POINTER(Csr), C.POINTER(Params), P, P, C.c_int32,
                                                  C.POINTER(P), *E]),
        "scxpca_plan_backward": (C.c_int32, [P, P, P, C.c_int32, P, P, P, *E]),
        "scxpca_batch_create": (C.c_int32, [C.POINTER(Csr), P, C.c_int64, C.POINTER(Params), C.c_int32,
                                            C.POINTER(P), *E]),
        "scxpca_batch_run": (C.c_int32, [P, C.c_int32, P, C.c_int32, P, P, P, P,
                                         C.POINTER(C.c_double), *E]),
        "scxpca_batch_info": (C.c_int32, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int64), P]),
        "scxpca_batch_destroy": (None, [P]),
        "scxpca_plan_info": (C.c_int32, [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int64)]),
        "scxpca_plan_matmat": (C.c_int32, [P, P, C.c_int64, P, C.c_int64, *E]),
        "scxpca_plan_rmatmat": (C.c_int32, [P, P, C.c_int64, P, C.c_int64, *E]),
        "scxpca_plan_qr": (C.c_int32, [P, P, C.c_int64, C.c_int64, *E]),
        "scxpca_plan_col_stats": (C.c_int32, [P, P, P, *E]),
        "scxpca_col_stats_noalloc": (C.c_int32, [C.c_int32, C.POINTER(Csr), P, P, *E]),
        "scxpca_plan_set_profiling": (C.c_int32, [P, C.c_int32]),
        "scxpca_plan_get_profile": (C.c_int32, [P, C.POINTER(Profile)]),
        "scxpca_gaussian": (C.c_int32, [C.c_int32, C.c_uint64, C.c_int64, C.c_int64, P, *E]),
        "scxpca_synth_nb_csr": (C.c_int32, [C.c_int32, C.c_uint64, C.c_int64, C.c_int64, C.c_double,
                                            C.c_double, P, P, P, C.POINTER(C.c_int64), *E]),
        "scxpca_wait_selftest": (C.c_int32, [C.c_int32, *E]),
        "scxpca_last_call_phases": (C.c_int32, [P, C.c_int32, C.POINTER(C.c_double)]),
        "scxpca_preprocess": (C.c_int32, [C.c_int32, C.POINTER(Csr), P, C.c_double, C.c_int32, P, P, *E]),
        "scxpca_project_columns": (C.c_int32, [C.c_int32, C.POINTER(Csr), P, C.c_int64, P, P, P,
                                               C.POINTER(C.c_int64), P, *E]),
        "scxpca_pflog_prepare": (C.c_int32, [C.c_int32, C.POINTER(Csr), C.c_double, P, P, P, *E]),
        "scxpca_pflog_pca": (C.c_int32, [C.POINTER(Csr), P, C.c_int32, C.POINTER(Params), C.POINTER(Result), *E]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class ScxPcaError(RuntimeError):
    """A non-OK status from the library (message kept verbatim)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int, err: C.Array) -> None:
    if status == OK:
        return
    msg = err.value.decode(errors="replace") or load().scxpca_status_string(status).decode()
    if status == INVALID_ARGUMENT:
        raise ValueError(msg)
    raise ScxPcaError(status, msg)


def errbuf() -> C.Array:
    return C.create_string_buffer(1024)
