"""Build and load the C++ CPU restatement (oracle/_build/librpca_cpu.so).

Test and baseline infrastructure only: the product never imports this.
"""

from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "rpca_cpu.cpp"
OUT = HERE / "_build" / "librpca_cpu.so"


def build(force: bool = False) -> Path:
    OUT.parent.mkdir(exist_ok=True)
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        raise RuntimeError("no C++ compiler to build the CPU baseline")
    subprocess.run([cxx, "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-shared", "-pthread",
                    str(SRC), "-o", str(OUT)], check=True)
    return OUT


_lib = None


def load():
    global _lib
    if _lib is None:
        if not OUT.exists():
            build()
        lib = C.CDLL(str(OUT))
        P = C.c_void_p
        lib.rpca_cpu_run.restype = C.c_int
        lib.rpca_cpu_run.argtypes = [C.c_int64, C.c_int64, P, P, P, C.c_int64, C.c_int64, C.c_int64,
                                     C.c_int, C.c_int, C.c_double, P, C.c_int, P, P, P, P]
        _lib = lib
    return _lib


def run(indptr, indices, values, shape, n_components, k, n_power_iterations, omega,
        zero_center=True, scale=False, clip_max=0.0, threads=1, want_embeddings=False):
    """Run the C++ FP64 randomized PCA; returns dict(singular_values, components, ...)."""
    lib = load()
    n, g = shape
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    values = np.ascontiguousarray(values, dtype=np.float32)
    om = np.ascontiguousarray(omega, dtype=np.float64)
    sigma = np.zeros(n_components)
    comps = np.zeros((n_components, g))
    emb = np.zeros((n, n_components), dtype=np.float32) if want_embeddings else None
    tv = C.c_double()
    st = lib.rpca_cpu_run(n, g, indptr.ctypes.data, indices.ctypes.data, values.ctypes.data,
                          n_components, k, n_power_iterations, int(zero_center), int(scale),
                          float(clip_max or 0.0), om.ctypes.data, threads, sigma.ctypes.data,
                          comps.ctypes.data, emb.ctypes.data if emb is not None else None,
                          C.byref(tv))
    if st != 0:
        raise RuntimeError(f"rpca_cpu_run failed with status {st}")
    return {"singular_values": sigma, "components": comps, "embeddings": emb,
            "total_var": tv.value}
