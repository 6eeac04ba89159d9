"""Build libscxpca.so (sm_100a) in-tree: scx_b200/libscxpca.so.

Usage: python -m scx_b200.csrc.build [--force] [--jobs N]

Each .cu translation unit is compiled by nvcc to an object under
scx_b200/csrc/_build/ (parallel), then linked into one shared library with
cudart and libcuda.  Objects are rebuilt when their source or any header in
this directory is newer.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
BUILD = HERE / "_build"
LIB = PKG / "libscxpca.so"

SOURCES = [
    "scxpca.cu",
    "kernels_sparse.cu",
    "kernels_dense.cu",
    "kernels_csr.cu",
    "synth.cu",
    "kernels_adjoint.cu",
    "noalloc.cu",
    "kernels_strict.cu",
    "kernels_preprocess.cu",
    "kernels_wide.cu",
]
EXTRA_SOURCES_OPTIONAL = ["kernels_tc.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libscxpca.so")
    return cand


def _headers_mtime() -> float:
    hs = list(HERE.glob("*.cuh")) + list(HERE.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, verbose: bool) -> str:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return res.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = [HERE / s for s in SOURCES] + [HERE / s for s in EXTRA_SOURCES_OPTIONAL if (HERE / s).exists()]
    hdr_t = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr_t):
            todo.append((s, o))
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            futs = [ex.submit(_compile, s, o, verbose) for s, o in todo]
            for f in futs:
                logs.append(f.result())
    if force or todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        for log in logs:
            sys.stderr.write(log)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.verbose))
