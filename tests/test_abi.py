"""The C ABI library loads, exports every symbol include/scxpca.h declares,
and rejects bad arguments before touching a device.  CPU only: no compute
call reaches a GPU here."""

import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from scx_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "scxpca.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(scxpca_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), f"{n} declared in scxpca.h but not exported"
    assert sorted(_lib.EXPORTED) == names


def test_abi_version_and_status_strings():
    lib = _lib.load()
    assert lib.scxpca_abi_version() == 2
    assert lib.scxpca_status_string(_lib.NOT_SPD) == b"not SPD"
    assert lib.scxpca_status_string(999) == b"unknown status"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "scxpca.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(scxpca_csr), sizeof(scxpca_params),"
        " sizeof(scxpca_result), offsetof(scxpca_params, stream), offsetof(scxpca_result, total_var),"
        " offsetof(scxpca_params, omega));return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(_lib.Csr), C.sizeof(_lib.Params), C.sizeof(_lib.Result),
            _lib.Params.stream.offset, _lib.Result.total_var.offset, _lib.Params.omega.offset]
    assert got == want


def _call(n_obs=4, n_vars=3, nc=2, over=1, dtype=_lib.F32, math=0, qr=0, clip=0.0):
    lib = _lib.load()
    indptr = np.array([0, 1, 2, 3, 3][: n_obs + 1] + [3] * max(0, n_obs + 1 - 5), dtype=np.int64)
    idx = np.array([0, 1, 2], dtype=np.int32)
    val = np.ones(3, dtype=np.float32)
    csr = _lib.Csr(n_obs, n_vars, 3, indptr.ctypes.data, idx.ctypes.data, val.ctypes.data, dtype,
                   _lib.MEM_HOST)
    p = _lib.Params()
    p.n_components, p.n_oversamples, p.n_power_iterations = nc, over, 2
    p.zero_center, p.math_mode, p.qr_method, p.clip_max = 1, math, qr, clip
    emb = np.zeros((max(n_obs, 1), max(nc, 1)), dtype=np.float32)
    res = _lib.Result()
    res.embeddings = emb.ctypes.data
    err = _lib.errbuf()
    st = lib.scxpca_randomized(C.byref(csr), C.byref(p), C.byref(res), err, len(err))
    return st, err.value.decode()


@pytest.mark.parametrize(
    "kw,status,msg",
    [
        (dict(nc=0), _lib.INVALID_ARGUMENT, "n_components must be > 0"),
        (dict(nc=4), _lib.INVALID_ARGUMENT, "exceeds matrix rank bound"),
        (dict(n_obs=0), _lib.INVALID_ARGUMENT, "non-empty"),
        (dict(dtype=7), _lib.INVALID_ARGUMENT, "values_dtype"),
        (dict(math=9), _lib.INVALID_ARGUMENT, "math_mode"),
        (dict(qr=5), _lib.INVALID_ARGUMENT, "qr_method"),
        (dict(clip=float("inf")), _lib.INVALID_ARGUMENT, "clip_max"),
    ],
)
def test_argument_validation_statuses(kw, status, msg):
    st, err = _call(**kw)
    assert st == status
    assert msg in err


def test_sketch_width_limit_is_reported():
    """k = min(n_components + n_oversamples, n_vars, n_obs) up to 256 is taken
    (two 128-column panels); a wider sketch is reported before any device work."""
    lib = _lib.load()
    n, g = 400, 400
    indptr = np.zeros(n + 1, dtype=np.int64)
    csr = _lib.Csr(n, g, 0, indptr.ctypes.data, None, None, 0, 0)
    p = _lib.Params()
    p.n_components, p.n_oversamples = 250, 10
    emb = np.zeros((n, 250), dtype=np.float32)
    res = _lib.Result()
    res.embeddings = emb.ctypes.data
    err = _lib.errbuf()
    st = lib.scxpca_randomized(C.byref(csr), C.byref(p), C.byref(res), err, len(err))
    assert st == _lib.UNSUPPORTED and "256" in err.value.decode()


def test_python_layer_maps_statuses():
    with pytest.raises(ValueError, match="n_components must be > 0"):
        _lib.check(_lib.INVALID_ARGUMENT, C.create_string_buffer(b"n_components must be > 0"))
    with pytest.raises(_lib.ScxPcaError, match="non-SPD"):
        _lib.check(_lib.NOT_SPD, C.create_string_buffer(b"CholeskyQR2 failed: non-SPD"))


def test_new_entry_points_reject_bad_arguments_without_a_device():
    """Null handles and contradictory arguments of the affine, backward and
    batch entry points return INVALID_ARGUMENT before any device call."""
    lib = _lib.load()
    err = _lib.errbuf()
    assert lib.scxpca_plan_backward(None, None, None, 8, None, None, None, err, len(err)) == _lib.INVALID_ARGUMENT
    assert lib.scxpca_batch_run(None, 1, None, 0, None, None, None, None, None, err, len(err)) == _lib.INVALID_ARGUMENT
    assert lib.scxpca_batch_info(None, None, None, None) == _lib.INVALID_ARGUMENT
    lib.scxpca_batch_destroy(None)  # no-op
    indptr = np.array([0, 1, 2, 3], dtype=np.int64)
    idx = np.array([0, 1, 2], dtype=np.int32)
    val = np.ones(3, dtype=np.float32)
    csr = _lib.Csr(3, 3, 3, indptr.ctypes.data, idx.ctypes.data, val.ctypes.data, _lib.F32, _lib.MEM_HOST)
    p = _lib.Params()
    p.n_components, p.n_oversamples, p.scale = 1, 1, 1
    h = C.c_void_p()
    st = lib.scxpca_plan_create_affine(C.byref(csr), C.byref(p), None, None, _lib.MEM_HOST, C.byref(h), err,
                                       len(err))
    assert st == _lib.INVALID_ARGUMENT and b"replace params.scale" in err.value
    p.scale = 0
    st = lib.scxpca_plan_create_affine(C.byref(csr), C.byref(p), None, None, 9, C.byref(h), err, len(err))
    assert st == _lib.INVALID_ARGUMENT and b"vectors_memory" in err.value
    offs = np.array([0, 3], dtype=np.int64)
    st = lib.scxpca_batch_create(C.byref(csr), offs.ctypes.data, 1, C.byref(p), 99, C.byref(h), err, len(err))
    assert st != _lib.OK  # bad branch count (or no device here): never a crash
