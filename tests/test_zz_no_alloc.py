"""scxpca_col_stats_noalloc: per-gene column statistics that allocate nothing.

The entry point exists for callers that cannot let a library call cudaMalloc
(a process whose device memory belongs to a caching pool such as PyTorch's or
RMM's, or a pipeline where cudaMalloc/cudaFree would synchronise the device
between its streams).  Its scratch is a static device array shared by every
call, so the GPU test runs it twice in a row on different matrices and
compares each result with the allocating entry point, scxpca_plan_col_stats,
on an unscaled FP32 plan of the same device CSR.

This file is named to be collected last, so that a run which stops at the
first failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

from scx_b200 import _lib

# FP64 sums over the same values in a different block partition: agreement to
# a few ulps of the column's sum of magnitudes.
RTOL = 1e-12


def _csr(indptr, indices, values, shape, memory=_lib.MEM_DEVICE, dtype=_lib.F32):
    return _lib.Csr(int(shape[0]), int(shape[1]), int(indices.numel() if hasattr(indices, "numel")
                                                      else len(indices)),
                    indptr.data_ptr(), indices.data_ptr(), values.data_ptr(), dtype, memory)


def test_noalloc_rejects_too_many_genes_before_touching_a_device():
    lib = _lib.load()
    err = _lib.errbuf()
    x = _lib.Csr(10, _lib.NOALLOC_MAX_VARS + 1, 0, 1, 0, 0, _lib.F32, _lib.MEM_DEVICE)
    st = lib.scxpca_col_stats_noalloc(0, C.byref(x), C.c_void_p(8), None, err, len(err))
    assert st == _lib.INVALID_ARGUMENT
    assert b"exceeds the no-allocation maximum" in err.value
    x = _lib.Csr(10, 20, 0, 1, 0, 0, _lib.F32, _lib.MEM_HOST)
    st = lib.scxpca_col_stats_noalloc(0, C.byref(x), C.c_void_p(8), None, err, len(err))
    assert st == _lib.INVALID_ARGUMENT
    assert b"device CSR" in err.value


@pytest.mark.gpu
def test_noalloc_col_stats_match_plan_col_stats_on_two_calls():
    import torch

    from scx_b200 import accel

    lib = _lib.load()
    torch.cuda.init()
    # the wider matrix first, so the second call runs over the first call's
    # leftover scratch contents
    cases = [(5000, 2000, 12), (3000, 700, 11)]
    mats, wants = [], []
    for n, g, seed in cases:
        ip, ix, vv = accel.synth_nb_csr_device(n, g, seed=seed, loc=-2.0)
        torch.cuda.synchronize()
        plan = accel.Plan(ip, ix, vv, (n, g), n_components=5, n_oversamples=5, zero_center=True,
                          scale=False, math_mode="strict_fp32")
        try:
            wants.append(plan.col_stats())
        finally:
            plan.close()
        mats.append((ip, ix, vv, (n, g)))
    outs = []
    for ip, ix, vv, shape in mats:  # two calls in a row
        out = torch.full((2 * shape[1],), float("nan"), dtype=torch.float64, device="cuda:0")
        x = _csr(ip, ix, vv, shape)
        err = _lib.errbuf()
        st = lib.scxpca_col_stats_noalloc(0, C.byref(x), C.c_void_p(out.data_ptr()), None, err, len(err))
        _lib.check(st, err)
        outs.append(out)
    for (ip, ix, vv, (n, g)), (want_s, want_q), out in zip(mats, wants, outs):
        got = out.cpu().numpy()
        scale_s = np.abs(want_s).max()
        scale_q = np.abs(want_q).max()
        np.testing.assert_allclose(got[:g], want_s, rtol=RTOL, atol=RTOL * scale_s)
        np.testing.assert_allclose(got[g:], want_q, rtol=RTOL, atol=RTOL * scale_q)
        # the same sums straight from the CSR values, in FP64 on the host
        idx = ix.cpu().numpy()
        val = vv.cpu().numpy().astype(np.float64)
        np.testing.assert_allclose(got[:g], np.bincount(idx, weights=val, minlength=g), rtol=1e-10,
                                   atol=1e-10 * scale_s)
        np.testing.assert_allclose(got[g:], np.bincount(idx, weights=val * val, minlength=g), rtol=1e-10,
                                   atol=1e-10 * scale_q)


@pytest.mark.gpu
def test_noalloc_at_the_gene_limit():
    """n_vars == NOALLOC_MAX_VARS: the widest matrix the static scratch serves
    (the fewest per-block partials, and more genes than one shared-memory
    accumulator pass holds).  Checked against the allocating entry point and
    against FP64 sums on the host, on two calls in a row."""
    import torch

    from scx_b200 import accel

    lib = _lib.load()
    torch.cuda.init()
    n, g = 2000, _lib.NOALLOC_MAX_VARS
    ip, ix, vv = accel.synth_nb_csr_device(n, g, seed=21, loc=-1.5)
    torch.cuda.synchronize()
    plan = accel.Plan(ip, ix, vv, (n, g), n_components=5, n_oversamples=5, zero_center=True, scale=False,
                      math_mode="strict_fp32")
    try:
        want_s, want_q = plan.col_stats()
    finally:
        plan.close()
    idx = ix.cpu().numpy()
    val = vv.cpu().numpy().astype(np.float64)
    host_s = np.bincount(idx, weights=val, minlength=g)
    host_q = np.bincount(idx, weights=val * val, minlength=g)
    for _ in range(2):
        out = torch.full((2 * g,), float("nan"), dtype=torch.float64, device="cuda:0")
        x = _csr(ip, ix, vv, (n, g))
        err = _lib.errbuf()
        st = lib.scxpca_col_stats_noalloc(0, C.byref(x), C.c_void_p(out.data_ptr()), None, err, len(err))
        _lib.check(st, err)
        got = out.cpu().numpy()
        # the same kernel over a different block partition (fewer partials)
        np.testing.assert_allclose(got[:g], want_s, rtol=RTOL, atol=RTOL * np.abs(want_s).max())
        np.testing.assert_allclose(got[g:], want_q, rtol=RTOL, atol=RTOL * np.abs(want_q).max())
        np.testing.assert_allclose(got[:g], host_s, rtol=1e-10, atol=1e-10 * np.abs(host_s).max())
        np.testing.assert_allclose(got[g:], host_q, rtol=1e-10, atol=1e-10 * np.abs(host_q).max())


@pytest.mark.gpu
def test_noalloc_reports_invalid_csr():
    import torch

    lib = _lib.load()
    ip = torch.tensor([0, 2, 3], dtype=torch.int64, device="cuda:0")
    ix = torch.tensor([0, 7, 1], dtype=torch.int32, device="cuda:0")  # 7 >= n_vars
    vv = torch.ones(3, dtype=torch.float32, device="cuda:0")
    out = torch.zeros(2 * 4, dtype=torch.float64, device="cuda:0")
    x = _csr(ip, ix, vv, (2, 4))
    err = _lib.errbuf()
    st = lib.scxpca_col_stats_noalloc(0, C.byref(x), C.c_void_p(out.data_ptr()), None, err, len(err))
    assert st == _lib.INVALID_CSR
    assert b"column index out of range" in err.value
