"""Upstream producers on the device (needs a B200): normalize_total + log1p with
an optional per-row factor (scxpca_preprocess) and the mask_var column
projection (scxpca_project_columns), against the FP64 restatements in
oracle/rpca.py on the same raw counts.

Tolerances: values 1e-6 relative (the reference's own GPU-vs-CPU rtol for this
transform, scx-gpu/kernels/normalize_log1p.cu:10-15); the projection is integer
and byte work, so it is checked bit-exact; the PCA of the projected,
normalised matrix agrees with the oracle's PCA of the same pipeline to 1e-4 on
singular values (the strict-path parity bar).
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel

pytestmark = pytest.mark.gpu


def _raw_counts(n=3000, g=900, seed=0):
    rng = np.random.default_rng(seed)
    mu = rng.lognormal(-1.0, 1.5, g)
    size = rng.lognormal(0.0, 0.5, n)
    lam = np.outer(size, mu)
    counts = rng.negative_binomial(1 / 0.3, 1 / (1 + 0.3 * lam)).astype(np.float32)
    counts[7, :] = 0.0  # empty rows
    counts[11, :] = 0.0
    rr, cc = np.nonzero(counts)
    indptr = np.r_[0, np.cumsum(np.bincount(rr, minlength=n))].astype(np.int64)
    return rpca.Csr(indptr, cc.astype(np.int32), counts[rr, cc], (n, g))


def _dev(c):
    import torch
    return (torch.from_numpy(c.indptr).cuda(), torch.from_numpy(c.indices).cuda(),
            torch.from_numpy(np.ascontiguousarray(c.data, dtype=np.float32)).cuda())


@pytest.mark.parametrize("target_sum,log1p,factors", [(1e4, True, False), (1e4, False, False),
                                                      (None, True, False), (1e4, True, True)])
def test_normalize_log1p_matches_oracle(target_sum, log1p, factors):
    import torch

    c = _raw_counts()
    ip, ix, vv = _dev(c)
    rf = np.random.default_rng(1).uniform(0.5, 2.0, c.shape[0]).astype(np.float32) if factors else None
    got = accel.preprocess(ip, ix, vv, c.shape, target_sum=target_sum, log1p=log1p,
                           row_factors=None if rf is None else torch.from_numpy(rf).cuda())
    want = rpca.normalize_log1p(c, target_sum, log1p, rf)
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-6, atol=0)
    # the input is untouched out of place; in place gives the same values
    np.testing.assert_array_equal(vv.cpu().numpy(), c.data)
    same = accel.preprocess(ip, ix, vv, c.shape, target_sum=target_sum, log1p=log1p,
                            row_factors=None if rf is None else torch.from_numpy(rf).cuda(), inplace=True)
    assert same.data_ptr() == vv.data_ptr()
    np.testing.assert_array_equal(vv.cpu().numpy(), got.cpu().numpy())


def test_project_columns_bit_exact():
    c = _raw_counts(seed=2)
    cols = np.flatnonzero(np.random.default_rng(3).random(c.shape[1]) < 0.3)
    ip, ix, vv = _dev(c)
    pip, pix, pvv, shape = accel.project_columns(ip, ix, vv, c.shape, cols)
    want = rpca.project_columns(c, cols)
    assert shape == want.shape
    np.testing.assert_array_equal(pip.cpu().numpy(), want.indptr)
    np.testing.assert_array_equal(pix.cpu().numpy(), want.indices)
    np.testing.assert_array_equal(pvv.cpu().numpy(), want.data)


def test_project_columns_rejects_bad_selections():
    c = _raw_counts(n=200, g=50, seed=4)
    ip, ix, vv = _dev(c)
    with pytest.raises(ValueError, match="sorted and unique"):
        accel.project_columns(ip, ix, vv, c.shape, [3, 2])
    with pytest.raises(ValueError, match="out of range"):
        accel.project_columns(ip, ix, vv, c.shape, [0, 50])


def test_raw_counts_to_pca_on_device_matches_oracle():
    """Raw counts resident on the device -> HVG column projection ->
    normalize_total(1e4) + log1p -> randomized PCA on the borrowed device CSR,
    against the oracle's run of the same pipeline with the same Omega."""
    c = _raw_counts(n=4000, g=1200, seed=5)
    cols = np.flatnonzero(np.random.default_rng(6).random(c.shape[1]) < 0.5)
    ip, ix, vv = _dev(c)
    pip, pix, pvv, shape = accel.project_columns(ip, ix, vv, c.shape, cols)
    accel.preprocess(pip, pix, pvv, shape, target_sum=1e4, log1p=True, inplace=True)
    k = 30
    om = rpca.gaussian_omega(shape[1], k, seed=0)
    res = accel.randomized_pca(pip, pix, pvv, shape, n_components=20, n_oversamples=10, n_power_iterations=4,
                               omega=om, math_mode="strict_fp32")
    pc = rpca.project_columns(c, cols)
    oc = pc.with_values(rpca.normalize_log1p(pc, 1e4, True))
    ref = rpca.randomized_pca(oc, 20, 10, 4, True, om)
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < 1e-4, rel.max()
    assert rpca.principal_angles(res.components.T, ref["components"].T).max() < 1e-3
