"""PFlog (v4) baseline-aware PCA on the device (needs a B200) against the FP64
restatement of pflog_pca (oracle/rpca.py; scx-accel/src/pca/cpu.rs:618-882,
scx-accel/src/pflog.rs:122-193) on the same raw counts and Omega.

Tolerances: delta and baseline 1e-6 relative (FP32 storage of delta; FP64
baseline); singular values 1e-4 relative and principal angles 1e-3 rad (the
strict-path parity bar); total variance 1e-6 relative; BF16 mode 1e-4 against
the oracle fed the same BF16-rounded working values (delta and baseline).
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel

pytestmark = pytest.mark.gpu

ALPHA = 0.3


def _raw(n=5000, g=800, seed=0):
    rng = np.random.default_rng(seed)
    mu = rng.lognormal(-1.5, 1.5, g)
    size = rng.lognormal(0.0, 0.5, n)
    lam = np.outer(size, mu)
    counts = rng.negative_binomial(1 / ALPHA, 1 / (1 + ALPHA * lam)).astype(np.float32)
    counts[3] = 0.0  # an empty cell: baseline 0
    rr, cc = np.nonzero(counts)
    ip = np.r_[0, np.cumsum(np.bincount(rr, minlength=n))].astype(np.int64)
    return rpca.Csr(ip, cc.astype(np.int32), counts[rr, cc], (n, g))


def _dev(c):
    import torch
    return (torch.from_numpy(c.indptr).cuda(), torch.from_numpy(c.indices).cuda(),
            torch.from_numpy(np.ascontiguousarray(c.data, dtype=np.float32)).cuda())


def test_pflog_prepare_matches_oracle():
    c = _raw()
    delta, base = accel.pflog_prepare(*_dev(c), c.shape, ALPHA)
    d_ref, b_ref = rpca.pflog_prepare(c, 4 * ALPHA)
    np.testing.assert_allclose(delta.cpu().numpy(), d_ref, rtol=1e-6)
    np.testing.assert_allclose(base.cpu().numpy(), b_ref, rtol=1e-10, atol=1e-12)
    assert base[3].item() == 0.0


def test_pflog_prepare_rejects_negative_and_non_finite_counts():
    c = _raw(n=200, g=50, seed=1)
    ip, ix, vv = _dev(c)
    bad = vv.clone()
    bad[5] = -1.0
    with pytest.raises(ValueError, match="negative count"):
        accel.pflog_prepare(ip, ix, bad, c.shape, ALPHA)
    bad = vv.clone()
    bad[7] = float("nan")
    with pytest.raises(ValueError, match="non-finite"):
        accel.pflog_prepare(ip, ix, bad, c.shape, ALPHA)


@pytest.mark.parametrize("zero_center", [True, False])
def test_pflog_pca_matches_oracle(zero_center):
    c = _raw(seed=2)
    k = 30
    om = rpca.gaussian_omega(c.shape[1], k, seed=0)
    res, base = accel.pflog_pca(*_dev(c), c.shape, ALPHA, n_components=20, n_oversamples=10,
                                n_power_iterations=4, zero_center=zero_center, omega=om)
    d_ref, b_ref = rpca.pflog_prepare(c, 4 * ALPHA)
    ref = rpca.pflog_pca(c.with_values(d_ref), b_ref, 20, 10, 4, zero_center, om)
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < 1e-4, rel.max()
    assert rpca.principal_angles(res.components.T, ref["components"].T).max() < 1e-3
    # closed forms: the oracle's S_dd - D B2 - n sum mu^2 assumes the baseline of
    # the FP64 delta; the library's general form takes the row sums of the
    # FP32-stored delta (sum_i b_i r_i), a 1e-7-relative difference
    np.testing.assert_allclose(res.total_var, ref["total_var"], rtol=1e-6)
    np.testing.assert_allclose(res.variance_ratio, ref["variance_ratio"], rtol=2e-4)
    if zero_center:  # the centring's mean baseline comes from the FP32-stored baseline column
        np.testing.assert_allclose(res.mean, ref["mean"], rtol=1e-6, atol=1e-9)
    assert res.components.shape == (20, c.shape[1])


def test_pflog_pca_mixed_bf16_matches_oracle_on_rounded_values():
    c = _raw(seed=3)
    k = 30
    om = rpca.gaussian_omega(c.shape[1], k, seed=0)
    res, _ = accel.pflog_pca(*_dev(c), c.shape, ALPHA, n_components=20, n_oversamples=10, n_power_iterations=4,
                             omega=om, math_mode="mixed_bf16")
    d_ref, b_ref = rpca.pflog_prepare(c, 4 * ALPHA)
    # the working values the tensor cores see: delta and the baseline column in BF16
    ref = rpca.pflog_pca(c.with_values(rpca.round_to_bf16(d_ref)), rpca.round_to_bf16(b_ref), 20, 10, 4, True, om)
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < 1e-4, rel.max()
