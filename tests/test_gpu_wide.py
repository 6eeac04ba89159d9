"""Sketches wider than 128 columns (needs a B200).

The reference sizes the sketch k = min(n_comps + n_oversamples, n_vars,
n_obs) with no cap (scx-gpu/src/gpu_pca.rs:433-446).  Here 128 < k <= 256
runs as two 128-column panels: the CUDA-core SpMM pair takes one panel per
launch (row stride 256), and the dense side uses the panel-shaped Gram,
Cholesky, right-multiplication and eigensolver paths.

Parity bars: operator products within 1e-5 of numpy FP64 (relative to the
output norm, as the single-panel seam test); singular values within 1e-4 of
the FP64 oracle with the same Omega (BF16 values: the oracle on the
BF16-rounded values); principal angles of the leading components below 1e-3
rad where the spectrum is gapped; QR of a tall matrix orthonormal to 1e-5.
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu

OP_RTOL = 1e-5
SV_RTOL = 1e-4


def _csr(n, g, seed, loc=-2.0):
    ip, ix, vv = synth_nb_csr(n, g, seed=seed, loc=loc)
    return rpca.Csr(ip, ix, vv, (n, g))


@pytest.mark.parametrize("k", [160, 256])
def test_wide_operator_seam(k):
    import torch

    n, g = 3001, 700
    c = _csr(n, g, seed=k)
    plan = accel.Plan(c.indptr, c.indices, c.data, c.shape, n_components=k, n_oversamples=0,
                      math_mode="strict_fp32")
    assert plan.k == k and plan.ld == 256
    mu = rpca.col_sums_and_sum_sq(c)[0] / n
    rng = np.random.default_rng(7)
    v = rng.standard_normal((g, k)).astype(np.float32)
    y = plan.matmat(torch.from_numpy(v).cuda()).cpu().numpy().astype(np.float64)
    y_ref = rpca.spmm_forward(c, v.astype(np.float64), mu)
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < OP_RTOL
    # every column of both panels
    col = np.linalg.norm(y - y_ref, axis=0) / np.linalg.norm(y_ref, axis=0)
    assert col.max() < 1e-4
    q = rng.standard_normal((n, k)).astype(np.float32)
    z = plan.rmatmat(torch.from_numpy(q).cuda()).cpu().numpy()
    z_ref = rpca.spmm_transpose(c, q.astype(np.float64), mu)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) < OP_RTOL
    col = np.linalg.norm(z - z_ref, axis=0) / np.linalg.norm(z_ref, axis=0)
    assert col.max() < 1e-4
    # tall QR through the operator seam: orthonormal columns spanning A
    a = rng.standard_normal((n, k)).astype(np.float32) @ np.diag(np.logspace(0, 3, k)).astype(np.float32)
    qa = plan.qr(torch.from_numpy(a).cuda()).cpu().numpy().astype(np.float64)
    assert np.abs(qa.T @ qa - np.eye(k)).max() < 1e-5
    proj = qa @ (qa.T @ a.astype(np.float64))
    assert np.linalg.norm(proj - a) / np.linalg.norm(a) < 1e-5
    plan.close()


@pytest.mark.parametrize("mode,nc,os_", [("strict_fp32", 150, 10), ("mixed_bf16", 150, 10),
                                         ("strict_fp32", 240, 16)])
def test_wide_pca_matches_oracle(mode, nc, os_):
    n, g = 4000, 600
    c = _csr(n, g, seed=11)
    k = nc + os_
    om = rpca.gaussian_omega(g, k, seed=3)
    res = accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, n_components=nc, n_oversamples=os_,
                               n_power_iterations=4, omega=om, math_mode=mode)
    rounder = rpca.round_to_bf16 if mode == "mixed_bf16" else None
    ref = rpca.randomized_pca(c, nc, os_, 4, True, om, value_dtype=rounder)
    sv = np.asarray(ref["singular_values"])
    np.testing.assert_allclose(res.singular_values, sv, rtol=SV_RTOL)
    # leading components where the spectrum is gapped
    s = sv[:20]
    gapped = [i for i in range(19) if (s[i] - s[i + 1]) / s[i] > 1e-2 and (i == 0 or (s[i - 1] - s[i]) / s[i - 1] > 1e-2)]
    assert gapped, "no isolated leading component to compare"
    ang = rpca.principal_angles(np.asarray(res.components, np.float64)[gapped].T,
                                np.asarray(ref["components"], np.float64)[gapped].T)
    assert ang.max() < 1e-3
    ve = np.asarray(res.variance_ratio)
    np.testing.assert_allclose(ve, np.asarray(ref["variance_ratio"]), rtol=2e-4)
    assert res.embeddings.shape == (n, nc) and np.isfinite(res.embeddings).all()


def test_wide_householder_contract_on_rank_deficient_input():
    """Rank-deficient columns force the shifted factorisation; the wide
    Cholesky's restart keeps the run finite and its Q orthonormal."""
    n, g = 3000, 300
    c = _csr(n, g, seed=5)
    dense_cols = np.repeat(np.arange(n), np.diff(c.indptr))
    # genes 100..299 repeat genes 0..99: rank <= 100 < k = 160
    x = np.zeros((n, g), dtype=np.float32)
    x[dense_cols, c.indices] = c.data
    x[:, 100:200] = x[:, 0:100]
    x[:, 200:300] = 2.0 * x[:, 0:100]
    rr, cc = np.nonzero(x)
    ip = np.r_[0, np.cumsum(np.bincount(rr, minlength=n))]
    d = rpca.Csr(ip, cc.astype(np.int32), x[rr, cc], (n, g))
    res = accel.randomized_pca(d.indptr, d.indices, d.data, d.shape, n_components=150, n_oversamples=10,
                               n_power_iterations=2, qr_method="householder", math_mode="strict_fp32", seed=1)
    assert np.isfinite(res.singular_values).all()
    assert np.isfinite(res.embeddings).all()
    full = np.linalg.svd(x - x.mean(0), compute_uv=False)
    np.testing.assert_allclose(res.singular_values[:10], full[:10], rtol=1e-3)
