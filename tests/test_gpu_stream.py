"""Streamed plans (needs a B200): a host matrix whose resident plan does not
fit the device budget stays in host memory and every product takes it in row
shards (the reference's StreamingPcaOperator, scx-gpu/src/linear_operator.rs:
61-288; resident vs streaming decision gpu_pca.rs:520-590).

A streamed run computes the same products as the resident one, shard by shard;
only the order in which the transposed product's partial sums are added
differs, so singular values agree to 1e-6 relative and components to 1e-4 rad.
The operator seam of a streamed plan is checked against the FP64 oracle.
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu

BUDGET = 150 << 20  # bytes: forces several shards for the 40,000-cell matrix


def _host(n=40000, g=2000, seed=0, loc=-2.5):
    ip, ix, vv = synth_nb_csr(n, g, seed=seed, loc=loc)
    return ip, ix, vv, (n, g)


@pytest.mark.parametrize("mode", ["strict_fp32", "mixed_bf16"])
def test_streamed_pca_equals_resident(mode):
    ip, ix, vv, shape = _host()
    kw = dict(n_components=30, n_oversamples=10, n_power_iterations=3, zero_center=True, scale=True,
              clip_max=10.0, seed=3, qr_method="cholesky", math_mode=mode)
    res = accel.randomized_pca(ip, ix, vv, shape, **kw)
    st = accel.randomized_pca(ip, ix, vv, shape, device_budget=BUDGET, **kw)
    assert res.resident_csr and res.n_shards == 0
    assert not st.resident_csr and st.n_shards >= 2, st.n_shards
    np.testing.assert_allclose(st.singular_values, res.singular_values, rtol=1e-6)
    assert rpca.principal_angles(st.components.T, res.components.T).max() < 1e-4
    np.testing.assert_allclose(st.total_var, res.total_var, rtol=1e-12)
    np.testing.assert_allclose(st.mean, res.mean, rtol=1e-12)
    np.testing.assert_allclose(st.std, res.std, rtol=1e-12)


def test_streaming_forced_by_environment_and_unsorted_rows(monkeypatch):
    """SCXPCA_RESIDENT=0 streams even what would fit; a matrix with unsorted
    rows is sorted shard by shard after every upload."""
    ip, ix, vv, shape = _host(n=6000, g=700, seed=1, loc=-2.0)
    rng = np.random.default_rng(2)
    ix2, vv2 = ix.copy(), vv.copy()
    for r in rng.choice(shape[0], 50, replace=False):  # shuffle some rows
        s, e = ip[r], ip[r + 1]
        perm = rng.permutation(e - s)
        ix2[s:e] = ix2[s:e][perm]
        vv2[s:e] = vv2[s:e][perm]
    kw = dict(n_components=20, n_oversamples=10, n_power_iterations=2, seed=5, math_mode="strict_fp32")
    res = accel.randomized_pca(ip, ix, vv, shape, **kw)
    monkeypatch.setenv("SCXPCA_RESIDENT", "0")
    st = accel.randomized_pca(ip, ix2, vv2, shape, **kw)
    assert not st.resident_csr and st.n_shards >= 1
    np.testing.assert_allclose(st.singular_values, res.singular_values, rtol=1e-6)


@pytest.mark.parametrize("mode,rounder,tol", [("strict_fp32", None, 1e-5),
                                              ("mixed_bf16", rpca.round_to_bf16, 1e-4)])
def test_streamed_operator_seam_matches_oracle(mode, rounder, tol):
    import torch

    ip, ix, vv, shape = _host()
    c = rpca.Csr(ip, ix, vv, shape)
    plan = accel.Plan(ip, ix, vv, shape, n_components=60, n_oversamples=0, math_mode=mode,
                      device_budget=BUDGET)
    cr = c if rounder is None else c.with_values(rounder(c.data))
    mu = rpca.col_sums_and_sum_sq(cr)[0] / shape[0]
    rng = np.random.default_rng(1)
    v = (rng.standard_normal((shape[1], 60)) / np.sqrt(shape[1])).astype(np.float32)
    y = plan.matmat(torch.from_numpy(v).cuda()).cpu().numpy().astype(np.float64)
    y_ref = rpca.spmm_forward(cr, v.astype(np.float64), mu)
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < tol
    q = (rng.standard_normal((shape[0], 60)) / np.sqrt(shape[0])).astype(np.float32)
    z = plan.rmatmat(torch.from_numpy(q).cuda()).cpu().numpy()
    z_ref = rpca.spmm_transpose(cr, q.astype(np.float64), mu)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) < tol
    s, sq = plan.col_stats()
    s_ref, sq_ref = rpca.col_sums_and_sum_sq(cr)
    np.testing.assert_allclose(s, s_ref, rtol=1e-10, atol=1e-10 * np.abs(s_ref).max())
    plan.close()
