"""CUDA path vs the FP64 oracle on the same seeded inputs (needs a B200).

Tolerances (stated per test): strict FP32 path vs FP64 oracle with the same
explicit Omega -- 1e-4 relative on singular values, 1e-3 rad on principal
angles of the sign-fixed components; operator-level products 1e-5 relative
to the output norm.  Mirrors scx's GPU tests: QR orthonormality at 1e-4
(scx-gpu/src/cusolver.rs:426-465), the non-SPD contract
(pyscx/tests/test_accel_pca_gpu.py:247-287), variance_ratio sanity
(scx-gpu/src/gpu_pca.rs:1176-1311), planted-cluster CPU/GPU parity
(test_accel_pca_gpu.py:128-202), Cholesky vs Householder (:210-239).
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel
from scx_b200.synth import LOC_8PCT, synth_nb_csr

pytestmark = pytest.mark.gpu

SIGMA_RTOL = 1e-4
ANGLE_TOL = 1e-3


@pytest.fixture(scope="module")
def cfg10k():
    """10,000 cells x 2,000 genes, ~8 % density (the CPU-runnable workload)."""
    n, g = 10_000, 2_000
    indptr, idx, val = synth_nb_csr(n, g, seed=0, loc=LOC_8PCT)
    return rpca.Csr(indptr, idx, val, (n, g))


@pytest.fixture(scope="module")
def oracle10k(cfg10k):
    n, g = cfg10k.shape
    k = 60
    om = rpca.gaussian_omega(g, k, seed=0)
    res = rpca.randomized_pca(cfg10k, 50, 10, 4, True, om)
    return om, res


def _angles(a_comps, b_comps):
    return rpca.principal_angles(np.asarray(a_comps, np.float64).T, np.asarray(b_comps, np.float64).T)


def _run(c, **kw):
    return accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, **kw)


def test_strict_fp32_matches_oracle_10k(cfg10k, oracle10k):
    om, ref = oracle10k
    res = _run(cfg10k, n_components=50, n_oversamples=10, n_power_iterations=4, omega=om,
               qr_method="cholesky")
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < SIGMA_RTOL, rel.max()
    assert _angles(res.components, ref["components"]).max() < ANGLE_TOL
    # sign-fixed component-wise angles on well-separated components
    a, ea = rpca.sign_fix(res.components, res.embeddings)
    b, eb = rpca.sign_fix(ref["components"], ref["embeddings"])
    sv = ref["singular_values"]
    gaps = np.minimum(np.r_[np.inf, -np.diff(sv)], np.r_[-np.diff(sv), np.inf]) / sv
    sep = gaps > 1e-2
    pc = rpca.per_component_angles(a.T, b.T)
    assert pc[sep].max() < ANGLE_TOL, pc[sep].max()
    np.testing.assert_allclose(res.variance_ratio, ref["variance_ratio"], rtol=2e-4)
    np.testing.assert_allclose(res.total_var, ref["total_var"], rtol=1e-10)
    np.testing.assert_allclose(res.mean, ref["mean"], rtol=1e-10, atol=1e-12)
    # embeddings: sign-fixed, relative to the column norm
    err = np.linalg.norm(ea[:, sep] - eb[:, sep], axis=0) / np.linalg.norm(eb[:, sep], axis=0)
    assert err.max() < 5e-3


def test_householder_mode_matches_cholesky_mode(cfg10k, oracle10k):
    om, ref = oracle10k
    a = _run(cfg10k, n_components=50, n_oversamples=10, n_power_iterations=4, omega=om,
             qr_method="householder")
    b = _run(cfg10k, n_components=50, n_oversamples=10, n_power_iterations=4, omega=om,
             qr_method="cholesky")
    np.testing.assert_allclose(a.singular_values, b.singular_values, rtol=1e-6)
    assert a.shifted_cholesky == 0


def test_variance_ratio_sanity(cfg10k, oracle10k):
    om, _ = oracle10k
    res = _run(cfg10k, n_components=50, n_oversamples=10, n_power_iterations=2, omega=om)
    vr = res.variance_ratio
    assert (vr >= 0).all() and (np.diff(vr) <= 1e-12).all() and vr.sum() <= 1 + 1e-3


def test_10x5_fixture_exact(csr_10x5, fixtures):
    res = _run(csr_10x5, n_components=3, n_oversamples=5, n_power_iterations=2, seed=42)
    exact = fixtures["csr_10x5"]["exact"]["centered"]
    np.testing.assert_allclose(res.singular_values, exact["singular_values"][:3], rtol=1e-5)
    np.testing.assert_allclose(res.components @ res.components.T, np.eye(3), atol=1e-5)
    res = _run(csr_10x5, n_components=2, n_oversamples=5, n_power_iterations=2, seed=42,
               zero_center=False)
    exact = fixtures["csr_10x5"]["exact"]["uncentered"]
    np.testing.assert_allclose(res.singular_values, exact["singular_values"][:2], rtol=1e-5)
    assert res.mean is None


def test_seeded_omega_matches_oracle_generator():
    import torch

    dev = accel.gaussian(2000, 60, seed=1234)
    host = rpca.gaussian_omega(2000, 60, seed=1234)
    np.testing.assert_allclose(dev.cpu().numpy(), host, rtol=0, atol=1e-6)
    # and the PCA seeded run equals the explicit-omega run with the same matrix
    torch.cuda.synchronize()


def test_seed_equals_explicit_omega(cfg10k):
    om = rpca.gaussian_omega(2000, 30, seed=9)
    a = _run(cfg10k, n_components=20, n_oversamples=10, n_power_iterations=2, seed=9)
    b = _run(cfg10k, n_components=20, n_oversamples=10, n_power_iterations=2, omega=om)
    np.testing.assert_allclose(a.singular_values, b.singular_values, rtol=1e-6)


def test_operator_seam_matches_oracle(cfg10k):
    import torch

    n, g = cfg10k.shape
    plan = accel.Plan(cfg10k.indptr, cfg10k.indices, cfg10k.data, cfg10k.shape, n_components=50,
                      n_oversamples=10)
    k = plan.k
    mu = cfg10k.to_dense().mean(0) if False else rpca.col_sums_and_sum_sq(cfg10k)[0] / n
    v = np.random.default_rng(1).standard_normal((g, k)).astype(np.float32)
    y = plan.matmat(torch.from_numpy(v).cuda()).cpu().numpy()
    y_ref = rpca.spmm_forward(cfg10k, v.astype(np.float64), mu)
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < 1e-5
    q = np.random.default_rng(2).standard_normal((n, k)).astype(np.float32)
    z = plan.rmatmat(torch.from_numpy(q).cuda()).cpu().numpy()
    z_ref = rpca.spmm_transpose(cfg10k, q.astype(np.float64), mu)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) < 1e-5
    a = torch.from_numpy(q).cuda()
    plan.qr(a)
    qa = a.cpu().numpy().astype(np.float64)
    np.testing.assert_allclose(qa.T @ qa, np.eye(k), atol=1e-4)
    assert rpca.principal_angles(qa, q).max() < 1e-3
    s, sq = plan.col_stats()
    s_ref, sq_ref = rpca.col_sums_and_sum_sq(cfg10k)
    np.testing.assert_allclose(s, s_ref, rtol=1e-12)
    np.testing.assert_allclose(sq, sq_ref, rtol=1e-12)
    plan.close()


def _rank5(n=1000, g=900, rank=5):
    rng = np.random.default_rng(7)
    u = rng.standard_normal((n, rank)).astype(np.float32)
    v = rng.standard_normal((g, rank)).astype(np.float32)
    dense = (u @ v.T).astype(np.float32)
    rows, cols = np.nonzero(dense)
    indptr = np.r_[0, np.cumsum(np.bincount(rows, minlength=n))]
    return rpca.Csr(indptr, cols, dense[rows, cols], (n, g)), dense


def test_cholesky_rank_deficient_raises_non_spd():
    c, _ = _rank5()
    with pytest.raises(RuntimeError, match="non-SPD"):
        _run(c, n_components=20, n_oversamples=10, n_power_iterations=2, seed=42, qr_method="cholesky")


def test_householder_rank_deficient_succeeds():
    c, dense = _rank5()
    res = _run(c, n_components=20, n_oversamples=10, n_power_iterations=2, seed=42,
               qr_method="householder")
    ex = rpca.dense_pca(dense, 5)
    np.testing.assert_allclose(res.singular_values[:5], ex["singular_values"], rtol=1e-4)
    assert res.shifted_cholesky > 0
    assert np.isfinite(res.embeddings).all()


@pytest.mark.parametrize("center", [True, False])
def test_scaled_clipped_matches_oracle(center):
    n, g = 4000, 500
    indptr, idx, val = synth_nb_csr(n, g, seed=4, loc=-2.0)
    c = rpca.Csr(indptr, idx, val, (n, g))
    om = rpca.gaussian_omega(g, 40, seed=3)
    ref = rpca.randomized_pca(c, 30, 10, 4, center, om, scale=True, clip_max=10.0)
    res = _run(c, n_components=30, n_oversamples=10, n_power_iterations=4, omega=om,
               zero_center=center, scale=True, clip_max=10.0)
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < SIGMA_RTOL
    assert _angles(res.components, ref["components"]).max() < ANGLE_TOL
    np.testing.assert_allclose(res.std, ref["std"], rtol=1e-10)
    np.testing.assert_allclose(res.total_var, ref["total_var"], rtol=1e-6)


@pytest.mark.parametrize("mode,rounder", [("mixed_bf16", rpca.round_to_bf16),
                                          ("mixed_f16", rpca.round_to_f16)])
def test_mixed_precision_matches_oracle_on_rounded_values(cfg10k, oracle10k, mode, rounder):
    om, exact = oracle10k
    ref = rpca.randomized_pca(cfg10k, 50, 10, 4, True, om, value_dtype=rounder)
    res = _run(cfg10k, n_components=50, n_oversamples=10, n_power_iterations=4, omega=om,
               math_mode=mode)
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < SIGMA_RTOL, rel.max()
    # against the unrounded FP64 result too (total error incl. value rounding)
    rel_tot = np.abs(res.singular_values - exact["singular_values"]) / exact["singular_values"]
    assert rel_tot.max() < 1e-3, rel_tot.max()


def test_device_and_host_entry_agree(cfg10k):
    import torch

    kw = dict(n_components=20, n_oversamples=10, n_power_iterations=2, seed=3)
    host = _run(cfg10k, **kw)
    ip = torch.from_numpy(cfg10k.indptr).cuda()
    ix = torch.from_numpy(cfg10k.indices).cuda()
    vv = torch.from_numpy(cfg10k.data).cuda()
    dev = accel.randomized_pca(ip, ix, vv, cfg10k.shape, device_embeddings=True, **kw)
    assert dev.embeddings.is_cuda
    np.testing.assert_allclose(dev.singular_values, host.singular_values, rtol=1e-6)
    np.testing.assert_allclose(np.abs(dev.embeddings.cpu().numpy()), np.abs(host.embeddings),
                               rtol=1e-3, atol=1e-3)


def test_unsorted_rows_and_empty_rows():
    n, g = 600, 80
    indptr, idx, val = synth_nb_csr(n, g, seed=8, loc=-2.0)
    # empty out every 7th row
    keep = np.repeat(np.arange(n) % 7 != 0, np.diff(indptr))
    counts = np.diff(indptr) * (np.arange(n) % 7 != 0)
    ip2 = np.r_[0, np.cumsum(counts)]
    ix2, v2 = idx[keep], val[keep]
    c_sorted = rpca.Csr(ip2, ix2, v2, (n, g))
    # reverse each row's order
    ix3, v3 = ix2.copy(), v2.copy()
    for r in range(n):
        s, e = ip2[r], ip2[r + 1]
        ix3[s:e] = ix3[s:e][::-1]
        v3[s:e] = v3[s:e][::-1]
    c_unsorted = rpca.Csr(ip2, ix3, v3, (n, g))
    om = rpca.gaussian_omega(g, 30, seed=1)
    a = _run(c_sorted, n_components=20, n_oversamples=10, n_power_iterations=3, omega=om)
    b = _run(c_unsorted, n_components=20, n_oversamples=10, n_power_iterations=3, omega=om)
    ref = rpca.randomized_pca(c_sorted, 20, 10, 3, True, om)
    np.testing.assert_allclose(a.singular_values, b.singular_values, rtol=1e-6)
    rel = np.abs(a.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < SIGMA_RTOL


def test_invalid_csr_rejected():
    indptr = np.array([0, 2, 1], dtype=np.int64)
    with pytest.raises(RuntimeError, match="invalid CSR"):
        accel.randomized_pca(indptr, np.array([0, 1], np.int32), np.ones(2, np.float32), (2, 3),
                             n_components=1, n_oversamples=0)
    with pytest.raises(RuntimeError, match="out of range"):
        accel.randomized_pca(np.array([0, 1, 2]), np.array([0, 9], np.int32), np.ones(2, np.float32),
                             (2, 3), n_components=1, n_oversamples=0)


def test_planted_clusters_top_pcs_match_dense():
    # planted low-rank programme: well separated top PCs (test_accel_pca_gpu.py:128-202)
    n, g = 3000, 400
    indptr, idx, val = synth_nb_csr(n, g, seed=21, loc=-1.5, planted_rank=4, planted_scale=1.5)
    c = rpca.Csr(indptr, idx, val, (n, g))
    res = _run(c, n_components=30, n_oversamples=10, n_power_iterations=4, seed=0)
    ex = rpca.dense_pca(c.to_dense(), 30)
    cos = np.abs(np.sum(res.components[:4] * ex["components"][:4], axis=1))
    assert (cos > 0.99).all(), cos
    vr_ex = ex["variance_explained"] / (np.sum((c.to_dense() - c.to_dense().mean(0)) ** 2) / (n - 1))
    assert np.abs(res.variance_ratio[:4] - vr_ex[:4]).max() < 1e-3


def test_device_synth_generator_properties():
    import torch

    ip, ix, vv = accel.synth_nb_csr_device(20_000, 2_000, seed=0, loc=-3.0)
    ip, ix, vv = ip.cpu().numpy(), ix.cpu().numpy(), vv.cpu().numpy()
    dens = ip[-1] / (20_000 * 2_000)
    assert 0.09 < dens < 0.125, dens
    assert np.isfinite(vv).all() and (vv > 0).all()
    assert (np.diff(ip) >= 0).all()
    # rows sorted strictly by gene
    starts = ip[:-1]
    d = np.diff(ix.astype(np.int64))
    row_break = np.zeros(len(ix), bool)
    row_break[starts[starts < len(ix)]] = True
    assert (d[~row_break[1:]] > 0).all()
    # deterministic
    ip2, ix2, vv2 = accel.synth_nb_csr_device(20_000, 2_000, seed=0, loc=-3.0)
    assert np.array_equal(ix, ix2.cpu().numpy()) and np.array_equal(vv, vv2.cpu().numpy())
    torch.cuda.synchronize()
