"""The FP64 oracle pinned against the reference's own fixtures and known answers.

Mirrors the CPU unit tests of scx-accel/src/pca/cpu.rs:2326-2514 (10x5
fixture, SpMM vs dense, QR, SVD reconstruction) and the cancellation-guard
tests (cpu.rs:2217-2323).  CPU only.
"""

import numpy as np
import pytest

from oracle import rpca


def _omega(n_vars, k, seed=42):
    return np.random.default_rng(seed).standard_normal((n_vars, k))


def test_10x5_structure_and_exactness(csr_10x5, fixtures):
    # cpu.rs:2342-2369 -- randomized_pca_inmemory(&csr, 3, 5, 2, true, 42)
    k = rpca.effective_k(10, 5, 3, 5)
    assert k == 5  # k == n_vars: the sketch spans everything, so the result is exact
    res = rpca.randomized_pca(csr_10x5, 3, 5, 2, True, _omega(5, k))
    assert res["embeddings"].shape == (10, 3)
    assert res["components"].shape == (3, 5)
    assert res["variance_explained"].shape == (3,)
    assert res["mean"] is not None
    ve = res["variance_explained"]
    assert (ve > 0).all() and (np.diff(ve) <= 0).all()
    assert 0 < res["variance_ratio"].sum() <= 1 + 1e-10
    exact = fixtures["csr_10x5"]["exact"]["centered"]
    np.testing.assert_allclose(res["singular_values"], exact["singular_values"][:3], rtol=1e-10)
    np.testing.assert_allclose(res["total_var"], exact["total_var"], rtol=1e-12)
    # components orthonormal (cpu.rs:2384-2399 asserts |dot| < 0.1; exact here)
    g = res["components"] @ res["components"].T
    np.testing.assert_allclose(g, np.eye(3), atol=1e-10)


def test_10x5_uncentered(csr_10x5, fixtures):
    res = rpca.randomized_pca(csr_10x5, 2, 5, 2, False, _omega(5, 5))
    assert res["mean"] is None
    assert (res["variance_explained"] > 0).all()
    exact = fixtures["csr_10x5"]["exact"]["uncentered"]
    np.testing.assert_allclose(res["singular_values"], exact["singular_values"][:2], rtol=1e-10)


@pytest.mark.parametrize("nc", [0, 6])
def test_10x5_errors(csr_10x5, nc):
    # cpu.rs:2402-2412
    with pytest.raises(ValueError):
        rpca.randomized_pca(csr_10x5, nc, 5, 2, True, _omega(5, 5))


def test_empty_matrix_error():
    c = rpca.Csr([0], [], np.zeros(0, np.float32), (0, 5))
    with pytest.raises(ValueError, match="non-empty"):
        rpca.randomized_pca(c, 1, 0, 0, True, np.zeros((5, 1)))


def test_spmm_matches_dense(csr_10x5):
    # cpu.rs:2415-2444 at 1e-10, both directions, with and without centring
    dense = csr_10x5.to_dense()
    m = _omega(5, 3)
    q = _omega(10, 3, 7)
    mu = dense.mean(axis=0)
    np.testing.assert_allclose(rpca.spmm_forward(csr_10x5, m, None), dense @ m, atol=1e-10)
    np.testing.assert_allclose(rpca.spmm_forward(csr_10x5, m, mu), (dense - mu) @ m, atol=1e-10)
    np.testing.assert_allclose(rpca.spmm_transpose(csr_10x5, q, None), dense.T @ q, atol=1e-10)
    np.testing.assert_allclose(rpca.spmm_transpose(csr_10x5, q, mu), (dense - mu).T @ q, atol=1e-10)


def test_qr_orthonormal(fixtures):
    f = fixtures["qr_4x2"]
    q = rpca.qr_thin_q(np.asarray(f["data"]).reshape(f["rows"], f["cols"]))
    np.testing.assert_allclose(q.T @ q, np.eye(2), atol=1e-10)


def test_svd_reconstruction(fixtures):
    f = fixtures["rowmajor_4x3"]
    a = np.asarray(f["data"]).reshape(f["rows"], f["cols"])
    u, s, vt = np.linalg.svd(a, full_matrices=False)
    np.testing.assert_allclose((u * s) @ vt, a, atol=1e-10)
    f = fixtures["svd_3x2"]
    s = np.linalg.svd(np.asarray(f["data"]).reshape(3, 2), compute_uv=False)
    assert s[0] >= s[1] > 0


def test_cancellation_guard_recomputes():
    # large mean, tiny variance: the closed form cancels (moments.rs:288-308)
    rng = np.random.default_rng(0)
    n, g = 400, 6
    dense = 1e5 + rng.standard_normal((n, g)) * 1e-2
    rows, cols = np.nonzero(dense)
    c = rpca.Csr(np.arange(0, n * g + 1, g), cols, dense[rows, cols].astype(np.float64), (n, g))
    s, sq = rpca.col_sums_and_sum_sq(c)
    mu = s / n
    assert rpca.closed_form_variance_health(sq, mu, n) == "cancelled"
    tv, recomputed = rpca.guarded_total_variance(c, sq, mu, n)
    assert recomputed
    np.testing.assert_allclose(tv, np.sum((dense - dense.mean(0)) ** 2) / (n - 1), rtol=1e-6)


def test_degenerate_matrix_is_not_cancelled():
    c = rpca.Csr([0, 1, 2], [0, 1], np.zeros(2, np.float32), (2, 2))
    s, sq = rpca.col_sums_and_sum_sq(c)
    assert rpca.closed_form_variance_health(sq, s / 2, 2) == "degenerate"


@pytest.mark.parametrize("center", [True, False])
def test_scale_values_matches_dense(center):
    from scx_b200.synth import synth_nb_csr

    indptr, idx, val = synth_nb_csr(300, 40, seed=3)
    c = rpca.Csr(indptr, idx, val, (300, 40))
    dense = c.to_dense()
    p, mu, std, cg = rpca.scale_values(c, 2.5, center)
    mu_d = dense.mean(0)
    sd = dense.std(0, ddof=1)
    sd[sd == 0] = 1
    if center:
        s = np.clip((dense - mu_d) / sd, -2.5, 2.5)
    else:
        s = np.minimum(dense / sd, 2.5)
    # S = P + 1 c^T (P sparse on X's pattern)
    recon = c.with_values(p).to_dense() + cg[None, :]
    np.testing.assert_allclose(recon, s, atol=1e-10)
    np.testing.assert_allclose(mu, mu_d, rtol=1e-12)


def test_scaled_pca_equals_dense_scaled_pca():
    from scx_b200.synth import synth_nb_csr

    n, g = 500, 60
    indptr, idx, val = synth_nb_csr(n, g, seed=5, planted_rank=3, planted_scale=1.0)
    c = rpca.Csr(indptr, idx, val, (n, g))
    res = rpca.randomized_pca(c, 10, 50, 0, True, _omega(g, 60), scale=True, clip_max=3.0)
    dense = c.to_dense()
    sd = dense.std(0, ddof=1)
    sd[sd == 0] = 1
    s = np.clip((dense - dense.mean(0)) / sd, -3, 3)
    ex = rpca.dense_pca(s, 10)
    np.testing.assert_allclose(res["singular_values"], ex["singular_values"], rtol=1e-9)


def test_oracle_converges_to_dense_on_gapped_spectrum():
    from scx_b200.synth import synth_nb_csr

    n, g = 3000, 200
    indptr, idx, val = synth_nb_csr(n, g, seed=11, loc=-1.5, planted_rank=5, planted_scale=1.5)
    c = rpca.Csr(indptr, idx, val, (n, g))
    res = rpca.randomized_pca(c, 5, 10, 4, True, _omega(g, 15))
    ex = rpca.dense_pca(c.to_dense(), 5)
    np.testing.assert_allclose(res["singular_values"], ex["singular_values"], rtol=1e-6)
    ang = rpca.principal_angles(res["components"].T, ex["components"].T)
    assert ang.max() < 1e-3


def test_gpu_and_cpu_orderings_agree_for_q_gt_2():
    from scx_b200.synth import synth_nb_csr

    indptr, idx, val = synth_nb_csr(800, 100, seed=2)
    c = rpca.Csr(indptr, idx, val, (800, 100))
    om = _omega(100, 30)
    a = rpca.randomized_pca(c, 20, 10, 3, True, om, ordering="gpu")
    b = rpca.randomized_pca(c, 20, 10, 3, True, om, ordering="cpu")
    np.testing.assert_allclose(a["singular_values"], b["singular_values"], rtol=1e-12)


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in kat:
        got = rpca.philox4x32_10(np.array([ctr[0]]), np.array([ctr[1]]), key[0], key[1], ctr[2], ctr[3])
        assert tuple(int(x[0]) for x in got) == want


def test_gaussian_omega_moments_and_determinism():
    a = rpca.gaussian_omega(2000, 60, seed=0)
    b = rpca.gaussian_omega(2000, 60, seed=0)
    c = rpca.gaussian_omega(2000, 60, seed=1)
    assert a.shape == (2000, 60)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    assert abs(a.mean()) < 0.01 and abs(a.std() - 1) < 0.01
    assert np.all(a == a.astype(np.float32))


def test_bf16_rounding_helper():
    x = np.array([1.0, 1.00390625, 1.001953125, -3.14159], dtype=np.float32)
    r = rpca.round_to_bf16(x)
    # bf16 spacing at 1 is 2^-7: 1 + 2^-8 is a tie and rounds to even (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


# --------------------------------------------------------------------------
# truncated-SVD adjoint (oracle/adjoint.py): pinned against torch autograd
# through torch.linalg.svd in FP64 and against central finite differences
# --------------------------------------------------------------------------

def _torch_reference_grads(ip, ix, vv, shape, center, scale, W, c):
    import torch

    n, g = shape
    rows = torch.from_numpy(np.repeat(np.arange(n), np.diff(ip)))
    cols = torch.from_numpy(ix.astype(np.int64))
    v = torch.tensor(vv, dtype=torch.float64, requires_grad=True)
    cen = torch.tensor(center, dtype=torch.float64, requires_grad=True)
    sca = torch.tensor(scale, dtype=torch.float64, requires_grad=True)
    X = torch.zeros((n, g), dtype=torch.float64).index_put((rows, cols), v, accumulate=True)
    Xt = (X - cen[None, :]) * sca[None, :]
    _, _, vh = torch.linalg.svd(Xt, full_matrices=False)
    S = Xt @ vh[:c].T
    loss = (torch.from_numpy(W) * S * S).sum()
    loss.backward()
    return v.grad.numpy(), cen.grad.numpy(), sca.grad.numpy()


def test_adjoint_matches_torch_svd_autograd():
    from oracle import adjoint as ad

    ip, ix, vv = ad.planted_csr(80, 24, 8, 0.5, seed=3, top=50.0, ratio=0.85, noise=0.2)
    shape = (80, 24)
    rng = np.random.default_rng(0)
    X = ad.dense(ip, ix, vv, shape)
    center = X.mean(axis=0)
    scale = 1.0 / (X.std(axis=0, ddof=1) + 0.5)
    W = rng.standard_normal((80, 6))
    gv, gc, gs = ad.grads(ip, ix, vv, shape, center, scale, W, 6)
    tv, tc, ts = _torch_reference_grads(ip, ix, vv.astype(np.float64), shape, center, scale, W, 6)
    for a, b in ((gv, tv), (gc, tc), (gs, ts)):
        assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b)


def test_adjoint_matches_finite_differences():
    from oracle import adjoint as ad

    n, g, c = 60, 20, 5
    ip, ix, vv = ad.planted_csr(n, g, 7, 0.6, seed=5, top=40.0, ratio=0.8, noise=0.1)
    rng = np.random.default_rng(1)
    X = ad.dense(ip, ix, vv, (n, g))
    center = X.mean(axis=0)
    scale = 1.0 / (X.std(axis=0, ddof=1) + 0.3)
    W = rng.standard_normal((n, c))
    gv, gc, gs = ad.grads(ip, ix, vv, (n, g), center, scale, W, c)
    vv64 = vv.astype(np.float64)

    def L(v, cen, sca):
        return ad.loss(ad.affine(ad.dense(ip, ix, v, (n, g)), cen, sca), W, c)

    eps = 1e-6
    for _ in range(3):
        dv, dc, ds = rng.standard_normal(len(vv)), rng.standard_normal(g), rng.standard_normal(g)
        fd_v = (L(vv64 + eps * dv, center, scale) - L(vv64 - eps * dv, center, scale)) / (2 * eps)
        fd_c = (L(vv64, center + eps * dc, scale) - L(vv64, center - eps * dc, scale)) / (2 * eps)
        fd_s = (L(vv64, center, scale + eps * ds) - L(vv64, center, scale - eps * ds)) / (2 * eps)
        assert abs(fd_v - gv @ dv) <= 1e-5 * max(1.0, abs(fd_v))
        assert abs(fd_c - gc @ dc) <= 1e-5 * max(1.0, abs(fd_c))
        assert abs(fd_s - gs @ ds) <= 1e-5 * max(1.0, abs(fd_s))


def test_cpp_restatement_matches_numpy_oracle():
    """The multithreaded C++ restatement (CPU baseline and full-size FP64
    reference of the bench) computes the same randomized PCA as the numpy
    oracle on the same Omega: scaled + clipped and plain centred."""
    from oracle import build_cpu
    from scx_b200.synth import synth_nb_csr

    n, g, nc, over, q = 3000, 400, 20, 10, 4
    ip, ix, vv = synth_nb_csr(n, g, seed=4, loc=-2.0)
    om = rpca.gaussian_omega(g, nc + over, seed=3)
    c = rpca.Csr(ip, ix, vv, (n, g))
    for scale, clip in ((False, 0.0), (True, 10.0)):
        ref = rpca.randomized_pca(c, nc, over, q, True, om, scale=scale, clip_max=clip)
        got = build_cpu.run(ip, ix, vv, (n, g), nc, nc + over, q, om, zero_center=True, scale=scale,
                            clip_max=clip, threads=4)
        np.testing.assert_allclose(got["singular_values"], ref["singular_values"], rtol=1e-9)
        assert rpca.principal_angles(got["components"].T, ref["components"].T).max() < 1e-6


def test_pflog_oracle_equals_dense_z():
    """The PFlog restatement's offset products are the products with the dense
    Z = delta + b 1^T, its closed-form total variance is the dense variance, and
    its PCA is the dense PCA of Z at k = n_vars (cpu.rs:618-786)."""
    rng = np.random.default_rng(4)
    n, g = 300, 40
    counts = rng.negative_binomial(3, 0.5, size=(n, g)).astype(np.float32) * (rng.random((n, g)) < 0.3)
    rr, cc = np.nonzero(counts)
    ip = np.r_[0, np.cumsum(np.bincount(rr, minlength=n))]
    raw = rpca.Csr(ip, cc, counts[rr, cc], (n, g))
    delta_v, base = rpca.pflog_prepare(raw, 4 * 0.3)
    delta = raw.with_values(delta_v)
    z = delta.to_dense() + base[:, None]
    # the baseline is minus the mean of each row of delta
    np.testing.assert_allclose(z.sum(axis=1), 0.0, atol=1e-6)
    om = rng.standard_normal((g, g))
    res = rpca.pflog_pca(delta, base, 10, g - 10, 2, True, om)
    ex = rpca.dense_pca(z, 10)
    np.testing.assert_allclose(res["singular_values"], ex["singular_values"], rtol=1e-8)
    zc = z - z.mean(axis=0)
    np.testing.assert_allclose(res["total_var"], (zc ** 2).sum() / (n - 1), rtol=1e-6)
    np.testing.assert_allclose(res["mean"], z.mean(axis=0), rtol=1e-10, atol=1e-12)
