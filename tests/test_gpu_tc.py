"""Tensor-core (tcgen05) SpMM path of the mixed-precision mode vs the FP64 oracle.

The oracle is fed the same 16-bit-rounded matrix values the tensor cores see;
the dense operand (V or Q) enters the tensor cores as a 16-bit image holding a
hi/lo pair per value (about 16 mantissa bits), so the forward product agrees to 1e-4 and
the transposed product to 1e-4 relative to the output norm.  Shapes cover
partial row tiles, partial gene chunks, a single tile, and both supported
sketch widths (ld 64 and 128).
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu

SHAPES = [
    (1000, 300, 20),    # partial tile and partial chunk, ld 64
    (128, 64, 30),      # exactly one tile and one chunk
    (77, 130, 10),      # fewer cells than a tile
    (4099, 2000, 60),   # the benchmark gene count
    (2500, 700, 100),   # ld 128
    (40000, 520, 30),   # more two-tile bands than SMs, odd chunk count
]


def _csr(n, g, seed=0):
    indptr, idx, val = synth_nb_csr(n, g, seed=seed, loc=-2.0)
    return rpca.Csr(indptr, idx, val, (n, g))


@pytest.mark.parametrize("mode,rounder", [("mixed_bf16", rpca.round_to_bf16),
                                          ("mixed_f16", rpca.round_to_f16)])
@pytest.mark.parametrize("n,g,k", SHAPES)
def test_tc_operator_seam(n, g, k, mode, rounder):
    import torch

    c = _csr(n, g)
    plan = accel.Plan(c.indptr, c.indices, c.data, c.shape, n_components=k, n_oversamples=0,
                      math_mode=mode)
    assert plan.k == k
    assert plan.ld == (k + 63) // 64 * 64  # tensor-core layout
    cr = c.with_values(rounder(c.data))
    mu = rpca.col_sums_and_sum_sq(cr)[0] / n
    rng = np.random.default_rng(1)
    v = (rng.standard_normal((g, k)) / np.sqrt(g)).astype(np.float32)
    y = plan.matmat(torch.from_numpy(v).cuda()).cpu().numpy().astype(np.float64)
    y_ref = rpca.spmm_forward(cr, v.astype(np.float64), mu)
    err = np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref)
    assert err < 1e-4, err
    q = (rng.standard_normal((n, k)) / np.sqrt(n)).astype(np.float32)
    z = plan.rmatmat(torch.from_numpy(q).cuda()).cpu().numpy()
    z_ref = rpca.spmm_transpose(cr, q.astype(np.float64), mu)
    err = np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref)
    assert err < 1e-4, err
    plan.close()


def test_tc_and_cuda_core_paths_agree(monkeypatch):
    n, g = 6000, 1500
    c = _csr(n, g, seed=4)
    om = rpca.gaussian_omega(g, 60, seed=2)
    kw = dict(n_components=50, n_oversamples=10, n_power_iterations=4, omega=om,
              math_mode="mixed_bf16", scale=True, clip_max=10.0)
    tc = accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, **kw)
    monkeypatch.setenv("SCXPCA_TC", "0")
    cc = accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, **kw)
    rel = np.abs(tc.singular_values - cc.singular_values) / cc.singular_values
    assert rel.max() < 1e-4, rel.max()
    # The tensor-core path also rounds V and the intermediate Y to 16 bits each
    # power iteration (~2^-9 per entry): the head of the subspace agrees to
    # 1e-3 rad, the near-degenerate tail to 2e-2 rad; sigma is second-order.
    assert rpca.principal_angles(tc.components[:20].T, cc.components[:20].T).max() < 1e-3
    assert rpca.principal_angles(tc.components.T, cc.components.T).max() < 2e-2


def test_tc_full_pca_matches_oracle_on_rounded_values():
    n, g = 8000, 2000
    c = _csr(n, g, seed=6)
    om = rpca.gaussian_omega(g, 60, seed=0)
    ref = rpca.randomized_pca(c, 50, 10, 4, True, om, value_dtype=rpca.round_to_bf16)
    res = accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, n_components=50,
                               n_oversamples=10, n_power_iterations=4, omega=om,
                               math_mode="mixed_bf16", qr_method="cholesky")
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < 1e-4, rel.max()
    assert rpca.principal_angles(res.components.T, ref["components"].T).max() < 1e-3
    emb_cos = np.abs(np.sum(res.embeddings * ref["embeddings"], 0)) / (
        np.linalg.norm(res.embeddings, axis=0) * np.linalg.norm(ref["embeddings"], axis=0))
    assert emb_cos[:10].min() > 0.9999


def test_tc_duplicates_use_cuda_cores_and_stay_correct():
    # duplicate coordinates: summed like the reference (cpu.rs:3224); the
    # tensor-core format needs unique entries, so this plan runs on CUDA cores
    n, g = 500, 100
    c = _csr(n, g, seed=9)
    ip, ix, vv = c.indptr.copy(), c.indices.copy(), c.data.copy()
    # duplicate the first entry of every non-empty row
    rows = np.flatnonzero(np.diff(ip) > 0)
    ins = ip[rows]
    ix2 = np.insert(ix, ins, ix[ins])
    vv2 = np.insert(vv, ins, np.float32(0.5))
    counts = np.diff(ip)
    counts[rows] += 1
    ip2 = np.r_[0, np.cumsum(counts)]
    dup = rpca.Csr(ip2, ix2, vv2, (n, g))
    dense = dup.to_dense()
    om = rpca.gaussian_omega(g, 40, seed=5)
    res = accel.randomized_pca(ip2, ix2, vv2, (n, g), n_components=10, n_oversamples=30,
                               n_power_iterations=4, omega=om, math_mode="mixed_bf16")
    ref = rpca.dense_pca(rpca.round_to_bf16(dense.astype(np.float32)), 10)
    rel = np.abs(res.singular_values - ref["singular_values"]) / ref["singular_values"]
    assert rel.max() < 5e-3


@pytest.mark.parametrize("n,nc,over,mode", [(3000, 50, 10, "mixed_bf16"), (100, 40, 24, "mixed_f16"),
                                            (20000, 64, 0, "mixed_bf16")])
def test_tensor_core_embeddings_match_cuda_core_product(monkeypatch, n, nc, over, mode):
    """The embeddings U = Q M on tensor cores (from Q's 16-bit image and the
    hi/lo image of M) against the CUDA-core FP32 product of the same run:
    a ragged last row tile, a single partial tile, more tiles than SMs, BF16
    and FP16 images, 40 to 64 components.  Everything before the embedding is
    the same launches, so sigma and the components are bit-identical."""
    g = 700
    c = _csr(n, g, seed=11)
    om = rpca.gaussian_omega(g, nc + over, seed=1)
    kw = dict(n_components=nc, n_oversamples=over, n_power_iterations=3, omega=om, math_mode=mode,
              qr_method="cholesky")
    tc = accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, **kw)
    monkeypatch.setenv("SCXPCA_EMBED_TC", "0")
    cc = accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, **kw)
    np.testing.assert_array_equal(tc.singular_values, cc.singular_values)
    np.testing.assert_array_equal(tc.components, cc.components)
    assert np.isfinite(tc.embeddings).all() and tc.embeddings.shape == (n, nc)
    # ~16 mantissa bits on both operands of the tensor-core product
    err = np.linalg.norm(tc.embeddings - cc.embeddings) / np.linalg.norm(cc.embeddings)
    assert err < 2e-4, err
    assert np.abs(tc.embeddings - cc.embeddings).max() < 2e-3 * np.abs(cc.embeddings).max()
