"""CUDA-core SpMM pair (strict FP32 path) and the fixed summation order (needs a B200).

Operator-level products against numpy FP64 on the same FP32 values, relative to
the output norm: 1e-5 (FP32 accumulation over rows of a few hundred entries).
Shapes cover every supported sketch width (ld 32, 64, 96, 128), partial row
tiles, gene counts that are not a multiple of the staged gene chunk, empty
rows, rows with more than 32 stored entries inside one gene chunk, and rows
with duplicate gene indices.  Determinism: with spmm_policy="deterministic"
(and on every other setting) two runs of the strict and of the mixed path are
bit-identical, as SpmmAlgPolicy::Deterministic asks of the reference
(scx-gpu/src/math_policy.rs:86-136).
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu

OP_RTOL = 1e-5


def _csr(n, g, seed=0, loc=-2.0):
    indptr, idx, val = synth_nb_csr(n, g, seed=seed, loc=loc)
    return rpca.Csr(indptr, idx, val, (n, g))


def _with_dense_block(c, rows, genes):
    """The CSR with rows `rows` made dense over genes [0, genes) (values 0.5 + gene / genes),
    so those rows hold more than 32 entries inside one staged gene chunk."""
    n, g = c.shape
    dense = np.zeros((n, g), dtype=np.float32)
    r = np.repeat(np.arange(n), np.diff(c.indptr))
    dense[r, c.indices] = c.data
    for i in rows:
        dense[i, :genes] = 0.5 + np.arange(genes, dtype=np.float32) / genes
    rr, cc = np.nonzero(dense)
    indptr = np.r_[0, np.cumsum(np.bincount(rr, minlength=n))]
    return rpca.Csr(indptr, cc.astype(np.int32), dense[rr, cc], (n, g))


SHAPES = [
    (1000, 300, 20),    # ld 32, partial tile
    (4099, 2000, 60),   # ld 64, the benchmark gene count, 16 gene chunks
    (777, 515, 90),     # ld 96, gene count off every chunk size
    (2500, 700, 120),   # ld 128
    (77, 130, 10),      # fewer cells than a tile
]


@pytest.mark.parametrize("n,g,k", SHAPES)
def test_strict_operator_seam(n, g, k):
    import torch

    c = _with_dense_block(_csr(n, g, seed=n), rows=[0, 5, n - 1], genes=min(g, 300))
    # empty rows
    ip = c.indptr.copy()
    for i in (1, n // 2):
        cnt = ip[i + 1] - ip[i]
        keep = np.ones(len(c.indices), dtype=bool)
        keep[ip[i]:ip[i + 1]] = False
        c = rpca.Csr(np.r_[ip[: i + 1], ip[i + 1:] - cnt], c.indices[keep], c.data[keep], (n, g))
        ip = c.indptr
    plan = accel.Plan(c.indptr, c.indices, c.data, c.shape, n_components=k, n_oversamples=0,
                      math_mode="strict_fp32")
    assert plan.k == k
    mu = rpca.col_sums_and_sum_sq(c)[0] / n
    rng = np.random.default_rng(3)
    v = rng.standard_normal((g, k)).astype(np.float32)
    y = plan.matmat(torch.from_numpy(v).cuda()).cpu().numpy().astype(np.float64)
    y_ref = rpca.spmm_forward(c, v.astype(np.float64), mu)
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < OP_RTOL
    q = rng.standard_normal((n, k)).astype(np.float32)
    z = plan.rmatmat(torch.from_numpy(q).cuda()).cpu().numpy()
    z_ref = rpca.spmm_transpose(c, q.astype(np.float64), mu)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) < OP_RTOL
    # row by row as well: no row may be dropped or doubled
    rel_rows = np.linalg.norm(y - y_ref, axis=1) / np.maximum(np.linalg.norm(y_ref, axis=1), 1e-30)
    assert rel_rows.max() < 1e-4
    plan.close()


def test_strict_duplicate_indices_sum():
    """A row that names a gene twice contributes both values (the sorted copy keeps both)."""
    import torch

    n, g = 300, 70
    c = _csr(n, g, seed=4)
    rows = np.repeat(np.arange(n), np.diff(c.indptr))
    # duplicate every third entry of row 3 and row 200, unsorted
    extra = [(r, j, 0.25) for r in (3, 200) for j in c.indices[c.indptr[r]:c.indptr[r + 1]][::3]]
    rr = np.r_[rows, [e[0] for e in extra]]
    cc = np.r_[c.indices, [e[1] for e in extra]].astype(np.int32)
    vv = np.r_[c.data, [e[2] for e in extra]].astype(np.float32)
    order = np.argsort(rr, kind="stable")
    rr, cc, vv = rr[order], cc[order], vv[order]
    indptr = np.r_[0, np.cumsum(np.bincount(rr, minlength=n))]
    d = rpca.Csr(indptr, cc, vv, (n, g))
    plan = accel.Plan(d.indptr, d.indices, d.data, d.shape, n_components=20, n_oversamples=0,
                      math_mode="strict_fp32")
    dense = np.zeros((n, g))
    np.add.at(dense, (rr, cc), vv.astype(np.float64))
    mu = dense.mean(0)
    v = np.random.default_rng(5).standard_normal((g, 20)).astype(np.float32)
    y = plan.matmat(torch.from_numpy(v).cuda()).cpu().numpy()
    y_ref = (dense - mu) @ v.astype(np.float64)
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < OP_RTOL
    q = np.random.default_rng(6).standard_normal((n, 20)).astype(np.float32)
    z = plan.rmatmat(torch.from_numpy(q).cuda()).cpu().numpy()
    z_ref = (dense - mu).T @ q.astype(np.float64)
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) < OP_RTOL
    plan.close()


@pytest.mark.parametrize("mode", ["strict_fp32", "mixed_bf16"])
def test_runs_are_bit_identical(mode):
    c = _csr(20000, 1500, seed=11, loc=-2.5)
    outs = []
    for _ in range(2):  # two plans (statistics, value transform, copies rebuilt) ...
        plan = accel.Plan(c.indptr, c.indices, c.data, c.shape, n_components=30, n_oversamples=10,
                          n_power_iterations=3, zero_center=True, scale=True, clip_max=10.0,
                          math_mode=mode, spmm_policy="deterministic", seed=5)
        outs.append(plan.run())
        outs.append(plan.run())  # ... and two runs of each
        plan.close()
    a = outs[0]
    for b in outs[1:]:
        assert np.array_equal(a.singular_values, b.singular_values)
        assert np.array_equal(a.components, b.components)
        assert np.array_equal(a.embeddings, b.embeddings)
        assert np.array_equal(a.mean, b.mean) and np.array_equal(a.std, b.std)
        assert a.total_var == b.total_var


def test_total_variance_cancellation_guard_on_device():
    """Closed-form total variance that cancels: every gene stored in every cell
    at a large mean with a tiny spread.  The library must take the recompute
    branch (scx-accel/src/pca/cpu.rs:1066-1092, scx-sparse/src/moments.rs:288-308)
    and agree with a two-pass FP64 variance of the same FP32 values."""
    n, g = 3000, 40
    rng = np.random.default_rng(8)
    dense = (4096.0 + rng.integers(-4, 5, size=(n, g)) * (1.0 / 256)).astype(np.float32)
    rr, cc = np.nonzero(dense)
    indptr = np.r_[0, np.cumsum(np.bincount(rr, minlength=n))]
    c = rpca.Csr(indptr, cc.astype(np.int32), dense[rr, cc], (n, g))
    res = accel.randomized_pca(c.indptr, c.indices, c.data, c.shape, n_components=5, n_oversamples=5,
                               n_power_iterations=1, seed=1, math_mode="strict_fp32")
    d64 = dense.astype(np.float64)
    want = ((d64 - d64.mean(0)) ** 2).sum() / (n - 1)
    sumsq = (d64 ** 2).sum()
    mu = d64.mean(0)
    assert sumsq - n * (mu ** 2).sum() <= 1e-7 * sumsq  # the closed form cancels here
    assert res.total_var_recomputed
    np.testing.assert_allclose(res.total_var, want, rtol=1e-6)
    assert np.all(res.variance_ratio >= 0) and res.variance_ratio.sum() <= 1 + 1e-6


@pytest.mark.parametrize("mode", ["strict_fp32", "mixed_bf16"])
def test_householder_qr_orthonormal_on_ill_conditioned(mode):
    """The Householder contract: qr returns an orthonormal Q spanning the input
    even at condition number 1e7 (QᵀQ ≈ I at 1e-4, the reference's GPU QR
    tolerance, scx-gpu/src/cusolver.rs:426-465)."""
    import torch

    c = _csr(500, 200, seed=2)
    plan = accel.Plan(c.indptr, c.indices, c.data, c.shape, n_components=50, n_oversamples=10,
                      qr_method="householder", math_mode=mode)
    m, k = 6000, plan.k
    rng = np.random.default_rng(12)
    u, _ = np.linalg.qr(rng.standard_normal((m, k)))
    w, _ = np.linalg.qr(rng.standard_normal((k, k)))
    y = (u * np.logspace(0, -7, k)) @ w.T
    y32 = y.astype(np.float32)
    a = torch.from_numpy(y32.copy()).cuda()
    plan.qr(a)
    q = a.cpu().numpy().astype(np.float64)
    np.testing.assert_allclose(q.T @ q, np.eye(k), atol=1e-4)
    # Q spans the input: the projection of Y onto Q's columns recovers Y
    y64 = y32.astype(np.float64)
    resid = np.linalg.norm(y64 - q @ (q.T @ y64)) / np.linalg.norm(y64)
    assert resid < 1e-5, resid
    plan.close()
