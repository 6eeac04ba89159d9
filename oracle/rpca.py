"""FP64 CPU restatement of scx's randomized PCA -- TEST INFRASTRUCTURE ONLY.

This module is the oracle the CUDA path is checked against.  Nothing in the
product (``scx_b200``) imports it; only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may call it, and only as the checker.

What it restates (paths are inside the ArcInstitute/scx tree):

* ``randomized_pca_inmemory``          scx-accel/src/pca/cpu.rs:887-952
* power-loop ordering of the GPU path  scx-gpu/src/pca_operator.rs:100-119
* ``validate_inputs``                  scx-accel/src/pca/cpu.rs:979-997
* ``col_sums_and_sum_sq``              scx-sparse/src/csr.rs:570-580
* ``spmm_forward_csr`` / ``_row``      scx-accel/src/pca/cpu.rs:1429-1523
* ``spmm_transpose_csr`` + ``apply_transpose_mean_correction``
                                       scx-accel/src/pca/cpu.rs:1238-1267, 1282-1389
* ``build_pca_result``                 scx-accel/src/pca/cpu.rs:1530-1585
* ``total_variance_from_col_sq``       scx-sparse/src/csr.rs:868-880
* ``closed_form_variance_health``      scx-sparse/src/moments.rs:288-308
* ``guarded_total_variance_inmemory``  scx-accel/src/pca/cpu.rs:1066-1092
* ``stable_centered_total_variance_inmemory``
                                       scx-accel/src/pca/cpu.rs:1130-1171

The reference takes Omega from ChaCha8 (CPU, rand_chacha 0.3.1 + rand_distr
0.4.3 StandardNormal) or cuRAND XORWOW (GPU); neither is reproducible here, so
this restatement takes an explicit Omega (``n_vars x k``), exactly like the
explicit-Omega argument of the CUDA entry point.  QR and SVD use numpy's LAPACK
in place of faer 0.24.0 (``qr_thin_q_row_major`` cpu.rs:118-122,
``thin_svd_decomp`` cpu.rs:458-472); both are pinned only by tolerances.

Parity pinning.  The reference is Rust and cannot be built or imported in this
environment (no cargo/rustc), and it ships no stored PCA outputs.  The oracle is
pinned against (1) the reference's own 10x5 CSR fixture and structural
assertions (cpu.rs:2326-2412), which at k == n_vars make randomized PCA exact,
so the oracle must equal a dense FP64 SVD there to 1e-10; (2) the SpMM-vs-dense
1e-10 and QR/SVD 1e-10 checks of cpu.rs:2415-2514; (3) dense FP64 PCA on gapped
spectra.  Parity with the reference's *numbers* is therefore partially pinned:
algorithm-level, not output-level.

The per-gene scale/clip transform (``scale_values``) has no reference
counterpart; it follows scanpy's ``pp.scale(zero_center, max_value)``
definition (ddof=1 standard deviation, zero std replaced by 1, two-sided clip
when centring, upper clip otherwise).
"""

from __future__ import annotations

import numpy as np

# scx-sparse/src/moments.rs:68
CLOSED_FORM_VAR_REL_EPS = 1e-7


# --------------------------------------------------------------------------
# Input validation (scx-accel/src/pca/cpu.rs:979-997)
# --------------------------------------------------------------------------

def validate_inputs(n_obs: int, n_vars: int, n_components: int) -> None:
    if n_components == 0:
        raise ValueError("n_components must be > 0")
    if n_obs == 0 or n_vars == 0:
        raise ValueError("matrix must be non-empty")
    if n_components > min(n_obs, n_vars):
        raise ValueError(
            f"n_components ({n_components}) exceeds matrix rank bound "
            f"min(n_obs, n_vars) = {min(n_obs, n_vars)}")


def effective_k(n_obs: int, n_vars: int, n_components: int, n_oversamples: int) -> int:
    """``k = min(n_components + n_oversamples, n_vars, n_obs)`` (cpu.rs:899)."""
    return min(n_components + n_oversamples, n_vars, n_obs)


# --------------------------------------------------------------------------
# CSR helpers
# --------------------------------------------------------------------------

class Csr:
    """Minimal CSR triple (int64 indptr, int32 indices, float values)."""

    def __init__(self, indptr, indices, data, shape):
        self.indptr = np.asarray(indptr, dtype=np.int64)
        self.indices = np.asarray(indices, dtype=np.int32)
        self.data = np.asarray(data)
        self.shape = (int(shape[0]), int(shape[1]))

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def row_ids(self) -> np.ndarray:
        return np.repeat(np.arange(self.shape[0], dtype=np.int64), np.diff(self.indptr))

    def to_dense(self) -> np.ndarray:
        out = np.zeros(self.shape, dtype=np.float64)
        np.add.at(out, (self.row_ids(), self.indices.astype(np.int64)),
                  self.data.astype(np.float64))
        return out

    def with_values(self, values) -> "Csr":
        return Csr(self.indptr, self.indices, values, self.shape)


def col_sums_and_sum_sq(csr: Csr):
    """Per-column sum and sum of squares in f64 (scx-sparse/src/csr.rs:570-580)."""
    v = csr.data.astype(np.float64)
    sums = np.bincount(csr.indices, weights=v, minlength=csr.shape[1])
    sum_sq = np.bincount(csr.indices, weights=v * v, minlength=csr.shape[1])
    return sums, sum_sq


# --------------------------------------------------------------------------
# Products with the implicitly centred matrix
# --------------------------------------------------------------------------

def spmm_forward(csr: Csr, m: np.ndarray, means):
    """``Y = (X - 1 mu^T) M`` (cpu.rs:1429-1523).

    ``mc = M^T mu`` is precomputed and subtracted from every output row, as in
    ``spmm_forward_csr`` (cpu.rs:1433-1441) and ``spmm_forward_row``.
    """
    n_obs = csr.shape[0]
    m = np.asarray(m, dtype=np.float64)
    prod = csr.data.astype(np.float64)[:, None] * m[csr.indices.astype(np.int64)]
    y = np.zeros((n_obs, m.shape[1]), dtype=np.float64)
    np.add.at(y, csr.row_ids(), prod) if csr.nnz < 4096 else _segment_sum(y, csr, prod)
    if means is not None:
        y -= (np.asarray(means, dtype=np.float64) @ m)[None, :]
    return y


def _segment_sum(out, csr: Csr, prod):
    # reduceat over row segments; empty rows keep zero.
    starts = csr.indptr[:-1]
    nonempty = np.diff(csr.indptr) > 0
    if prod.shape[0]:
        sums = np.add.reduceat(prod, starts[nonempty], axis=0)
        out[nonempty] = sums
    return out


def spmm_transpose(csr: Csr, q: np.ndarray, means):
    """``Z = (X - 1 mu^T)^T Q = X^T Q - mu (1^T Q)`` (cpu.rs:1238-1267, 1282-1389)."""
    q = np.asarray(q, dtype=np.float64)
    n_vars = csr.shape[1]
    prod = csr.data.astype(np.float64)[:, None] * q[csr.row_ids()]
    z = np.zeros((n_vars, q.shape[1]), dtype=np.float64)
    order = np.argsort(csr.indices, kind="stable")
    cols = csr.indices[order]
    if prod.shape[0]:
        starts = np.flatnonzero(np.r_[True, cols[1:] != cols[:-1]])
        z[cols[starts]] = np.add.reduceat(prod[order], starts, axis=0)
    if means is not None:
        z -= np.outer(np.asarray(means, dtype=np.float64), q.sum(axis=0))
    return z


def qr_thin_q(a: np.ndarray) -> np.ndarray:
    """Thin Householder Q (LAPACK geqrf/orgqr, standing in for faer's QR)."""
    q, _ = np.linalg.qr(np.asarray(a, dtype=np.float64), mode="reduced")
    return q


# --------------------------------------------------------------------------
# Total variance (scx-sparse csr.rs:868-880, moments.rs:288-308, cpu.rs:1066-1171)
# --------------------------------------------------------------------------

def total_variance_from_col_sq(col_sum_sq, means, n_obs: int) -> float:
    col_sum_sq = np.asarray(col_sum_sq, dtype=np.float64)
    if means is not None:
        total = float(np.sum(col_sum_sq - n_obs * np.asarray(means) ** 2))
    else:
        total = float(np.sum(col_sum_sq))
    return total / max(n_obs - 1.0, 1.0)


def closed_form_variance_health(col_sum_sq, means, n_obs: int) -> str:
    sum_sq = float(np.sum(col_sum_sq))
    if sum_sq <= 0.0:
        return "degenerate"
    mean_sq = float(np.sum(np.asarray(means) ** 2)) * n_obs
    residual = sum_sq - mean_sq
    if sum_sq > 0.0 and residual <= CLOSED_FORM_VAR_REL_EPS * sum_sq:
        return "cancelled"
    return "usable"


def stable_centered_total_variance(csr: Csr, means, n_obs: int) -> float:
    means = np.asarray(means, dtype=np.float64)
    d = csr.data.astype(np.float64) - means[csr.indices]
    total = float(np.sum(d * d))
    col_nnz = np.bincount(csr.indices, minlength=csr.shape[1])
    n_zeros = np.maximum(n_obs - col_nnz, 0).astype(np.float64)
    total += float(np.sum(n_zeros * means * means))
    return total / max(n_obs - 1.0, 1.0)


def guarded_total_variance(csr: Csr, col_sum_sq, means, n_obs: int):
    closed = total_variance_from_col_sq(col_sum_sq, means, n_obs)
    if means is None:
        return closed, False
    if closed_form_variance_health(col_sum_sq, means, n_obs) != "cancelled":
        return closed, False
    return stable_centered_total_variance(csr, means, n_obs), True


# --------------------------------------------------------------------------
# Per-gene scaling (no reference counterpart; scanpy pp.scale semantics)
# --------------------------------------------------------------------------

def scale_values(csr: Csr, clip_max: float, zero_center: bool):
    """Return (P values, mu, std, c) for ``S = clip((X - mu) / std)``.

    With centring, every stored zero maps to the per-gene constant
    ``c = clip(-mu / std)``, so ``S = P + 1 c^T`` with ``P`` sparse on X's
    pattern, holding ``clip((x - mu) / std) - c``.  Centred PCA of S equals
    centred PCA of P.  Without centring ``S = min(x / std, clip)`` keeps the
    sparsity pattern directly (c = 0).
    """
    n_obs = csr.shape[0]
    sums, sum_sq = col_sums_and_sum_sq(csr)
    mu = sums / n_obs
    var = (sum_sq - n_obs * mu * mu) / max(n_obs - 1, 1)
    var = np.maximum(var, 0.0)
    std = np.sqrt(var)
    std[std == 0.0] = 1.0
    x = csr.data.astype(np.float64)
    g = csr.indices.astype(np.int64)
    if zero_center:
        s = (x - mu[g]) / std[g]
        c = -mu / std
        if clip_max > 0:
            s = np.clip(s, -clip_max, clip_max)
            c = np.clip(c, -clip_max, clip_max)
        p = s - c[g]
    else:
        p = x / std[g]
        c = np.zeros_like(mu)
        if clip_max > 0:
            p = np.minimum(p, clip_max)
    return p, mu, std, c


# --------------------------------------------------------------------------
# Randomized PCA (cpu.rs:887-952 with the GPU ordering of pca_operator.rs)
# --------------------------------------------------------------------------

def randomized_pca(csr: Csr, n_components: int, n_oversamples: int,
                   n_power_iterations: int, zero_center: bool, omega,
                   scale: bool = False, clip_max: float = 0.0,
                   ordering: str = "gpu", value_dtype=None):
    """FP64 randomized PCA with an explicit ``omega`` (n_vars x k).

    ``ordering="gpu"`` follows ``run_power_loop`` (pca_operator.rs:100-119):
    ``matmat(Omega) -> qr(Y) -> [rmatmat -> qr(Z) -> matmat(Z) -> qr(Y)] x N ->
    rmatmat``.  ``ordering="cpu"`` follows cpu.rs:920-936, which skips the QR
    of Z when ``n_power_iterations <= 2``.

    ``value_dtype`` rounds the stored values first (e.g. ``bfloat16`` emulation
    via :func:`round_to_bf16`) so the algorithmic error of a mixed-precision
    run can be separated from the data rounding.
    """
    n_obs, n_vars = csr.shape
    validate_inputs(n_obs, n_vars, n_components)
    k = effective_k(n_obs, n_vars, n_components, n_oversamples)
    omega = np.asarray(omega, dtype=np.float64)
    if omega.shape != (n_vars, k):
        raise ValueError(f"omega must be ({n_vars}, {k}), got {omega.shape}")

    work = csr
    mu_x = std = None
    if scale:
        p, mu_x, std, _c = scale_values(csr, clip_max, zero_center)
        work = csr.with_values(p)
    if value_dtype is not None:
        work = work.with_values(value_dtype(work.data))

    col_sums, col_sum_sq = col_sums_and_sum_sq(work)
    means = col_sums / n_obs if zero_center else None

    y = spmm_forward(work, omega, means)
    q = qr_thin_q(y)
    for _ in range(n_power_iterations):
        z = spmm_transpose(work, q, means)
        if ordering == "gpu" or n_power_iterations > 2:
            z = qr_thin_q(z)
        y = spmm_forward(work, z, means)
        q = qr_thin_q(y)
    b = spmm_transpose(work, q, means)

    total_var, recomputed = guarded_total_variance(work, col_sum_sq, means, n_obs)
    res = build_pca_result(q, b, n_components, n_obs, total_var)
    res["mean"] = means if not scale else mu_x
    res["std"] = std
    res["k"] = k
    res["total_var"] = total_var
    res["total_var_recomputed"] = recomputed
    return res


def build_pca_result(q, b, n_components: int, n_obs: int, total_var: float):
    """SVD of B -> embeddings ``Q V sigma``, components ``U_hat^T`` (cpu.rs:1530-1585)."""
    u_hat, sigma, vt = np.linalg.svd(b, full_matrices=False)
    v = vt.T
    emb = (q @ v[:, :n_components]) * sigma[None, :n_components]
    components = u_hat[:, :n_components].T.copy()
    denom = max(n_obs - 1.0, 1.0)
    ve = sigma[:n_components] ** 2 / denom
    ratio = ve / total_var if total_var > 0.0 else np.zeros(n_components)
    return {
        "embeddings": emb,
        "components": components,
        "variance_explained": ve,
        "variance_ratio": ratio,
        "singular_values": sigma[:n_components].copy(),
    }


# --------------------------------------------------------------------------
# Exact dense oracle and comparison metrics
# --------------------------------------------------------------------------

def dense_pca(dense: np.ndarray, n_components: int, zero_center: bool = True):
    """Exact PCA of a dense FP64 matrix (numpy SVD)."""
    x = np.asarray(dense, dtype=np.float64)
    if zero_center:
        x = x - x.mean(axis=0, keepdims=True)
    u, s, vt = np.linalg.svd(x, full_matrices=False)
    n = x.shape[0]
    return {
        "embeddings": u[:, :n_components] * s[None, :n_components],
        "components": vt[:n_components].copy(),
        "singular_values": s[:n_components].copy(),
        "variance_explained": s[:n_components] ** 2 / max(n - 1.0, 1.0),
    }


def sign_fix(components: np.ndarray, embeddings: np.ndarray | None = None):
    """Make the largest-|loading| entry of every component positive."""
    comps = np.array(components, dtype=np.float64, copy=True)
    idx = np.argmax(np.abs(comps), axis=1)
    signs = np.sign(comps[np.arange(comps.shape[0]), idx])
    signs[signs == 0] = 1.0
    comps *= signs[:, None]
    if embeddings is None:
        return comps, None
    emb = np.array(embeddings, dtype=np.float64, copy=True) * signs[None, :]
    return comps, emb


def principal_angles(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Principal angles (radians) between the column spaces of a and b."""
    qa, _ = np.linalg.qr(np.asarray(a, dtype=np.float64))
    qb, _ = np.linalg.qr(np.asarray(b, dtype=np.float64))
    s = np.linalg.svd(qa.T @ qb, compute_uv=False)
    return np.arccos(np.clip(s, -1.0, 1.0))


def per_component_angles(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Angle (radians) between matching columns of a and b, sign-agnostic."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = np.abs(np.sum(a * b, axis=0))
    den = np.linalg.norm(a, axis=0) * np.linalg.norm(b, axis=0)
    return np.arccos(np.clip(num / np.maximum(den, 1e-300), 0.0, 1.0))


def round_to_bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (round-to-nearest-even), returned as f32."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    r = ((u + rounding) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def round_to_f16(x) -> np.ndarray:
    return np.asarray(x, dtype=np.float32).astype(np.float16).astype(np.float32)


# --------------------------------------------------------------------------
# Seeded Gaussian test matrix: restatement of the device generator
# --------------------------------------------------------------------------

_PHILOX_M0 = np.uint64(0xD2511F53)
_PHILOX_M1 = np.uint64(0xCD9E8D57)
_PHILOX_W0 = np.uint64(0x9E3779B9)
_PHILOX_W1 = np.uint64(0xBB67AE85)
_MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr0, ctr1, key0: int, key1: int, ctr2=0, ctr3=0):
    """Philox4x32-10 (Salmon et al., SC'11) on arrays of counters."""
    c0 = np.asarray(ctr0, dtype=np.uint64) & _MASK32
    c1 = np.asarray(ctr1, dtype=np.uint64) & _MASK32
    c2 = (np.zeros_like(c0) + np.uint64(ctr2)) & _MASK32
    c3 = (np.zeros_like(c0) + np.uint64(ctr3)) & _MASK32
    k0 = np.uint64(key0 & 0xFFFFFFFF)
    k1 = np.uint64(key1 & 0xFFFFFFFF)
    for _ in range(10):
        p0 = _PHILOX_M0 * c0
        p1 = _PHILOX_M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK32
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & _MASK32, lo1, (hi0 ^ c3 ^ k1) & _MASK32, lo0
        k0 = (k0 + _PHILOX_W0) & _MASK32
        k1 = (k1 + _PHILOX_W1) & _MASK32
    return c0, c1, c2, c3


def gaussian_omega(n_vars: int, k: int, seed: int) -> np.ndarray:
    """Seeded N(0,1) test matrix, ``n_vars x k`` (float32 values, FP64 array).

    Element (i, j) sits at flat column-major index ``e = j * n_vars + i``.  Pair
    ``p = e // 2`` draws one Philox4x32-10 block with counter (p_lo, p_hi, 0, 0)
    and key (seed_lo, seed_hi); two 53-bit uniforms in (0, 1) feed Box-Muller
    in FP64, ``z0`` for even e and ``z1`` for odd e, rounded to float32.
    """
    n = n_vars * k
    e = np.arange(n, dtype=np.uint64)
    p = e >> np.uint64(1)
    x0, x1, x2, x3 = philox4x32_10(p & _MASK32, p >> np.uint64(32),
                                   seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    a = ((x0 << np.uint64(32)) | x1) >> np.uint64(11)
    b = ((x2 << np.uint64(32)) | x3) >> np.uint64(11)
    u1 = (a.astype(np.float64) + 0.5) * 2.0 ** -53
    u2 = (b.astype(np.float64) + 0.5) * 2.0 ** -53
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.where((e & np.uint64(1)) == 0, r * np.cos(2.0 * np.pi * u2), r * np.sin(2.0 * np.pi * u2))
    z = z.astype(np.float32).astype(np.float64)
    return z.reshape(k, n_vars).T.copy()


# --------------------------------------------------------------------------
# Upstream producers (scx-gpu/kernels/normalize_log1p.cu:17-140 dispatched by
# gpu_apply_fused_ops, scx-gpu/src/gpu_preprocess.rs:340-391; the CPU
# counterpart scx-engine fused_normalize_log1p forms value_f64 * factor, rounds
# to f32 and takes ln_1p) and the column projection of ProjectedShardSource
# (scx-accel/src/projected_source.rs:28-80 over scx_engine::project_csr)
# --------------------------------------------------------------------------

def normalize_log1p(csr: Csr, target_sum=1e4, log1p=True, row_factors=None) -> np.ndarray:
    """New FP32 values: per row v * target_sum / rowsum (FP64 factor, result
    rounded to f32; rows summing to zero untouched), then log1p, then the
    explicit per-row factor."""
    v = csr.data.astype(np.float64)
    rows = csr.row_ids()
    out = csr.data.astype(np.float32).copy()
    if target_sum and target_sum > 0:
        rs = np.bincount(rows, weights=v, minlength=csr.shape[0])
        nz = rs[rows] != 0.0
        scaled = (v * (target_sum / np.where(rs == 0.0, 1.0, rs))[rows]).astype(np.float32)
        out = np.where(nz, scaled, out)
        if log1p:
            out = np.where(nz, np.log1p(out.astype(np.float64)).astype(np.float32), out)
    elif log1p:
        out = np.log1p(out.astype(np.float64)).astype(np.float32)
    if row_factors is not None:
        out = (out * np.asarray(row_factors, dtype=np.float32)[rows]).astype(np.float32)
    return out


def project_columns(csr: Csr, cols) -> Csr:
    """Keep the sorted unique columns ``cols``; column cols[i] becomes i."""
    cols = np.asarray(cols, dtype=np.int64)
    cmap = np.full(csr.shape[1], -1, dtype=np.int64)
    cmap[cols] = np.arange(len(cols))
    new = cmap[csr.indices.astype(np.int64)]
    keep = new >= 0
    rows = csr.row_ids()[keep]
    indptr = np.r_[0, np.cumsum(np.bincount(rows, minlength=csr.shape[0]))].astype(np.int64)
    return Csr(indptr, new[keep].astype(np.int32), csr.data[keep], (csr.shape[0], len(cols)))


# --------------------------------------------------------------------------
# PFlog (v4) baseline-aware PCA (scx-accel/src/pflog.rs:122-193,
# scx-accel/src/pca/cpu.rs:618-882)
# --------------------------------------------------------------------------

def pflog_prepare(csr: Csr, four_alpha: float):
    """delta = log1p(four_alpha * x) at the stored entries (FP64, rounded to
    f32 as the reference stores it) and b_i = -(1/D) sum_j delta_ij in FP64
    (pflog_baseline_from_raw, pflog.rs:122-193)."""
    x = csr.data.astype(np.float64)
    if not np.all(np.isfinite(x)):
        raise ValueError("PFlog input contains a non-finite value")
    if np.any(x < 0):
        raise ValueError("PFlog: negative count")
    d = np.log1p(four_alpha * x)
    base = -np.bincount(csr.row_ids(), weights=d, minlength=csr.shape[0]) / csr.shape[1]
    return d.astype(np.float32), base


def pflog_total_variance(col_sum_sq_delta, colmean_delta, baseline, n_obs: int, n_vars: int) -> float:
    """Closed form of pflog_total_variance (cpu.rs:689-786)."""
    s_dd = float(np.sum(col_sum_sq_delta))
    b2 = float(np.sum(np.asarray(baseline) ** 2))
    denom = max(n_obs - 1.0, 1.0)
    if colmean_delta is None:
        tss = s_dd - n_vars * b2
    else:
        mu = np.asarray(colmean_delta) + float(np.sum(baseline)) / max(n_obs, 1)
        tss = s_dd - n_vars * b2 - n_obs * float(np.sum(mu * mu))
    return max(tss / denom, 0.0)


def pflog_pca(delta: Csr, baseline, n_components: int, n_oversamples: int, n_power_iterations: int,
              zero_center: bool, omega, ordering: str = "gpu"):
    """Randomized PCA of Z = delta + b 1^T with the offset products
    streaming_spmm_forward_offset / streaming_spmm_transpose_offset
    (cpu.rs:618-687) and the loop of pflog_pca_with_depth (cpu.rs:815-882);
    explicit Omega, GPU step order by default (as randomized_pca)."""
    n_obs, n_vars = delta.shape
    validate_inputs(n_obs, n_vars, n_components)
    k = effective_k(n_obs, n_vars, n_components, n_oversamples)
    b = np.asarray(baseline, dtype=np.float64)
    omega = np.asarray(omega, dtype=np.float64)
    col_sums, col_sum_sq = col_sums_and_sum_sq(delta)
    colmean = col_sums / n_obs if zero_center else None
    means = colmean + b.mean() if zero_center else None

    def fwd(m):  # (delta + b 1^T - 1 mu^T) m
        return spmm_forward(delta, m, means) + np.outer(b, m.sum(axis=0))

    def tr(q):  # (delta + b 1^T - 1 mu^T)^T q
        return spmm_transpose(delta, q, means) + (b @ q)[None, :]

    q = qr_thin_q(fwd(omega))
    for _ in range(n_power_iterations):
        z = tr(q)
        if ordering == "gpu" or n_power_iterations > 2:
            z = qr_thin_q(z)
        q = qr_thin_q(fwd(z))
    bm = tr(q)
    total_var = pflog_total_variance(col_sum_sq, colmean, b, n_obs, n_vars)
    res = build_pca_result(q, bm, n_components, n_obs, total_var)
    res["mean"] = means
    res["total_var"] = total_var
    res["k"] = k
    return res
