"""FP64 CPU restatement of the truncated-SVD adjoint -- TEST INFRASTRUCTURE ONLY.

Checks the CUDA backward pass (scxpca_plan_backward).  Nothing in the product
imports this module.  The reference PCA (scx-gpu/src/gpu_pca.rs:706-763,
scx-accel/src/pca/cpu.rs:887-952) is not differentiable, so there is no
reference gradient to restate; the gradient is pinned instead against
automatic differentiation of ``torch.linalg.svd`` in FP64 and against central
finite differences of the dense FP64 loss (tests/test_oracle.py).

Function (dense, exact): X~ = (X - 1 c^T) diag(s) with X the CSR matrix made
dense, V_c the top-c right singular vectors of X~, scores S = X~ V_c, and the
loss L = sum(W * S**2) (invariant to the sign of each singular vector).

Adjoint, for dL/dS = G:  with H = X~^T G, C = X~^T X~ = V diag(lambda) V^T
(all n_vars eigenpairs), a_i = sum_{j != i} v_j (v_j^T h_i) / (lambda_i -
lambda_j) and A = [a_1 .. a_c],
    dL/dX~ = D = (G + X~ A) V_c^T + S A^T,
    dL/dx_rj (stored) = D_rj s_j,
    dL/dc_j = -s_j sum_r D_rj,
    dL/ds_j = sum_r D_rj (x_rj - c_j).
"""

from __future__ import annotations

import numpy as np


def dense(indptr, indices, values, shape) -> np.ndarray:
    n, g = int(shape[0]), int(shape[1])
    X = np.zeros((n, g), dtype=np.float64)
    rows = np.repeat(np.arange(n), np.diff(np.asarray(indptr)))
    np.add.at(X, (rows, np.asarray(indices)), np.asarray(values, dtype=np.float64))
    return X


def affine(X: np.ndarray, center, scale) -> np.ndarray:
    Xt = X.copy()
    if center is not None:
        Xt -= np.asarray(center, dtype=np.float64)[None, :]
    if scale is not None:
        Xt *= np.asarray(scale, dtype=np.float64)[None, :]
    return Xt


def top_right_vectors(Xt: np.ndarray, c: int) -> np.ndarray:
    _, _, vt = np.linalg.svd(Xt, full_matrices=False)
    return vt[:c].T


def scores(Xt: np.ndarray, c: int) -> np.ndarray:
    return Xt @ top_right_vectors(Xt, c)


def loss(Xt: np.ndarray, W: np.ndarray, c: int) -> float:
    S = scores(Xt, c)
    return float(np.sum(W * S * S))


def grad_wrt_matrix(Xt: np.ndarray, grad_of_scores, c: int) -> np.ndarray:
    """dL/dX~ from the full eigendecomposition of X~^T X~.

    ``grad_of_scores(S)`` returns dL/dS for scores S computed with this
    function's own singular vectors (G must follow the same sign choice)."""
    lam, V = np.linalg.eigh(Xt.T @ Xt)
    order = np.argsort(lam)[::-1]
    lam, V = lam[order], V[:, order]
    Vc = V[:, :c]
    S = Xt @ Vc
    G = grad_of_scores(S)
    H = Xt.T @ G
    coef = V.T @ H  # (g, c): v_j^T h_i
    gap = lam[None, :c] - lam[:, None]  # (g, c): lambda_i - lambda_j
    with np.errstate(divide="ignore", invalid="ignore"):
        F = np.where(np.abs(gap) > 0, coef / gap, 0.0)
    F[np.arange(c), np.arange(c)] = 0.0
    A = V @ F
    return (G + Xt @ A) @ Vc.T + S @ A.T


def grads(indptr, indices, values, shape, center, scale, W, c):
    """(dL/dvalues at the stored entries, dL/dcenter, dL/dscale) in FP64."""
    X = dense(indptr, indices, values, shape)
    Xt = affine(X, center, scale)
    D = grad_wrt_matrix(Xt, lambda S: 2.0 * W * S, c)
    g = int(shape[1])
    s = np.ones(g) if scale is None else np.asarray(scale, dtype=np.float64)
    cv = np.zeros(g) if center is None else np.asarray(center, dtype=np.float64)
    rows = np.repeat(np.arange(int(shape[0])), np.diff(np.asarray(indptr)))
    gv = D[rows, np.asarray(indices)] * s[np.asarray(indices)]
    gc = -s * D.sum(axis=0)
    gs = (D * (X - cv[None, :])).sum(axis=0)
    return gv, gc, gs


def planted_csr(n: int, g: int, rank: int, density: float, seed: int, top: float = 40.0,
                ratio: float = 0.95, noise: float = 0.3):
    """Sparse matrix whose leading spectrum is a planted rank-``rank`` component.

    The stored entries are those of a Bernoulli(density) mask; their values are
    the planted component U diag(sigma) V^T (sigma geometric from ``top`` with
    step ``ratio``, so neighbouring singular values differ by ~(1 - ratio)),
    scaled by 1 / density so the masked matrix keeps the planted spectrum in
    expectation, plus N(0, noise) entries.  Rows sorted by gene, float32.
    """
    rng = np.random.default_rng(seed)
    U = np.linalg.qr(rng.standard_normal((n, rank)))[0]
    V = np.linalg.qr(rng.standard_normal((g, rank)))[0]
    sig = top * ratio ** np.arange(rank) * np.sqrt(n * g / (n + g))
    L = (U * sig) @ V.T / np.sqrt(n * g / (n + g))
    mask = rng.random((n, g)) < density
    vals = (L / density + noise * rng.standard_normal((n, g)))[mask]
    rows, cols = np.nonzero(mask)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(indptr, rows + 1, 1)
    indptr = np.cumsum(indptr)
    return indptr, cols.astype(np.int32), vals.astype(np.float32)
