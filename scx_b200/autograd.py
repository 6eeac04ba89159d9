"""Differentiable PCA scores: a ``torch.autograd.Function`` over the C ABI.

``pca_scores`` returns S = X~ V (n_obs x n_components), the PCA embeddings of
X~ = (X - 1 center^T) diag(scale) for a CUDA CSR matrix X, differentiable
with respect to the stored values of X and the per-gene ``center`` and
``scale`` vectors.  The forward pass is the plan's randomized PCA
(scxpca_plan_create_affine + scxpca_plan_run); the backward pass is the
hand-written truncated-SVD adjoint scxpca_plan_backward (an SDDMM over the
stored entries plus the gradients of the two gene vectors).  The reference's
PCA (scx-gpu/src/gpu_pca.rs:706-763) has no gradient; the forward arguments
keep its names and meaning.

Sign convention: singular vectors are defined up to sign, so only losses that
are invariant to flipping the sign of a score column (for example
sum(W * S**2)) have a well-defined gradient.
"""

from __future__ import annotations

import torch

from . import accel


class _PcaScores(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, center, scale, indptr, indices, shape, opts):
        plan = accel.Plan(indptr, indices, values.detach(), shape,
                          center=None if center is None else center.detach(),
                          gene_scale=None if scale is None else scale.detach(), **opts["plan"])
        scores = torch.empty((int(shape[0]), plan.n_components), dtype=torch.float32,
                             device=values.device)
        plan.run(embeddings_out=scores, omega=opts["omega"])
        ctx.plan = plan
        ctx.solve_iterations = opts["solve_iterations"]
        ctx.value_dtype = values.dtype
        ctx.center_dtype = None if center is None else center.dtype
        ctx.scale_dtype = None if scale is None else scale.dtype
        ctx.save_for_backward(scores)
        return scores

    @staticmethod
    def backward(ctx, grad_scores):
        (scores,) = ctx.saved_tensors
        plan = ctx.plan
        try:
            gv, gc, gs = plan.backward(scores, grad_scores, ctx.solve_iterations)
        finally:
            plan.close()
            ctx.plan = None
        gv = gv.to(ctx.value_dtype)
        gc = None if ctx.center_dtype is None else gc.to(ctx.center_dtype)
        gs = None if ctx.scale_dtype is None else gs.to(ctx.scale_dtype)
        return gv, gc, gs, None, None, None, None


def pca_scores(indptr, indices, values, shape, center=None, scale=None, n_components: int = 50,
               n_oversamples: int = 10, n_power_iterations: int = 4, seed: int = 0, omega=None,
               qr_method: str = "householder", math_mode: str = "strict_fp32",
               solve_iterations: int = 8, device: int | None = None):
    """Differentiable randomized-PCA scores of a CUDA CSR matrix.

    ``values`` (nnz,), ``center`` and ``scale`` (n_vars,) may require grad;
    ``center=None`` means no centring and ``scale=None`` a unit scale.  The
    plan is built in the forward pass and released after the backward pass.
    ``solve_iterations`` bounds the conjugate-gradient steps of the adjoint
    (each one X~^T X~ product) for the part of the singular-vector derivatives
    outside the sketch subspace.
    """
    if not (torch.is_tensor(values) and values.is_cuda):
        raise ValueError("pca_scores needs CUDA tensors (the CSR stays on the device)")
    dev = values.device.index if device is None else device
    opts = {
        "plan": dict(n_components=n_components, n_oversamples=n_oversamples,
                     n_power_iterations=n_power_iterations, seed=seed, qr_method=qr_method,
                     math_mode=math_mode, device=dev or 0),
        "omega": omega,
        "solve_iterations": int(solve_iterations),
    }
    return _PcaScores.apply(values, center, scale, indptr, indices, tuple(shape), opts)
