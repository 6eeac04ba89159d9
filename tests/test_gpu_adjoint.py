"""Backward pass of the PCA scores on the GPU (scxpca_plan_backward) against
the FP64 adjoint oracle and FP64 central finite differences.

Loss: L = sum(W * S**2), S the n_components scores, W seeded N(0, 1).
Inputs: 2,000 cells x 500 genes slices with a planted low-rank component, so
the singular values that matter are separated by relative gaps >= 1e-3
(asserted) and the randomized forward pass has converged to the exact
truncated SVD the oracle differentiates.

Tolerances (FP32 sparse products, FP64 gene-side algebra): each gradient
vector within 2e-3 relative (2-norm) of the FP64 oracle; directional
derivatives within 2e-3 of the finite differences.
"""

import numpy as np
import pytest

from oracle import adjoint as ad

pytestmark = pytest.mark.gpu

GRAD_RTOL = 2e-3


def _case(n, g, rank, density, c, seed, ratio, noise, top=100.0):
    ip, ix, vv = ad.planted_csr(n, g, rank, density, seed=seed, top=top, ratio=ratio, noise=noise)
    X = ad.dense(ip, ix, vv, (n, g))
    center = X.mean(axis=0)
    scale = 1.0 / (X.std(axis=0, ddof=1) + 0.1)
    s = np.linalg.svd(ad.affine(X, center, scale), compute_uv=False)
    gaps = (s[:c] - s[1:c + 1]) / s[:c]
    assert gaps.min() >= 1e-3, f"planted spectrum not gapped: {gaps.min():.2e}"
    return ip, ix, vv, center, scale


def _gpu_grads(ip, ix, vv, shape, center, scale, W, c, k, q, math_mode="strict_fp32", solve_iterations=8):
    import torch

    from scx_b200.autograd import pca_scores

    dev = "cuda:0"
    tip = torch.from_numpy(ip).to(dev)
    tix = torch.from_numpy(ix).to(dev)
    vals = torch.from_numpy(vv).to(dev)
    if math_mode == "mixed_bf16":
        vals = vals.to(torch.bfloat16)
    vals.requires_grad_(True)
    tc = torch.tensor(center, dtype=torch.float64, device=dev, requires_grad=True)
    ts = torch.tensor(scale, dtype=torch.float64, device=dev, requires_grad=True)
    S = pca_scores(tip, tix, vals, shape, center=tc, scale=ts, n_components=c, n_oversamples=k - c,
                   n_power_iterations=q, seed=1, math_mode=math_mode, solve_iterations=solve_iterations)
    loss = (torch.from_numpy(W).to(dev, torch.float32) * S * S).sum()
    loss.backward()
    return (vals.grad.float().cpu().numpy().astype(np.float64), tc.grad.cpu().numpy(),
            ts.grad.cpu().numpy(), float(loss.detach()))


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name,args,c,k,q", [
    ("sparse_30pct_c10", dict(n=2000, g=500, rank=12, density=0.3, seed=0, ratio=0.97, noise=0.1), 10, 20, 8),
    ("stored_dense_c50", dict(n=2000, g=500, rank=60, density=1.0, seed=1, ratio=0.97, noise=0.05), 50, 60, 6),
])
def test_backward_matches_fp64_adjoint_and_finite_differences(name, args, c, k, q):
    n, g = args["n"], args["g"]
    ip, ix, vv, center, scale = _case(c=c, **args)
    rng = np.random.default_rng(7)
    W = rng.standard_normal((n, c))
    gv, gc, gs, loss = _gpu_grads(ip, ix, vv, (n, g), center, scale, W, c, k, q)
    ov, oc, os_ = ad.grads(ip, ix, vv, (n, g), center, scale, W, c)
    Xt = ad.affine(ad.dense(ip, ix, vv, (n, g)), center, scale)
    assert abs(loss - ad.loss(Xt, W, c)) <= 1e-4 * abs(ad.loss(Xt, W, c))
    assert _rel(gv, ov) < GRAD_RTOL, f"values gradient off by {_rel(gv, ov):.2e}"
    assert _rel(gc, oc) < GRAD_RTOL, f"center gradient off by {_rel(gc, oc):.2e}"
    assert _rel(gs, os_) < GRAD_RTOL, f"scale gradient off by {_rel(gs, os_):.2e}"

    # directional finite differences of the FP64 dense loss
    vv64 = vv.astype(np.float64)

    def L(v, cen, sca):
        return ad.loss(ad.affine(ad.dense(ip, ix, v, (n, g)), cen, sca), W, c)

    eps = 1e-6
    dv, dc, ds = rng.standard_normal(len(vv)), rng.standard_normal(g), rng.standard_normal(g)
    fd_v = (L(vv64 + eps * dv, center, scale) - L(vv64 - eps * dv, center, scale)) / (2 * eps)
    fd_c = (L(vv64, center + eps * dc, scale) - L(vv64, center - eps * dc, scale)) / (2 * eps)
    fd_s = (L(vv64, center, scale + eps * ds) - L(vv64, center, scale - eps * ds)) / (2 * eps)
    for fd, got in ((fd_v, gv @ dv), (fd_c, gc @ dc), (fd_s, gs @ ds)):
        assert abs(fd - got) <= GRAD_RTOL * abs(fd), (fd, got)


def test_backward_mixed_bf16_matches_oracle_on_rounded_values():
    import torch

    n, g, c, k = 2000, 500, 10, 20
    ip, ix, vv, center, scale = _case(n, g, 12, 0.3, c, 0, 0.97, 0.1)
    vb = torch.from_numpy(vv).to(torch.bfloat16).float().numpy()
    W = np.random.default_rng(8).standard_normal((n, c))
    gv, gc, gs, _ = _gpu_grads(ip, ix, vb, (n, g), center, scale, W, c, k, 8, math_mode="mixed_bf16")
    # the mixed path stores the working values x s in bf16: the oracle takes
    # the same rounded matrix, expressed back in the input's units
    s_j = scale[ix]
    xs = torch.from_numpy(vb.astype(np.float64) * s_j).float().to(torch.bfloat16).double().numpy()
    ov, oc, os_ = ad.grads(ip, ix, xs / s_j, (n, g), center, scale, W, c)
    # the value gradient itself is returned in bf16 (the values' dtype)
    assert _rel(gv, ov) < 1e-2
    assert _rel(gc, oc) < GRAD_RTOL
    assert _rel(gs, os_) < GRAD_RTOL


def test_backward_contract_errors():
    import torch

    from scx_b200 import accel

    ip, ix, vv = ad.planted_csr(300, 60, 5, 0.3, seed=2, top=20.0)
    dev = "cuda:0"
    tip, tix, tvv = (torch.from_numpy(a).to(dev) for a in (ip, ix, vv))
    plan = accel.Plan(tip, tix, tvv, (300, 60), n_components=4, n_oversamples=4)
    S = torch.zeros((300, 4), dtype=torch.float32, device=dev)
    with pytest.raises(ValueError, match="completed run"):
        plan.backward(S, S)
    plan.run(embeddings_out=S)
    plan.backward(S, torch.ones_like(S))
    with pytest.raises(ValueError, match="completed run"):  # one backward per run
        plan.backward(S, S)
    plan.close()
    clipped = accel.Plan(tip, tix, tvv, (300, 60), n_components=4, n_oversamples=4, scale=True, clip_max=1.0)
    clipped.run(embeddings_out=S)
    with pytest.raises(RuntimeError, match="clipped"):
        clipped.backward(S, S)
    clipped.close()
