"""The device-resident embedding hand-off to a kNN consumer (needs a B200).

The reference's fused path hands gpu_randomized_pca_device's row-major
(n_obs x n_components) f32 device embedding straight to CAGRA
(scx-gpu/src/gpu_pca.rs:775-838 -> scx-accel/src/fused/gpu.rs:36-60,
pca_then_knn_gpu).  Here the contract is: embeddings_memory = DEVICE writes a
caller-owned, row-major, contiguous float32 buffer on the plan's device, in
place (no intermediate host copy), complete when the call returns.  A CUDA
torch tensor passed as the output is that buffer, and DLPack exports it to any
consumer without a copy.  The consumer here is an exact kNN on the device; its
neighbours equal those computed from the host-embedding run of the same PCA.
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu


def _knn(x, k):
    import torch
    d = torch.cdist(x, x)
    d.fill_diagonal_(float("inf"))
    return torch.topk(d, k, dim=1, largest=False).indices


def test_device_embeddings_feed_a_device_knn_without_a_host_copy():
    import torch
    from torch.utils import dlpack

    n, g, nc = 3000, 600, 20
    ip, ix, vv = synth_nb_csr(n, g, seed=4, loc=-2.0)
    om = rpca.gaussian_omega(g, nc + 10, seed=0)
    dev_csr = (torch.from_numpy(ip).cuda(), torch.from_numpy(ix).cuda(), torch.from_numpy(vv).cuda())
    out = torch.full((n, nc), float("nan"), dtype=torch.float32, device="cuda:0")
    ptr = out.data_ptr()
    res = accel.randomized_pca(*dev_csr, (n, g), n_components=nc, n_oversamples=10, n_power_iterations=4,
                               omega=om, embeddings_out=out)
    emb = res.embeddings
    assert emb is out and emb.data_ptr() == ptr  # written in place
    assert emb.is_cuda and emb.dtype == torch.float32 and emb.stride() == (nc, 1)
    assert torch.isfinite(emb).all()
    # zero-copy export to a consumer
    shared = dlpack.from_dlpack(dlpack.to_dlpack(emb))
    assert shared.data_ptr() == ptr
    nbr_dev = _knn(shared, 15).cpu().numpy()
    # the same PCA with host embeddings, neighbours computed from the host copy
    host = accel.randomized_pca(ip, ix, vv, (n, g), n_components=nc, n_oversamples=10, n_power_iterations=4,
                                omega=om)
    np.testing.assert_allclose(emb.cpu().numpy(), host.embeddings, rtol=1e-5, atol=1e-5 * np.abs(host.embeddings).max())
    nbr_host = _knn(torch.from_numpy(host.embeddings).cuda(), 15).cpu().numpy()
    agree = np.mean([len(set(a) & set(b)) / 15 for a, b in zip(nbr_dev, nbr_host)])
    assert agree > 0.99, agree
