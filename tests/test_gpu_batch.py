"""Batched sub-PCAs (scxpca_batch_*): every row segment gets its own centred
randomized PCA; the single graph launch, the plain per-segment launches and a
standalone one-shot PCA of each segment must agree, and each segment must
match the FP64 oracle run on that segment alone with the same test matrix.

Tolerances: graph vs plain launches bit-identical on the tensor-core path
(fixed-order accumulation), 1e-6 relative on the strict FP32 path (its
CUDA-core transposed product adds in shared-memory atomics, in no fixed
order); vs a standalone call 1e-6 relative on the
singular values; vs the FP64 oracle 1e-4 relative (strict FP32, and BF16 on
the BF16-rounded values).
"""

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu

SIZES = (300, 1000, 2500, 700, 4100, 129)
N_VARS = 300


def _clusters():
    parts = [synth_nb_csr(n, N_VARS, seed=100 + i, loc=-2.0) for i, n in enumerate(SIZES)]
    indptr = [np.zeros(1, dtype=np.int64)]
    base = 0
    for ip, _, _ in parts:
        indptr.append(ip[1:] + base)
        base += ip[-1]
    ip = np.concatenate(indptr)
    ix = np.concatenate([p[1] for p in parts])
    vv = np.concatenate([p[2] for p in parts])
    offs = np.r_[0, np.cumsum(SIZES)]
    return ip, ix, vv, offs


@pytest.mark.parametrize("mode", ["strict_fp32", "mixed_bf16"])
def test_batch_graph_plain_standalone_and_oracle_agree(mode):
    import torch

    ip, ix, vv, offs = _clusters()
    n = int(offs[-1])
    dev = "cuda:0"
    tv = torch.from_numpy(vv).to(dev)
    if mode == "mixed_bf16":
        tv = tv.to(torch.bfloat16)
    tip, tix = torch.from_numpy(ip).to(dev), torch.from_numpy(ix).to(dev)
    nc, over, q, seed = 10, 10, 3, 5
    b = accel.Batch(tip, tix, tv, (n, N_VARS), offs, n_components=nc, n_oversamples=over,
                    n_power_iterations=q, seed=seed, math_mode=mode, branches=0)
    assert 1 <= abs(b.branches) <= len(SIZES) and b.graph_nodes > 0 and b.tuned_ms
    assert any(t < 0 for t in b.tuned_ms) and any(t > 0 for t in b.tuned_ms)  # both schedules timed
    emb_g, comp_g, sv_g, vr_g, _ = b.run(use_graph=True)
    emb_p, comp_p, sv_p, vr_p, _ = b.run(use_graph=False)
    emb_g2, _, sv_g2, _, _ = b.run(use_graph=True)  # a second launch of the same graph
    b.close()
    # every path adds in a fixed order: the graph launches equal the plain
    # per-segment launches bit for bit
    np.testing.assert_array_equal(sv_g, sv_p)
    np.testing.assert_array_equal(sv_g2, sv_g)
    np.testing.assert_array_equal(emb_g, emb_p)
    np.testing.assert_array_equal(comp_g, comp_p)
    np.testing.assert_array_equal(vr_g, vr_p)
    k = nc + over
    om = rpca.gaussian_omega(N_VARS, k, seed)
    for s in range(len(SIZES)):
        r0, r1 = offs[s], offs[s + 1]
        e0, e1 = ip[r0], ip[r1]
        sip, six, svv = ip[r0:r1 + 1] - e0, ix[e0:e1], vv[e0:e1]
        if mode == "mixed_bf16":
            svv = torch.from_numpy(svv).to(torch.bfloat16).float().numpy()
        one = accel.randomized_pca(torch.from_numpy(sip).to(dev), torch.from_numpy(six).to(dev),
                                   tv[e0:e1], (r1 - r0, N_VARS), n_components=nc, n_oversamples=over,
                                   n_power_iterations=q, seed=seed, math_mode=mode)
        np.testing.assert_allclose(sv_g[s], one.singular_values, rtol=1e-6)
        ref = rpca.randomized_pca(rpca.Csr(sip, six, svv, (r1 - r0, N_VARS)), nc, over, q, True, om)
        rel = np.abs(sv_g[s] - ref["singular_values"]) / ref["singular_values"]
        assert rel.max() < 1e-4, (s, rel.max())


def test_batch_rejects_bad_segments():
    import torch

    ip, ix, vv, offs = _clusters()
    n = int(offs[-1])
    dev = "cuda:0"
    args = (torch.from_numpy(ip).to(dev), torch.from_numpy(ix).to(dev), torch.from_numpy(vv).to(dev),
            (n, N_VARS))
    with pytest.raises(ValueError, match="end at n_obs"):
        accel.Batch(*args, offs[:-1], n_components=5, math_mode="strict_fp32")
    bad = offs.copy()
    bad[2] = bad[1]
    with pytest.raises(ValueError, match="increase strictly"):
        accel.Batch(*args, bad, n_components=5, math_mode="strict_fp32")


@pytest.mark.parametrize("branches", [-1, -3])
def test_lockstep_tensor_core_products_ld64(branches):
    """k = 60 (ld 64) under the lockstep schedule: the forward product, the
    transposed product and the Gram of all segments run as one launch each
    (segments of 2 to 33 row tiles, odd and even).  Their results must equal
    the plain per-segment launches bit for bit and match the FP64 oracle."""
    import torch

    ip, ix, vv, offs = _clusters()
    n = int(offs[-1])
    dev = "cuda:0"
    tv = torch.from_numpy(vv).to(dev).to(torch.bfloat16)
    tip, tix = torch.from_numpy(ip).to(dev), torch.from_numpy(ix).to(dev)
    nc, over, q, seed = 50, 10, 2, 3
    b = accel.Batch(tip, tix, tv, (n, N_VARS), offs, n_components=nc, n_oversamples=over,
                    n_power_iterations=q, seed=seed, math_mode="mixed_bf16", branches=branches)
    assert b.lockstep
    emb_g, comp_g, sv_g, vr_g, _ = b.run(use_graph=True)
    emb_p, comp_p, sv_p, _, _ = b.run(use_graph=False)
    emb_g2, _, sv_g2, _, _ = b.run(use_graph=True)
    b.close()
    np.testing.assert_array_equal(sv_g, sv_p)
    np.testing.assert_array_equal(sv_g2, sv_g)
    np.testing.assert_array_equal(emb_g, emb_p)
    np.testing.assert_array_equal(emb_g2, emb_g)
    np.testing.assert_array_equal(comp_g, comp_p)
    om = rpca.gaussian_omega(N_VARS, nc + over, seed)
    for s in range(len(SIZES)):
        r0, r1 = offs[s], offs[s + 1]
        e0, e1 = ip[r0], ip[r1]
        svv = torch.from_numpy(vv[e0:e1]).to(torch.bfloat16).float().numpy()
        ref = rpca.randomized_pca(rpca.Csr(ip[r0:r1 + 1] - e0, ix[e0:e1], svv, (r1 - r0, N_VARS)), nc, over, q,
                                  True, om)
        rel = np.abs(sv_g[s] - ref["singular_values"]) / ref["singular_values"]
        assert rel.max() < 1e-4, (s, rel.max())
