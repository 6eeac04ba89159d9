"""Argument checks of the Python mirror (scx_b200.accel) on CPU: the shape and
option errors the reference's Python layer raises as ValueError
(pyscx/src/accel/pca.rs) come back as ValueError here too, before any device
work, and the C ABI's own parameter validation surfaces the same way."""

import numpy as np
import pytest

from scx_b200 import accel


def _csr(n=20, g=8, seed=0):
    rng = np.random.default_rng(seed)
    dense = (rng.random((n, g)) < 0.4) * rng.random((n, g))
    ip = np.r_[0, np.cumsum((dense != 0).sum(1))].astype(np.int64)
    rows, cols = np.nonzero(dense)
    return ip, cols.astype(np.int32), dense[rows, cols].astype(np.float32), (n, g)


@pytest.mark.parametrize("kw,match", [
    (dict(qr_method="lu"), "Invalid qr_method"),
    (dict(math_mode="tf32_everywhere"), "Invalid math_mode"),
    (dict(spmm_policy="fastest"), "Invalid spmm_policy"),
])
def test_invalid_options(kw, match):
    ip, ix, vv, shape = _csr()
    with pytest.raises(ValueError, match=match):
        accel.randomized_pca(ip, ix, vv, shape, n_components=3, **kw)


def test_indptr_length_must_be_n_obs_plus_one():
    ip, ix, vv, shape = _csr()
    with pytest.raises(ValueError, match="indptr must have n_obs"):
        accel.randomized_pca(ip[:-1], ix, vv, shape, n_components=3)


def test_indices_and_values_lengths_must_agree():
    ip, ix, vv, shape = _csr()
    with pytest.raises(ValueError, match="lengths differ"):
        accel.randomized_pca(ip, ix[:-1], vv, shape, n_components=3)


def test_omega_shape_is_checked():
    ip, ix, vv, shape = _csr()
    with pytest.raises(ValueError, match="omega must have shape"):
        accel.randomized_pca(ip, ix, vv, shape, n_components=3, n_oversamples=2,
                             omega=np.zeros((shape[1], 4)))


@pytest.mark.parametrize("device,ok", [("gpu", 0), ("auto", 0), ("gpu:1", 1)])
def test_device_strings(device, ok):
    assert accel._resolve_device(device) == ok


@pytest.mark.parametrize("device,match", [("cpu", "GPU path only"), ("tpu", "Invalid device")])
def test_device_strings_rejected(device, match):
    with pytest.raises(ValueError, match=match):
        accel._resolve_device(device)


@pytest.mark.parametrize("n_components", [0, 9])
def test_component_count_checked_by_the_library(n_components):
    # n_comps = 0 and n_comps > min(n_obs, n_vars) are shape errors (cpu.rs:979-997)
    ip, ix, vv, shape = _csr()
    with pytest.raises(ValueError):
        accel.randomized_pca(ip, ix, vv, shape, n_components=n_components)


def test_host_bf16_values_pass_by_pointer():
    """Host BF16 values (a torch CPU bfloat16 tensor) reach the C ABI as
    values_dtype BF16 in host memory, without a conversion copy."""
    import torch

    from scx_b200 import _lib

    ip, ix, vv, shape = _csr()
    t = torch.from_numpy(vv).to(torch.bfloat16)
    csr, keep, mem, dev = accel._prepare_csr(torch.from_numpy(ip), torch.from_numpy(ix), t, shape)
    assert mem == _lib.MEM_HOST and dev is None
    assert csr.values_dtype == _lib.BF16 and csr.values == t.data_ptr()
    assert csr.nnz == len(vv)
    with pytest.raises(ValueError, match="indptr must have n_obs"):
        accel._prepare_csr(ip[:-1], ix, t, shape)
