"""The give-up path of the bounded pipeline wait (needs a B200).

Every mbarrier wait of the tensor-core kernels is bounded (about 1 s); when
one runs out the block raises its abort flag, the other roles leave their own
waits, the kernel records the wait site and the host turns it into
SCXPCA_TIMEOUT.  scxpca_wait_selftest runs that wait on a barrier that no
thread ever arrives on, with no copy or MMA in flight, so the failure is made
without any fault.  The test checks the status and message, that the wait ran
for its limit (not less), and that a PCA on the same device afterwards runs
normally and matches the oracle.
"""

import time

import numpy as np
import pytest

from oracle import rpca
from scx_b200 import _lib, accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu


def test_wait_that_never_completes_returns_timeout_and_context_stays_usable():
    import torch

    torch.cuda.init()
    t0 = time.perf_counter()
    with pytest.raises(_lib.ScxPcaError) as ei:
        accel.wait_selftest(0)
    waited = time.perf_counter() - t0
    assert ei.value.status == _lib.TIMEOUT
    assert "site 99" in str(ei.value)
    assert 0.2 < waited < 30.0, waited  # ran to its limit (~1 s at 2 GHz), then returned

    # the same context afterwards: no sticky error, a normal PCA matches the oracle
    assert torch.cuda.is_available()
    torch.cuda.synchronize()
    n, g, nc = 2000, 300, 10
    ip, ix, vv = synth_nb_csr(n, g, seed=9, loc=-2.0)
    om = rpca.gaussian_omega(g, nc + 10, seed=0)
    res = accel.randomized_pca(ip, ix, vv, (n, g), n_components=nc, n_oversamples=10, n_power_iterations=4,
                               omega=om, math_mode="strict_fp32")
    ref = rpca.randomized_pca(rpca.Csr(ip, ix, vv, (n, g)), nc, 10, 4, True, om)
    sv = np.asarray(ref["singular_values"])
    np.testing.assert_allclose(res.singular_values, sv, rtol=1e-4)
