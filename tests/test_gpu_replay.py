"""Repeated plan runs replayed as a CUDA graph (needs a B200).

A plan run again with the same power iterations, seed, omega and embeddings
buffer records its run on the second occurrence and replays the graph from
then on.  The replay must give the bits of the plain launches, count the same
kernels, follow a change of seed, and stay off under stage profiling or
SCXPCA_GRAPH=0.
"""

import numpy as np
import pytest

from scx_b200 import accel
from scx_b200.synth import synth_nb_csr

pytestmark = pytest.mark.gpu


def _plan(mode):
    n, g = 6000, 800
    ip, ix, vv = synth_nb_csr(n, g, seed=21, loc=-2.2)
    return accel.Plan(ip, ix, vv, (n, g), n_components=20, n_oversamples=10, n_power_iterations=3,
                      zero_center=True, scale=True, clip_max=10.0, seed=5, math_mode=mode)


def _same(a, b):
    np.testing.assert_array_equal(a.embeddings, b.embeddings)
    np.testing.assert_array_equal(a.singular_values, b.singular_values)
    np.testing.assert_array_equal(a.components, b.components)


@pytest.mark.parametrize("mode", ["mixed_bf16", "strict_fp32"])
def test_replayed_runs_equal_plain_launches(mode, monkeypatch):
    plan = _plan(mode)
    counts = []
    runs = []
    for _ in range(4):  # plain, recorded, replayed, replayed
        before = plan.profile()["kernel_launches"]
        runs.append(plan.run())
        counts.append(plan.profile()["kernel_launches"] - before)
    for r in runs[1:]:
        _same(runs[0], r)
    assert len(set(counts)) == 1 and counts[0] > 0, counts
    # a new seed: plain, then recorded and replayed again
    other = [plan.run(seed=9) for _ in range(3)]
    for r in other[1:]:
        _same(other[0], r)
    assert not np.array_equal(other[0].singular_values, runs[0].singular_values)
    back = plan.run()
    _same(runs[0], back)
    plan.close()
    # the plain path everywhere
    monkeypatch.setenv("SCXPCA_GRAPH", "0")
    plain = _plan(mode)
    for _ in range(3):
        _same(runs[0], plain.run())
    plain.close()


def test_profiled_runs_stay_plain_and_time_every_stage():
    plan = _plan("mixed_bf16")
    r0 = plan.run()
    plan.run()
    plan.set_profiling(True)
    for _ in range(2):
        r = plan.run()
        _same(r0, r)
    prof = plan.profile()
    assert prof["runs"] == 2
    assert prof["stages"]["forward"]["launches"] > 0 and prof["stages"]["forward"]["device_ms"] > 0
    plan.close()
