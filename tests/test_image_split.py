"""Error bound of the 16-bit image the tensor-core path multiplies.

The dense operand of both sparse products (V, and the tall Y / Q) enters the
tensor cores as an image that holds, for each value x, hi = round16(x) and
lo = round16(x - hi) in adjacent columns; the MMA multiplies both and the
epilogue adds the two halves.  The only quantity the mixed-precision path
rounds to 16 bits is then the matrix value itself.  This CPU test checks the
bound that design rests on, with torch's round-to-nearest-even conversions
(the same rounding as the kernels' cvt.rn):

* bf16: |x - (hi + lo)| <= 2^-16 |x| (two 8-bit significands);
* f16 : |x - (hi + lo)| <= 2^-21 |x| for |x| >= 2^-3; for values near
  1e-3 (a tall operand's entries at a million cells) the lo half falls into
  f16's subnormal range and the pair is exact to half a subnormal step (2^-25).
"""

import numpy as np
import pytest
import torch


def _split(x, dtype):
    t = torch.from_numpy(x)
    hi = t.to(dtype)
    lo = (t - hi.float()).to(dtype)
    return hi.double().numpy(), lo.double().numpy()


@pytest.mark.parametrize("scale", [1e-3, 1.0, 30.0])
def test_bf16_pair_keeps_16_bits(scale):
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(200_000) * scale).astype(np.float32)
    hi, lo = _split(x, torch.bfloat16)
    err = np.abs(x.astype(np.float64) - (hi + lo))
    assert (err <= 2.0 ** -16 * np.abs(x) + 1e-45).all()
    # the hi half alone is only an 8-bit significand
    assert np.max(np.abs(x - hi) / np.abs(x)) > 2.0 ** -10


def test_f16_pair_error():
    rng = np.random.default_rng(1)
    x = rng.uniform(0.125, 8.0, 200_000).astype(np.float32) * rng.choice([-1, 1], 200_000)
    hi, lo = _split(x, torch.float16)
    err = np.abs(x.astype(np.float64) - (hi + lo))
    assert (err <= 2.0 ** -21 * np.abs(x)).all()
    # tall operands near 1/sqrt(n) at n = 1e6: the lo half reaches f16's
    # subnormal range, so the pair is exact only to the subnormal step
    y = (rng.standard_normal(200_000) * 1e-3).astype(np.float32)
    hi, lo = _split(y, torch.float16)
    assert (np.abs(y.astype(np.float64) - (hi + lo)) <= 2.0 ** -25 + 2.0 ** -21 * np.abs(y)).all()
