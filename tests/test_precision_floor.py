"""CPU tests of the FP32 arithmetic floor of the precision configuration, on the exact column reduction of the
384x384x192 channel (tests/channel_column.py: the paired dense kernel's arithmetic emulated operation by operation):

- with the momentum rounded at every operation, FP32 arithmetic alone drifts away from FP64 by more than the 1e-4
  target after the 20,000 steps (the stored values' rounding contributes less than 1e-6: the drift is the rounding of
  the momentum sums and of j + F, which the force changes by a few hundred ulps per step, every step alike);
- with the kernel's two-number momentum (TwoSum of the momentum sums and of j + F, the low parts added to the odd
  part of every direction) the same arithmetic stays within 3e-5 of FP64, the bound the GPU storage tests use for
  FP32 storage.

The FP64 column is also checked against the start-up series of the channel."""
import numpy as np
import pytest

import channel_column as cc
from cases import CHANNEL_G, CHANNEL_STEPS, CHANNEL_TAU, channel_startup_profile

NZ = 192


def relative(u, ref):
    return np.linalg.norm(u[1:-1] - ref[1:-1])/np.linalg.norm(ref[1:-1])


@pytest.fixture(scope='module')
def fp64_column():
    return cc.run(NZ, CHANNEL_STEPS, np.float64, tau=CHANNEL_TAU, gx=CHANNEL_G)


def test_fp64_column_follows_startup_series(fp64_column):
    exact = channel_startup_profile(NZ, CHANNEL_TAU, CHANNEL_G, CHANNEL_STEPS)
    assert relative(fp64_column, exact) <= 1.5e-4


def test_rounded_momentum_floor_is_above_target(fp64_column):
    u = cc.run(NZ, CHANNEL_STEPS, np.float32, tau=CHANNEL_TAU, gx=CHANNEL_G, compensated=False)
    error = relative(u, fp64_column)
    print('FP32 arithmetic, rounded momentum: %.3e' % error)
    assert 1e-4 < error < 5e-4
    # a bias of the whole profile, not noise
    bias = (u - fp64_column)[1:-1].mean()/fp64_column[1:-1].mean()
    assert bias > 0.8*error


def test_compensated_momentum_meets_target(fp64_column):
    u = cc.run(NZ, CHANNEL_STEPS, np.float32, tau=CHANNEL_TAU, gx=CHANNEL_G, compensated=True)
    error = relative(u, fp64_column)
    print('FP32 arithmetic, two-number momentum: %.3e' % error)
    assert error <= 3e-5
