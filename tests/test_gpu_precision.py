"""GPU tests of the storage formats on the precision channel: a 384x384x192 Poiseuille channel between bounce-back
planes z = 0 and z = 191, Guo body force g_x = 5e-7, tau 0.55, started from rest, 20,000 steps, in FP64, FP32, FP16 and
BF16 storage (FP32 collide arithmetic for the last three).  After 20,000 steps the flow is still in start-up
(H^2/nu = 2.2e6 steps), so the analytic reference is the start-up series of the channel with halfway walls.

Errors are relative L2 norms over the fluid nodes, ||u - u_ref||/||u_ref||; the profile error compares the
xy-averaged profiles u_x(z), which removes the node-to-node scatter of the stochastic rounding.  Measured on B200:

    storage    vs FP64     vs analytic   profile vs FP64
    double     0           1.11e-4       0
    single     1.75e-4     2.09e-4       1.75e-4
    half       2.47e-4     2.73e-4       1.00e-4
    bfloat16   1.82e-3     1.82e-3       1.09e-4

The tolerances below are about twice these.  FP32 arithmetic alone drifts by ~1e-4 over 20,000 steps of this flow
(a uniform periodic fluid accelerated by the same force drifts by 2e-4), so no storage format with FP32 collide
arithmetic reaches 1e-4 here; round-to-nearest 16-bit storage stalls the flow (errors 0.22 and 0.88), which the
stochastic rounding of the stores prevents."""
import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from cases import (CHANNEL_G, CHANNEL_SHAPE, CHANNEL_STEPS, CHANNEL_TAU, channel_kernel, channel_startup_profile)

pytestmark = pytest.mark.gpu

TOL_VS_FP64 = {'single': 4e-4, 'half': 5e-4, 'bfloat16': 4e-3}
TOL_PROFILE = {'single': 4e-4, 'half': 2.5e-4, 'bfloat16': 2.5e-4}
TOL_ANALYTIC_FP64 = 2.5e-4


def run_channel(precision, shape=CHANNEL_SHAPE, steps=CHANNEL_STEPS):
    kernel = channel_kernel(shape, precision)
    for s in range(steps):
        kernel.begin_step(s)
        kernel.execute(s)
    _, velocity = kernel.get_fluid_fields()
    kernel.close()
    nx, ny, nz = shape
    return velocity.reshape(nz, ny, nx, 3)[1:-1]


@pytest.fixture(scope='module')
def channel_runs():
    return {p: run_channel(p) for p in ('double', 'single', 'half', 'bfloat16')}


def relative(u, ref):
    return np.linalg.norm(u - ref)/np.linalg.norm(ref)


def test_fp64_channel_follows_startup_series(channel_runs):
    nz = CHANNEL_SHAPE[2]
    exact = channel_startup_profile(nz, CHANNEL_TAU, CHANNEL_G, CHANNEL_STEPS)[1:-1]
    u = channel_runs['double']
    ref = np.zeros_like(u)
    ref[..., 0] = exact[:, None, None]
    assert relative(u, ref) <= TOL_ANALYTIC_FP64


@pytest.mark.parametrize('precision', ['single', 'half', 'bfloat16'])
def test_storage_error_against_fp64(channel_runs, precision):
    u, ref = channel_runs[precision], channel_runs['double']
    error = relative(u, ref)
    profile = relative(u[..., 0].mean(axis=(1, 2)), ref[..., 0].mean(axis=(1, 2)))
    print('%s: |u - u64|/|u64| = %.3e, profile %.3e' % (precision, error, profile))
    assert error <= TOL_VS_FP64[precision]
    assert profile <= TOL_PROFILE[precision]


@pytest.mark.parametrize('precision', ['half', 'bfloat16'])
def test_small_accelerations_are_not_rounded_away(precision):
    """A periodic fluid accelerated from rest by g = 5e-7: the populations change by 1.5e-6 of w_q per step, far
    below half an ulp of FP16 (and BF16) once |u| > 1e-3.  With unbiased rounding u keeps following g t."""
    n, g, steps = 16, 5e-7, 4000
    force = LBMForce()
    force.setGridSize(n, n, n)
    force.setFluidDensity(1.0)
    force.setKinematicViscosity((0.8 - 0.5)/3.0)
    force.setBodyAcceleration((g, 0.0, 0.0))
    force.setFluidMomentumRemovalFrequency(0)
    lattice = force.latticeParameters(np.array([n, n, n], dtype=float), 1.0, np.ones(1))
    kernel = lbm_b200.B200Kernel(lattice, [], [], precision)
    for s in range(steps):
        kernel.begin_step(s)
        kernel.execute(s)
    density, velocity = kernel.get_fluid_fields()
    kernel.close()
    mean = (density[:, None]*velocity).sum(axis=0)/density.sum()
    # u = (j + F/2)/rho after `steps` steps of the force: g (steps + 1/2).
    assert abs(mean[0]/(g*(steps + 0.5)) - 1) <= 2e-3
