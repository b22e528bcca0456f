"""GPU tests of the storage formats on the precision channel: a 384x384x192 Poiseuille channel between bounce-back
planes z = 0 and z = 191, Guo body force g_x = 5e-7, tau 0.55, started from rest, 20,000 steps, in FP64, FP32, FP16 and
BF16 storage (FP32 collide arithmetic for the last three, with the momentum carried in two floats).  After 20,000 steps
the flow is still in start-up (H^2/nu = 2.2e6 steps), so the analytic reference is the start-up series of the channel
with halfway walls.

Errors are relative L2 norms over the fluid nodes, ||u - u_ref||/||u_ref||; the profile error compares the
xy-averaged profiles u_x(z), which removes the node-to-node scatter of the stochastic rounding.

Bounds:
- the target of 1e-4 against FP64 for FP32 storage (pointwise) and for the profile of every format: the systematic
  error, which the two-float momentum brings from the FP32 arithmetic floor of 2.5e-4 to 1.6e-5 (tests/
  test_precision_floor.py, on the exact column reduction of this channel);
- for FP16 and BF16 the pointwise error is the scatter of the stochastic rounding, unbiased noise whose size the
  16-bit quantum sets: each step every stored value is off by at most one quantum, with variance q^2/6 averaged over
  the dither, and the velocity of a node sums 10 such values per component.  That one-step scatter, computed here
  from the FP64 fields (the equilibrium populations of each node), is a lower bound: the momentum that a rounding adds
  is conserved by the collision and carried over to later steps.  The test requires the scatter to lie between 1 and
  3 times the one-step value, for both formats (on B200 both measure 2.2 times it)."""
import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from cases import (CHANNEL_G, CHANNEL_SHAPE, CHANNEL_STEPS, CHANNEL_TAU, channel_kernel, channel_startup_profile)

pytestmark = pytest.mark.gpu

TARGET = 1e-4
TOL_ANALYTIC_FP64 = 2.5e-4
# D3Q19 velocities and weights in the kernel's order, and the 16-bit storage factors: the stored value of direction q
# is (f_q - w_q) k_q (times 2^10 for FP16).
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1])
W = np.array([1/3] + [1/18]*6 + [1/36]*12)
K = np.array([4.0] + [16.0]*6 + [32.0]*12)


def one_step_scatter(u, fmt):
    """The relative node scatter of the velocity that one step of stochastically rounded 16-bit stores gives:
    sqrt(mean over nodes of sum_a sum_q c_qa^2 q_q^2/6)/rms(u), with q_q the quantum of the stored value of the
    node's equilibrium population f_q - w_q = w_q (3 c.u + 4.5 (c.u)^2 - 1.5 u.u) (rho = 1)."""
    ux, uy, uz = (u[..., a].reshape(-1) for a in range(3))
    var = np.zeros_like(ux)
    scale = 1024.0 if fmt == 'half' else 1.0
    mantissa = 10 if fmt == 'half' else 7
    for q in range(19):
        cu = CX[q]*ux + CY[q]*uy + CZ[q]*uz
        dev = W[q]*(3*cu + 4.5*cu*cu - 1.5*(ux*ux + uy*uy + uz*uz))
        v = np.abs(dev*K[q]*scale)
        e = np.floor(np.log2(np.maximum(v, 1e-300)))
        if fmt == 'half':
            e = np.maximum(e, -14)
        quantum = 2.0**(e - mantissa)/(K[q]*scale)
        var += (CX[q]**2 + CY[q]**2 + CZ[q]**2)*quantum**2/6
    return np.sqrt(var.mean())/np.sqrt((u**2).sum(axis=-1).mean())


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
    assert profile <= TARGET
    if precision == 'single':
        assert error <= TARGET
        return
    # The scatter: the pointwise error without the profile's part.
    scatter = np.sqrt(max(error**2 - profile**2, 0.0))
    estimate = one_step_scatter(ref, precision)
    print('%s: scatter %.3e = %.2f x the one-step quantization scatter %.3e' % (precision, scatter,
                                                                              scatter/estimate, estimate))
    assert estimate <= scatter <= 3*estimate


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
