"""GPU parity over a long run: a 32^3 lattice between bounce-back planes z = 0 and z = 31 (periodic in x and y), tau 0.8,
rho0 = 1, body force g_x = 1e-6, no fluctuations and no momentum removal, with 64 particles of mass 1 (= the node mass)
started at rest at seeded uniform positions (x, y in [0, 32), z in [2, 29]; numpy PCG64 seed 2026), coupled through
the trilinear stencil with the explicit drag, friction 0.5 per step.  2000 steps in lattice units (dx = 1 nm,
dt = 1 ps), the GPU against the oracle: the u_x(z) profile and the particle velocities agree within 1e-12 relative
(FP64 storage) and 1e-5 (FP32 storage)."""
import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from oracle import OracleKernel

pytestmark = pytest.mark.gpu

N, TAU, G, FRICTION, STEPS, PARTICLES = 32, 0.8, 1e-6, 0.5, 2000, 64
TOL = {'double': 1e-12, 'single': 1e-5}


def particle_channel(kernel_factory=None, properties=None):
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((N, 0, 0), (0, N, 0), (0, 0, N))
    force = LBMForce()
    force.setGridSize(N, N, N)
    force.setFluidDensity(1.0)
    force.setKinematicViscosity((TAU - 0.5)/3.0)
    force.setBodyAcceleration((G, 0.0, 0.0))
    force.setFluidMomentumRemovalFrequency(0)
    force.setSolidNodes([i + N*(j + N*k) for k in (0, N - 1) for j in range(N) for i in range(N)])
    force.setFriction(FRICTION)
    force.setDragScheme(LBMForce.Explicit)
    force.setInterpolationStencil(LBMForce.Trilinear)
    force.setTemperature(0.0)
    for i in range(PARTICLES):
        system.addParticle(1.0)
        force.addParticle(i)
    system.addForce(force)
    context = lbm_b200.Context(system, lbm_b200.VerletIntegrator(1.0), kernel_factory, properties)
    rng = np.random.Generator(np.random.PCG64(2026))
    positions = np.column_stack([rng.uniform(0, N, PARTICLES), rng.uniform(0, N, PARTICLES),
                                 rng.uniform(2, N - 3, PARTICLES)])
    context.setPositions(positions)
    context.setVelocities(np.zeros((PARTICLES, 3)))
    return context, force


def run(kernel_factory, properties):
    context, force = particle_channel(kernel_factory, properties)
    context.integrator.step(STEPS)
    _, velocity = force.getFluidFields(context)
    profile = velocity.reshape(N, N, N, 3)[:, :, :, 0].mean(axis=(1, 2))
    out = profile, context.velocities.copy()
    context.close()
    return out


@pytest.fixture(scope='module')
def oracle_run():
    return run(OracleKernel, None)


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_long_particle_channel_agrees_with_oracle(oracle_run, precision):
    (ref_profile, ref_velocities), (profile, velocities) = oracle_run, run(None, {'Precision': precision})
    assert abs(ref_profile).max() > 1e-5                 # the flow has developed
    assert abs(profile - ref_profile).max() <= TOL[precision]*abs(ref_profile).max()
    assert abs(velocities - ref_velocities).max() <= TOL[precision]*abs(ref_velocities).max()
