"""GPU tests of the fluctuating fluid and its coupled beads, statistically, with block-average error bars: a reduced
instance of the scale configuration's observables (free beads of mass 20 in a 16^3 periodic fluctuating fluid,
tau 0.8, kT = 1e-4, Keys stencil, centred drag 0.5 per step; lattice units dx = 1 nm, dt = 1 ps, rho0 = 1 Da/nm^3).

- the fluid temperature <rho (u - <u>)^2> and the bead temperature <m v^2>/3 agree with kT;
- the beads' velocity autocorrelation agrees with the oracle's (the reference's algorithm on the CPU, with its own
  sequential random stream, so the two runs are independent samples of the same process) within the combined error
  bars of the two."""
import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from oracle import OracleKernel

pytestmark = pytest.mark.gpu

BOLTZ = 6.02214076e23*1.380649e-23/1000.0
N, TAU, KT, FRICTION, MASS, SIDE = 16, 0.8, 1e-4, 0.5, 20.0, 3


def free_beads(kernel_factory=None, properties=None, seed=11):
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((N, 0, 0), (0, N, 0), (0, 0, N))
    force = LBMForce()
    force.setGridSize(N, N, N)
    force.setFluidDensity(1.0)
    force.setKinematicViscosity((TAU - 0.5)/3.0)
    force.setFluidFluctuations(True)
    force.setTemperature(KT/BOLTZ)
    force.setRandomNumberSeed(seed)
    force.setInterpolationStencil(LBMForce.Keys)
    force.setDragScheme(LBMForce.Centered)
    force.setFriction(FRICTION)
    count = SIDE**3
    for i in range(count):
        system.addParticle(MASS)
        force.addParticle(i)
    system.addForce(force)
    context = lbm_b200.Context(system, lbm_b200.VerletIntegrator(1.0), kernel_factory, properties)
    g = (np.arange(SIDE) + 0.5)*N/SIDE
    context.setPositions(np.array([(x, y, z) for z in g for y in g for x in g]))
    context.setVelocities(np.zeros((count, 3)))
    return context, force


def block_mean(samples, blocks=10):
    """Mean and standard error of the mean over `blocks` consecutive blocks of the samples (first axis)."""
    s = np.asarray(samples)
    m = len(s)//blocks
    means = s[:m*blocks].reshape((blocks, m) + s.shape[1:]).mean(axis=1)
    return means.mean(axis=0), means.std(axis=0, ddof=1)/np.sqrt(blocks)


def velocity_record(context, steps, equilibrate):
    context.integrator.step(equilibrate)
    record = []
    for _ in range(steps):
        context.integrator.step(1)
        record.append(context.velocities.copy())
    return np.array(record)


def vacf(record, lags):
    """C(lag) = <v(t) . v(t + lag)>/3 per time origin (averaged over beads)."""
    t = len(record) - max(lags)
    return np.stack([(record[:t]*record[lag:lag + t]).sum(axis=2).mean(axis=1)/3 for lag in lags], axis=1)


@pytest.mark.parametrize('precision', ['single', 'half'])
def test_fluid_and_bead_temperatures(precision):
    """400 snapshots 20 steps apart after 1000 steps, in 20 blocks.  The standard error comes from the spread of the
    block means, so the bound is the two-sided 99.9 % quantile of Student's t with 19 degrees of freedom (3.88) times
    that error, not a normal 3 sigma."""
    from scipy.stats import t as student
    blocks = 20
    bound = student.ppf(0.9995, blocks - 1)
    context, force = free_beads(properties={'Precision': precision})
    context.integrator.step(1000)
    fluid, beads = [], []
    for _ in range(400):
        context.integrator.step(20)
        density, velocity = force.getFluidFields(context)
        u = velocity - (velocity*density[:, None]).sum(axis=0)/density.sum()
        fluid.append((density[:, None]*u*u).mean())
        beads.append(MASS*(context.velocities**2).sum(axis=1).mean()/3)
    context.close()
    for name, samples in (('fluid', fluid), ('beads', beads)):
        mean, err = block_mean(samples, blocks)
        print('%s temperature %.4f +- %.4f kT' % (name, mean/KT, err/KT))
        assert abs(mean/KT - 1) <= max(bound*err/KT, 0.02), name


def test_bead_velocity_autocorrelation_agrees_with_oracle():
    lags = [0, 2, 5, 10, 20]
    results = []
    for factory, props in ((lambda l, m, s: OracleKernel(l, m, s, random='sequential'), None),
                           (None, {'Precision': 'double'})):
        context, _ = free_beads(factory, props)
        record = velocity_record(context, 3000, 500)
        context.close()
        results.append(block_mean(vacf(record, lags)))
    (ref, ref_err), (got, got_err) = results
    print('VACF/(kT/m) oracle', np.round(ref/(KT/MASS), 3), 'GPU', np.round(got/(KT/MASS), 3))
    assert abs(ref[0]/(KT/MASS) - 1) < 0.15
    assert np.all(abs(got - ref) <= 3*np.sqrt(ref_err**2 + got_err**2) + 0.02*KT/MASS)
