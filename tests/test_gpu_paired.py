"""GPU tests of the paired dense kernel (two x-adjacent nodes per thread, tiles of 64 x 8 nodes) on lattices wider
than one tile: FP32 storage follows the oracle (1e-5 of the largest population of the fluid nodes, as the other FP32
parity tests) with ragged tiles (ny not a multiple of the 8 rows of a tile), several tiles along x (the pulls across
the tile edges and the periodic wrap at both ends), solid nodes (pairs with one or both nodes solid) under bounce-back
or regularized walls, open faces, fluctuations and coupled particles.

The quad kernel of 16-bit storage (four x-adjacent nodes per thread, nx a multiple of 4, no fluctuations) collides
its nodes as two pairs with the paired kernel's arithmetic and dither bits, so without the momentum removal (whose
sums the two kernels add in different orders) its runs are bitwise those of the paired kernel, which a subprocess
selects with LBM_B200_QUAD16=0."""
import os
import subprocess
import sys

import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from oracle import OracleKernel

pytestmark = pytest.mark.gpu

DX, DT = 0.5, 0.01


def solid_nodes(shape, walls):
    """The wall plane j = 0 and a block of solid nodes (x = 2, 3 and nx - 1; y = 2, 3; z = 1, 2)."""
    nx, ny, nz = shape
    if walls == 'periodic':
        return []
    return ([i + nx*ny*k for k in range(nz) for i in range(nx)] +
            [i + nx*(j + ny*k) for k in (1, 2) for j in (2, 3) for i in (2, 3, nx - 1)])


def wide_case(shape, walls, fluct, particles, kernel_factory=None, properties=None, removal=None):
    """A perturbed fluid of `shape` nodes (tau 0.8, body force, momentum removal every third step unless faces are
    open), with the wall plane j = 0 and a block of solid nodes, bounce-back ('walls') or regularized
    ('regularized', 'dvfaces'), open x faces ('dvfaces'), fluctuations and particle noise at 300 K (else 0 K), and
    `particles` coupled particles under explicit drag.  Returns (context, force)."""
    nx, ny, nz = shape
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((nx*DX, 0, 0), (0, ny*DX, 0), (0, 0, nz*DX))
    force = LBMForce()
    force.setGridSize(nx, ny, nz)
    force.setKinematicViscosity((0.8 - 0.5)/3*DX*DX/DT)
    force.setBodyAcceleration((0.5, -0.2, 0.1))
    force.setInitialFluidVelocity((0.5, 0.2, -0.3))
    force.setFluidMomentumRemovalFrequency(removal if removal is not None else (0 if walls == 'dvfaces' else 3))
    if walls != 'periodic':
        force.setSolidNodes(solid_nodes(shape, walls))
    if walls in ('regularized', 'dvfaces'):
        force.setWallScheme(LBMForce.Regularized)
    if walls == 'dvfaces':
        force.setFaceBoundary(LBMForce.XMin, LBMForce.DensityVelocity)
        force.setFaceBoundary(LBMForce.XMax, LBMForce.Velocity)
        force.setFaceVelocity(LBMForce.XMin, (0.5, 0.1, 0.0))
        force.setFaceDensity(LBMForce.XMin, 605.0)
        force.setFaceVelocity(LBMForce.XMax, (0.4, 0.0, 0.1))
    force.setFluidFluctuations(fluct)
    force.setTemperature(300.0 if fluct else 0.0)
    force.setRandomNumberSeed(2024)
    for i in range(particles):
        system.addParticle(100.0)
        force.addParticle(i)
    if particles == 0:
        system.addParticle(1.0)
    force.setFriction(10.0)
    system.addForce(force)
    context = lbm_b200.Context(system, lbm_b200.VerletIntegrator(DT), kernel_factory, properties)
    rng = np.random.default_rng(5)
    box = np.array(shape)*DX
    positions = rng.uniform(0.1, 0.9, (system.getNumParticles(), 3))*box
    positions[:, 1] = np.maximum(positions[:, 1], 1.5*DX)    # clear of the wall plane (the block is at x < 4 and x = nx - 1)
    context.setPositions(positions)
    context.setVelocities(rng.normal(0.0, 0.5, (system.getNumParticles(), 3)))
    state = force.getFluidState(context)
    force.setFluidState(context, state + 1e-3*np.sin(1.3*np.arange(len(state))))
    return context, force


PARITY_CASES = [((64, 13, 5), 'periodic', False, 0), ((64, 13, 5), 'walls', False, 3),
                ((128, 9, 4), 'regularized', True, 0), ((128, 9, 4), 'dvfaces', False, 2),
                ((64, 8, 6), 'walls', True, 3)]


@pytest.mark.parametrize('shape,walls,fluct,particles', PARITY_CASES)
def test_paired_fp32_agrees_with_oracle(shape, walls, fluct, particles):
    results = []
    for factory, props in ((OracleKernel, None), (None, {'Precision': 'single'})):
        context, force = wide_case(shape, walls, fluct, particles, factory, props)
        context.integrator.step(20)
        results.append((force.getFluidState(context), context.positions.copy(), force.getWallForce(context)))
        context.close()
    (ref, ref_pos, ref_wall), (got, pos, wall) = results
    # Populations of the fluid nodes, relative to the largest of them (solid nodes hold -w_q, far larger).
    fluid = np.ones(int(np.prod(shape)), dtype=bool)
    fluid[solid_nodes(shape, walls)] = False
    ref, got = ref.reshape(19, -1)[:, fluid], got.reshape(19, -1)[:, fluid]
    assert abs(got - ref).max() <= 1e-5*abs(ref).max()
    assert abs(pos - ref_pos).max() <= 1e-6*abs(ref_pos).max()
    assert abs(wall - ref_wall).max() <= 1e-5*max(1.0, abs(ref_wall).max())


QUAD_CASES = [((64, 13, 5), 'walls', 3), ((128, 9, 4), 'regularized', 0), ((128, 9, 4), 'dvfaces', 2),
              ((256, 6, 3), 'periodic', 0)]


def run_wide_16bit(shape, walls, particles, precision, steps=30):
    context, force = wide_case(shape, walls, False, particles, None, {'Precision': precision}, removal=0)
    context.integrator.step(steps)
    result = (force.getFluidState(context), context.positions.copy())
    context.close()
    return result


@pytest.mark.parametrize('precision', ['half', 'bfloat16'])
@pytest.mark.parametrize('shape,walls,particles', QUAD_CASES)
def test_quad_kernel_is_bitwise_the_paired_kernel(shape, walls, particles, precision, tmp_path):
    """Quads with one to three solid nodes (the block at x = 2, 3 and nx - 1), pulls across the 128-node row tiles and
    the periodic wrap, open faces and coupled particles (the reaction forces of the quad's nodes)."""
    out = str(tmp_path/'paired.npz')
    code = ('import sys; sys.path.insert(0, %r); import conftest, numpy; from test_gpu_paired import run_wide_16bit; '
            'state, positions = run_wide_16bit(%r, %r, %d, %r); numpy.savez(%r, state=state, positions=positions)'
            % (os.path.dirname(os.path.abspath(__file__)), shape, walls, particles, precision, out))
    env = dict(os.environ, LBM_B200_QUAD16='0')
    subprocess.run([sys.executable, '-c', code], env=env, check=True, timeout=300)
    paired = np.load(out)
    state, positions = run_wide_16bit(shape, walls, particles, precision)
    assert np.array_equal(state, paired['state'])
    assert np.array_equal(positions, paired['positions'])
