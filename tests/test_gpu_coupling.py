"""GPU tests of the particle coupling through the C ABI: parity with the oracle on the reference's coupling cases
(TestLBMForce.py:573-635: both drags, every stencil, walls and open faces, a soft pair force and a field), pathwise
agreement with noise (the same Philox numbers), and the reference's known answers (tests/TestLBMCoupling.h)."""
import numpy as np
import pytest

from cases import (COUPLING_CASES, COUPLING_MASS, FLUID_DT, coupled_system, coupling_case, make_context,
                   total_momentum, uniform_state)
from oracle import OracleKernel
from lbm_b200 import LBMForce

pytestmark = pytest.mark.gpu


def run_case(walls, drag, stencil, factory, props, temperature=0.0, steps=60):
    context, force = coupling_case(walls, drag, stencil, factory, props, temperature=temperature, seed=77)
    context.integrator.step(steps)
    out = (context.positions.copy(), context.velocities.copy(), force.getFluidState(context),
           force.getWallForce(context))
    if factory is None and drag == 'Centered' and stencil != 'NearestNode':
        # Every step solved through the explicit coupling matrix (4 particles: no cell or row over capacity).
        assert context.kernel.solver_fallback_steps() == 0
    context.close()
    return out


def cluster_case(count, spread, stencil, factory, props, seed=3):
    """`count` particles of mass 100 within a cube of `spread` nm (lattice spacing 0.5 nm) in the middle of a 16^3
    lattice, centred drag with friction 10/ps, a field and random velocities: more particles than a cell of the
    explicit coupling matrix holds (64, cells of 4^3 nodes) or more overlapping stencils than a row holds (128)."""
    import lbm_b200
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((8, 0, 0), (0, 8, 0), (0, 0, 8))
    force = LBMForce()
    force.setGridSize(16, 16, 16)
    for i in range(count):
        system.addParticle(100.0)
        force.addParticle(i)
    system.addForce(lbm_b200.ExternalForce(lambda p: np.tile([3.0, -2.0, 1.0], (len(p), 1))))
    system.addForce(force)
    force.setDragScheme(LBMForce.Centered)
    force.setInterpolationStencil(getattr(LBMForce, stencil))
    force.setFriction(10.0)
    force.setTemperature(0.0)
    force.setFluidMomentumRemovalFrequency(0)
    context = lbm_b200.Context(system, lbm_b200.VerletIntegrator(0.01), factory, props)
    rng = np.random.default_rng(seed)
    context.setPositions(4.55 + rng.uniform(0.0, spread, (count, 3)))
    context.setVelocities(rng.normal(0.0, 0.5, (count, 3)))
    return context, force


def chain_case(stencil, factory, props):
    """Five random-walk chains of 12 beads (bond 0.5 nm, one lattice spacing) and 8 free beads in a 12^3 lattice,
    centred drag with friction 10/ps and a field: rows of the coupling matrix along the chains and between chains
    that come within a stencil width, as for the beads of the scale configuration."""
    import lbm_b200
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((6, 0, 0), (0, 6, 0), (0, 0, 6))
    force = LBMForce()
    force.setGridSize(12, 12, 12)
    rng = np.random.default_rng(17)
    positions = []
    for chain in range(5):
        x = rng.uniform(0.0, 6.0, 3)
        for bead in range(12):
            positions.append(x.copy())
            step = rng.normal(size=3)
            x = x + 0.5*step/np.linalg.norm(step)
    positions += list(rng.uniform(0.0, 6.0, (8, 3)))
    for i in range(len(positions)):
        system.addParticle(100.0)
        force.addParticle(i)
    system.addForce(lbm_b200.ExternalForce(lambda p: np.tile([3.0, -2.0, 1.0], (len(p), 1))))
    system.addForce(force)
    force.setDragScheme(LBMForce.Centered)
    force.setInterpolationStencil(getattr(LBMForce, stencil))
    force.setFriction(10.0)
    force.setTemperature(0.0)
    force.setFluidMomentumRemovalFrequency(0)
    context = lbm_b200.Context(system, lbm_b200.VerletIntegrator(0.01), factory, props)
    context.setPositions(np.mod(np.array(positions), 6.0))
    context.setVelocities(rng.normal(0.0, 0.5, (len(positions), 3)))
    return context, force


@pytest.mark.parametrize('stencil', ['Trilinear', 'ThreePoint', 'Keys'])
def test_centred_drag_of_bead_chains_agrees_with_oracle(stencil):
    """The centred stencil drag of bead chains through the explicit coupling matrix gives the trajectory of the
    oracle's spread-and-gather solve (FP64, 1e-10)."""
    results = []
    for factory, props in ((OracleKernel, None), (None, {'Precision': 'double'})):
        context, force = chain_case(stencil, factory, props)
        context.integrator.step(10)
        results.append((context.positions.copy(), context.velocities.copy(), force.getFluidState(context)))
        if factory is None:
            assert context.kernel.solver_fallback_steps() == 0
            assert context.kernel.solver_iterations() > 0
        context.close()
    for a, b, name in zip(results[0], results[1], ('positions', 'velocities', 'state')):
        assert abs(b - a).max() <= 1e-10*max(1.0, abs(a).max()), name


@pytest.mark.parametrize('count,spread,stencil', [(80, 1.9, 'Keys'), (200, 3.4, 'Keys'), (160, 2.4, 'ThreePoint')])
def test_crowded_centred_drag_agrees_with_oracle(count, spread, stencil):
    """Crowded particles overflow the capacity of the explicit coupling matrix (a cell of 80 in 2^3 nm; 200 and 160
    particles whose stencils overlap more than 128 others), so those steps take the spread-and-gather solve: both
    solves give the oracle's trajectory (FP64, 1e-10)."""
    results = []
    for factory, props in ((OracleKernel, None), (None, {'Precision': 'double'})):
        context, force = cluster_case(count, spread, stencil, factory, props)
        context.integrator.step(10)
        results.append((context.positions.copy(), context.velocities.copy(), force.getFluidState(context)))
        if factory is None:
            assert context.kernel.solver_fallback_steps() > 0
        context.close()
    for a, b, name in zip(results[0], results[1], ('positions', 'velocities', 'state')):
        assert abs(b - a).max() <= 1e-10*max(1.0, abs(a).max()), name


@pytest.mark.parametrize('stencil', ['Trilinear', 'ThreePoint', 'Keys'])
def test_centred_stencil_at_open_faces_agrees_with_oracle(stencil):
    """The centred drag with a stencil next to open x faces, where the stencil's indices are clamped to the last
    node (repeated entries of weight zero): the coupling matrix matches the oracle's spread-and-gather solve."""
    ref = run_case('faces', 'Centered', stencil, OracleKernel, None)
    got = run_case('faces', 'Centered', stencil, None, {'Precision': 'double'})
    for a, b, name in zip(ref, got, ('positions', 'velocities', 'state', 'wall')):
        assert abs(b - a).max() <= 1e-10*max(1.0, abs(a).max()), name


@pytest.mark.parametrize('walls,drag,stencil', COUPLING_CASES)
def test_coupling_agrees_with_oracle_double(walls, drag, stencil):
    ref = run_case(walls, drag, stencil, OracleKernel, None)
    got = run_case(walls, drag, stencil, None, {'Precision': 'double'})
    for a, b, name in zip(ref, got, ('positions', 'velocities', 'state', 'wall')):
        # TestLBMForce.py:633-635.
        assert abs(b - a).max() <= 1e-10*max(1.0, abs(a).max()), name


@pytest.mark.parametrize('walls,drag,stencil', [c for c in COUPLING_CASES if c[0] != 'faces'])
def test_coupling_agrees_with_oracle_single(walls, drag, stencil):
    ref = run_case(walls, drag, stencil, OracleKernel, None)
    got = run_case(walls, drag, stencil, None, {'Precision': 'single'})
    for a, b, name in zip(ref, got, ('positions', 'velocities', 'state', 'wall')):
        # The wall force is a sum of populations with cancellations: in single precision the reference allows it
        # 5e-5 (TestLBMFluid.h:530-534, 623-626).
        tol = 5e-5 if name == 'wall' else 1e-5
        assert abs(b - a).max() <= tol*max(1.0, abs(a).max()), name


@pytest.mark.parametrize('drag,stencil', [('Explicit', 'NearestNode'), ('Centered', 'NearestNode'),
                                          ('Explicit', 'Keys'), ('Centered', 'ThreePoint')])
def test_noisy_coupling_follows_oracle_pathwise(drag, stencil):
    """At 300 K the random forces of the particles come from the same Philox counters on the GPU and in the oracle."""
    ref = run_case(True, drag, stencil, OracleKernel, None, temperature=300.0, steps=20)
    got = run_case(True, drag, stencil, None, {'Precision': 'double'}, temperature=300.0, steps=20)
    for a, b, name in zip(ref, got, ('positions', 'velocities', 'state', 'wall')):
        assert abs(b - a).max() <= 1e-10*max(1.0, abs(a).max()), name


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_first_step_drag(precision):
    """testFirstStepDrag (TestLBMCoupling.h:84-103): v1 = v0 (1 - gamma dt); the force between steps is that of the
    next step."""
    friction = 5.0
    system, force = coupled_system(1, friction, 0.0)
    context = make_context(system, properties={'Precision': precision})
    context.setPositions([(1.1, 1.3, 1.7)])
    v0 = np.array([0.3, -0.2, 0.1])
    context.setVelocities([v0])
    assert not context.getForces().any()
    context.integrator.step(1)
    v1 = context.velocities[0].copy()
    forces = context.getForces()
    tol = 1e-14 if precision == 'double' else 2e-6
    assert abs(v1 - v0*(1.0 - friction*FLUID_DT)).max() <= tol
    context.integrator.step(1)
    v2 = context.velocities[0].copy()
    assert abs((v2 - v1)*(COUPLING_MASS/FLUID_DT) - forces[0]).max() <= (1e-12 if precision == 'double' else 2e-6)*100


@pytest.mark.parametrize('drag', ['Explicit', 'Centered'])
@pytest.mark.parametrize('rho0', [1.0, 1.2])
def test_momentum_conservation(drag, rho0):
    """testMomentumConservation (TestLBMCoupling.h:146-172): particles and fluid together conserve momentum with drag
    and random forces; two particles share a node and one crosses the periodic boundary."""
    system, force = coupled_system(4, 10.0, 300.0)
    force.setDragScheme(getattr(LBMForce, drag))
    context = make_context(system, properties={'Precision': 'double'})
    positions = [(1.02, 2.01, 0.98), (0.97, 1.99, 1.03), (3.98, 0.02, 3.96), (2.3, 1.1, 0.6)]
    velocities = np.array([(0.5, -0.2, 0.3), (-0.4, 0.1, 0.2), (2.0, -1.5, 1.0), (0.0, 0.3, -0.6)])
    context.setPositions(positions)
    context.setVelocities(velocities)
    force.setFluidState(context, uniform_state(512, rho0, [0, 0, 0]))
    scale = (COUPLING_MASS*np.sqrt((velocities**2).sum(axis=1))).sum()
    p0 = total_momentum(context, force)
    context.integrator.step(50)
    p1 = total_momentum(context, force)
    assert np.sqrt(((p1 - p0)**2).sum())/scale <= 1e-11
    assert context.positions[2][0] > 4.0


@pytest.mark.parametrize('drag', ['Explicit', 'Centered'])
@pytest.mark.parametrize('stencil', ['NearestNode', 'Trilinear', 'Keys'])
def test_comoving_particle_feels_no_force(drag, stencil):
    """testComoving (TestLBMCoupling.h:178-193)."""
    for u in ([1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0], [0.6, -0.5, 0.6]):
        system, force = coupled_system(1, 10.0, 0.0)
        force.setDragScheme(getattr(LBMForce, drag))
        force.setInterpolationStencil(getattr(LBMForce, stencil))
        force.setInitialFluidVelocity(u)
        context = make_context(system, properties={'Precision': 'double'})
        context.setPositions([(1.1, 1.3, 1.7)])
        context.setVelocities([u])
        context.integrator.step(100)
        assert abs(context.velocities[0] - np.array(u)).max() <= 1e-13
        context.close()
