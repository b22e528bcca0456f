"""The parity cases of the tests, built like the reference's cross-platform tests
(python/tests/TestLBMForce.py:501-635): the same Systems, in the harness of lbm_b200."""
import numpy as np

import lbm_b200
from lbm_b200 import LBMForce

FLUID_WALLS = ('periodic', 'walls', 'regularized', 'faces', 'dvfaces')


def fluid_case(walls, kernel_factory=None, properties=None):
    """test_fluid_agrees_with_reference (TestLBMForce.py:505-570): a 6x5x4 lattice with a perturbed fluid, a body
    force and the removal of the momentum every third step, with solid nodes (the plane j = 0 and a block),
    bounce-back or regularized walls, and open faces.  Returns (context, force); the fluid is perturbed."""
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((3, 0, 0), (0, 2.5, 0), (0, 0, 2))
    system.addParticle(1.0)
    force = LBMForce()
    force.setGridSize(6, 5, 4)
    force.setKinematicViscosity((0.8 - 0.5)/3*0.25/0.01)
    force.setBodyAcceleration((0.5, -0.2, 0.1))
    force.setInitialFluidVelocity((0.5, 0.2, -0.3))
    force.setFluidMomentumRemovalFrequency(0 if walls in ('faces', 'dvfaces') else 3)
    if walls != 'periodic':
        force.setSolidNodes([i + 6*5*k for k in range(4) for i in range(6)] +
                            [i + 6*(j + 5*k) for k in (1, 2) for j in (2, 3) for i in (2, 3)])
    if walls in ('regularized', 'faces', 'dvfaces'):
        force.setWallScheme(LBMForce.Regularized)
    if walls == 'dvfaces':
        force.setFaceBoundary(LBMForce.XMin, LBMForce.DensityVelocity)
        force.setFaceBoundary(LBMForce.XMax, LBMForce.Velocity)
        force.setFaceBoundary(LBMForce.ZMin, LBMForce.Density)
        force.setFaceBoundary(LBMForce.ZMax, LBMForce.DensityVelocity)
        force.setFaceVelocity(LBMForce.XMin, (0.5, 0.1, 0.0))
        force.setFaceDensity(LBMForce.XMin, 605.0)
        force.setFaceVelocity(LBMForce.XMax, (0.4, 0.0, 0.1))
        force.setFaceDensity(LBMForce.ZMax, 600.0)
        force.setFaceVelocity(LBMForce.ZMax, (0.2, -0.1, 0.0))
    if walls == 'faces':
        force.setFaceBoundary(LBMForce.XMin, LBMForce.Velocity)
        force.setFaceBoundary(LBMForce.XMax, LBMForce.Density)
        force.setFaceVelocity(LBMForce.XMin, (0.5, 0.1, 0.0))
        force.setFaceDensity(LBMForce.XMax, 605.0)
    system.addForce(force)
    integrator = lbm_b200.VerletIntegrator(0.01)
    context = lbm_b200.Context(system, integrator, kernel_factory, properties)
    context.setPositions([(0.1, 0.7, 0.3)])
    state = force.getFluidState(context)
    state = state + 1e-3*np.sin(1.3*np.arange(len(state)))
    force.setFluidState(context, state)
    return context, force


COUPLING_CASES = ([(walls, drag, 'NearestNode') for walls in (False, True, 'faces') for drag in ('Explicit', 'Centered')] +
                  [(walls, drag, stencil) for walls in (False, True) for drag in ('Explicit', 'Centered')
                   for stencil in ('Trilinear', 'ThreePoint', 'Keys')])


def coupling_case(walls, drag, stencil, kernel_factory=None, properties=None, temperature=0.0, seed=0, removal=0):
    """test_coupling_agrees_with_reference (TestLBMForce.py:573-635): 4 particles of mass 100 on an 8^3 lattice,
    friction 10/ps, a constant external field and a soft pair force, explicit or centred drag, every stencil,
    with the wall plane j = 0 or open faces along x."""
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((4, 0, 0), (0, 4, 0), (0, 0, 4))
    force = LBMForce()
    force.setGridSize(8, 8, 8)
    for i in range(4):
        system.addParticle(100.0)
        force.addParticle(i)
    # CustomExternalForce('-3*x+2*y-z'): F = -grad U = (3, -2, 1).
    system.addForce(lbm_b200.ExternalForce(lambda p: np.tile([3.0, -2.0, 1.0], (len(p), 1))))
    # CustomNonbondedForce('50*(1-r)^2') with a periodic cutoff 1: dU/dr = -100 (1 - r).
    system.addForce(lbm_b200.PairForce(lambda r: -100.0*(1.0 - r), 1.0))
    system.addForce(force)
    force.setDragScheme(getattr(LBMForce, drag))
    force.setInterpolationStencil(getattr(LBMForce, stencil))
    force.setFriction(10.0)
    force.setTemperature(temperature)
    force.setRandomNumberSeed(seed)
    force.setFluidMomentumRemovalFrequency(removal)
    if walls == 'faces':
        force.setFaceBoundary(LBMForce.XMin, LBMForce.Velocity)
        force.setFaceBoundary(LBMForce.XMax, LBMForce.Density)
        force.setFaceVelocity(LBMForce.XMin, (0.2, 0.0, 0.0))
        force.setFaceDensity(LBMForce.XMax, 603.0)
    elif walls:
        force.setSolidNodes([i + 64*k for k in range(8) for i in range(8)])
    integrator = lbm_b200.VerletIntegrator(0.01)
    context = lbm_b200.Context(system, integrator, kernel_factory, properties)
    context.setPositions([(1.02, 2.01, 0.98), (0.97, 1.99, 1.03), (3.98, 0.52, 3.96),
                          (3.55 if walls == 'faces' else 2.3, 0.6, 0.6)])
    context.setVelocities([(0.5, -0.2, 0.3), (-0.4, 0.1, 0.2), (2.0, -1.5, 1.0), (0.0, -2.0, -0.6)])
    return context, force


# The fluid tests of the reference (tests/TestLBMFluid.h:22-50): lattice spacing (nm), time step (ps), density.
FLUID_DX, FLUID_DT, FLUID_DENSITY = 0.5, 0.01, 602.2


def fluid_system(nx, ny, nz, tau):
    """createFluidSystem (TestLBMFluid.h:41-52): a fluid of nx*ny*nz nodes with relaxation time tau, no momentum
    removal, one particle that is not coupled.  Returns (system, force)."""
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((nx*FLUID_DX, 0, 0), (0, ny*FLUID_DX, 0), (0, 0, nz*FLUID_DX))
    system.addParticle(1.0)
    force = LBMForce()
    force.setGridSize(nx, ny, nz)
    force.setFluidDensity(FLUID_DENSITY)
    force.setKinematicViscosity((tau - 0.5)/3.0*FLUID_DX*FLUID_DX/FLUID_DT)
    force.setFluidMomentumRemovalFrequency(0)
    system.addForce(force)
    return system, force


def make_context(system, kernel_factory=None, properties=None):
    context = lbm_b200.Context(system, lbm_b200.VerletIntegrator(FLUID_DT), kernel_factory, properties)
    context.setPositions([(0.1, 0.2, 0.3)]*system.getNumParticles())
    return context


W = np.array([1/3] + [1/18]*6 + [1/36]*12)
C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0], [-1, -1, 0],
              [1, -1, 0], [-1, 1, 0], [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1], [1, 0, 1], [-1, 0, -1],
              [-1, 0, 1], [1, 0, -1]], dtype=float)


def uniform_state(num_nodes, rho, u):
    """uniformState (TestLBMFluid.h:58-73): equilibrium deviations at density rho and velocity u."""
    u = np.asarray(u, dtype=float)
    cu = C @ u
    dfeq = W*((rho - 1.0) + rho*(3.0*cu + 4.5*cu*cu - 1.5*u.dot(u)))
    return np.repeat(dfeq, num_nodes)


def total_moments(state):
    """totalMoments (TestLBMFluid.h:76-91): mass = numNodes + sum(f - w) and momentum, lattice units."""
    f = state.reshape(19, -1)
    return f.shape[1] + f.sum(), C.T @ f.sum(axis=1)


def wall_plane(nx, ny, nz):
    """wallPlane (TestLBMFluid.h:450-456): the nodes of the plane j = 0."""
    return [i + nx*ny*k for k in range(nz) for i in range(nx)]


def wall_test_nodes(nx, ny, nz):
    """wallTestNodes (TestLBMFluid.h:632-641): the plane i = 0 and a 2x2x2 block."""
    return [i + nx*(j + ny*k) for k in range(nz) for j in range(ny) for i in range(nx)
            if i == 0 or (2 <= i < 4 and 1 <= j < 3 and 1 <= k < 3)]


COUPLING_MASS = 100.0


def coupled_system(num_particles, friction, temperature, coupled=None, seed=1):
    """createCoupledSystem (TestLBMCoupling.h:39-61): particles of mass 100 on an 8^3 fluid (tau = 0.8), no momentum
    removal, a fixed seed.  Returns (system, force)."""
    n = 8
    system = lbm_b200.System()
    system.setDefaultPeriodicBoxVectors((n*FLUID_DX, 0, 0), (0, n*FLUID_DX, 0), (0, 0, n*FLUID_DX))
    force = LBMForce()
    force.setGridSize(n, n, n)
    force.setFluidDensity(FLUID_DENSITY)
    force.setKinematicViscosity((0.8 - 0.5)/3.0*FLUID_DX*FLUID_DX/FLUID_DT)
    force.setFluidMomentumRemovalFrequency(0)
    force.setFriction(friction)
    force.setTemperature(temperature)
    force.setRandomNumberSeed(seed)
    for _ in range(num_particles):
        system.addParticle(COUPLING_MASS)
    for particle in (coupled if coupled is not None else range(num_particles)):
        force.addParticle(particle)
    system.addForce(force)
    return system, force


def total_momentum(context, force):
    """totalMomentum (TestLBMCoupling.h:64-79): particles (half step) plus fluid, Da nm/ps."""
    p = (context.velocities*np.array(context.system.masses)[:, None]).sum(axis=0)
    mass, j = total_moments(force.getFluidState(context))
    cell_mass = force.getFluidDensity()*FLUID_DX**3
    return p + j*(cell_mass*FLUID_DX/FLUID_DT)


# The precision channel: a Poiseuille channel between bounce-back planes z = 0 and z = nz - 1 driven by the Guo body
# force g_x, in lattice units (dx = dt = rho0 = 1), no momentum removal, no fluctuations, started from rest.
CHANNEL_SHAPE, CHANNEL_TAU, CHANNEL_G, CHANNEL_STEPS = (384, 384, 192), 0.55, 5e-7, 20000


def channel_kernel(shape, precision, tau=CHANNEL_TAU, g=CHANNEL_G):
    nx, ny, nz = shape
    force = LBMForce()
    force.setGridSize(nx, ny, nz)
    force.setFluidDensity(1.0)
    force.setKinematicViscosity((tau - 0.5)/3.0)
    force.setBodyAcceleration((g, 0.0, 0.0))
    force.setFluidMomentumRemovalFrequency(0)
    lattice = force.latticeParameters(np.array(shape, dtype=float), 1.0, np.ones(1))
    plane = np.arange(nx*ny, dtype=np.int64)
    solids = np.concatenate([plane, plane + nx*ny*(nz - 1)])
    return lbm_b200.B200Kernel(lattice, [], solids, precision)


def channel_startup_profile(nz, tau, g, t, terms=4001):
    """u_x(z) at time t of the channel flow started from rest, walls halfway between the solid and the first fluid
    planes (h = nz - 2): the steady parabola minus its decaying odd sine modes,
    u = g/(2 nu) s (h - s) - sum_{n odd} 4 g h^2/(nu pi^3 n^3) sin(n pi s/h) exp(-nu n^2 pi^2 t/h^2), s = z - 1/2."""
    nu, h = (tau - 0.5)/3.0, nz - 2
    s = np.arange(nz) - 0.5
    u = g/(2*nu)*s*(h - s)
    n = np.arange(1, terms + 1, 2, dtype=float)[:, None]
    u -= (4*g*h*h/(nu*np.pi**3*n**3)*np.sin(n*np.pi*s/h)*np.exp(-nu*n*n*np.pi**2*t/(h*h))).sum(axis=0)
    u[0] = u[-1] = 0.0
    return u


def step_with_repeated_evaluation(context):
    """One integration step whose force evaluation is repeated before the step count advances, as the GPU platforms
    of OpenMM do when they enlarge their neighbour list (ReferenceLBMKernels.cpp:341-365): returns the coupled forces of
    both evaluations; the step integrates with the first."""
    p, v, f = context._coupled_arrays(np.zeros_like(context.positions))
    context.kernel.begin_step(context.step_count, p, v, f)
    if v is not None:
        context.velocities[context.coupled] = v
    first = context._forces()
    again = context._forces()
    dt = context.integrator.step_size
    context.velocities += dt*first/context.masses[:, None]
    context.positions += dt*context.velocities
    context.step_count += 1
    return first, again


def evaluation_sequence(context):
    """The force evaluations of the kernel's evaluation rules (ReferenceLBMKernels.cpp:341-401), in order: before the
    first step (no coupling force yet), between steps (the next step's forces, twice), a step with a repeated
    evaluation (the same forces again), and between steps after more steps; then the state.  Returns a dict of
    arrays."""
    out = {'before_first_step': context.getForces()}
    context.integrator.step(2)
    out['between_steps'] = context.getForces()
    out['between_steps_again'] = context.getForces()
    out['step_first_evaluation'], out['step_repeated_evaluation'] = step_with_repeated_evaluation(context)
    context.integrator.step(2)
    out['between_steps_later'] = context.getForces()
    context.integrator.step(1)
    out['positions'] = context.positions.copy()
    out['velocities'] = context.velocities.copy()
    return out


# The cases of the evaluation-sequence fixture: (walls, drag, stencil); momentum removal every 2 steps (none with open
# faces, where it is not allowed), so that the next-step forces of odd and even step counts differ in the removal.
EVALUATION_CASES = [(False, 'Explicit', 'NearestNode'), (True, 'Explicit', 'Keys'), (False, 'Centered', 'NearestNode'),
                    (True, 'Centered', 'ThreePoint'), ('faces', 'Centered', 'Keys'), ('faces', 'Explicit', 'Trilinear')]


def evaluation_case(walls, drag, stencil, kernel_factory=None, properties=None, temperature=0.0):
    return coupling_case(walls, drag, stencil, kernel_factory, properties, temperature=temperature, seed=5,
                         removal=0 if walls == 'faces' else 2)
