"""GPU tests of the fluid path through the C ABI: parity with the oracle on the reference's cross-platform cases,
and the reference's analytic known answers (tests/TestLBMFluid.h), for FP64 and FP32 storage.

Tolerances (as the reference's): FP64 storage 1e-12 of the largest population for 40 steps of parity
(TestLBMForce.py:567-570); FP32 storage 1e-5 relative."""
import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from cases import (FLUID_DENSITY, FLUID_DT, FLUID_DX, FLUID_WALLS, fluid_case, fluid_system, make_context,
                   total_moments, uniform_state, wall_plane, wall_test_nodes)
from oracle import OracleKernel

pytestmark = pytest.mark.gpu

TOL = {'double': 1e-12, 'single': 1e-5}


def storage_tolerance(precision, tolerance, single=None):
    return tolerance if precision == 'double' else (single if single is not None else 2e-6)


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('walls', FLUID_WALLS)
def test_fluid_agrees_with_oracle(walls, precision):
    results = []
    for factory, props in ((OracleKernel, None), (None, {'Precision': precision})):
        context, force = fluid_case(walls, factory, props)
        context.integrator.step(40)
        results.append((force.getFluidState(context), force.getWallForce(context)))
        context.close()
    (ref_state, ref_wall), (state, wall) = results
    assert abs(state - ref_state).max() <= TOL[precision]*abs(ref_state).max()
    wall_tol = 1e-10 if precision == 'double' else 1e-5
    assert abs(wall - ref_wall).max() <= wall_tol*max(1.0, abs(ref_wall).max())


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_uniform_flow_is_steady(precision):
    """testUniformFlowIsSteady (TestLBMFluid.h:93-108)."""
    system, force = fluid_system(6, 5, 4, 0.8)
    force.setInitialFluidVelocity(np.array([0.03, -0.02, 0.01])*(FLUID_DX/FLUID_DT))
    context = make_context(system, properties={'Precision': precision})
    before = force.getFluidState(context)
    context.integrator.step(50)
    after = force.getFluidState(context)
    assert abs(before - after).max() <= storage_tolerance(precision, 1e-13)


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_fluid_conservation(precision):
    """testFluidConservation (TestLBMFluid.h:113-135)."""
    system, force = fluid_system(6, 5, 4, 0.7)
    context = make_context(system, properties={'Precision': precision})
    state = force.getFluidState(context)
    i = np.arange(state.size)
    state = state + 1e-3*np.sin(1.3*i + 0.7*(i % 11))
    force.setFluidState(context, state)
    mass0, p0 = total_moments(force.getFluidState(context))
    context.integrator.step(100)
    mass1, p1 = total_moments(force.getFluidState(context))
    tol = storage_tolerance(precision, 1e-13, 2e-5)
    assert abs(mass0 - mass1) <= tol*mass0
    assert np.dot(p0, p0) > 1e-10
    assert abs(p0 - p1).max() <= tol*mass0


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('rho0', [1.0, 1.3])
def test_body_force(precision, rho0):
    """testBodyForce (TestLBMFluid.h:141-169): momentum n rho g per node, u = (n + 1/2) g dt."""
    system, force = fluid_system(4, 3, 5, 0.9)
    g = np.array([0.5, -0.3, 0.2])
    force.setBodyAcceleration(g)
    context = make_context(system, properties={'Precision': precision})
    n = 4*3*5
    force.setFluidState(context, uniform_state(n, rho0, [0, 0, 0]))
    steps = 20
    context.integrator.step(steps)
    mass, p = total_moments(force.getFluidState(context))
    g_lattice = g*(FLUID_DT*FLUID_DT/FLUID_DX)
    tol = storage_tolerance(precision, 1e-13, 2e-5)
    assert abs(rho0*n - mass) <= tol*rho0*n
    assert abs(g_lattice*steps*rho0*n - p).max() <= tol*max(1.0, abs(g_lattice*steps*rho0*n).max())
    density, velocity = force.getFluidFields(context)
    assert abs(density - rho0*FLUID_DENSITY).max() <= tol*FLUID_DENSITY
    assert abs(velocity - g*((steps + 0.5)*FLUID_DT)).max() <= storage_tolerance(precision, 1e-12, 2e-5)*abs(g).max()


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_fluid_momentum_removal(precision):
    """testFluidMomentumRemoval (TestLBMFluid.h:176-199): removal at steps that are multiples of 3."""
    system, force = fluid_system(4, 4, 4, 1.0)
    g = np.array([0.5, 0.0, 0.0])
    force.setBodyAcceleration(g)
    force.setInitialFluidVelocity(np.array([0.01, 0.02, -0.01])*(FLUID_DX/FLUID_DT))
    force.setFluidMomentumRemovalFrequency(3)
    context = make_context(system, properties={'Precision': precision})
    g_lattice = g[0]*FLUID_DT*FLUID_DT/FLUID_DX
    for n in range(1, 8):
        context.integrator.step(1)
        mass, p = total_moments(force.getFluidState(context))
        expected = np.array([((n - 1) % 3 + 1)*g_lattice*64, 0, 0])
        assert abs(p - expected).max() <= storage_tolerance(precision, 1e-13, 2e-6)


@pytest.mark.parametrize('precision,tau', [('double', 0.6), ('double', 1.2), ('single', 0.8)])
def test_shear_wave_viscosity(precision, tau):
    """testShearWaveViscosity (TestLBMFluid.h:205-251): nu = (tau - 1/2)/3 to 2e-3."""
    nx, ny, nz = 2, 64, 2
    system, force = fluid_system(nx, ny, nz, tau)
    context = make_context(system, properties={'Precision': precision})
    n = nx*ny*nz
    k = 2*np.pi/ny
    amp = 1e-3
    state = np.zeros(19*n)
    for j in range(ny):
        col = uniform_state(1, 1.0, [amp*np.sin(k*j), 0, 0])
        for kk in range(nz):
            for i in range(nx):
                state[np.arange(19)*n + i + nx*(j + ny*kk)] = col
    force.setFluidState(context, state)

    def measure():
        density, velocity = force.getFluidFields(context)
        j = (np.arange(n)//nx) % ny
        return 2*(velocity[:, 0]*np.sin(k*j)).sum()/n/(FLUID_DX/FLUID_DT)
    context.integrator.step(200)
    a1 = measure()
    context.integrator.step(1000)
    a2 = measure()
    nu_measured = -np.log(a2/a1)/(1000*k*k)
    assert abs(nu_measured/((tau - 0.5)/3.0) - 1.0) < 2e-3


def test_queries_do_not_advance_fluid():
    """testQueriesDoNotAdvanceFluid (TestLBMFluid.h:257-280): evaluations between steps leave the fluid unchanged,
    bit for bit."""
    states = []
    for run in range(2):
        system, force = fluid_system(4, 4, 4, 0.8)
        force.setBodyAcceleration((0.5, -0.2, 0.1))
        force.setInitialFluidVelocity(np.array([0.01, 0.0, 0.0])*(FLUID_DX/FLUID_DT))
        context = make_context(system, properties={'Precision': 'double'})
        for _ in range(10):
            context.integrator.step(1)
            if run == 1:
                context.getForces()
                force.getFluidMachNumber(context)
                force.getWallForce(context)
        states.append(force.getFluidState(context))
    assert np.array_equal(states[0], states[1])


@pytest.mark.parametrize('precision', ['double', 'single', 'half'])
def test_restart_from_checkpoint_is_bitwise(precision):
    """testRestartFromCheckpoint (TestLBMFluid.h:287-320): a run restarted from a checkpoint at a step that is not a
    multiple of the removal frequency is identical to the uninterrupted one."""
    steps, split = 35, 13
    results = {}
    checkpoint = None
    for run in range(3):
        system, force = fluid_system(4, 4, 4, 0.8)
        force.setBodyAcceleration((0.5, -0.2, 0.1))
        force.setInitialFluidVelocity(np.array([0.01, 0.0, 0.0])*(FLUID_DX/FLUID_DT))
        force.setFluidMomentumRemovalFrequency(5)
        context = make_context(system, properties={'Precision': precision})
        if run == 0:
            context.integrator.step(steps)
            results['uninterrupted'] = force.getFluidState(context)
        elif run == 1:
            context.integrator.step(split)
            checkpoint = (force.createCheckpoint(context), context.getStepCount(), force.getFluidState(context))
        else:
            data, count, saved = checkpoint
            force.loadCheckpoint(context, data)
            context.setStepCount(count)
            force.setFluidState(context, saved)
            context.integrator.step(steps - split)
            results['restarted'] = force.getFluidState(context)
        context.close()
    assert np.array_equal(results['uninterrupted'], results['restarted'])


@pytest.mark.parametrize('variant', [0, 1, 2])
def test_mach_number_check(variant):
    """testMachNumberCheck (TestLBMFluid.h:383-407)."""
    mach = 0.35
    speed = mach/np.sqrt(3.0)
    system, force = fluid_system(4, 4, 4, 0.8)
    force.setInitialFluidVelocity(np.array([speed, 0, 0])*(FLUID_DX/FLUID_DT))
    force.setMachCheckFrequency(0 if variant == 1 else 10)
    if variant == 2:
        force.setMachNumberLimit(0.5)
    context = make_context(system, properties={'Precision': 'double'})
    assert abs(force.getFluidMachNumber(context) - mach) < 1e-12
    context.integrator.step(9)
    thrown = False
    try:
        context.integrator.step(1)
    except lbm_b200.LbmError as e:
        thrown = 'Mach number' in str(e) and e.status == 2
    assert thrown == (variant == 0)


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('tau', [0.6, 0.875, 1.4])
def test_poiseuille_bounce_back(precision, tau):
    """testPoiseuille (TestLBMFluid.h:495-535): exact steady profile with the slip term of the scheme, and the walls
    carry the body force."""
    nx, ny, nz = 2, 12, 2
    system, force = fluid_system(nx, ny, nz, tau)
    g = 1e-5
    force.setBodyAcceleration((g*FLUID_DX/(FLUID_DT*FLUID_DT), 0, 0))
    force.setSolidNodes(wall_plane(nx, ny, nz))
    context = make_context(system, properties={'Precision': precision})
    nu, lam, h = (tau - 0.5)/3.0, (tau - 0.5)/2.0, ny - 1
    context.integrator.step(int(4*h*h/nu))
    density, velocity = force.getFluidFields(context)
    umax = g/(2*nu)*(0.5*h)**2 + g*(16*lam - 3)/(24*nu)
    tol = storage_tolerance(precision, 1e-9, 5e-5)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                node = i + nx*(j + ny*k)
                u = velocity[node]*(FLUID_DT/FLUID_DX)
                if j == 0:
                    assert density[node] == 0.0 and not u.any()
                    continue
                exact = g/(2*nu)*(j - 0.5)*(ny - 0.5 - j) + g*(16*lam - 3)/(24*nu)
                assert abs(u/umax - np.array([exact/umax, 0, 0])).max() <= tol
    mass = density.sum()*FLUID_DX**3
    body = np.array([g*FLUID_DX/(FLUID_DT*FLUID_DT)*mass, 0, 0])
    assert abs(force.getWallForce(context) - body).max() <= storage_tolerance(precision, 1e-8, 5e-5)*abs(body).max()


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('tau', [0.7, 1.0, 1.6])
def test_regularized_poiseuille(precision, tau):
    """testRegularizedPoiseuille (TestLBMFluid.h:590-627)."""
    nx, ny, nz = 2, 12, 2
    system, force = fluid_system(nx, ny, nz, tau)
    g = 1e-5
    force.setBodyAcceleration((g*FLUID_DX/(FLUID_DT*FLUID_DT), 0, 0))
    force.setSolidNodes(wall_plane(nx, ny, nz))
    force.setWallScheme(LBMForce.Regularized)
    context = make_context(system, properties={'Precision': precision})
    nu, h = (tau - 0.5)/3.0, ny
    context.integrator.step(int(4*h*h/nu))
    density, velocity = force.getFluidFields(context)
    umax = g/(2*nu)*(0.5*h)**2
    tol = storage_tolerance(precision, 1e-9, 5e-5)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                node = i + nx*(j + ny*k)
                u = velocity[node]*(FLUID_DT/FLUID_DX)
                if j == 0:
                    assert density[node] == 0.0 and not u.any()
                    continue
                assert abs(density[node]/FLUID_DENSITY - 1.0) <= tol
                exact = g/(2*nu)*j*(ny - j) + 3*g*(tau - 1)/(tau - 0.5)
                assert abs(u/umax - np.array([exact/umax, 0, 0])).max() <= tol
    mass = density.sum()*FLUID_DX**3
    body = np.array([g*FLUID_DX/(FLUID_DT*FLUID_DT)*mass, 0, 0])
    assert abs(force.getWallForce(context) - body).max() <= storage_tolerance(precision, 1e-8, 5e-5)*abs(body).max()


@pytest.mark.parametrize('scheme', [LBMForce.BounceBack, LBMForce.Regularized])
def test_wall_balance(scheme):
    """testWallBalance (TestLBMFluid.h:648-685): P(t+dt) - P(t) = (M g - F_wall) dt at every step."""
    nx, ny, nz = 6, 5, 4
    system, force = fluid_system(nx, ny, nz, 0.7)
    force.setSolidNodes(wall_test_nodes(nx, ny, nz))
    force.setWallScheme(scheme)
    force.setInitialFluidVelocity(np.array([0.02, -0.01, 0.005])*(FLUID_DX/FLUID_DT))
    g = np.array([1e-5, 2e-5, -1e-5])*(FLUID_DX/(FLUID_DT*FLUID_DT))
    force.setBodyAcceleration(g)
    context = make_context(system, properties={'Precision': 'double'})
    vol = FLUID_DX**3

    def moments():
        density, velocity = force.getFluidFields(context)
        return (density*vol).sum(), (velocity*(density*vol)[:, None]).sum(axis=0)
    mass0, p0 = moments()
    scale = mass0*0.02*FLUID_DX/FLUID_DT
    for _ in range(30):
        context.integrator.step(1)
        mass, p = moments()
        assert abs(mass - mass0) <= 1e-13*mass0
        balance = p - p0 - (g*mass - force.getWallForce(context))*FLUID_DT
        assert np.sqrt(balance.dot(balance))/scale <= 1e-12
        p0 = p


def test_invalid_solid_nodes_are_rejected():
    """testSolidNodeChecks (TestLBMFluid.h:462-482)."""
    for nodes in ([-1], [64], [3, 5, 3], list(range(64))):
        system, force = fluid_system(4, 4, 4, 0.8)
        force.setSolidNodes(nodes)
        with pytest.raises(lbm_b200.LbmError):
            make_context(system)


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_fluctuating_fluid_follows_oracle_pathwise(precision):
    """With the same Philox counters, the fluctuating fluid of the GPU follows the oracle step by step (normals in
    double for FP64 storage, in float for FP32), with regularized walls and DensityVelocity faces whose rebuilt
    populations carry equilibrium noise."""
    results = []
    for factory, props in ((OracleKernel, None), (None, {'Precision': precision})):
        system, force = fluid_system(8, 6, 5, 0.8)
        force.setFluidFluctuations(True)
        force.setTemperature(300.0)
        force.setRandomNumberSeed(4321)
        force.setSolidNodes(wall_plane(8, 6, 5))
        force.setWallScheme(LBMForce.Regularized)
        force.setFaceBoundary(LBMForce.XMin, LBMForce.DensityVelocity)
        force.setFaceBoundary(LBMForce.XMax, LBMForce.Velocity)
        force.setFaceVelocity(LBMForce.XMin, (0.2, 0.0, 0.0))
        context = make_context(system, factory, props)
        context.integrator.step(15)
        results.append((force.getFluidState(context), force.getWallForce(context)))
    scale = abs(results[0][0]).max()
    tol = 1e-12 if precision == 'double' else 1e-5
    assert abs(results[1][0] - results[0][0]).max() <= tol*scale
