"""GPU tests of the failure paths, made to fire without any fault: the iteration cap of the centred stencil drag's
conjugate gradients (LBM_ERR_CG_NOT_CONVERGED with the reference's message, ReferenceLBMKernels.cpp:864-866), the
bounded grid barrier of its cooperative solve (LBM_ERR_DEVICE_TIMEOUT), and the bounded wait for the tensor cores of
the warm start's convolutions.  The limits are lowered through the ABI; every wait still ends, and the tests check
that a failed call leaves nothing behind: the next call gives what a run without the failure gives."""
import numpy as np
import pytest
import torch

from cases import coupling_case
from lbm_b200.abi import LBM_ERR_CG_NOT_CONVERGED, LBM_ERR_DEVICE_TIMEOUT, LbmError

pytestmark = pytest.mark.gpu


def centred_case():
    return coupling_case(False, 'Centered', 'Keys', None, {'Precision': 'double'}, seed=3)


def uninterrupted(steps):
    context, force = centred_case()
    context.integrator.step(steps)
    out = (context.positions.copy(), context.velocities.copy(), force.getFluidState(context))
    context.close()
    return out


def test_cg_iteration_cap_reports_non_convergence_and_leaves_no_reaction():
    expected = uninterrupted(5)
    context, force = centred_case()
    context.integrator.step(2)
    context.kernel.set_solver_limits(max_iterations=1)
    with pytest.raises(LbmError) as failure:
        context.integrator.step(1)
    assert failure.value.status == LBM_ERR_CG_NOT_CONVERGED
    assert 'did not converge in 1 iterations of the conjugate gradients' in str(failure.value)
    assert context.getStepCount() == 2
    # The step is taken again with the default cap: the failed solve left no reaction on the fluid.
    context.kernel.set_solver_limits()
    context.integrator.step(3)
    got = (context.positions, context.velocities, force.getFluidState(context))
    context.close()
    for a, b, name in zip(expected, got, ('positions', 'velocities', 'state')):
        assert abs(b - a).max() <= 1e-13*max(1.0, abs(a).max()), name


def crowded_case(count=600):
    """`count` particles of mass 100 spread over a 16^3 lattice, Keys stencil, centred drag with friction 10/ps and a
    field: the cooperative solve runs on count/32 blocks of 1024 threads (one warp per particle)."""
    import lbm_b200
    from lbm_b200 import LBMForce
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
    force.setInterpolationStencil(LBMForce.Keys)
    force.setFriction(10.0)
    force.setTemperature(0.0)
    force.setFluidMomentumRemovalFrequency(0)
    context = lbm_b200.Context(system, lbm_b200.VerletIntegrator(0.01), None, {'Precision': 'double'})
    rng = np.random.default_rng(21)
    context.setPositions(rng.uniform(0.0, 8.0, (count, 3)))
    context.setVelocities(rng.normal(0.0, 0.5, (count, 3)))
    return context, force


def test_grid_barrier_timeout_is_reported_and_the_next_solve_succeeds():
    """A limit of one poll makes the blocks that wait at a grid barrier of the cooperative solve (19 blocks here) give
    up: the solve leaves with LBM_ERR_DEVICE_TIMEOUT, the barrier starts the next solve from zero, and the run goes on
    as if the failed attempt had not been made."""
    context, force = crowded_case()
    context.integrator.step(5)
    assert context.kernel.solver_fallback_steps() == 0
    expected = (context.positions.copy(), context.velocities.copy(), force.getFluidState(context))
    context.close()
    context, force = crowded_case()
    context.integrator.step(2)
    context.kernel.set_solver_limits(barrier_polls=1)
    timeouts = 0
    for _ in range(5):
        try:
            context.integrator.step(1)
        except LbmError as failure:
            assert failure.status == LBM_ERR_DEVICE_TIMEOUT
            assert 'grid barrier' in str(failure)
            timeouts += 1
            break
    assert timeouts == 1
    steps_done = context.getStepCount()
    context.kernel.set_solver_limits()
    context.integrator.step(5 - steps_done)
    got = (context.positions, context.velocities, force.getFluidState(context))
    context.close()
    for a, b, name in zip(expected, got, ('positions', 'velocities', 'state')):
        assert abs(b - a).max() <= 1e-13*max(1.0, abs(a).max()), name


def test_tensor_core_wait_timeout_is_reported_and_the_next_convolution_succeeds():
    """With a wait limit of 0 every convolution gives up at its first wait for the tensor cores (after they finish the
    stage in flight, so that the tensor memory is freed only when they are done): lbm_conv3d_status reports the
    timeout; with the default limit the same convolution gives its normal result."""
    from lbm_b200 import warmstart as ws
    lib = ws._lib()
    rng = np.random.default_rng(7)
    x = ws._volume(torch.as_tensor(rng.standard_normal((1, 16, 6, 7, 8)), dtype=torch.float32).to(torch.bfloat16).cuda())
    w = torch.as_tensor(rng.standard_normal((32, 27, 16))*0.2, dtype=torch.float32).to(torch.bfloat16).cuda()
    expected = ws.conv3d_forward(x, w, None, False)
    ws.conv_status()
    try:
        assert lib.lbm_conv3d_set_wait_limit(0) == 0
        ws.conv3d_forward(x, w, None, False)
        with pytest.raises(LbmError) as failure:
            ws.conv_status()
        assert failure.value.status == LBM_ERR_DEVICE_TIMEOUT
    finally:
        assert lib.lbm_conv3d_set_wait_limit(-1) == 0
    again = ws.conv3d_forward(x, w, None, False)
    ws.conv_status()
    assert torch.equal(again, expected)
