"""GPU tests of the checkpoint format: the B200 kernel writes the kernel stream of the reference's GPU platforms
(CommonCalcLBMForceKernel::createCheckpoint, platforms/common/src/CommonLBMKernels.cpp:2019-2034) after
LBMForceImpl's header (openmmapi/src/LBMForceImpl.cpp:514-528), and reads such a stream as the reference's CUDA kernel
writes it (:2036-2058), without the B200 trailer.

The stream is read and built with the oracle's restatement (oracle/checkpoint_format.py).  A stream "of the
reference's CUDA kernel" is built from the state of the reference's own kernel (oracle/_ref, the Reference platform
compiled from its sources) after some steps: its populations, its wall force split over the wall entries as that
kernel keeps it (one entry per solid node, one per boundary node, less the static parts), and the flag of a fluid that
has advanced.  Loaded into the B200 kernel, the run continues as the reference's run does, within the tolerances of
the reference's cross-platform tests (python/tests/TestLBMForce.py:505-635: 1e-12 for the fluid, 1e-10 for the
coupling)."""
import numpy as np
import pytest

import oracle
import checkpoint_format
from cases import coupling_case, fluid_case
from lbm_b200 import checkpoint
from lbm_b200.abi import LbmError

pytestmark = pytest.mark.gpu


def lattice_momentum(force, context):
    """getWallForce() as a momentum in lattice units: F dt / (rho dx^3 dx/dt)."""
    lat = context.lattice
    return np.array(force.getWallForce(context))*lat.dt*lat.dt/(lat.density*lat.dx**4)


def geometry(force, context):
    solid = force.getSolidNodes()
    bits = oracle.find_boundaries(context.lattice, solid)[2]
    return solid, len(bits), checkpoint_format.static_wall_momentum(context.lattice, solid, bits)


def split_entries(total, count, rng):
    """`total` (3,) spread over `count` entries with random shares that sum to it."""
    shares = rng.random(count)
    shares /= shares.sum()
    entries = np.outer(total, shares)
    entries[:, -1] = total - entries[:, :-1].sum(axis=1)
    return entries


@pytest.mark.parametrize('walls,precision', [('walls', 'double'), ('regularized', 'single'), ('dvfaces', 'double'),
                                             ('faces', 'half'), ('periodic', 'bfloat16')])
def test_checkpoint_is_the_reference_stream(walls, precision):
    context, force = fluid_case(walls, None, {'Precision': precision})
    context.integrator.step(5)
    data = force.createCheckpoint(context)
    start = checkpoint.read_header(data, 'CUDA', context.lattice, 0)
    assert data[:8] == b'LBMCKPT1'
    stream = data[start:]
    n = context.lattice.nx*context.lattice.ny*context.lattice.nz
    solid, num_boundary, static = geometry(force, context)
    arrays = checkpoint_format.read_stream(stream, n, 0, len(solid), num_boundary)
    e = 8 if precision == 'double' else 4
    assert (arrays['element_size'], arrays['noise_drawn'], arrays['has_advanced']) == (e, 0, 1)
    state = force.getFluidState(context)
    # FP32, FP16 and BF16 storage hold values that a float represents exactly.
    assert np.array_equal(arrays['populations'], state)
    wall = checkpoint_format.stored_wall_momentum(arrays, len(solid)) + (static if solid else 0)
    expected = lattice_momentum(force, context)
    tol = 1e-12 if e == 8 else 1e-6
    assert abs(wall - expected).max() <= tol*max(1.0, abs(expected).max())
    assert stream[arrays['end']:arrays['end'] + 8] == b'B200LBM1'
    assert len(stream) == sum(context.kernel.checkpoint_layout())
    context.close()


@pytest.mark.parametrize('walls', ['walls', 'regularized', 'dvfaces'])
def test_reference_stream_continues_the_reference_run(walls):
    rng = np.random.default_rng(11)
    ref, ref_force = fluid_case(walls, oracle.ReferenceKernel)
    ref.integrator.step(5)
    state = ref_force.getFluidState(ref)
    solid, num_boundary, static = geometry(ref_force, ref)
    stored = lattice_momentum(ref_force, ref) - static
    if num_boundary:
        wall_part = rng.random()*stored
        boundary = split_entries(stored - wall_part, num_boundary, rng)
    else:
        wall_part, boundary = stored, None
    entries = split_entries(wall_part, len(solid), rng)
    data = (checkpoint.write_header('CUDA', ref.lattice, 0) +
            checkpoint_format.write_stream(8, state, True, entries, 0, len(solid), num_boundary, boundary=boundary))
    context, force = fluid_case(walls, None, {'Precision': 'double'})
    context.setStepCount(ref.getStepCount())
    force.loadCheckpoint(context, data)
    assert np.array_equal(force.getFluidState(context), state)
    ref_wall = np.array(ref_force.getWallForce(ref))
    assert abs(np.array(force.getWallForce(context)) - ref_wall).max() <= 1e-12*max(1.0, abs(ref_wall).max())
    ref.integrator.step(7)
    context.integrator.step(7)
    ref_state, got = ref_force.getFluidState(ref), force.getFluidState(context)
    assert abs(got - ref_state).max() <= 1e-12*abs(ref_state).max()
    ref_wall = np.array(ref_force.getWallForce(ref))
    assert abs(np.array(force.getWallForce(context)) - ref_wall).max() <= 1e-10*max(1.0, abs(ref_wall).max())
    ref.close()
    context.close()


@pytest.mark.parametrize('drag,stencil', [('Centered', 'Keys'), ('Explicit', 'NearestNode')])
def test_reference_stream_continues_the_coupled_reference_run(drag, stencil):
    """Four coupled particles next to the wall plane: the particles' wall momentum is one of the arrays."""
    rng = np.random.default_rng(12)
    ref, ref_force = coupling_case(True, drag, stencil, oracle.ReferenceKernel)
    ref.integrator.step(10)
    state = ref_force.getFluidState(ref)
    solid, num_boundary, static = geometry(ref_force, ref)
    stored = lattice_momentum(ref_force, ref) - static
    particle_share = rng.random()*stored
    particle_wall = split_entries(particle_share, 4, rng)
    entries = split_entries(stored - particle_share, len(solid), rng)
    data = (checkpoint.write_header('CUDA', ref.lattice, 4) +
            checkpoint_format.write_stream(8, state, True, entries, 4, len(solid), num_boundary,
                                           particle_wall=particle_wall))
    context, force = coupling_case(True, drag, stencil, None, {'Precision': 'double'})
    context.setPositions(ref.positions)
    context.setVelocities(ref.velocities)
    context.setStepCount(ref.getStepCount())
    force.loadCheckpoint(context, data)
    ref_wall = np.array(ref_force.getWallForce(ref))
    assert abs(np.array(force.getWallForce(context)) - ref_wall).max() <= 1e-12*max(1.0, abs(ref_wall).max())
    ref.integrator.step(10)
    context.integrator.step(10)
    for got, expected, name in ((context.positions, ref.positions, 'positions'),
                                (context.velocities, ref.velocities, 'velocities'),
                                (force.getFluidState(context), ref_force.getFluidState(ref), 'state'),
                                (force.getWallForce(context), ref_force.getWallForce(ref), 'wall')):
        got, expected = np.asarray(got), np.asarray(expected)
        assert abs(got - expected).max() <= 1e-10*max(1.0, abs(expected).max()), name
    ref.close()
    context.close()


def test_stream_of_another_storage_loads_without_its_trailer():
    """A checkpoint of FP16 storage (element size 4, the trailer of FP16) loads into FP32 storage through the stream:
    the FP16 values are floats, so the state is the same, and the runs continue alike within the FP16 rounding."""
    a, force_a = fluid_case('regularized', None, {'Precision': 'half'})
    a.integrator.step(4)
    data = force_a.createCheckpoint(a)
    b, force_b = fluid_case('regularized', None, {'Precision': 'single'})
    b.setStepCount(a.getStepCount())
    force_b.loadCheckpoint(b, data)
    assert np.array_equal(force_b.getFluidState(b), force_a.getFluidState(a))
    wall_a, wall_b = np.array(force_a.getWallForce(a)), np.array(force_b.getWallForce(b))
    assert abs(wall_b - wall_a).max() <= 1e-6*abs(wall_a).max()
    a.close()
    b.close()


def test_checkpoint_mismatches_are_rejected():
    context, force = fluid_case('walls', None, {'Precision': 'double'})
    context.integrator.step(2)
    data = force.createCheckpoint(context)
    start = checkpoint.read_header(data, 'CUDA', context.lattice, 0)
    single, force_single = fluid_case('walls', None, {'Precision': 'single'})
    with pytest.raises(LbmError, match='written with a different precision'):
        force_single.loadCheckpoint(single, data)
    with pytest.raises(LbmError, match='the checkpoint is truncated'):
        force.loadCheckpoint(context, data[:start + 100])
    other = checkpoint.write_header('Reference', context.lattice, 0) + data[start:]
    with pytest.raises(LbmError, match='written on the platform Reference, not on CUDA'):
        force.loadCheckpoint(context, other)
    regularized, force_reg = fluid_case('regularized', None, {'Precision': 'double'})
    with pytest.raises(LbmError, match='different wall scheme'):
        force_reg.loadCheckpoint(regularized, data)
    for c in (context, single, regularized):
        c.close()
