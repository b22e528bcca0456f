"""GPU tests of the drop-in: the B200 platform kernel (openmm-lbm_b200/openmm/B200LBMKernels.cpp, the reference's
CalcLBMForceKernel interface over liblbm_b200.so), created by its kernel factory and driven through OpenMM's kernel
interface (initialize, beginStep, execute, getFluidState, getWallForce, getFluidFields, createCheckpoint,
loadCheckpoint) exactly as the reference's ReferenceCalcLBMForceKernel is driven, by the same driver
(oracle/ref_driver.cpp built as oracle/_ref/libadapter_lbm.so).  Expectations: the outputs of the reference's own kernel
on the reference's cross-platform cases (tests/golden/, python/tests/TestLBMForce.py:505-635, with its tolerances 1e-12
for the fluid and 1e-10 for the coupling), its evaluation sequence, and its getFluidFields() with the halo."""
import os

import numpy as np
import pytest

import oracle
from cases import (COUPLING_CASES, EVALUATION_CASES, FLUID_WALLS, coupling_case, evaluation_case, evaluation_sequence,
                   fluid_case)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.adapter_available(), reason='oracle/_ref/libadapter_lbm.so is not built')]

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_cases.npz'))
SEQUENCES = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'evaluation_sequences.npz'))


def adapter(lattice, masses, solid):
    return oracle.AdapterKernel(lattice, masses, solid, 'double')


@pytest.mark.parametrize('walls', FLUID_WALLS)
def test_adapter_fluid_matches_reference(walls):
    context, force = fluid_case(walls, adapter)
    context.integrator.step(40)
    state, wall = force.getFluidState(context), force.getWallForce(context)
    context.close()
    ref_state, ref_wall = GOLDEN['fluid_%s_state' % walls], GOLDEN['fluid_%s_wall' % walls]
    assert abs(state - ref_state).max() <= 1e-12*abs(ref_state).max()
    assert abs(wall - ref_wall).max() <= 1e-10*max(1.0, abs(ref_wall).max())


@pytest.mark.parametrize('walls,drag,stencil', COUPLING_CASES)
def test_adapter_coupling_matches_reference(walls, drag, stencil):
    context, force = coupling_case(walls, drag, stencil, adapter)
    context.integrator.step(60)
    key = 'coupling_%s_%s_%s' % (walls, drag, stencil)
    for value, name in ((context.positions, 'positions'), (context.velocities, 'velocities'),
                        (force.getFluidState(context), 'state'), (force.getWallForce(context), 'wall')):
        ref = GOLDEN[key + '_' + name]
        assert abs(value - ref).max() <= 1e-10*max(1.0, abs(ref).max()), name
    context.close()


@pytest.mark.parametrize('walls,drag,stencil', EVALUATION_CASES)
def test_adapter_evaluation_rules_match_reference(walls, drag, stencil):
    context, force = evaluation_case(walls, drag, stencil, adapter)
    got = evaluation_sequence(context)
    context.close()
    for name, value in got.items():
        ref = SEQUENCES['%s_%s_%s_%s' % (walls, drag, stencil, name)]
        assert abs(value - ref).max() <= 1e-10*max(1.0, abs(ref).max()), name


@pytest.mark.skipif(not oracle.reference_available(), reason='oracle/_ref/libref_lbm.so is not built')
@pytest.mark.parametrize('walls', ['faces', 'walls'])
def test_adapter_fields_with_halo_match_reference(walls):
    """getFluidFields() with the halo (LBMKernels.h:139-144): the lattice extended by one node on every side, the
    nodes across a periodic boundary for the density (whose halo the driver exchanges), NaN for the velocity (whose
    halo it does not) and beyond open faces."""
    results = []
    for factory in (oracle.ReferenceKernel, adapter):
        context, force = fluid_case(walls, factory)
        context.integrator.step(5)
        results.append(oracle.fields_with_halo(context.kernel))
        context.close()
    (d_ref, v_ref), (d, v) = results
    assert (np.isnan(d) == np.isnan(d_ref)).all() and (np.isnan(v) == np.isnan(v_ref)).all()
    assert np.isnan(v_ref).any() and not np.isnan(d_ref[1:-1, 1:-1, 1:-1]).any()
    ok = ~np.isnan(d_ref)
    assert abs(d[ok] - d_ref[ok]).max() <= 1e-12*abs(d_ref[ok]).max()
    ok = ~np.isnan(v_ref)
    assert abs(v[ok] - v_ref[ok]).max() <= 1e-12*max(1e-30, abs(v_ref[ok]).max())


def test_adapter_checkpoint_restarts_bit_for_bit():
    """createCheckpoint() / loadCheckpoint() of the platform kernel through OpenMM's streams: a run restarted from a
    checkpoint continues as the uninterrupted run, bit for bit."""
    context, force = coupling_case(True, 'Centered', 'Keys', adapter)
    context.integrator.step(10)
    data = context.kernel.create_checkpoint()
    positions, velocities, step = context.positions.copy(), context.velocities.copy(), context.getStepCount()
    context.integrator.step(10)
    expected = force.getFluidState(context), context.positions.copy()
    context.close()
    context, force = coupling_case(True, 'Centered', 'Keys', adapter)
    context.kernel.load_checkpoint(data)
    context.setPositions(positions)
    context.setVelocities(velocities)
    context.setStepCount(step)
    context.integrator.step(10)
    got = force.getFluidState(context), context.positions.copy()
    context.close()
    assert (got[0] == expected[0]).all() and (got[1] == expected[1]).all()


def test_checkpoint_reporter_and_load_continue_bit_for_bit(tmp_path):
    """saveCheckpoint / loadCheckpoint (python/openmmlbm.i:513-586) and LBMCheckpointReporter on the B200 kernel: a
    run rebuilt from the reporter's last file continues as the uninterrupted run, bit for bit."""
    import lbm_b200
    path = os.path.join(str(tmp_path), 'run.chk')
    context, force = coupling_case(True, 'Centered', 'Keys', None, {'Precision': 'single'}, temperature=300.0)
    simulation = lbm_b200.Simulation(context)
    simulation.reporters.append(lbm_b200.LBMCheckpointReporter(path, 6, force))
    simulation.step(12)
    simulation.reporters = []
    simulation.step(6)
    expected = force.getFluidState(context), context.positions.copy(), context.velocities.copy()
    context.close()
    context, force = coupling_case(True, 'Centered', 'Keys', None, {'Precision': 'single'}, temperature=300.0)
    lbm_b200.loadCheckpoint(path, context, force)
    assert context.getStepCount() == 12
    context.integrator.step(6)
    got = force.getFluidState(context), context.positions.copy(), context.velocities.copy()
    context.close()
    for a, b in zip(expected, got):
        assert (a == b).all()


def test_adapter_checkpoint_is_the_reference_stream():
    """Through OpenMM's stream interface the platform kernel writes what the library writes (the kernel stream of
    the reference's GPU platforms, CommonLBMKernels.cpp:2019-2034, then the B200 trailer), and it reads the stream
    alone, as the reference's CUDA kernel writes it, from a stream that ends there."""
    context, force = fluid_case('regularized', adapter)
    context.integrator.step(5)
    data = context.kernel.create_checkpoint()
    state, wall = force.getFluidState(context), np.array(force.getWallForce(context))
    context.close()
    library, library_force = fluid_case('regularized', None, {'Precision': 'double'})
    library.integrator.step(5)
    stream_bytes, trailer_bytes = library.kernel.checkpoint_layout()
    # The same stream; the trailers differ in the seed, which each kernel drew for itself (seed 0).
    assert data[:stream_bytes] == library.kernel.create_checkpoint()[:stream_bytes]
    assert len(data) == stream_bytes + trailer_bytes and data[stream_bytes:stream_bytes + 8] == b'B200LBM1'
    library.close()
    fresh, fresh_force = fluid_case('regularized', adapter)
    fresh.kernel.load_checkpoint(data[:stream_bytes])
    assert np.array_equal(fresh_force.getFluidState(fresh), state)
    assert abs(np.array(fresh_force.getWallForce(fresh)) - wall).max() <= 1e-12*abs(wall).max()
    fresh.close()
