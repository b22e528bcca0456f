"""CPU tests of the oracle: the C restatement (oracle/lbm_oracle.c) against the golden outputs of the reference's
own kernel (tests/golden/reference_cases.npz, made by tests/golden/make_golden.py from oracle/_ref), against the
reference build itself where it is present, and against published known answers (Philox4x32-10, the stencil
moments of tests/TestLBMStencils.h, the orthogonality of the fluctuation basis of TestLBMFluctuations.h)."""
import os

import numpy as np
import pytest

from cases import (COUPLING_CASES, EVALUATION_CASES, FLUID_WALLS, coupling_case, evaluation_case, evaluation_sequence,
                   fluid_case)
import oracle
from oracle import OracleKernel

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_cases.npz'))
SEQUENCES = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'evaluation_sequences.npz'))


def sequential(lattice, masses, solid):
    return OracleKernel(lattice, masses, solid, random='sequential')


@pytest.mark.parametrize('walls', FLUID_WALLS)
def test_oracle_fluid_matches_reference_golden(walls):
    context, force = fluid_case(walls, sequential)
    context.integrator.step(40)
    state, wall = force.getFluidState(context), force.getWallForce(context)
    ref_state, ref_wall = GOLDEN['fluid_%s_state' % walls], GOLDEN['fluid_%s_wall' % walls]
    # The tolerance of the reference's cross-platform test (TestLBMForce.py:567-570).
    assert abs(state - ref_state).max() <= 1e-12*abs(ref_state).max()
    assert abs(wall - ref_wall).max() <= 1e-10*max(1.0, abs(ref_wall).max())


@pytest.mark.parametrize('walls,drag,stencil', COUPLING_CASES)
def test_oracle_coupling_matches_reference_golden(walls, drag, stencil):
    context, force = coupling_case(walls, drag, stencil, sequential)
    context.integrator.step(60)
    key = 'coupling_%s_%s_%s' % (walls, drag, stencil)
    for value, name in ((context.positions, 'positions'), (context.velocities, 'velocities'),
                        (force.getFluidState(context), 'state'), (force.getWallForce(context), 'wall')):
        ref = GOLDEN[key + '_' + name]
        # TestLBMForce.py:633-635.
        assert abs(value - ref).max() <= 1e-10*max(1.0, abs(ref).max()), name


@pytest.mark.parametrize('walls,drag,stencil', EVALUATION_CASES)
def test_oracle_evaluation_rules_match_reference_golden(walls, drag, stencil):
    """The evaluation rules (ReferenceLBMKernels.cpp:341-401): no coupling force before the first step, the next
    step's forces between steps (with the momentum removal of that step), the same forces on a repeated evaluation,
    and a run that queries between steps ends where the reference's does."""
    context, force = evaluation_case(walls, drag, stencil, sequential)
    got = evaluation_sequence(context)
    for name, value in got.items():
        ref = SEQUENCES['%s_%s_%s_%s' % (walls, drag, stencil, name)]
        assert abs(value - ref).max() <= 1e-10*max(1.0, abs(ref).max()), name
    assert (got['step_repeated_evaluation'] == got['step_first_evaluation']).all()


@pytest.mark.skipif(not oracle.reference_available(), reason='the reference build (oracle/_ref) is absent')
def test_oracle_fluctuating_matches_reference_bitwise():
    """With the shim's generator stream, the restatement draws the same normal numbers as the reference, in the
    same order, for the particles, the collision and the boundary nodes."""
    from cases import coupling_case as cc
    for walls in ('regularized', 'dvfaces'):
        results = []
        for factory in (oracle.ReferenceKernel, sequential):
            context, force = fluid_case(walls, factory)
            force.setFluidFluctuations(True)
            context.close()
            import lbm_b200
            system = context.system
            for f in system.forces:
                if isinstance(f, lbm_b200.LBMForce):
                    f.setFluidFluctuations(True)
                    f.setTemperature(300.0)
                    f.setRandomNumberSeed(1234)
                    if walls == 'dvfaces':
                        f.setFaceBoundary(f.ZMin, f.DensityVelocity)
            ctx = lbm_b200.Context(system, lbm_b200.VerletIntegrator(0.01), factory)
            ctx.setPositions([(0.1, 0.7, 0.3)])
            ctx.integrator.step(10)
            results.append(f.getFluidState(ctx))
        assert abs(results[0] - results[1]).max() <= 1e-12*abs(results[0]).max()
    results = []
    for factory in (oracle.ReferenceKernel, sequential):
        context, force = cc(True, 'Explicit', 'Keys', factory, temperature=300.0)
        context.integrator.step(10)
        results.append(context.velocities.copy())
    assert abs(results[0] - results[1]).max() <= 1e-12*abs(results[0]).max()


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors published with the Random123 library (kat_vectors)."""
    assert oracle.philox4x32_10([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle.philox4x32_10([0xffffffff]*4, [0xffffffff]*2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert oracle.philox4x32_10([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_philox_normals_are_standard():
    values = np.array([oracle.philox_normal(7, 0, i, 3, m) for i in range(2000) for m in range(15)])
    assert abs(values.mean()) < 0.02 and abs(values.std() - 1.0) < 0.02


@pytest.mark.parametrize('stencil', [1, 2, 3])
def test_stencil_weight_moments(stencil):
    """testStencilMoments (TestLBMStencils.h:27-63): sum 1, first moment 0; the three-point kernel has sum of
    squares 1/2."""
    for s in np.linspace(3.0, 4.0, 23):
        index, weight = oracle.axis_weights(stencil, s, 16, False)
        weight = np.array(weight)
        assert abs(weight.sum() - 1.0) < 1e-14
        assert abs(np.dot(weight, np.array(index) - s)) < 1e-14
        if stencil == 2:
            assert abs((weight**2).sum() - 0.5) < 1e-14


def test_stencil_open_axis_merges_weights():
    """Open faces: the stencil stops at the last node and merges the weights (LBMStencils.h:73-95)."""
    index, weight = oracle.axis_weights(3, 0.3, 8, True)
    assert index == [0, 0, 1, 2] and weight[1] == 0.0 and abs(sum(weight) - 1.0) < 1e-14


def test_fluctuation_basis_orthogonal():
    """testBasisOrthogonality (TestLBMFluctuations.h:58-69), through the random part: it carries no mass and no
    momentum, and mode k receives phi_k r_k."""
    c = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
                  [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1], [1, 0, 1],
                  [-1, 0, -1], [-1, 0, 1], [1, 0, -1]])
    rng = np.random.default_rng(1)
    for _ in range(5):
        xi = oracle.fluctuation(rng.normal(size=15), 0.7, 1.3)
        assert abs(xi.sum()) < 1e-15 and abs(c.T @ xi).max() < 1e-15
        assert abs(xi).max() > 0.01
