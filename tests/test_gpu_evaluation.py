"""GPU tests of the evaluation rules of the kernel (ReferenceLBMKernels.cpp:341-401) through the C ABI: the coupled
forces of a scripted sequence of evaluations -- before the first step (no coupling force), between steps (the next
step's forces, with that step's momentum removal), a repeated evaluation within a step (the same forces) -- against
the reference's own outputs (tests/golden/evaluation_sequences.npz, made by tests/golden/make_golden.py from the
reference's kernel), and with random forces path by path against the oracle's Philox mode.

Tolerances: those of the reference's cross-platform coupling test in double precision (TestLBMForce.py:633-635,
1e-10 of the largest value); 1e-5 for single-precision storage."""
import os

import numpy as np
import pytest

from cases import EVALUATION_CASES, evaluation_case, evaluation_sequence
from oracle import OracleKernel

pytestmark = pytest.mark.gpu

SEQUENCES = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'evaluation_sequences.npz'))


@pytest.mark.parametrize('precision,tolerance', [('double', 1e-10), ('single', 1e-5)])
@pytest.mark.parametrize('walls,drag,stencil', EVALUATION_CASES)
def test_evaluation_rules_match_reference(walls, drag, stencil, precision, tolerance):
    context, force = evaluation_case(walls, drag, stencil, None, {'Precision': precision})
    got = evaluation_sequence(context)
    context.close()
    for name, value in got.items():
        ref = SEQUENCES['%s_%s_%s_%s' % (walls, drag, stencil, name)]
        assert abs(value - ref).max() <= tolerance*max(1.0, abs(ref).max()), name
    # A repeated evaluation reuses the forces of the step (ReferenceLBMKernels.cpp:352-365), bit for bit.
    assert (got['step_repeated_evaluation'] == got['step_first_evaluation']).all()
    assert (got['between_steps_again'] == got['between_steps']).all()


@pytest.mark.parametrize('walls,drag,stencil', EVALUATION_CASES)
def test_noisy_evaluation_rules_follow_oracle_pathwise(walls, drag, stencil):
    """At 300 K the next-step forces between steps carry the random forces of that step, drawn once per step: the
    query, the step that follows and a repeated evaluation all see the same numbers (the same Philox counters on
    the GPU and in the oracle)."""
    results = []
    for factory, props in ((OracleKernel, None), (None, {'Precision': 'double'})):
        context, force = evaluation_case(walls, drag, stencil, factory, props, temperature=300.0)
        results.append(evaluation_sequence(context))
        context.close()
    for name in results[0]:
        a, b = results[0][name], results[1][name]
        assert abs(b - a).max() <= 1e-10*max(1.0, abs(a).max()), name
    assert (results[1]['between_steps'] == results[1]['step_first_evaluation']).all()
