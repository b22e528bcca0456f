"""Generate tests/golden/reference_cases.npz and tests/golden/evaluation_sequences.npz: outputs of the reference's own Reference-platform kernel
(ReferenceCalcLBMForceKernel, compiled unmodified from the reference sources into oracle/_ref by
`make -C oracle ref`) on the cases of the reference's cross-platform tests (python/tests/TestLBMForce.py:
505-635), driven by the OpenMM call order of lbm_b200.harness; and the coupled forces of a scripted sequence of force
evaluations (before the first step, between steps, a repeated evaluation within a step) that pins the evaluation rules
of ReferenceCalcLBMForceKernel (platforms/reference/src/ReferenceLBMKernels.cpp:341-401).

    python tests/golden/make_golden.py

The fixtures pin the C restatement (oracle/lbm_oracle.c) where the reference build is absent (the GPU box).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import conftest  # noqa: E402,F401  (imports lbm_b200 and puts oracle/ on the path)
from cases import (COUPLING_CASES, EVALUATION_CASES, FLUID_WALLS, coupling_case, evaluation_case,  # noqa: E402
                   evaluation_sequence, fluid_case)
from oracle import ReferenceKernel  # noqa: E402


def main():
    out = {}
    for walls in FLUID_WALLS:
        context, force = fluid_case(walls, ReferenceKernel)
        context.integrator.step(40)
        out['fluid_%s_state' % walls] = force.getFluidState(context)
        out['fluid_%s_wall' % walls] = force.getWallForce(context)
    for walls, drag, stencil in COUPLING_CASES:
        key = 'coupling_%s_%s_%s' % (walls, drag, stencil)
        context, force = coupling_case(walls, drag, stencil, ReferenceKernel)
        context.integrator.step(60)
        out[key + '_positions'] = context.positions.copy()
        out[key + '_velocities'] = context.velocities.copy()
        out[key + '_state'] = force.getFluidState(context).astype(np.float64)
        out[key + '_wall'] = force.getWallForce(context)
    np.savez_compressed(os.path.join(HERE, 'reference_cases.npz'), **out)
    sequences = {}
    for walls, drag, stencil in EVALUATION_CASES:
        context, force = evaluation_case(walls, drag, stencil, ReferenceKernel)
        for name, value in evaluation_sequence(context).items():
            sequences['%s_%s_%s_%s' % (walls, drag, stencil, name)] = value
        context.close()
    np.savez_compressed(os.path.join(HERE, 'evaluation_sequences.npz'), **sequences)


if __name__ == '__main__':
    main()
