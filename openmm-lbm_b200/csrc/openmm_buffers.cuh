// Device gathers and scatters between the buffers of an OpenMM CUDA-platform Context (LbmOpenMMBuffers) and the
// coupling-order particle arrays of the kernel (openmm_buffers.cu).
#pragma once

#include "lbm_internal.h"
#include <cuda_runtime.h>
#include <algorithm>

namespace lbm {

// Checks the buffers of a call (atoms as given to lbm_set_coupled_atoms); throws Error.
void validateOpenMMBuffers(const LbmOpenMMBuffers* buffers, int couplingAtoms);
// Positions and velocities (and with withForces the fixed-point forces, times 2^-32) of the coupled atoms, in coupling
// order, into 3-double-per-particle device arrays.
void gatherOpenMM(const LbmOpenMMBuffers& buffers, const int* couplingIndex, double* positions, double* velocities,
                  double* forces, bool withForces, cudaStream_t stream);
// The coupled atoms' velocities back into velm (the fourth component, 1/m, is kept).
void scatterVelocitiesOpenMM(const LbmOpenMMBuffers& buffers, const int* couplingIndex, const double* velocities,
                             cudaStream_t stream);
// forces (kJ/mol/nm, coupling order) added to the fixed-point force buffer.
void addForcesFixedPoint(const LbmOpenMMBuffers& buffers, const int* couplingIndex, const double* forces,
                         cudaStream_t stream);

} // namespace lbm
