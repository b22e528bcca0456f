// The particle buffers of an OpenMM CUDA-platform Context (include/lbm_b200.h, LbmOpenMMBuffers): gathers of the
// coupled atoms' positions, velocities and fixed-point forces into coupling order, the velocities written back after
// the reflection at the walls, and the coupling forces added to the fixed-point force buffer.  These are the reads and
// writes of OpenMM's buffers that the reference's CUDA kernels make (platforms/common/src/kernels/lbmCoupling.cc:
// loadPosition :47-54, reflectParticles :148-171, applyCouplingForces :2043-2053): the atoms are in the platform's
// storage order, atom_index[j] is the System index of the atom stored at slot j, and couplingIndex[atom] is the
// coupling index of a coupled atom or -1.  One thread per storage slot.
#include "openmm_buffers.cuh"
#include <cuda_runtime.h>
#include <string>

namespace lbm {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void position(const LbmOpenMMBuffers& b, int j, double out[3]) {
    if (b.precision == LBM_OPENMM_DOUBLE) {
        const double4 p = reinterpret_cast<const double4*>(b.posq)[j];
        out[0] = p.x; out[1] = p.y; out[2] = p.z;
        return;
    }
    const float4 p = reinterpret_cast<const float4*>(b.posq)[j];
    out[0] = p.x; out[1] = p.y; out[2] = p.z;
    if (b.precision == LBM_OPENMM_MIXED && b.posq_correction != nullptr) {
        // Mixed precision: the position is posq + posqCorrection, summed in double (lbmCoupling.cc:47-54).
        const float4 c = reinterpret_cast<const float4*>(b.posq_correction)[j];
        out[0] += (double) c.x; out[1] += (double) c.y; out[2] += (double) c.z;
    }
}

__device__ __forceinline__ void velocity(const LbmOpenMMBuffers& b, int j, double out[3]) {
    if (b.precision == LBM_OPENMM_SINGLE) {
        const float4 v = reinterpret_cast<const float4*>(b.velm)[j];
        out[0] = v.x; out[1] = v.y; out[2] = v.z;
    }
    else {
        const double4 v = reinterpret_cast<const double4*>(b.velm)[j];
        out[0] = v.x; out[1] = v.y; out[2] = v.z;
    }
}

__global__ void __launch_bounds__(kThreads) gatherKernel(LbmOpenMMBuffers b, const int* __restrict__ couplingIndex,
                                                         double* pos, double* vel, double* force, int withForces) {
    for (int j = blockIdx.x*blockDim.x + threadIdx.x; j < b.num_atoms; j += gridDim.x*blockDim.x) {
        const int i = couplingIndex[b.atom_index[j]];
        if (i < 0)
            continue;
        double p[3], v[3];
        position(b, j, p);
        velocity(b, j, v);
        for (int k = 0; k < 3; k++) {
            pos[3*i + k] = p[k];
            vel[3*i + k] = v[k];
        }
        if (withForces)
            for (int k = 0; k < 3; k++)
                force[3*i + k] = (double) b.force[j + (long long) k*b.padded_num_atoms]*(1.0/4294967296.0);
    }
}

__global__ void __launch_bounds__(kThreads) scatterVelocityKernel(LbmOpenMMBuffers b,
                                                                  const int* __restrict__ couplingIndex,
                                                                  const double* __restrict__ vel) {
    for (int j = blockIdx.x*blockDim.x + threadIdx.x; j < b.num_atoms; j += gridDim.x*blockDim.x) {
        const int i = couplingIndex[b.atom_index[j]];
        if (i < 0)
            continue;
        if (b.precision == LBM_OPENMM_SINGLE) {
            float4* v = reinterpret_cast<float4*>(b.velm) + j;
            *v = make_float4((float) vel[3*i], (float) vel[3*i + 1], (float) vel[3*i + 2], v->w);
        }
        else {
            double4* v = reinterpret_cast<double4*>(b.velm) + j;
            *v = make_double4(vel[3*i], vel[3*i + 1], vel[3*i + 2], v->w);
        }
    }
}

// forceBuffers[j + k padded] += (long long) (F_k 2^32), truncated toward zero as the reference's cast.
__global__ void __launch_bounds__(kThreads) addFixedPointKernel(LbmOpenMMBuffers b, const int* __restrict__ couplingIndex,
                                                                const double* __restrict__ force) {
    for (int j = blockIdx.x*blockDim.x + threadIdx.x; j < b.num_atoms; j += gridDim.x*blockDim.x) {
        const int i = couplingIndex[b.atom_index[j]];
        if (i < 0)
            continue;
        for (int k = 0; k < 3; k++)
            b.force[j + (long long) k*b.padded_num_atoms] += (long long) (force[3*i + k]*4294967296.0);
    }
}

int gridFor(int atoms) {
    return std::max(1, std::min(1184, (atoms + kThreads - 1)/kThreads));
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw Error(LBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace

void validateOpenMMBuffers(const LbmOpenMMBuffers* b, int couplingAtoms) {
    if (b == nullptr || b->posq == nullptr || b->velm == nullptr || b->force == nullptr || b->atom_index == nullptr)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_*_openmm: a buffer of the OpenMM Context is missing");
    if (b->precision != LBM_OPENMM_SINGLE && b->precision != LBM_OPENMM_MIXED && b->precision != LBM_OPENMM_DOUBLE)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_*_openmm: unknown precision of the OpenMM Context");
    if (b->num_atoms != couplingAtoms || b->padded_num_atoms < b->num_atoms)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_*_openmm: the number of atoms differs from lbm_set_coupled_atoms()");
}

void gatherOpenMM(const LbmOpenMMBuffers& b, const int* couplingIndex, double* pos, double* vel, double* force,
                  bool withForces, cudaStream_t s) {
    gatherKernel<<<gridFor(b.num_atoms), kThreads, 0, s>>>(b, couplingIndex, pos, vel, force, withForces ? 1 : 0);
    check(cudaGetLastError(), "gatherKernel");
}

void scatterVelocitiesOpenMM(const LbmOpenMMBuffers& b, const int* couplingIndex, const double* vel, cudaStream_t s) {
    scatterVelocityKernel<<<gridFor(b.num_atoms), kThreads, 0, s>>>(b, couplingIndex, vel);
    check(cudaGetLastError(), "scatterVelocityKernel");
}

void addForcesFixedPoint(const LbmOpenMMBuffers& b, const int* couplingIndex, const double* force, cudaStream_t s) {
    addFixedPointKernel<<<gridFor(b.num_atoms), kThreads, 0, s>>>(b, couplingIndex, force);
    check(cudaGetLastError(), "addFixedPointKernel");
}

} // namespace lbm
