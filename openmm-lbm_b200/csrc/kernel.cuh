// The B200 LBM force kernel: the host object behind the C ABI.  It mirrors the platform kernel
// interface CalcLBMForceKernel (openmmapi/include/LBMKernels.h:97-189) and the evaluation rules of the
// reference's ReferenceCalcLBMForceKernel (platforms/reference/src/ReferenceLBMKernels.cpp:308-401):
// the fluid advances once per integration step, on the first evaluation after beginStep(); evaluations
// between steps give the coupling force of the next step without its reaction; a repeated evaluation of a
// step reuses its forces.
#pragma once

#include "fluid.cuh"
#include <memory>

namespace lbm {

class CouplingEngine;

class B200Kernel {
public:
    B200Kernel(const LbmLatticeParameters& lattice, const LbmOptions& options, int numParticles, const double* masses,
               int numSolid, const int* solid);
    ~B200Kernel();
    void beginStep(long long stepCount, const LbmParticleArrays* particles);
    double execute(long long stepCount, const LbmParticleArrays* particles, bool includeForces, bool includeEnergy);
    void copyParameters(const LbmLatticeParameters& lattice);
    void getFluidFields(double* density, double* velocity);
    double getFluidMachNumber();
    void getWallForce(double force[3]);
    void getFluidState(double* state);
    void setFluidState(const double* state);
    size_t checkpointSize();
    void createCheckpoint(void* buffer, size_t bytes);
    void loadCheckpoint(const void* buffer, size_t bytes);
    void setCheckpointElementSize(int elementSize);
    void checkpointLayout(size_t& streamBytes, size_t& trailerBytes);
    long long numNodes() const { return fluid->numNodes(); }
    int storage() const { return fluid->storage(); }
    cudaStream_t getStream() const { return stream; }
    FluidEngine& fluidEngine() { return *fluid; }
    int solverIterations() const;
    long long solverFallbackSteps() const;
    void setSolverLimits(int maxIterations, long long barrierPolls);
    // The OpenMM Context interface: coupled atoms as System indices, then beginStep/execute on its buffers.
    void setCoupledAtoms(int numAtoms, int numCoupled, const int* particles);
    void beginStepOpenMM(long long stepCount, const LbmOpenMMBuffers* buffers);
    double executeOpenMM(long long stepCount, const LbmOpenMMBuffers* buffers, bool includeForces);
    void setFluidEquilibrium(const double* density, const double* velocity, bool onDevice, bool strain);
    long long steadySolve(long long firstStep, int interval, double tolerance, long long maxSteps, double* residual);
private:
    // The evaluation rules of execute(); returns whether the coupling forces are to be added to the caller's forces.
    bool evaluate(long long stepCount, const LbmParticleArrays* particles, bool includeForces);
    LbmParticleArrays stagingArrays();
    void advanceFluid(const LbmParticleArrays* particles);
    void computeNextStepForces(long long stepCount, const LbmParticleArrays* particles);
    void checkMachNumber();
    LbmLatticeParameters lattice;
    Geometry geometry;
    cudaStream_t stream;
    bool ownStream;
    int device;
    std::unique_ptr<FluidEngine> fluid;
    std::unique_ptr<CouplingEngine> coupling;
    int numParticles;
    bool stepPending, stepForcesCurrent, stepWallValid;
    long long stepIndex;
    double hostWallMomentum[3];     // reflection at the walls and reactions on solid nodes, Da nm/ps
    // The checkpoint stream of the reference's GPU platforms: its element size, and the static wall momentum (the part
    // w_q of the populations, the same in every step) that its readers add to the stored momentum, lattice units.
    int checkpointElementSize;
    double staticWall[3];
    bool rawPopulationsInTrailer() const;
    double wallMomentumScale() const;
    // The OpenMM Context interface: couplingIndex[atom] (-1 for an atom that is not coupled) and the coupled atoms'
    // positions, velocities and other forces gathered into coupling order (device memory).
    int openmmAtoms = 0;
    int* couplingIndexDev = nullptr;
    double* stageDev = nullptr;
};

} // namespace lbm
