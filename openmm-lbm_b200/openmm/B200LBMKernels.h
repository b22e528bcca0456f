/*
 * The B200 platform kernel of openmm-lbm: LBMPlugin::CalcLBMForceKernel (openmmapi/include/LBMKernels.h:97-189)
 * implemented over the C ABI of liblbm_b200.so (include/lbm_b200.h), to be registered where the reference registers
 * its CUDA kernel (platforms/cuda/src/CudaLBMKernelFactory.cpp:42-72).
 *
 * B200CalcLBMForceKernel does everything that does not depend on where OpenMM keeps the particles; a subclass reads
 * and writes them:
 *   B200HostDataLBMKernel  the particles in host vectors in System order (OpenMM's ReferencePlatform::PlatformData:
 *                          positions, velocities, forces), copied through the host arrays of lbm_begin_step and
 *                          lbm_execute;
 *   B200CudaDataLBMKernel  the particles in the device buffers of OpenMM's CUDA platform (posq, posqCorrection,
 *                          velm, the fixed-point force buffer, the atom order), read and written on the device by
 *                          lbm_begin_step_openmm and lbm_execute_openmm; compiled with LBM_B200_WITH_OPENMM_CUDA
 *                          against OpenMM's CUDA platform headers.
 */
#ifndef OPENMM_LBM_B200_KERNELS_H_
#define OPENMM_LBM_B200_KERNELS_H_

#include "LBMKernels.h"
#include "lbm_b200.h"
#include "openmm/internal/ContextImpl.h"
#include <string>
#include <vector>

namespace LBMPlugin {

/* The lattice parameters in the flat form of the C ABI (one domain). */
LbmLatticeParameters toLbmLatticeParameters(const LBMLatticeParameters& lattice);

class B200CalcLBMForceKernel : public CalcLBMForceKernel {
public:
    /* storage: LBM_STORAGE_*; device: CUDA device ordinal; stream: cudaStream_t to launch on (NULL: the kernel's own). */
    B200CalcLBMForceKernel(std::string name, const OpenMM::Platform& platform, int storage, int device, void* stream);
    ~B200CalcLBMForceKernel();
    void initialize(const OpenMM::System& system, const LBMForce& force, const LBMLatticeParameters& lattice);
    void beginStep(OpenMM::ContextImpl& context);
    double execute(OpenMM::ContextImpl& context, bool includeForces, bool includeEnergy);
    void copyParametersToContext(OpenMM::ContextImpl& context, const LBMLatticeParameters& lattice);
    void getFluidFields(OpenMM::ContextImpl& context, std::vector<double>& density, std::vector<OpenMM::Vec3>& velocity,
                        bool halo);
    double getFluidMachNumber(OpenMM::ContextImpl& context);
    OpenMM::Vec3 getWallForce(OpenMM::ContextImpl& context);
    void getFluidState(OpenMM::ContextImpl& context, std::vector<double>& state);
    void setFluidState(OpenMM::ContextImpl& context, const std::vector<double>& state);
    void createCheckpoint(OpenMM::ContextImpl& context, std::ostream& stream);
    void loadCheckpoint(OpenMM::ContextImpl& context, std::istream& stream);
    /* The files of the domain decomposition (MPI) are not supported: one GPU holds the whole lattice. */
    void createRankCheckpoint(OpenMM::ContextImpl& context, std::ostream& stream);
    void loadRankCheckpoint(OpenMM::ContextImpl& context, std::istream& stream);
    void resetRankState(OpenMM::ContextImpl& context);
    LbmKernel* handle() const { return kernel; }
    /* The element size of the checkpoint stream, as the reference's GPU platforms write it: 8 in double and mixed
       precision, 4 in single (CommonLBMKernels.cpp:243-244).  The kernel factory sets it from the Context. */
    void setCheckpointElementSize(int size) { checkpointElementSize = size; }
protected:
    /* Called by initialize() once the kernel exists: the platform's particle data set-up. */
    virtual void initializeParticles(const OpenMM::System& system, const LBMForce& force) = 0;
    virtual void beginStepParticles(OpenMM::ContextImpl& context, long long step) = 0;
    virtual void executeParticles(OpenMM::ContextImpl& context, long long step, bool includeForces) = 0;
    /* Throws OpenMMException with lbm_last_error() unless status is LBM_OK. */
    static void check(LbmStatus status);
    LbmKernel* kernel;
    LBMLatticeParameters lattice;
    std::vector<int> particles;    // System indices of the coupled particles, in coupling order
    long long numNodes;
private:
    int storage, device;
    void* stream;
    int checkpointElementSize;
};

class B200HostDataLBMKernel : public B200CalcLBMForceKernel {
public:
    B200HostDataLBMKernel(std::string name, const OpenMM::Platform& platform, int storage, int device, void* stream)
        : B200CalcLBMForceKernel(name, platform, storage, device, stream) {}
protected:
    void initializeParticles(const OpenMM::System& system, const LBMForce& force);
    void beginStepParticles(OpenMM::ContextImpl& context, long long step);
    void executeParticles(OpenMM::ContextImpl& context, long long step, bool includeForces);
private:
    void gather(OpenMM::ContextImpl& context);
    std::vector<double> positions, velocities, forces;
};

#ifdef LBM_B200_WITH_OPENMM_CUDA
/* The buffers of one OpenMM CUDA-platform Context; the platform kernel fills them before every call. */
class B200CudaDataLBMKernel : public B200CalcLBMForceKernel {
public:
    B200CudaDataLBMKernel(std::string name, const OpenMM::Platform& platform, OpenMM::CudaContext& cc, int storage);
protected:
    void initializeParticles(const OpenMM::System& system, const LBMForce& force);
    void beginStepParticles(OpenMM::ContextImpl& context, long long step);
    void executeParticles(OpenMM::ContextImpl& context, long long step, bool includeForces);
private:
    LbmOpenMMBuffers buffers();
    OpenMM::CudaContext& cc;
};
#endif

} // namespace LBMPlugin

#endif
