/*
 * The kernel factory of the B200 platform kernel, the counterpart of the reference's CudaLBMKernelFactory
 * (platforms/cuda/src/CudaLBMKernelFactory.cpp:42-72): it creates the CalcLBMForce kernel of a Context.
 */
#ifndef OPENMM_LBM_B200_KERNEL_FACTORY_H_
#define OPENMM_LBM_B200_KERNEL_FACTORY_H_

#include "openmm/KernelFactory.h"
#include <string>

namespace LBMPlugin {

class B200LBMKernelFactory : public OpenMM::KernelFactory {
public:
    /* storage: LBM_STORAGE_* of the populations, or -1 for the storage that the Context's precision gives (the
       reference's: FP32 in single precision, FP64 in mixed and double precision, docs/theory.md:899-910), unless the
       environment variable OPENMM_LBM_B200_STORAGE (f64, f32, f16 or bf16) names another. */
    explicit B200LBMKernelFactory(int storage = -1) : storage(storage) {}
    OpenMM::KernelImpl* createKernelImpl(std::string name, const OpenMM::Platform& platform,
                                         OpenMM::ContextImpl& context) const;
    /* The storage of a Context of the given precision ("single", "mixed" or "double"). */
    int storageFor(const std::string& precision) const;
private:
    int storage;
};

} // namespace LBMPlugin

#endif
