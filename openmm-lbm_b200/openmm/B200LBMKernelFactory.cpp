/*
 * The kernel factory of the B200 platform kernel and its registration (CudaLBMKernelFactory.cpp:42-72).  On OpenMM's
 * CUDA platform (built with LBM_B200_WITH_OPENMM_CUDA) the kernel reads the particles from the Context's device
 * buffers; on a platform that keeps them in host vectors in System order (OpenMM's Reference platform) it copies them
 * through host memory.
 */
#include "B200LBMKernelFactory.h"
#include "B200LBMKernels.h"
#include "openmm/OpenMMException.h"
#include <cstdlib>
#include <cstring>

using namespace OpenMM;

namespace LBMPlugin {

int B200LBMKernelFactory::storageFor(const std::string& precision) const {
    if (storage >= 0)
        return storage;
    const char* name = std::getenv("OPENMM_LBM_B200_STORAGE");
    if (name != NULL) {
        if (std::strcmp(name, "f64") == 0) return LBM_STORAGE_F64;
        if (std::strcmp(name, "f32") == 0) return LBM_STORAGE_F32;
        if (std::strcmp(name, "f16") == 0) return LBM_STORAGE_F16;
        if (std::strcmp(name, "bf16") == 0) return LBM_STORAGE_BF16;
        throw OpenMMException("OPENMM_LBM_B200_STORAGE must be f64, f32, f16 or bf16");
    }
    return precision == "single" ? LBM_STORAGE_F32 : LBM_STORAGE_F64;
}

KernelImpl* B200LBMKernelFactory::createKernelImpl(std::string name, const Platform& platform,
                                                   ContextImpl& context) const {
    if (name != CalcLBMForceKernel::Name())
        throw OpenMMException((std::string("Tried to create kernel with illegal kernel name '") + name + "'").c_str());
#ifdef LBM_B200_WITH_OPENMM_CUDA
    if (platform.getName() == "CUDA") {
        CudaPlatform::PlatformData* data = static_cast<CudaPlatform::PlatformData*>(context.getPlatformData());
        if (data->contexts.size() > 1)
            throw OpenMMException("LBMForce does not support running on multiple devices");
        CudaContext& cc = *data->contexts[0];
        std::string precision = cc.getUseDoublePrecision() ? "double" : cc.getUseMixedPrecision() ? "mixed" : "single";
        B200CalcLBMForceKernel* kernel = new B200CudaDataLBMKernel(name, platform, cc, storageFor(precision));
        kernel->setCheckpointElementSize(precision == "single" ? 4 : 8);
        return kernel;
    }
#endif
    return new B200HostDataLBMKernel(name, platform, storageFor("double"), 0, NULL);
}

} // namespace LBMPlugin

#ifdef LBM_B200_WITH_OPENMM_CUDA
extern "C" OPENMM_EXPORT void registerKernelFactories() {
    try {
        Platform& platform = Platform::getPlatformByName("CUDA");
        platform.registerKernelFactory(LBMPlugin::CalcLBMForceKernel::Name(), new LBMPlugin::B200LBMKernelFactory());
    }
    catch (const std::exception& ex) {
        // No CUDA platform: nothing to register.
    }
}
#endif
