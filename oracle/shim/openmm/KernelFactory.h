/* Minimal stand-in for OpenMM's KernelFactory (oracle harness only). */
#ifndef SHIM_OPENMM_KERNELFACTORY_H_
#define SHIM_OPENMM_KERNELFACTORY_H_
#include "openmm/KernelImpl.h"
#include <string>
namespace OpenMM {
class ContextImpl;
class KernelFactory {
public:
    virtual ~KernelFactory() {}
    virtual KernelImpl* createKernelImpl(std::string name, const Platform& platform, ContextImpl& context) const = 0;
};
}
#endif
