/* Minimal stand-in for OpenMM's Platform (oracle harness only): a named platform object. */
#ifndef SHIM_OPENMM_PLATFORM_H_
#define SHIM_OPENMM_PLATFORM_H_
#include <string>
namespace OpenMM {
class Platform {
public:
    virtual ~Platform() {}
    virtual std::string getName() const { return "Reference"; }
};
}
#endif
