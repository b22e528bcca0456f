/* Minimal stand-in for OpenMM's Force base class (oracle harness only). */
#ifndef SHIM_OPENMM_FORCE_H_
#define SHIM_OPENMM_FORCE_H_
namespace OpenMM {
class ForceImpl;
class Context;
class ContextImpl;
class Force {
public:
    virtual ~Force() {}
protected:
    virtual ForceImpl* createImpl() const = 0;
    virtual bool usesPeriodicBoundaryConditions() const { return true; }
};
}
#endif
