/*
 * Minimal stand-in for OpenMM's ReferencePlatform::PlatformData (oracle harness only): the
 * arrays of positions (nm), velocities (nm/ps) and forces (kJ/mol/nm) of all particles.
 */
#ifndef SHIM_OPENMM_REFERENCEPLATFORM_H_
#define SHIM_OPENMM_REFERENCEPLATFORM_H_
#include "openmm/Platform.h"
#include "openmm/Vec3.h"
#include <vector>
namespace OpenMM {
class ReferencePlatform : public Platform {
public:
    class PlatformData {
    public:
        std::vector<Vec3>* positions;
        std::vector<Vec3>* velocities;
        std::vector<Vec3>* forces;
    };
};
}
#endif
