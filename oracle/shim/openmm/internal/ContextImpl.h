/*
 * Minimal stand-in for OpenMM's ContextImpl (oracle harness only): the step count of the
 * integrator and the platform data pointer through which the Reference-platform kernel reads
 * positions, velocities and forces.
 */
#ifndef SHIM_OPENMM_CONTEXTIMPL_H_
#define SHIM_OPENMM_CONTEXTIMPL_H_
namespace OpenMM {
class ContextImpl {
public:
    ContextImpl() : stepCount(0), platformData(0) {}
    long long getStepCount() const { return stepCount; }
    void setStepCount(long long count) { stepCount = count; }
    void* getPlatformData() { return platformData; }
    void setPlatformData(void* data) { platformData = data; }
private:
    long long stepCount;
    void* platformData;
};
}
#endif
