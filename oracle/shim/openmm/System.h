/* Minimal stand-in for OpenMM's System (oracle harness only): particle masses. */
#ifndef SHIM_OPENMM_SYSTEM_H_
#define SHIM_OPENMM_SYSTEM_H_
#include <vector>
namespace OpenMM {
class System {
public:
    int addParticle(double mass) { masses.push_back(mass); return (int) masses.size()-1; }
    int getNumParticles() const { return (int) masses.size(); }
    double getParticleMass(int index) const { return masses[index]; }
private:
    std::vector<double> masses;
};
}
#endif
