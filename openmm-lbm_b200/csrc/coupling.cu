// Particle coupling (placeholder until the coupling kernels are in place).
#include "coupling.cuh"

namespace lbm {

CouplingEngine::CouplingEngine(const LbmLatticeParameters& l, FluidEngine& f, const Geometry&, int n, const double*,
                               cudaStream_t s) : lattice(l), fluid(f), stream(s), np(n) {
    throw Error(LBM_ERR_NOT_SUPPORTED, "coupled particles are not supported yet");
}
CouplingEngine::~CouplingEngine() {}
void CouplingEngine::setParameters(const LbmLatticeParameters& l) { lattice = l; }
void CouplingEngine::load(const LbmParticleArrays*, bool) {}
void CouplingEngine::reflect(const LbmParticleArrays*, double w[3]) { w[0] = w[1] = w[2] = 0; }
void CouplingEngine::couple(long long, bool, bool) {}
void CouplingEngine::addForces(const LbmParticleArrays*) {}
void CouplingEngine::clearReaction() {}
void CouplingEngine::reactionWallMomentum(double out[3]) { out[0] = out[1] = out[2] = 0; }

} // namespace lbm
