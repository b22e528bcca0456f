// Internal host-side declarations of the B200 LBM force kernel library.
#pragma once

#include "lbm_b200.h"
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define LBM_HOST_DEVICE __host__ __device__
#else
#define LBM_HOST_DEVICE
#endif

namespace lbm {

// An error with the status code that the C ABI returns.
class Error : public std::runtime_error {
public:
    Error(LbmStatus status, const std::string& message) : std::runtime_error(message), status(status) {}
    LbmStatus status;
};

// The message that lbm_last_error() returns on this thread.
void setLastError(const std::string& message);

void defaultForceDescription(LbmForceDescription* force);
void computeLatticeParameters(const LbmForceDescription& force, const double box[3], double stepSize,
                              int numSystemParticles, const double* systemMasses, int numCoupled,
                              const int* coupled, int numSolid, const int* solid, LbmLatticeParameters& lattice);

// Boundary node kinds (the reference's LBMBoundaries::Kind, openmmapi/include/internal/LBMBoundaries.h:30).
enum BoundaryKind { KindWall = 0, KindVelocity = 1, KindDensity = 2, KindDensityAtRest = 3, KindDensityVelocity = 4 };

LBM_HOST_DEVICE inline bool hasEquilibriumNoise(int kind) {
    return kind == KindWall || kind == KindDensityVelocity;
}

// The geometry derived from the solid nodes and the faces (host side, computed once).
struct Geometry {
    std::vector<char> fluid;                   // empty without solid nodes
    std::vector<int> solidNodes;               // sorted
    // Bounce-back: fluid nodes next to solid nodes and, per node, the bits 1 << q of the directions q whose
    // node x + c_q is solid, without links that cross an open face (LBMBoundaries::findWallLinks).
    std::vector<int> wallNodes, wallLinks;
    // Regularized walls and open faces (LBMBoundaries::find): boundary nodes, unknown and solid direction
    // bits, kind and face.
    std::vector<int> boundaryNodes, unknown, solidBits, kind, face;
};

void buildGeometry(const LbmLatticeParameters& lattice, int numSolid, const int* solid, Geometry& geometry);
void staticWallMomentum(const LbmLatticeParameters& lattice, const Geometry& geometry, double momentum[3]);

} // namespace lbm
