// Particle coupling of the B200 LBM force kernel: drag and random force through the nearest node or an
// interpolation stencil (trilinear, three-point, Keys), explicit or centred, and the reaction of the
// particles on the fluid (the reference's coupling, platforms/reference/src/ReferenceLBMKernels.cpp:503-1018).
#pragma once

#include "fluid.cuh"

namespace lbm {

struct CouplingView;

// Limits of the centred stencil drag's conjugate gradients: the iteration cap of the reference
// (ReferenceLBMKernels.cpp:864-866) and the polls after which a block waiting at a grid barrier gives up.
constexpr int kDefaultCgIterations = 1000;
constexpr long long kDefaultBarrierPolls = 1LL << 26;

class CouplingEngine {
public:
    CouplingEngine(const LbmLatticeParameters& lattice, FluidEngine& fluid, const Geometry& geometry, int numParticles,
                   const double* masses, cudaStream_t stream);
    ~CouplingEngine();
    void setParameters(const LbmLatticeParameters& lattice);
    // Load the particle arrays of a call into the device buffers (copies for host arrays).
    void load(const LbmParticleArrays* particles, bool withForces);
    // Reflection at the walls (beginStep, ReferenceLBMKernels.cpp:315-338): reverses velocities on the device and
    // returns the momentum given to the wall, Da nm/ps (synchronizes).  The velocities are stored back.
    void reflect(const LbmParticleArrays* particles, double wallMomentum[3]);
    // Coupling forces of step `step` on the current fluid (isStep: also the reaction on the fluid, with the
    // momentum removal `remove`).  Returns the momentum of the reactions on solid nodes, Da nm/ps (isStep only).
    void couple(long long step, bool isStep, bool remove);
    // The part of step `step`'s coupling that needs only the positions and the fluid (the stencil pass and, for the
    // centred stencil drag, the cell list and the rows of the coupling matrix), launched at beginStep on a second
    // stream, so that it runs while the caller computes its other forces; couple() of that step continues from it.
    void prepare(const LbmParticleArrays* particles, long long step, bool remove);
    // The kernel's stream waits for prepared work (before anything that changes its inputs); discardPrepared() also
    // forgets it (the fluid or the parameters changed, or another evaluation comes first).
    void joinPrepared();
    void discardPrepared();
    // Add the coupling forces to the force array of the call.
    void addForces(const LbmParticleArrays* particles);
    // Clear the reaction of the last step from the fluid's reaction buffers.
    void clearReaction();
    // Clear the flags of the last step's reactions (the next step's stencil pass zeroes the reactions it flags).
    void clearReactionFlags();
    // Momentum given to solid nodes by the reactions of the last coupling step (lattice units), read on demand.
    void reactionWallMomentum(double out[3]);
    int numParticles() const { return np; }
    // Conjugate-gradient iterations of the last centred stencil solve.
    int lastIterations = 0;
    long long spreadSteps = 0;   // steps whose centred drag ran the spread-and-gather solve
    // The coupling forces of the last evaluation (kJ/mol/nm, 3 doubles per particle in coupling order, device memory).
    const double* couplingForces() const { return forceOutDev; }
    // Lower limits make the failure paths reachable in tests; 0 restores a default.
    void setSolverLimits(int maxIterations, long long barrierPolls);
private:
    struct Device;
    void release();
    template <typename R>
    void coupleWith(long long step, bool isStep, const CouplingView* view, bool matrixReady);
    template <typename R>
    void launchMatrix(const CouplingView* view, cudaStream_t s);
    void launchStencilPass(const CouplingView& view, bool remove, bool mark, cudaStream_t s);
    bool matrixSolve() const;
    void launchSlotMomentsNow();
    bool slotMomentsPending = false;      // the last stencil pass left the per-slot moments out (the matrix reads nodes)
    cudaStream_t side = nullptr;          // stream of the prepared work
    cudaEvent_t begun = nullptr, ready = nullptr;
    bool prepared = false, preparedRemove = false;
    long long preparedStep = -1;
    LbmLatticeParameters lattice;
    FluidEngine& fluid;
    cudaStream_t stream;
    int np;
    int storageType;
    // device buffers (double precision for the particles)
    double *posDev, *velDev, *forceInDev, *forceOutDev, *massDev;
    double* wallDev;           // 3 doubles: momentum of reactions on solid nodes
    int* statusDev;            // device status word of the conjugate gradients
    double* pinned;            // pinned staging for host particle arrays
    Device* dev;               // slot, sort and solver buffers
    int stencilSlots;
    int cgMaxIterations = kDefaultCgIterations;
    long long barrierPollLimit = kDefaultBarrierPolls;
};

} // namespace lbm
