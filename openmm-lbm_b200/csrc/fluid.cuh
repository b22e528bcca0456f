// The fluid engine of the B200 LBM force kernel: device state of the lattice and the launches of one
// lattice step, in pull form with two population arrays.
//
// Layout in HBM.  Two arrays A and B of 19*N deviations f_q - w_q in the storage type, [q*N + node],
// node = x + nx*(y + ny*z) (the reference's layout, openmmapi/include/internal/D3Q19.h:16-25).  The input
// array of a step holds the post-collision populations of the previous step at the node that produced
// them: the population that node x receives in direction q at step n is A_q(x - c_q) (pull streaming).
// Every population slot is read by exactly one node, so halfway bounce-back, regularized walls and
// open faces are applied by sparse passes that write the value node x must receive into the slot it
// pulls (the slot of a solid node, or of the node across an open face), and the dense kernel needs no
// geometry but a one-bit solid mask per node.
#pragma once

#include "lbm_internal.h"
#include <cuda_runtime.h>
#include <functional>
#include <vector>

namespace lbm {

// Statistics of a step, computed on the device (double precision).
struct StepStats {
    double mass;         // sum of the deviations of the fluid nodes after the step (mass - number of fluid nodes)
    double momentum[3];  // total momentum of the fluid after the step (deviations), lattice units
    double ucm[3];       // momentum / mass: the velocity that the next removal subtracts
    double wall[3];      // momentum exchanged with the walls by the streaming of the step, lattice units
    double maxSpeed2;    // max |j/rho|^2 (only from the moments pass)
    double pad[3];
};

// Everything the fluid kernels need, by value.
struct FluidView {
    int nx, ny, nz;
    long long n;               // nodes
    int wordsPerRow;           // 32-bit words per row of the node bitmaps
    int tilesX, tilesY;
    long long numTiles;        // 32 x 8 node tiles
    double omega;
    double g[3];
    double numFluid;
    uint32_t seed;
    double mu;                 // 3 kT of the fluid fluctuations in lattice units (0: no fluctuations)
    int faceOpen;              // some face is not periodic
    const uint32_t* solidMask; // bit per node, rows padded to 32 bits; NULL without solid nodes
    const uint32_t* reactMask; // bit per node with a coupling reaction; NULL without particles
    const void* reaction;      // 4 values (R) per node, lattice units
    double* partials;          // 4 doubles per block of the dense kernels
    StepStats* stats;          // statistics of the last step (ucm read by the next removal)
};

class FluidEngine {
public:
    FluidEngine(const LbmLatticeParameters& lattice, int storage, const Geometry& geometry, cudaStream_t stream);
    ~FluidEngine();
    int storage() const { return storageType; }
    long long numNodes() const { return view.n; }
    // Populations as deviations [q*N + node] in double, from or to host memory (the reference's state layout).
    void getState(double* host);
    void setState(const double* host);
    // The state one direction q at a time, each plane f_q(x) of view.n doubles in node order (getState's layout).
    void getStateByDirection(const std::function<void(int, const double*)>& sink);
    void setStateByDirection(const std::function<void(int, double*)>& source);
    // One lattice step: stream+collide (with momentum removal when `remove`), bounce-back, boundaries and the
    // reduction of the step statistics.  The coupling reaction is read from the reaction buffers when `react`.
    void step(long long stepIndex, bool remove, bool react);
    // Full moments pass over the current state: the largest speed, and with setSums the mass, momentum and ucm.
    void momentsPass(bool setSums);
    // The steady-state residual max|u - u_prev|/(interval max|u|) in FP64 against the velocities of the previous call
    // (u = j/rho of the post-stream state, fluid nodes); the first call records the velocities and returns infinity.
    double steadyResidual(int interval);
    void restoreStats(const StepStats& stats);
    // Download the stats (synchronizes the stream).
    StepStats readStats();
    void fields(double* density, double* velocity, double densityScale, double velocityScale);
    // Sets the state to the equilibrium of the fields (density [N], velocity [N][3], divided by the scales into lattice
    // units), from host or device memory.
    void setEquilibrium(const double* density, const double* velocity, bool onDevice, double densityScale,
                        double velocityScale, bool strain);
    void setParameters(const LbmLatticeParameters& lattice);
    size_t stateBytes() const { return (size_t) 19*view.n*elementSize; }
    void* currentState() const { return pop[cur]; }
    void copyStateOut(void* host);    // raw storage bytes of the current input array
    void copyStateIn(const void* host);
    // Reaction buffers, owned here so that the dense kernel reads them directly.
    void enableReaction();
    uint32_t* reactMask() { return reactMaskDev; }
    void clearReactMask(cudaStream_t s);
    void* reactionBuffer() { return reactionDev; }
    const FluidView& deviceView() const { return view; }
    const void* inputArray() const { return pop[cur]; }
    cudaStream_t getStream() const { return stream; }
    int wordsPerRow() const { return view.wordsPerRow; }
    int numSolid() const { return (int) solidNodes.size(); }
    // CUDA events around each dense launch (profiling of the step, lbm_profile_dense_kernel).
    void profileDense(bool enable);
    void denseTime(long long* launches, double* totalMs);
    // Kernels launched by the engines of this lattice (fluid and coupling).
    long long launches;
private:
    void launchStreamCollide(long long stepIndex, bool remove, bool react);
    void launchFinish(int numBlocks, int numExtra);
    LbmLatticeParameters lattice;
    int storageType;
    size_t elementSize;
    cudaStream_t stream;
    FluidView view;
    void* pop[2];
    int cur;
    int gridBlocks;            // persistent grid of the dense kernel
    uint32_t* solidMaskDev;
    uint32_t* reactMaskDev;
    void* reactionDev;
    double* partialsDev;
    StepStats* statsDev;
    int numWall, numBoundary;
    int* wallDev;              // [node, links] pairs
    int* boundaryDev;          // [node, unknown, solid, kind | face << 8] quadruples
    bool equilibriumNoise;
    std::vector<int> solidNodes;
    void* stagingDev;          // N doubles for state transfer
    int extraBlocks;           // blocks of the sparse passes that write partials
    double* faceDev;           // face velocities/densities and the boundary stress weight
    double* residualPrevDev = nullptr;   // 3N velocities of the last residual call
    double faceHost[32];
    StepStats statsHost;
    bool profiling;
    std::vector<cudaEvent_t> profileEvents;   // start/stop pairs
    size_t profileUsed;
};

} // namespace lbm
