// Host object of the B200 LBM force kernel (see kernel.cuh).
#include "kernel.cuh"
#include "coupling.cuh"
#include "openmm_buffers.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <sstream>
#include <vector>

namespace lbm {

#define CUDA_CHECK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    throw Error(LBM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

namespace {

// The trailer that follows the reference's kernel stream in a checkpoint: what a bitwise restart needs beyond it.
const char kTrailerTag[8] = {'B', '2', '0', '0', 'L', 'B', 'M', '1'};
const int kTrailerVersion = 1;

struct CheckpointTrailer {
    char tag[8];
    int version, storage;
    int nx, ny, nz, numParticles;
    int stepWallValid, rawPopulations;    // rawPopulations: the raw storage bytes follow the trailer
    int seed, pad;                        // the seed in use (a seed of 0 was replaced by a unique one at creation)
    long long stepIndex;
    double hostWall[3];
    StepStats stats;
};

// Element counts of the arrays of the reference's kernel stream (CommonLBMKernels.cpp:251, 378, 401, 666, 723).
struct StreamLayout {
    size_t populations, particles, solidEntries, boundaryNodes;
    size_t bytes(size_t elementSize) const {
        size_t b = 3*sizeof(int) + populations*elementSize;
        if (particles > 0)
            b += 16*particles + 3*particles*elementSize;
        b += 3*solidEntries*elementSize;
        if (boundaryNodes > 0)
            b += 3*boundaryNodes*elementSize;
        return b;
    }
};

void putValue(char*& out, int elementSize, double value) {
    if (elementSize == 8)
        std::memcpy(out, &value, 8);
    else {
        float f = (float) value;
        std::memcpy(out, &f, 4);
    }
    out += elementSize;
}

double getValue(const char*& in, int elementSize) {
    double value;
    if (elementSize == 8)
        std::memcpy(&value, in, 8);
    else {
        float f;
        std::memcpy(&f, in, 4);
        value = f;
    }
    in += elementSize;
    return value;
}

} // namespace

B200Kernel::B200Kernel(const LbmLatticeParameters& l, const LbmOptions& options, int np, const double* masses,
                       int numSolid, const int* solid)
        : lattice(l), stream(nullptr), ownStream(false), device(options.device), numParticles(np), stepPending(false),
          stepForcesCurrent(false), stepWallValid(false), stepIndex(0),
          checkpointElementSize(options.storage == LBM_STORAGE_F64 ? 8 : 4) {
    hostWallMomentum[0] = hostWallMomentum[1] = hostWallMomentum[2] = 0;
    if (l.nx <= 0 || l.ny <= 0 || l.nz <= 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the grid size must be set to positive values with setGridSize()");
    if (!(l.tau > 0.5) || std::fabs(l.omega*l.tau - 1.0) > 1e-12)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the relaxation time must exceed 1/2 and omega must be 1/tau");
    if (np < 0 || numSolid < 0 || (np > 0 && masses == nullptr) || (numSolid > 0 && solid == nullptr))
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_create: invalid particle or solid node arrays");
    long long n = (long long) l.nx*l.ny*l.nz;
    for (int i = 0; i < numSolid; i++)
        if (solid[i] < 0 || solid[i] >= n)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: a solid node index is out of range");
    for (int i = 0; i < np; i++)
        if (!(masses[i] > 0))
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: coupled particles must have a positive mass");
    // The coupling keeps the node of each stencil slot as a 32-bit signed index (and the solid nodes are ints at the
    // interface), so a lattice with coupled particles is limited to 2^31 - 1 nodes; the fluid alone goes to 2^32.
    if (np > 0 && n > 2147483647LL)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: a lattice with coupled particles may have at most 2^31 - 1 nodes");
    CUDA_CHECK(cudaSetDevice(device));
    if (options.stream != nullptr)
        stream = (cudaStream_t) options.stream;
    else {
        CUDA_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        ownStream = true;
    }
    // A seed of 0 asks for a unique one, chosen when the kernel is created (ReferenceLBMKernels.cpp:293-295).  The
    // random numbers are a function of (seed, step, node or particle), so the seed is the whole generator state.
    if (lattice.random_number_seed == 0) {
        std::random_device device;
        do
            lattice.random_number_seed = (int) (device() & 0x7fffffffu);
        while (lattice.random_number_seed == 0);
    }
    buildGeometry(l, numSolid, solid, geometry);
    for (size_t i = 1; i < geometry.solidNodes.size(); i++)
        if (geometry.solidNodes[i] == geometry.solidNodes[i-1])
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: a solid node is listed more than once");
    if ((long long) geometry.solidNodes.size() == n)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: all lattice nodes are solid");
    staticWallMomentum(lattice, geometry, staticWall);
    fluid.reset(new FluidEngine(lattice, options.storage, geometry, stream));
    if (np > 0) {
        fluid->enableReaction();
        coupling.reset(new CouplingEngine(lattice, *fluid, geometry, np, masses, stream));
    }
}

B200Kernel::~B200Kernel() {
    cudaFree(couplingIndexDev);
    cudaFree(stageDev);
    coupling.reset();
    fluid.reset();
    if (ownStream && stream != nullptr)
        cudaStreamDestroy(stream);
}

// beginStep (ReferenceLBMKernels.cpp:308-339).
void B200Kernel::beginStep(long long stepCount, const LbmParticleArrays* particles) {
    CUDA_CHECK(cudaSetDevice(device));
    stepIndex = stepCount;
    stepPending = true;
    stepWallValid = false;
    hostWallMomentum[0] = hostWallMomentum[1] = hostWallMomentum[2] = 0;
    if (!geometry.solidNodes.empty() && numParticles > 0) {
        if (particles == nullptr)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_begin_step: the particle arrays are missing");
        coupling->reflect(particles, hostWallMomentum);
    }
    // The positions are those of the step's evaluation: the stencil pass (and the coupling matrix) of the step starts
    // now, beside the caller's other forces.
    if (numParticles > 0 && particles != nullptr) {
        bool remove = lattice.momentum_removal_frequency > 0 && stepCount%lattice.momentum_removal_frequency == 0;
        coupling->prepare(particles, stepCount, remove);
    }
}

// execute (ReferenceLBMKernels.cpp:341-365).
double B200Kernel::execute(long long stepCount, const LbmParticleArrays* particles, bool includeForces, bool) {
    CUDA_CHECK(cudaSetDevice(device));
    if (numParticles > 0 && particles == nullptr)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_execute: the particle arrays are missing");
    if (evaluate(stepCount, particles, includeForces))
        coupling->addForces(particles);
    return 0.0;
}

bool B200Kernel::evaluate(long long stepCount, const LbmParticleArrays* particles, bool includeForces) {
    bool repeatedStep = (stepForcesCurrent && stepCount == stepIndex-1);
    if (stepPending) {
        stepPending = false;
        advanceFluid(particles);
    }
    else if (includeForces && numParticles > 0 && stepCount > 0 && !repeatedStep)
        computeNextStepForces(stepCount, particles);
    return includeForces && numParticles > 0;
}

// The OpenMM Context interface.  couplingIndex[atom] is built once from the coupled particles' System indices; every
// call gathers the coupled atoms from the Context's buffers (the storage order changes when OpenMM reorders the atoms)
// into device arrays in coupling order, and writes back what the reference's CUDA kernels write: the reflected
// velocities, and the coupling forces in fixed point.
void B200Kernel::setCoupledAtoms(int numAtoms, int numCoupled, const int* particles) {
    CUDA_CHECK(cudaSetDevice(device));
    if (numAtoms < 0 || numCoupled != numParticles || (numCoupled > 0 && particles == nullptr))
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_set_coupled_atoms: the coupled particles differ from lbm_create()");
    std::vector<int> index(std::max(1, numAtoms), -1);
    for (int i = 0; i < numCoupled; i++) {
        if (particles[i] < 0 || particles[i] >= numAtoms || index[particles[i]] >= 0)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_set_coupled_atoms: a particle index is out of range or repeated");
        index[particles[i]] = i;
    }
    cudaFree(couplingIndexDev);
    couplingIndexDev = nullptr;
    CUDA_CHECK(cudaMalloc(&couplingIndexDev, sizeof(int)*index.size()));
    CUDA_CHECK(cudaMemcpy(couplingIndexDev, index.data(), sizeof(int)*index.size(), cudaMemcpyHostToDevice));
    if (stageDev == nullptr)
        CUDA_CHECK(cudaMalloc(&stageDev, sizeof(double)*9*(size_t) std::max(1, numParticles)));
    openmmAtoms = numAtoms;
}

LbmParticleArrays B200Kernel::stagingArrays() {
    LbmParticleArrays a;
    a.positions = stageDev;
    a.velocities = stageDev + 3*(size_t) numParticles;
    a.forces = stageDev + 6*(size_t) numParticles;
    a.memory = LBM_MEMORY_DEVICE;
    return a;
}

void B200Kernel::beginStepOpenMM(long long stepCount, const LbmOpenMMBuffers* buffers) {
    CUDA_CHECK(cudaSetDevice(device));
    if (numParticles == 0) {
        beginStep(stepCount, nullptr);
        return;
    }
    if (couplingIndexDev == nullptr)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_begin_step_openmm: call lbm_set_coupled_atoms() first");
    validateOpenMMBuffers(buffers, openmmAtoms);
    LbmParticleArrays a = stagingArrays();
    bool reflects = !geometry.solidNodes.empty();
    // The positions also start the step's coupling (beginStep prepares it).
    gatherOpenMM(*buffers, couplingIndexDev, a.positions, a.velocities, nullptr, false, stream);
    beginStep(stepCount, &a);
    if (reflects)
        scatterVelocitiesOpenMM(*buffers, couplingIndexDev, a.velocities, stream);
}

double B200Kernel::executeOpenMM(long long stepCount, const LbmOpenMMBuffers* buffers, bool includeForces) {
    CUDA_CHECK(cudaSetDevice(device));
    if (numParticles == 0) {
        evaluate(stepCount, nullptr, includeForces);
        return 0.0;
    }
    if (couplingIndexDev == nullptr)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_execute_openmm: call lbm_set_coupled_atoms() first");
    validateOpenMMBuffers(buffers, openmmAtoms);
    LbmParticleArrays a = stagingArrays();
    gatherOpenMM(*buffers, couplingIndexDev, a.positions, a.velocities, a.forces,
                 lattice.drag_scheme == LBM_DRAG_CENTERED, stream);
    if (evaluate(stepCount, &a, includeForces))
        addForcesFixedPoint(*buffers, couplingIndexDev, coupling->couplingForces(), stream);
    return 0.0;
}

// advanceFluid (ReferenceLBMKernels.cpp:367-389).
void B200Kernel::advanceFluid(const LbmParticleArrays* particles) {
    bool remove = lattice.momentum_removal_frequency > 0 && stepIndex%lattice.momentum_removal_frequency == 0;
    bool react = false;
    if (numParticles > 0) {
        coupling->joinPrepared();
        coupling->load(particles, lattice.drag_scheme == LBM_DRAG_CENTERED);
        try {
            coupling->couple(stepIndex, true, remove);
        }
        catch (const Error&) {
            // A failed solve may have written part of the reactions: clear them, so that no later step sees them.
            coupling->clearReaction();
            cudaStreamSynchronize(stream);
            throw;
        }
        react = true;
    }
    fluid->step(stepIndex, remove, react);
    if (react)
        coupling->clearReactionFlags();
    stepWallValid = true;
    stepForcesCurrent = true;
    stepIndex++;
    if (lattice.mach_check_frequency > 0 && stepIndex%lattice.mach_check_frequency == 0)
        checkMachNumber();
}

// computeNextStepForces (ReferenceLBMKernels.cpp:391-401).
void B200Kernel::computeNextStepForces(long long stepCount, const LbmParticleArrays* particles) {
    stepForcesCurrent = false;
    bool remove = lattice.momentum_removal_frequency > 0 && stepCount%lattice.momentum_removal_frequency == 0;
    coupling->discardPrepared();
    coupling->load(particles, lattice.drag_scheme == LBM_DRAG_CENTERED);
    coupling->couple(stepCount, false, remove);
}

// checkMachNumber (ReferenceLBMKernels.cpp:412-428).
void B200Kernel::checkMachNumber() {
    double mach = getFluidMachNumber();
    if (mach > lattice.mach_number_limit) {
        std::stringstream msg;
        msg << "LBMForce: the Mach number of the fluid is " << mach << " after " << stepIndex << " lattice steps, "
            << "above the limit " << lattice.mach_number_limit << " (docs/theory.md, section 6). Reduce the forces on the "
            << "fluid, the time step or the friction.";
        throw Error(LBM_ERR_MACH_LIMIT, msg.str());
    }
}

void B200Kernel::copyParameters(const LbmLatticeParameters& l) {
    CUDA_CHECK(cudaSetDevice(device));
    // The fluid or the parameters change: prepared coupling work is waited for and dropped.
    if (coupling)
        coupling->discardPrepared();
    if (l.nx != lattice.nx || l.ny != lattice.ny || l.nz != lattice.nz)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "updateParametersInContext: the grid size cannot be changed");
    if (l.density != lattice.density || l.tau != lattice.tau)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "updateParametersInContext: the fluid density and viscosity cannot be changed");
    if (l.wall_scheme != lattice.wall_scheme)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "updateParametersInContext: the wall scheme cannot be changed");
    for (int f = 0; f < 6; f++)
        if (l.face_boundary[f] != lattice.face_boundary[f])
            throw Error(LBM_ERR_INVALID_ARGUMENT, "updateParametersInContext: the boundary types of the faces cannot be changed");
    if (l.drag_scheme != lattice.drag_scheme)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "updateParametersInContext: the drag scheme cannot be changed");
    if (l.interpolation_stencil != lattice.interpolation_stencil)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "updateParametersInContext: the interpolation stencil cannot be changed");
    if (l.fluid_fluctuations != lattice.fluid_fluctuations)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "updateParametersInContext: the fluid fluctuations cannot be switched on or off");
    // The generator is not reseeded by a parameter update: it keeps the seed of the kernel's creation, as the
    // reference's kernel keeps its generator state.
    int seed = lattice.random_number_seed;
    lattice = l;
    lattice.random_number_seed = seed;
    fluid->setParameters(lattice);
    if (coupling)
        coupling->setParameters(lattice);
}

void B200Kernel::getFluidFields(double* density, double* velocity) {
    CUDA_CHECK(cudaSetDevice(device));
    fluid->fields(density, velocity, lattice.density, lattice.dx/lattice.dt);
}

void B200Kernel::setFluidEquilibrium(const double* density, const double* velocity, bool onDevice, bool strain) {
    CUDA_CHECK(cudaSetDevice(device));
    // The fluid or the parameters change: prepared coupling work is waited for and dropped.
    if (coupling)
        coupling->discardPrepared();
    fluid->setEquilibrium(density, velocity, onDevice, lattice.density, lattice.dx/lattice.dt, strain);
}

// Steps the fluid from step firstStep until the steady residual, taken every `interval` steps against the velocities
// of the previous check (the first check is the state at the start), is at most `tolerance`, or maxSteps steps.
long long B200Kernel::steadySolve(long long firstStep, int interval, double tolerance, long long maxSteps,
                                  double* residual) {
    CUDA_CHECK(cudaSetDevice(device));
    // The fluid or the parameters change: prepared coupling work is waited for and dropped.
    if (coupling)
        coupling->discardPrepared();
    if (numParticles > 0)
        throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_steady_solve: the steady solve advances a fluid without coupled particles");
    if (interval <= 0 || maxSteps < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_steady_solve: the interval must be positive");
    double r = fluid->steadyResidual(interval);
    long long s = 0;
    while (s < maxSteps && !(r <= tolerance)) {
        for (int i = 0; i < interval && s < maxSteps; i++, s++) {
            beginStep(firstStep + s, nullptr);
            execute(firstStep + s, nullptr, false, false);
        }
        r = fluid->steadyResidual(interval);
    }
    if (residual)
        *residual = r;
    return s;
}

double B200Kernel::getFluidMachNumber() {
    CUDA_CHECK(cudaSetDevice(device));
    // The pass keeps the sums of the last step for the next removal, so that the result of a run does not
    // depend on when the Mach number is read.
    fluid->momentsPass(false);
    StepStats s = fluid->readStats();
    return std::sqrt(3.0*s.maxSpeed2);
}

// getWallForce (ReferenceLBMKernels.cpp:1438-1443): the momentum given to the solid nodes in the last step,
// divided by the time step.
void B200Kernel::getWallForce(double force[3]) {
    CUDA_CHECK(cudaSetDevice(device));
    double cellMass = lattice.density*lattice.dx*lattice.dx*lattice.dx;
    double scale = cellMass*lattice.dx/lattice.dt;
    double total[3] = {hostWallMomentum[0], hostWallMomentum[1], hostWallMomentum[2]};
    if (stepWallValid) {
        StepStats s = fluid->readStats();
        for (int a = 0; a < 3; a++)
            total[a] += s.wall[a]*scale;
        if (coupling) {
            double r[3];
            coupling->reactionWallMomentum(r);
            for (int a = 0; a < 3; a++)
                total[a] += r[a]*scale;
        }
    }
    for (int a = 0; a < 3; a++)
        force[a] = total[a]/lattice.dt;
}

int B200Kernel::solverIterations() const {
    return coupling ? coupling->lastIterations : 0;
}

long long B200Kernel::solverFallbackSteps() const {
    return coupling ? coupling->spreadSteps : 0;
}

void B200Kernel::setSolverLimits(int maxIterations, long long barrierPolls) {
    if (maxIterations < 0 || barrierPolls < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_set_solver_limits: the limits must not be negative");
    if (coupling)
        coupling->setSolverLimits(maxIterations, barrierPolls);
}

void B200Kernel::getFluidState(double* state) {
    CUDA_CHECK(cudaSetDevice(device));
    fluid->getState(state);
}

// setFluidState (ReferenceLBMKernels.cpp:1488-1505).
void B200Kernel::setFluidState(const double* state) {
    CUDA_CHECK(cudaSetDevice(device));
    // The fluid or the parameters change: prepared coupling work is waited for and dropped.
    if (coupling)
        coupling->discardPrepared();
    fluid->setState(state);
    stepForcesCurrent = false;
}

// The checkpoint (LBMKernels.h:170-174): the kernel stream of the reference's GPU platforms (CommonLBMKernels.cpp:
// 2019-2058), then this kernel's trailer.  With one domain the reference stores one wall entry per solid node and one
// boundary entry per boundary node; only the sums of the entries matter to its readers (getWallForce,
// CommonLBMKernels.cpp:1918-1945), so the dynamic wall momentum goes into the first wall entry.
void B200Kernel::setCheckpointElementSize(int elementSize) {
    if (elementSize != 4 && elementSize != 8)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_set_checkpoint_element_size: the element size must be 4 or 8");
    checkpointElementSize = elementSize;
}

bool B200Kernel::rawPopulationsInTrailer() const {
    return fluid->storage() == LBM_STORAGE_F64 && checkpointElementSize == 4;
}

double B200Kernel::wallMomentumScale() const {
    return lattice.density*lattice.dx*lattice.dx*lattice.dx*lattice.dx/lattice.dt;
}

static StreamLayout streamLayout(long long numNodes, int numParticles, const Geometry& g) {
    StreamLayout s;
    s.populations = 19*(size_t) numNodes;
    s.particles = (size_t) numParticles;
    s.solidEntries = std::max<size_t>(1, g.solidNodes.size());
    s.boundaryNodes = g.boundaryNodes.size();
    return s;
}

void B200Kernel::checkpointLayout(size_t& streamBytes, size_t& trailerBytes) {
    streamBytes = streamLayout(numNodes(), numParticles, geometry).bytes(checkpointElementSize);
    trailerBytes = sizeof(CheckpointTrailer) + (rawPopulationsInTrailer() ? fluid->stateBytes() : 0);
}

size_t B200Kernel::checkpointSize() {
    size_t streamBytes, trailerBytes;
    checkpointLayout(streamBytes, trailerBytes);
    return streamBytes + trailerBytes;
}

void B200Kernel::createCheckpoint(void* buffer, size_t bytes) {
    CUDA_CHECK(cudaSetDevice(device));
    if (bytes < checkpointSize())
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_create_checkpoint: the buffer is too small");
    const int e = checkpointElementSize;
    const long long n = numNodes();
    StreamLayout layout = streamLayout(n, numParticles, geometry);
    char* out = (char*) buffer;
    int head[3] = {e, 0, stepWallValid ? 1 : 0};
    std::memcpy(out, head, sizeof(head));
    out += sizeof(head);
    fluid->getStateByDirection([&](int q, const double* values) {
        char* plane = out + (size_t) q*n*e;
        for (long long x = 0; x < n; x++)
            putValue(plane, e, values[x]);
    });
    out += layout.populations*e;
    if (numParticles > 0) {
        std::memset(out, 0, 16*layout.particles + 3*layout.particles*e);
        out += 16*layout.particles + 3*layout.particles*e;
    }
    // The wall momentum of the last step in lattice units, without the static part that the reader adds.
    double wall[3] = {0, 0, 0};
    StepStats stats = fluid->readStats();
    if (!geometry.solidNodes.empty() && stepWallValid) {
        double reaction[3] = {0, 0, 0};
        if (coupling)
            coupling->reactionWallMomentum(reaction);
        for (int a = 0; a < 3; a++)
            wall[a] = hostWallMomentum[a]/wallMomentumScale() + stats.wall[a] + reaction[a] - staticWall[a];
    }
    for (int a = 0; a < 3; a++)
        for (size_t i = 0; i < layout.solidEntries; i++)
            putValue(out, e, i == 0 ? wall[a] : 0.0);
    if (layout.boundaryNodes > 0) {
        std::memset(out, 0, 3*layout.boundaryNodes*e);
        out += 3*layout.boundaryNodes*e;
    }
    CheckpointTrailer h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.tag, kTrailerTag, sizeof(kTrailerTag));
    h.version = kTrailerVersion;
    h.storage = fluid->storage();
    h.nx = lattice.nx; h.ny = lattice.ny; h.nz = lattice.nz;
    h.numParticles = numParticles;
    h.stepWallValid = stepWallValid;
    h.rawPopulations = rawPopulationsInTrailer() ? 1 : 0;
    h.seed = lattice.random_number_seed;
    h.stepIndex = stepIndex;
    for (int a = 0; a < 3; a++)
        h.hostWall[a] = hostWallMomentum[a];
    h.stats = stats;
    std::memcpy(out, &h, sizeof(h));
    out += sizeof(h);
    if (h.rawPopulations)
        fluid->copyStateOut(out);
}

void B200Kernel::loadCheckpoint(const void* buffer, size_t bytes) {
    CUDA_CHECK(cudaSetDevice(device));
    // The fluid or the parameters change: prepared coupling work is waited for and dropped.
    if (coupling)
        coupling->discardPrepared();
    const char* in = (const char*) buffer;
    int head[3];
    if (bytes < sizeof(head))
        throw Error(LBM_ERR_CHECKPOINT, "LBMForce: the checkpoint is truncated");
    std::memcpy(head, in, sizeof(head));
    const int e = head[0];
    if (e != checkpointElementSize)
        throw Error(LBM_ERR_CHECKPOINT, "LBMForce: the checkpoint was written with a different precision");
    const long long n = numNodes();
    StreamLayout layout = streamLayout(n, numParticles, geometry);
    size_t streamBytes = layout.bytes(e);
    if (bytes < streamBytes)
        throw Error(LBM_ERR_CHECKPOINT, "LBMForce: the checkpoint is truncated");
    // This kernel's trailer, when it describes this kernel (another storage type reads the stream alone).
    CheckpointTrailer h;
    bool exact = false;
    if (bytes >= streamBytes + sizeof(h)) {
        std::memcpy(&h, in + streamBytes, sizeof(h));
        exact = std::memcmp(h.tag, kTrailerTag, sizeof(kTrailerTag)) == 0 && h.version == kTrailerVersion &&
                h.storage == fluid->storage() && h.nx == lattice.nx && h.ny == lattice.ny && h.nz == lattice.nz &&
                h.numParticles == numParticles &&
                (h.rawPopulations == 0 || bytes >= streamBytes + sizeof(h) + fluid->stateBytes());
    }
    const char* populations = in + sizeof(head);
    if (exact && h.rawPopulations)
        fluid->copyStateIn(in + streamBytes + sizeof(h));
    else
        fluid->setStateByDirection([&](int q, double* values) {
            const char* plane = populations + (size_t) q*n*e;
            for (long long x = 0; x < n; x++)
                values[x] = getValue(plane, e);
        });
    stepForcesCurrent = false;
    if (exact) {
        // The random numbers are a function of (seed, step, index): the seed of the run continues it, as the
        // reference's generator state does.
        if (h.seed != 0 && h.seed != lattice.random_number_seed) {
            lattice.random_number_seed = h.seed;
            fluid->setParameters(lattice);
            if (coupling)
                coupling->setParameters(lattice);
        }
        fluid->restoreStats(h.stats);
        stepWallValid = h.stepWallValid != 0;
        stepIndex = h.stepIndex;
        for (int a = 0; a < 3; a++)
            hostWallMomentum[a] = h.hostWall[a];
        return;
    }
    // A stream without the trailer: the wall momentum of the last step is the sum of the stored entries plus the
    // static part (getWallForce, CommonLBMKernels.cpp:1918-1945), kept on the host until the next step.
    double wall[3] = {0, 0, 0};
    bool advanced = head[2] != 0;
    if (advanced && !geometry.solidNodes.empty()) {
        const char* p = populations + layout.populations*e;
        std::vector<double> values;
        if (numParticles > 0) {
            p += 16*layout.particles;
            for (size_t i = 0; i < 3*layout.particles; i++)
                values.push_back(getValue(p, e));
            for (int a = 0; a < 3; a++)
                for (size_t i = 0; i < layout.particles; i++)
                    wall[a] += values[a*layout.particles + i];
        }
        for (int a = 0; a < 3; a++)
            for (size_t i = 0; i < layout.solidEntries; i++)
                wall[a] += getValue(p, e);
        for (int a = 0; a < 3; a++)
            for (size_t i = 0; i < layout.boundaryNodes; i++)
                wall[a] += getValue(p, e);
        for (int a = 0; a < 3; a++)
            wall[a] += staticWall[a];
    }
    stepWallValid = false;
    for (int a = 0; a < 3; a++)
        hostWallMomentum[a] = wall[a]*wallMomentumScale();
}

} // namespace lbm
