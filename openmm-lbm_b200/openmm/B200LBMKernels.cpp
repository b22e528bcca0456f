/*
 * The B200 platform kernel of openmm-lbm over the C ABI of liblbm_b200.so (B200LBMKernels.h).  The evaluation rules
 * (which evaluation advances the fluid, next-step forces between steps, repeated evaluations) are those of the library
 * (lbm_begin_step / lbm_execute follow ReferenceLBMKernels.cpp:308-401); this class converts OpenMM's objects into the
 * ABI's plain arrays and the ABI's status codes into OpenMMException.
 */
#include "B200LBMKernels.h"
#include "openmm/OpenMMException.h"
#include "openmm/System.h"
#include "openmm/reference/ReferencePlatform.h"
#include <cmath>
#include <cstring>
#include <istream>
#include <limits>
#include <ostream>

using namespace OpenMM;
using namespace std;

namespace LBMPlugin {

LbmLatticeParameters toLbmLatticeParameters(const LBMLatticeParameters& l) {
    LbmLatticeParameters p;
    p.nx = l.nx; p.ny = l.ny; p.nz = l.nz;
    p.dx = l.dx; p.dt = l.dt; p.density = l.density;
    p.tau = l.tau; p.omega = l.omega;
    for (int a = 0; a < 3; a++) {
        p.initial_velocity[a] = l.initialVelocity[a];
        p.body_acceleration[a] = l.bodyAcceleration[a];
    }
    p.friction = l.friction;
    p.kT = l.kT;
    p.drag_scheme = (int) l.dragScheme;
    p.interpolation_stencil = (int) l.interpolationStencil;
    p.fluid_fluctuations = l.fluidFluctuations ? 1 : 0;
    p.fluid_kT = l.fluidKT;
    p.random_number_seed = l.randomNumberSeed;
    p.momentum_removal_frequency = l.momentumRemovalFrequency;
    p.mach_check_frequency = l.machCheckFrequency;
    p.mach_number_limit = l.machNumberLimit;
    p.wall_scheme = (int) l.wallScheme;
    for (int f = 0; f < 6; f++) {
        p.face_boundary[f] = (int) l.faceBoundary[f];
        for (int a = 0; a < 3; a++)
            p.face_velocity[f][a] = l.faceVelocity[f][a];
        p.face_density[f] = l.faceDensity[f];
    }
    return p;
}

B200CalcLBMForceKernel::B200CalcLBMForceKernel(string name, const Platform& platform, int storage, int device,
                                               void* stream)
        : CalcLBMForceKernel(name, platform), kernel(NULL), numNodes(0), storage(storage), device(device),
          stream(stream), checkpointElementSize(8) {
}

B200CalcLBMForceKernel::~B200CalcLBMForceKernel() {
    lbm_destroy(kernel);
}

void B200CalcLBMForceKernel::check(LbmStatus status) {
    if (status != LBM_OK)
        throw OpenMMException(lbm_last_error());
}

void B200CalcLBMForceKernel::initialize(const System& system, const LBMForce& force, const LBMLatticeParameters& l) {
    if (l.isDecomposed())
        throw OpenMMException("LBMForce: the B200 platform kernel runs the whole lattice on one GPU; the domain "
                              "decomposition is not supported");
    lattice = l;
    particles = l.particles;
    LbmLatticeParameters p = toLbmLatticeParameters(l);
    LbmOptions options;
    options.storage = storage;
    options.device = device;
    options.stream = stream;
    vector<double> masses;
    for (int i : particles)
        masses.push_back(system.getParticleMass(i));
    check(lbm_create(&p, &options, (int) masses.size(), masses.empty() ? NULL : masses.data(),
                     (int) l.solidNodes.size(), l.solidNodes.empty() ? NULL : l.solidNodes.data(), &kernel));
    numNodes = (long long) l.nx*l.ny*l.nz;
    check(lbm_set_checkpoint_element_size(kernel, checkpointElementSize));
    initializeParticles(system, force);
}

void B200CalcLBMForceKernel::beginStep(ContextImpl& context) {
    beginStepParticles(context, context.getStepCount());
}

double B200CalcLBMForceKernel::execute(ContextImpl& context, bool includeForces, bool includeEnergy) {
    executeParticles(context, context.getStepCount(), includeForces);
    return 0.0;
}

void B200CalcLBMForceKernel::copyParametersToContext(ContextImpl& context, const LBMLatticeParameters& l) {
    LbmLatticeParameters p = toLbmLatticeParameters(l);
    check(lbm_copy_parameters(kernel, &p));
    lattice = l;
}

void B200CalcLBMForceKernel::getFluidFields(ContextImpl& context, vector<double>& density, vector<Vec3>& velocity,
                                            bool halo) {
    vector<double> rho(numNodes), u(3*numNodes);
    check(lbm_get_fluid_fields(kernel, rho.data(), u.data()));
    if (!halo) {
        density = rho;
        velocity.resize(numNodes);
        for (long long n = 0; n < numNodes; n++)
            velocity[n] = Vec3(u[3*n], u[3*n+1], u[3*n+2]);
        return;
    }
    // The lattice extended by one node on every side (CalcLBMForceKernel::getFluidFields, LBMKernels.h:139-144): with
    // one domain a node of the extension takes the fields of the node across the periodic boundary, if the halo of the
    // field is exchanged, and NaN beyond an open face or for a field whose halo is not exchanged.
    const double nan = numeric_limits<double>::quiet_NaN();
    const int size[3] = {lattice.nx, lattice.ny, lattice.nz};
    const int ex = lattice.nx + 2, ey = lattice.ny + 2, ez = lattice.nz + 2;
    density.assign((size_t) ex*ey*ez, nan);
    velocity.assign((size_t) ex*ey*ez, Vec3(nan, nan, nan));
    for (int k = -1; k <= lattice.nz; k++)
        for (int j = -1; j <= lattice.ny; j++)
            for (int i = -1; i <= lattice.nx; i++) {
                int c[3] = {i, j, k};
                bool inside = true, valid = true;
                for (int a = 0; a < 3; a++) {
                    if (c[a] >= 0 && c[a] < size[a])
                        continue;
                    inside = false;
                    if (lattice.isOpenAxis(a))
                        valid = false;
                    else
                        c[a] = (c[a] + size[a])%size[a];
                }
                if (!valid)
                    continue;
                long long node = c[0] + (long long) lattice.nx*(c[1] + (long long) lattice.ny*c[2]);
                size_t l = (size_t) (i + 1) + (size_t) ex*((j + 1) + (size_t) ey*(k + 1));
                if (inside || lattice.densityHaloExchange)
                    density[l] = rho[node];
                if (inside || lattice.velocityHaloExchange)
                    velocity[l] = Vec3(u[3*node], u[3*node+1], u[3*node+2]);
            }
}

double B200CalcLBMForceKernel::getFluidMachNumber(ContextImpl& context) {
    double mach;
    check(lbm_get_fluid_mach_number(kernel, &mach));
    return mach;
}

Vec3 B200CalcLBMForceKernel::getWallForce(ContextImpl& context) {
    double f[3];
    check(lbm_get_wall_force(kernel, f));
    return Vec3(f[0], f[1], f[2]);
}

void B200CalcLBMForceKernel::getFluidState(ContextImpl& context, vector<double>& state) {
    state.resize(LBM_NUM_VELOCITIES*(size_t) numNodes);
    check(lbm_get_fluid_state(kernel, state.data()));
}

void B200CalcLBMForceKernel::setFluidState(ContextImpl& context, const vector<double>& state) {
    if (state.size() != LBM_NUM_VELOCITIES*(size_t) numNodes)
        throw OpenMMException("LBMForce: setFluidState() was called with a state of the wrong size");
    check(lbm_set_fluid_state(kernel, state.data()));
}

void B200CalcLBMForceKernel::createCheckpoint(ContextImpl& context, ostream& stream) {
    // The kernel stream of the reference's GPU platforms (CommonLBMKernels.cpp:2019-2034), which LBMForceImpl writes
    // after its header (LBMForceImpl.cpp:568-573), then this kernel's trailer, which the reference does not read.
    size_t bytes = 0;
    check(lbm_checkpoint_size(kernel, &bytes));
    vector<char> buffer(bytes);
    check(lbm_create_checkpoint(kernel, buffer.data(), bytes));
    stream.write(buffer.data(), bytes);
}

void B200CalcLBMForceKernel::loadCheckpoint(ContextImpl& context, istream& stream) {
    // The stream has no length: its size follows from the lattice and the precision (CommonLBMKernels.cpp:2036-2058).
    // The trailer is read when it is there; a stream of the reference's CUDA kernel ends without it.
    size_t streamBytes = 0, trailerBytes = 0;
    check(lbm_checkpoint_layout(kernel, &streamBytes, &trailerBytes));
    vector<char> buffer(streamBytes + trailerBytes);
    stream.read(buffer.data(), sizeof(int));
    if (!stream)
        throw OpenMMException("LBMForce: the checkpoint is truncated");
    int elementSize;
    memcpy(&elementSize, buffer.data(), sizeof(int));
    if (elementSize != checkpointElementSize)
        throw OpenMMException("LBMForce: the checkpoint was written with a different precision");
    stream.read(buffer.data() + sizeof(int), streamBytes - sizeof(int));
    if (!stream)
        throw OpenMMException("LBMForce: the checkpoint is truncated");
    stream.read(buffer.data() + streamBytes, trailerBytes);
    size_t length = streamBytes + (size_t) stream.gcount();
    if (!stream)
        stream.clear();
    check(lbm_load_checkpoint(kernel, buffer.data(), length));
}

void B200CalcLBMForceKernel::createRankCheckpoint(ContextImpl& context, ostream& stream) {
    throw OpenMMException("LBMForce: the checkpoint files of the domain decomposition are not supported by the B200 "
                          "platform kernel (one GPU); use createCheckpoint()");
}

void B200CalcLBMForceKernel::loadRankCheckpoint(ContextImpl& context, istream& stream) {
    throw OpenMMException("LBMForce: the checkpoint files of the domain decomposition are not supported by the B200 "
                          "platform kernel (one GPU); use loadCheckpoint()");
}

void B200CalcLBMForceKernel::resetRankState(ContextImpl& context) {
    throw OpenMMException("LBMForce: the checkpoint files of the domain decomposition are not supported by the B200 "
                          "platform kernel (one GPU)");
}

// ------------------------------------------------------------------------------------------------------------------
// Particles in host vectors of the System's order (ReferencePlatform::PlatformData).
// ------------------------------------------------------------------------------------------------------------------

void B200HostDataLBMKernel::initializeParticles(const System& system, const LBMForce& force) {
    positions.assign(3*particles.size(), 0.0);
    velocities.assign(3*particles.size(), 0.0);
    forces.assign(3*particles.size(), 0.0);
}

void B200HostDataLBMKernel::gather(ContextImpl& context) {
    ReferencePlatform::PlatformData* data = static_cast<ReferencePlatform::PlatformData*>(context.getPlatformData());
    const vector<Vec3>& pos = *data->positions;
    const vector<Vec3>& vel = *data->velocities;
    const vector<Vec3>& frc = *data->forces;
    for (size_t i = 0; i < particles.size(); i++)
        for (int k = 0; k < 3; k++) {
            positions[3*i+k] = pos[particles[i]][k];
            velocities[3*i+k] = vel[particles[i]][k];
            forces[3*i+k] = frc[particles[i]][k];
        }
}

void B200HostDataLBMKernel::beginStepParticles(ContextImpl& context, long long step) {
    if (particles.empty()) {
        check(lbm_begin_step(kernel, step, NULL));
        return;
    }
    gather(context);
    LbmParticleArrays a = {positions.data(), velocities.data(), forces.data(), LBM_MEMORY_HOST};
    check(lbm_begin_step(kernel, step, &a));
    // The reflection at the walls may have reversed velocities.
    vector<Vec3>& vel = *static_cast<ReferencePlatform::PlatformData*>(context.getPlatformData())->velocities;
    for (size_t i = 0; i < particles.size(); i++)
        vel[particles[i]] = Vec3(velocities[3*i], velocities[3*i+1], velocities[3*i+2]);
}

void B200HostDataLBMKernel::executeParticles(ContextImpl& context, long long step, bool includeForces) {
    if (particles.empty()) {
        check(lbm_execute(kernel, step, NULL, includeForces ? 1 : 0, 0, NULL));
        return;
    }
    gather(context);
    LbmParticleArrays a = {positions.data(), velocities.data(), forces.data(), LBM_MEMORY_HOST};
    check(lbm_execute(kernel, step, &a, includeForces ? 1 : 0, 0, NULL));
    if (includeForces) {
        vector<Vec3>& frc = *static_cast<ReferencePlatform::PlatformData*>(context.getPlatformData())->forces;
        for (size_t i = 0; i < particles.size(); i++)
            frc[particles[i]] = Vec3(forces[3*i], forces[3*i+1], forces[3*i+2]);
    }
}

#ifdef LBM_B200_WITH_OPENMM_CUDA
// ------------------------------------------------------------------------------------------------------------------
// Particles in the device buffers of OpenMM's CUDA platform.  With the centred drag the evaluation needs the other
// forces of the step, so it runs in a post-computation after all of them, as the reference's does
// (CommonLBMKernels.cpp:107-126): execute() then does nothing.
// ------------------------------------------------------------------------------------------------------------------

namespace {
class CenteredDragPostComputation : public ComputeContext::ForcePostComputation {
public:
    CenteredDragPostComputation(CudaContext& cc, int group, LbmKernel* kernel, LbmOpenMMBuffers (*buffers)(CudaContext&))
        : cc(cc), group(group), kernel(kernel), buffers(buffers) {}
    double computeForceAndEnergy(bool includeForces, bool includeEnergy, int groups) {
        if ((groups&(1<<group)) == 0 || !cc.getForcesValid())
            return 0.0;
        LbmOpenMMBuffers b = buffers(cc);
        LbmStatus status = lbm_execute_openmm(kernel, cc.getStepCount(), &b, includeForces ? 1 : 0, 0, NULL);
        if (status != LBM_OK)
            throw OpenMMException(lbm_last_error());
        return 0.0;
    }
private:
    CudaContext& cc;
    int group;
    LbmKernel* kernel;
    LbmOpenMMBuffers (*buffers)(CudaContext&);
};

LbmOpenMMBuffers cudaBuffers(CudaContext& cc) {
    LbmOpenMMBuffers b;
    b.posq = (const void*) cc.getPosq().getDevicePointer();
    b.posq_correction = cc.getUseMixedPrecision() ? (const void*) cc.getPosqCorrection().getDevicePointer() : NULL;
    b.velm = (void*) cc.getVelm().getDevicePointer();
    b.force = (long long*) cc.getLongForceBuffer().getDevicePointer();
    b.atom_index = (const int*) cc.getAtomIndexArray().getDevicePointer();
    b.num_atoms = cc.getNumAtoms();
    b.padded_num_atoms = cc.getPaddedNumAtoms();
    b.precision = cc.getUseDoublePrecision() ? LBM_OPENMM_DOUBLE : cc.getUseMixedPrecision() ? LBM_OPENMM_MIXED :
                  LBM_OPENMM_SINGLE;
    return b;
}
} // namespace

B200CudaDataLBMKernel::B200CudaDataLBMKernel(string name, const Platform& platform, CudaContext& cc, int storage)
        : B200CalcLBMForceKernel(name, platform, storage, cc.getDeviceIndex(), (void*) cc.getCurrentStream()), cc(cc) {
}

LbmOpenMMBuffers B200CudaDataLBMKernel::buffers() {
    return cudaBuffers(cc);
}

void B200CudaDataLBMKernel::initializeParticles(const System& system, const LBMForce& force) {
    ContextSelector selector(cc);
    check(lbm_set_coupled_atoms(kernel, system.getNumParticles(), (int) particles.size(),
                                particles.empty() ? NULL : particles.data()));
    if (lattice.dragScheme == LBMForce::Centered)
        cc.addPostComputation(new CenteredDragPostComputation(cc, force.getForceGroup(), kernel, cudaBuffers));
}

void B200CudaDataLBMKernel::beginStepParticles(ContextImpl& context, long long step) {
    ContextSelector selector(cc);
    LbmOpenMMBuffers b = buffers();
    check(lbm_begin_step_openmm(kernel, step, &b));
}

void B200CudaDataLBMKernel::executeParticles(ContextImpl& context, long long step, bool includeForces) {
    if (lattice.dragScheme == LBMForce::Centered)
        return;
    ContextSelector selector(cc);
    LbmOpenMMBuffers b = buffers();
    check(lbm_execute_openmm(kernel, step, &b, includeForces ? 1 : 0, 0, NULL));
}
#endif

} // namespace LBMPlugin
