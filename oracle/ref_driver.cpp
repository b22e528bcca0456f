/*
 * ref_driver.cpp -- TEST INFRASTRUCTURE (oracle): drives the reference's own Reference-platform
 * kernel, ReferenceCalcLBMForceKernel (platforms/reference/src/ReferenceLBMKernels.cpp), compiled
 * unmodified from the reference sources against the minimal OpenMM shim in oracle/shim/.
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark use this file; it is the
 * checker, never the product.  It exposes the entry points of include/lbm_b200.h with the prefix
 * refdrv_ and host particle arrays only, so that the same Python harness can drive the reference,
 * the C restatement (lbm_oracle.c) and the CUDA library.
 *
 * OpenMM's ContextImpl is replaced by the shim's ContextImpl: the step count is set from the
 * step_count argument of each call, and the Reference platform data points at vectors of Vec3
 * that are filled from, and copied back to, the caller's arrays around each call.  The coupled
 * particles are particles 0..num_particles-1 of a System that holds them alone.
 */
#include "LBMForce.h"
#include "LBMKernels.h"
#include "ReferenceLBMKernels.h"
#include "openmm/internal/ContextImpl.h"
#include "openmm/reference/ReferencePlatform.h"
#include "lbm_b200.h"
#include <algorithm>
#include <cstring>
#include <exception>
#include <new>
#include <sstream>
#include <string>
#include <vector>

using namespace LBMPlugin;
using namespace OpenMM;

namespace {

thread_local std::string lastError;

struct RefKernel {
    ReferencePlatform platform;
    System system;
    ContextImpl context;
    ReferencePlatform::PlatformData data;
    std::vector<Vec3> positions, velocities, forces;
    ReferenceCalcLBMForceKernel* kernel;
    int numParticles;
    long long numNodes;
    RefKernel() : kernel(NULL), numParticles(0), numNodes(0) {
        data.positions = &positions;
        data.velocities = &velocities;
        data.forces = &forces;
        context.setPlatformData(&data);
    }
    ~RefKernel() { delete kernel; }
    void load(const LbmParticleArrays* p) {
        for (int i = 0; i < numParticles; i++) {
            positions[i] = Vec3(p->positions[3*i], p->positions[3*i+1], p->positions[3*i+2]);
            velocities[i] = Vec3(p->velocities[3*i], p->velocities[3*i+1], p->velocities[3*i+2]);
            forces[i] = Vec3(p->forces[3*i], p->forces[3*i+1], p->forces[3*i+2]);
        }
    }
    void store(const LbmParticleArrays* p) {
        for (int i = 0; i < numParticles; i++)
            for (int k = 0; k < 3; k++) {
                p->velocities[3*i+k] = velocities[i][k];
                p->forces[3*i+k] = forces[i][k];
            }
    }
};

LBMLatticeParameters toLattice(const LbmLatticeParameters* in, int numParticles, int numSolid, const int* solid) {
    LBMLatticeParameters l;
    l.nx = in->nx; l.ny = in->ny; l.nz = in->nz;
    l.procs[0] = l.procs[1] = l.procs[2] = 1;
    l.particleCopiesCheck = false;
    l.densityHaloExchange = l.velocityHaloExchange = false;
    l.dx = in->dx; l.dt = in->dt; l.density = in->density;
    l.tau = in->tau; l.omega = in->omega;
    l.initialVelocity = Vec3(in->initial_velocity[0], in->initial_velocity[1], in->initial_velocity[2]);
    l.bodyAcceleration = Vec3(in->body_acceleration[0], in->body_acceleration[1], in->body_acceleration[2]);
    l.friction = in->friction;
    l.kT = in->kT;
    l.dragScheme = (LBMForce::DragScheme) in->drag_scheme;
    l.interpolationStencil = (LBMForce::InterpolationStencil) in->interpolation_stencil;
    l.fluidFluctuations = in->fluid_fluctuations != 0;
    l.fluidKT = in->fluid_kT;
    l.randomNumberSeed = in->random_number_seed;
    l.momentumRemovalFrequency = in->momentum_removal_frequency;
    l.machCheckFrequency = in->mach_check_frequency;
    l.machNumberLimit = in->mach_number_limit;
    l.particles.clear();
    for (int i = 0; i < numParticles; i++)
        l.particles.push_back(i);
    l.solidNodes.assign(solid, solid + numSolid);
    std::sort(l.solidNodes.begin(), l.solidNodes.end());
    l.wallScheme = (LBMForce::WallScheme) in->wall_scheme;
    for (int f = 0; f < 6; f++) {
        l.faceBoundary[f] = (LBMForce::BoundaryType) in->face_boundary[f];
        l.faceVelocity[f] = Vec3(in->face_velocity[f][0], in->face_velocity[f][1], in->face_velocity[f][2]);
        l.faceDensity[f] = in->face_density[f];
    }
    return l;
}

LbmStatus fail(const std::exception& e) {
    lastError = e.what();
    std::string m = lastError;
    if (m.find("Mach number") != std::string::npos)
        return LBM_ERR_MACH_LIMIT;
    if (m.find("did not converge") != std::string::npos)
        return LBM_ERR_CG_NOT_CONVERGED;
    return LBM_ERR_INVALID_ARGUMENT;
}

} // namespace

#define GUARD_BEGIN try {
#define GUARD_END } catch (const std::exception& e) { return fail(e); } return LBM_OK;

extern "C" {

const char* refdrv_last_error(void) {
    return lastError.c_str();
}

LbmStatus refdrv_create(const LbmLatticeParameters* lattice, int num_particles, const double* masses,
                        int num_solid, const int* solid, RefKernel** out) {
    GUARD_BEGIN
    RefKernel* k = new RefKernel();
    k->numParticles = num_particles;
    k->numNodes = (long long) lattice->nx*lattice->ny*lattice->nz;
    for (int i = 0; i < num_particles; i++)
        k->system.addParticle(masses[i]);
    k->positions.resize(num_particles);
    k->velocities.resize(num_particles);
    k->forces.resize(num_particles);
    k->kernel = new ReferenceCalcLBMForceKernel("CalcLBMForce", k->platform);
    LBMLatticeParameters l = toLattice(lattice, num_particles, num_solid, solid);
    // The Reference kernel never reads the LBMForce object it is given (its parameters come in l).
    alignas(LBMForce) static char forceStorage[sizeof(LBMForce)];
    const LBMForce& force = *reinterpret_cast<const LBMForce*>(forceStorage);
    try {
        k->kernel->initialize(k->system, force, l);
    }
    catch (...) {
        delete k;
        throw;
    }
    *out = k;
    GUARD_END
}

void refdrv_destroy(RefKernel* k) {
    delete k;
}

LbmStatus refdrv_begin_step(RefKernel* k, long long step, const LbmParticleArrays* p) {
    GUARD_BEGIN
    k->context.setStepCount(step);
    if (k->numParticles > 0)
        k->load(p);
    k->kernel->beginStep(k->context);
    if (k->numParticles > 0)
        k->store(p);
    GUARD_END
}

LbmStatus refdrv_execute(RefKernel* k, long long step, const LbmParticleArrays* p, int include_forces,
                         int include_energy, double* energy) {
    GUARD_BEGIN
    k->context.setStepCount(step);
    if (k->numParticles > 0)
        k->load(p);
    double e = k->kernel->execute(k->context, include_forces != 0, include_energy != 0);
    if (energy)
        *energy = e;
    if (k->numParticles > 0)
        k->store(p);
    GUARD_END
}

LbmStatus refdrv_copy_parameters(RefKernel* k, const LbmLatticeParameters* lattice, int num_solid, const int* solid) {
    GUARD_BEGIN
    k->kernel->copyParametersToContext(k->context, toLattice(lattice, k->numParticles, num_solid, solid));
    GUARD_END
}

LbmStatus refdrv_get_fluid_fields(RefKernel* k, double* density, double* velocity) {
    GUARD_BEGIN
    std::vector<double> d;
    std::vector<Vec3> v;
    k->kernel->getFluidFields(k->context, d, v, false);
    for (size_t i = 0; i < d.size(); i++) {
        density[i] = d[i];
        for (int a = 0; a < 3; a++)
            velocity[3*i+a] = v[i][a];
    }
    GUARD_END
}

LbmStatus refdrv_get_fluid_mach_number(RefKernel* k, double* mach) {
    GUARD_BEGIN
    *mach = k->kernel->getFluidMachNumber(k->context);
    GUARD_END
}

LbmStatus refdrv_get_wall_force(RefKernel* k, double* force) {
    GUARD_BEGIN
    Vec3 f = k->kernel->getWallForce(k->context);
    for (int a = 0; a < 3; a++)
        force[a] = f[a];
    GUARD_END
}

LbmStatus refdrv_get_fluid_state(RefKernel* k, double* state) {
    GUARD_BEGIN
    std::vector<double> s;
    k->kernel->getFluidState(k->context, s);
    std::memcpy(state, s.data(), sizeof(double)*s.size());
    GUARD_END
}

LbmStatus refdrv_set_fluid_state(RefKernel* k, const double* state) {
    GUARD_BEGIN
    std::vector<double> s(state, state + LBM_NUM_VELOCITIES*k->numNodes);
    k->kernel->setFluidState(k->context, s);
    GUARD_END
}

/* The checkpoint of the reference kernel, as bytes: the first call with buffer == NULL gives the size. */
LbmStatus refdrv_create_checkpoint(RefKernel* k, void* buffer, size_t* bytes) {
    GUARD_BEGIN
    std::stringstream stream;
    k->kernel->createCheckpoint(k->context, stream);
    std::string s = stream.str();
    if (buffer != NULL) {
        if (*bytes < s.size())
            throw std::runtime_error("checkpoint buffer too small");
        std::memcpy(buffer, s.data(), s.size());
    }
    *bytes = s.size();
    GUARD_END
}

LbmStatus refdrv_load_checkpoint(RefKernel* k, const void* buffer, size_t bytes) {
    GUARD_BEGIN
    std::stringstream stream(std::string((const char*) buffer, bytes));
    k->kernel->loadCheckpoint(k->context, stream);
    GUARD_END
}

} // extern "C"
