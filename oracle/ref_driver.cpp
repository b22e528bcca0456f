/*
 * ref_driver.cpp -- TEST INFRASTRUCTURE (oracle): drives the reference's own Reference-platform
 * kernel, ReferenceCalcLBMForceKernel (platforms/reference/src/ReferenceLBMKernels.cpp), compiled
 * unmodified from the reference sources against the minimal OpenMM shim in oracle/shim/.
 *
 * Compiled with LBM_DRIVER_ADAPTER it drives instead the B200 platform kernel of this project
 * (openmm-lbm_b200/openmm/, CalcLBMForceKernel over liblbm_b200.so), created by its kernel factory,
 * with the entry points prefixed adapterdrv_: the same harness then runs the reference's kernel and
 * the drop-in through the same OpenMM interface.
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
#ifdef LBM_DRIVER_ADAPTER
#include "B200LBMKernelFactory.h"
#include "B200LBMKernels.h"
#define DRV(name) adapterdrv_##name
#else
#include "ReferenceLBMKernels.h"
#define DRV(name) refdrv_##name
#endif
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
    CalcLBMForceKernel* kernel;
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
    // The density halo is exchanged and the velocity halo is not, so that getFluidFields() with the halo shows both
    // kinds of halo node (one domain: no exchange takes place).
    l.densityHaloExchange = true;
    l.velocityHaloExchange = false;
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

LbmStatus DRV(create_with_storage)(const LbmLatticeParameters* lattice, int num_particles, const double* masses,
                                   int num_solid, const int* solid, int storage, RefKernel** out);

const char* DRV(last_error)(void) {
    return lastError.c_str();
}

LbmStatus DRV(create)(const LbmLatticeParameters* lattice, int num_particles, const double* masses,
                      int num_solid, const int* solid, RefKernel** out) {
    return DRV(create_with_storage)(lattice, num_particles, masses, num_solid, solid, LBM_STORAGE_F64, out);
}

/* The storage type matters only for the B200 platform kernel (the reference's Reference kernel stores doubles). */
LbmStatus DRV(create_with_storage)(const LbmLatticeParameters* lattice, int num_particles, const double* masses,
                                   int num_solid, const int* solid, int storage, RefKernel** out) {
    (void) storage;
    GUARD_BEGIN
    RefKernel* k = new RefKernel();
    k->numParticles = num_particles;
    k->numNodes = (long long) lattice->nx*lattice->ny*lattice->nz;
    for (int i = 0; i < num_particles; i++)
        k->system.addParticle(masses[i]);
    k->positions.resize(num_particles);
    k->velocities.resize(num_particles);
    k->forces.resize(num_particles);
#ifdef LBM_DRIVER_ADAPTER
    // The B200 platform kernel, created by its factory for a platform that keeps the particles in host vectors.
    LBMPlugin::B200LBMKernelFactory factory(storage);
    k->kernel = dynamic_cast<CalcLBMForceKernel*>(factory.createKernelImpl(CalcLBMForceKernel::Name(), k->platform,
                                                                           k->context));
#else
    k->kernel = new ReferenceCalcLBMForceKernel("CalcLBMForce", k->platform);
#endif
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

void DRV(destroy)(RefKernel* k) {
    delete k;
}

LbmStatus DRV(begin_step)(RefKernel* k, long long step, const LbmParticleArrays* p) {
    GUARD_BEGIN
    k->context.setStepCount(step);
    if (k->numParticles > 0)
        k->load(p);
    k->kernel->beginStep(k->context);
    if (k->numParticles > 0)
        k->store(p);
    GUARD_END
}

LbmStatus DRV(execute)(RefKernel* k, long long step, const LbmParticleArrays* p, int include_forces,
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

LbmStatus DRV(copy_parameters)(RefKernel* k, const LbmLatticeParameters* lattice, int num_solid, const int* solid) {
    GUARD_BEGIN
    k->kernel->copyParametersToContext(k->context, toLattice(lattice, k->numParticles, num_solid, solid));
    GUARD_END
}

LbmStatus DRV(get_fluid_fields)(RefKernel* k, double* density, double* velocity) {
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

/* getFluidFields() with the halo: (nx + 2)(ny + 2)(nz + 2) values, i fastest, NaN where the kernel gives none. */
LbmStatus DRV(get_fluid_fields_halo)(RefKernel* k, double* density, double* velocity) {
    GUARD_BEGIN
    std::vector<double> d;
    std::vector<Vec3> v;
    k->kernel->getFluidFields(k->context, d, v, true);
    for (size_t i = 0; i < d.size(); i++) {
        density[i] = d[i];
        for (int a = 0; a < 3; a++)
            velocity[3*i+a] = v[i][a];
    }
    GUARD_END
}

LbmStatus DRV(get_fluid_mach_number)(RefKernel* k, double* mach) {
    GUARD_BEGIN
    *mach = k->kernel->getFluidMachNumber(k->context);
    GUARD_END
}

LbmStatus DRV(get_wall_force)(RefKernel* k, double* force) {
    GUARD_BEGIN
    Vec3 f = k->kernel->getWallForce(k->context);
    for (int a = 0; a < 3; a++)
        force[a] = f[a];
    GUARD_END
}

LbmStatus DRV(get_fluid_state)(RefKernel* k, double* state) {
    GUARD_BEGIN
    std::vector<double> s;
    k->kernel->getFluidState(k->context, s);
    std::memcpy(state, s.data(), sizeof(double)*s.size());
    GUARD_END
}

LbmStatus DRV(set_fluid_state)(RefKernel* k, const double* state) {
    GUARD_BEGIN
    std::vector<double> s(state, state + LBM_NUM_VELOCITIES*k->numNodes);
    k->kernel->setFluidState(k->context, s);
    GUARD_END
}

/* The checkpoint of the reference kernel, as bytes: the first call with buffer == NULL gives the size. */
LbmStatus DRV(create_checkpoint)(RefKernel* k, void* buffer, size_t* bytes) {
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

LbmStatus DRV(load_checkpoint)(RefKernel* k, const void* buffer, size_t bytes) {
    GUARD_BEGIN
    std::stringstream stream(std::string((const char*) buffer, bytes));
    k->kernel->loadCheckpoint(k->context, stream);
    GUARD_END
}

} // extern "C"
