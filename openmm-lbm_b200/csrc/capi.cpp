// The C ABI of the B200 LBM force kernel (include/lbm_b200.h): status codes, a thread-local error message,
// and no C++ exception crossing the boundary.
#include "kernel.cuh"
#include <cstring>
#include <new>
#include <string>

struct LbmKernel {
    lbm::B200Kernel* impl;
};

namespace {

thread_local std::string lastError;

LbmStatus fail(LbmStatus status, const std::string& message) {
    lastError = message;
    return status;
}

template <typename F>
LbmStatus guard(F&& f) {
    try {
        lastError.clear();
        f();
        return LBM_OK;
    }
    catch (const lbm::Error& e) {
        return fail(e.status, e.what());
    }
    catch (const std::bad_alloc&) {
        return fail(LBM_ERR_OUT_OF_MEMORY, "out of host memory");
    }
    catch (const std::exception& e) {
        return fail(LBM_ERR_INVALID_ARGUMENT, e.what());
    }
}

} // namespace

namespace lbm {
void setLastError(const std::string& message) {
    lastError = message;
}
}

extern "C" {

const char* lbm_last_error(void) {
    return lastError.c_str();
}

void lbm_default_force_description(LbmForceDescription* force) {
    if (force)
        lbm::defaultForceDescription(force);
}

LbmStatus lbm_compute_lattice_parameters(const LbmForceDescription* force, const double box[3], double step_size,
                                         int num_system_particles, const double* system_masses,
                                         int num_coupled, const int* coupled_particles,
                                         int num_solid_nodes, const int* solid_nodes,
                                         LbmLatticeParameters* lattice) {
    if (!force || !box || !lattice || num_system_particles < 0 || num_coupled < 0 || num_solid_nodes < 0 ||
            (num_system_particles > 0 && !system_masses) || (num_coupled > 0 && !coupled_particles) ||
            (num_solid_nodes > 0 && !solid_nodes))
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_compute_lattice_parameters: null argument");
    return guard([&] {
        lbm::computeLatticeParameters(*force, box, step_size, num_system_particles, system_masses, num_coupled,
                                      coupled_particles, num_solid_nodes, solid_nodes, *lattice);
    });
}

LbmStatus lbm_create(const LbmLatticeParameters* lattice, const LbmOptions* options, int num_particles,
                     const double* particle_masses, int num_solid_nodes, const int* solid_nodes, LbmKernel** kernel) {
    if (!lattice || !kernel)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_create: null argument");
    LbmOptions opts;
    if (options)
        opts = *options;
    else {
        opts.storage = LBM_STORAGE_F32;
        opts.device = 0;
        opts.stream = nullptr;
    }
    *kernel = nullptr;
    return guard([&] {
        LbmKernel* k = new LbmKernel;
        try {
            k->impl = new lbm::B200Kernel(*lattice, opts, num_particles, particle_masses, num_solid_nodes, solid_nodes);
        }
        catch (...) {
            delete k;
            throw;
        }
        *kernel = k;
    });
}

void lbm_destroy(LbmKernel* kernel) {
    if (kernel) {
        delete kernel->impl;
        delete kernel;
    }
}

#define CHECK_HANDLE(k) if (!(k) || !(k)->impl) return fail(LBM_ERR_INVALID_ARGUMENT, "null kernel handle")

LbmStatus lbm_begin_step(LbmKernel* kernel, long long step_count, const LbmParticleArrays* particles) {
    CHECK_HANDLE(kernel);
    return guard([&] { kernel->impl->beginStep(step_count, particles); });
}

LbmStatus lbm_execute(LbmKernel* kernel, long long step_count, const LbmParticleArrays* particles, int include_forces,
                      int include_energy, double* energy) {
    CHECK_HANDLE(kernel);
    return guard([&] {
        double e = kernel->impl->execute(step_count, particles, include_forces != 0, include_energy != 0);
        if (energy)
            *energy = e;
    });
}

LbmStatus lbm_copy_parameters(LbmKernel* kernel, const LbmLatticeParameters* lattice) {
    CHECK_HANDLE(kernel);
    if (!lattice)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_copy_parameters: null argument");
    return guard([&] { kernel->impl->copyParameters(*lattice); });
}

LbmStatus lbm_get_fluid_fields(LbmKernel* kernel, double* density, double* velocity) {
    CHECK_HANDLE(kernel);
    if (!density || !velocity)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_get_fluid_fields: null argument");
    return guard([&] { kernel->impl->getFluidFields(density, velocity); });
}

LbmStatus lbm_get_fluid_mach_number(LbmKernel* kernel, double* mach) {
    CHECK_HANDLE(kernel);
    if (!mach)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_get_fluid_mach_number: null argument");
    return guard([&] { *mach = kernel->impl->getFluidMachNumber(); });
}

LbmStatus lbm_get_wall_force(LbmKernel* kernel, double force[3]) {
    CHECK_HANDLE(kernel);
    if (!force)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_get_wall_force: null argument");
    return guard([&] { kernel->impl->getWallForce(force); });
}

LbmStatus lbm_get_fluid_state(LbmKernel* kernel, double* state) {
    CHECK_HANDLE(kernel);
    if (!state)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_get_fluid_state: null argument");
    return guard([&] { kernel->impl->getFluidState(state); });
}

LbmStatus lbm_set_fluid_state(LbmKernel* kernel, const double* state) {
    CHECK_HANDLE(kernel);
    if (!state)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_set_fluid_state: null argument");
    return guard([&] { kernel->impl->setFluidState(state); });
}

LbmStatus lbm_checkpoint_size(LbmKernel* kernel, size_t* bytes) {
    CHECK_HANDLE(kernel);
    if (!bytes)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_checkpoint_size: null argument");
    return guard([&] { *bytes = kernel->impl->checkpointSize(); });
}

LbmStatus lbm_create_checkpoint(LbmKernel* kernel, void* buffer, size_t bytes) {
    CHECK_HANDLE(kernel);
    if (!buffer)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_create_checkpoint: null argument");
    return guard([&] { kernel->impl->createCheckpoint(buffer, bytes); });
}

LbmStatus lbm_load_checkpoint(LbmKernel* kernel, const void* buffer, size_t bytes) {
    CHECK_HANDLE(kernel);
    if (!buffer)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_load_checkpoint: null argument");
    return guard([&] { kernel->impl->loadCheckpoint(buffer, bytes); });
}

LbmStatus lbm_set_checkpoint_element_size(LbmKernel* kernel, int element_size) {
    CHECK_HANDLE(kernel);
    return guard([&] { kernel->impl->setCheckpointElementSize(element_size); });
}

LbmStatus lbm_checkpoint_layout(LbmKernel* kernel, size_t* stream_bytes, size_t* trailer_bytes) {
    CHECK_HANDLE(kernel);
    if (!stream_bytes || !trailer_bytes)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_checkpoint_layout: null argument");
    return guard([&] { kernel->impl->checkpointLayout(*stream_bytes, *trailer_bytes); });
}

LbmStatus lbm_get_info(LbmKernel* kernel, long long* num_nodes, int* storage) {
    CHECK_HANDLE(kernel);
    if (num_nodes)
        *num_nodes = kernel->impl->numNodes();
    if (storage)
        *storage = kernel->impl->storage();
    return LBM_OK;
}

void* lbm_get_stream(LbmKernel* kernel) {
    if (!kernel || !kernel->impl)
        return nullptr;
    return (void*) kernel->impl->getStream();
}

LbmStatus lbm_profile_dense_kernel(LbmKernel* kernel, int enable) {
    CHECK_HANDLE(kernel);
    return guard([&] { kernel->impl->fluidEngine().profileDense(enable != 0); });
}

LbmStatus lbm_dense_kernel_time(LbmKernel* kernel, long long* launches, double* total_ms) {
    CHECK_HANDLE(kernel);
    if (!launches || !total_ms)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_dense_kernel_time: null argument");
    return guard([&] { kernel->impl->fluidEngine().denseTime(launches, total_ms); });
}

LbmStatus lbm_solver_iterations(LbmKernel* kernel, int* iterations) {
    CHECK_HANDLE(kernel);
    if (!iterations)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_solver_iterations: null argument");
    *iterations = kernel->impl->solverIterations();
    return LBM_OK;
}

LbmStatus lbm_set_coupled_atoms(LbmKernel* kernel, int num_atoms, int num_coupled, const int* particles) {
    CHECK_HANDLE(kernel);
    return guard([&] { kernel->impl->setCoupledAtoms(num_atoms, num_coupled, particles); });
}

LbmStatus lbm_begin_step_openmm(LbmKernel* kernel, long long step_count, const LbmOpenMMBuffers* buffers) {
    CHECK_HANDLE(kernel);
    return guard([&] { kernel->impl->beginStepOpenMM(step_count, buffers); });
}

LbmStatus lbm_execute_openmm(LbmKernel* kernel, long long step_count, const LbmOpenMMBuffers* buffers,
                             int include_forces, int include_energy, double* energy) {
    CHECK_HANDLE(kernel);
    (void) include_energy;
    return guard([&] {
        double e = kernel->impl->executeOpenMM(step_count, buffers, include_forces != 0);
        if (energy)
            *energy = e;
    });
}

LbmStatus lbm_set_solver_limits(LbmKernel* kernel, int max_iterations, long long barrier_polls) {
    CHECK_HANDLE(kernel);
    return guard([&] { kernel->impl->setSolverLimits(max_iterations, barrier_polls); });
}

LbmStatus lbm_solver_fallback_steps(LbmKernel* kernel, long long* steps) {
    CHECK_HANDLE(kernel);
    if (!steps)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_solver_fallback_steps: null argument");
    *steps = kernel->impl->solverFallbackSteps();
    return LBM_OK;
}

LbmStatus lbm_steady_residual(LbmKernel* kernel, int interval, double* residual) {
    CHECK_HANDLE(kernel);
    if (!residual || interval <= 0)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_steady_residual: null residual or interval not positive");
    return guard([&] { *residual = kernel->impl->fluidEngine().steadyResidual(interval); });
}

LbmStatus lbm_steady_solve(LbmKernel* kernel, long long first_step, int interval, double tolerance, long long max_steps,
                           long long* steps_taken, double* residual) {
    CHECK_HANDLE(kernel);
    return guard([&] {
        long long s = kernel->impl->steadySolve(first_step, interval, tolerance, max_steps, residual);
        if (steps_taken)
            *steps_taken = s;
    });
}

LbmStatus lbm_set_fluid_equilibrium(LbmKernel* kernel, const double* density, const double* velocity, int memory,
                                    int strain) {
    CHECK_HANDLE(kernel);
    if (!density || !velocity)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_set_fluid_equilibrium: null argument");
    return guard([&] { kernel->impl->setFluidEquilibrium(density, velocity, memory == LBM_MEMORY_DEVICE, strain != 0); });
}

LbmStatus lbm_kernel_launches(LbmKernel* kernel, long long* launches) {
    CHECK_HANDLE(kernel);
    if (!launches)
        return fail(LBM_ERR_INVALID_ARGUMENT, "lbm_kernel_launches: null argument");
    *launches = kernel->impl->fluidEngine().launches;
    return LBM_OK;
}

} // extern "C"
