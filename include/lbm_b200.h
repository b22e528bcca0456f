/*
 * lbm_b200.h -- C ABI of the B200 lattice-Boltzmann force kernel.
 *
 * This is the drop-in boundary for the per-step fluid and particle-coupling path of openmm-lbm.
 * Each entry point replaces one method of the plugin kernel interface
 * `LBMPlugin::CalcLBMForceKernel` (openmmapi/include/LBMKernels.h:97-189) and takes the
 * lattice-unit parameter block `LBMPlugin::LBMLatticeParameters` (LBMKernels.h:30-92) flattened
 * into a plain C struct.  Everything crossing the boundary is a plain pointer, a size or a POD
 * struct: no C++ or torch types.
 *
 * OpenMM's ContextImpl is replaced by explicit arguments: the step count of the integrator
 * (ContextImpl::getStepCount) and the particle arrays (positions, velocities, forces of the coupled
 * particles, in the order in which they were coupled) that the Reference platform reads from
 * ReferencePlatform::PlatformData and the CUDA platform from its posq/velm/force buffers.
 *
 * Units are those of LBMLatticeParameters: dx (nm), dt (ps), density (Da/nm^3), friction (1/ps),
 * kT (kJ/mol); velocities and accelerations of the fluid in lattice units; particle positions in
 * nm, velocities in nm/ps, forces in kJ/mol/nm.
 *
 * Every call returns an LbmStatus; on failure lbm_last_error() gives the message (thread-local).
 * A handle is driven by one host thread at a time; distinct handles are independent.
 */
#ifndef LBM_B200_H_
#define LBM_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_NUM_VELOCITIES 19

/* Status codes.  The reference throws OpenMMException with a message in each of these cases. */
typedef enum LbmStatus {
    LBM_OK = 0,
    LBM_ERR_INVALID_ARGUMENT = 1,   /* bad setup (LBMForceImpl.cpp:44-214 checks), wrong sizes, null pointers */
    LBM_ERR_MACH_LIMIT = 2,         /* Mach number above the limit (ReferenceLBMKernels.cpp:412-420) */
    LBM_ERR_CG_NOT_CONVERGED = 3,   /* centred stencil drag: no convergence in 1000 iterations (:864-866) */
    LBM_ERR_DEVICE_TIMEOUT = 4,     /* a bounded device-side wait ran out */
    LBM_ERR_CUDA = 5,               /* a CUDA runtime call failed */
    LBM_ERR_OUT_OF_MEMORY = 6,
    LBM_ERR_NOT_SUPPORTED = 7,      /* e.g. a storage type that the option set does not allow */
    LBM_ERR_CHECKPOINT = 8          /* a checkpoint of another lattice, precision or particle count */
} LbmStatus;

/* Enumerations with the values of LBMForce.h:46-138. */
enum { LBM_DRAG_EXPLICIT = 0, LBM_DRAG_CENTERED = 1 };
enum { LBM_STENCIL_NEAREST = 0, LBM_STENCIL_TRILINEAR = 1, LBM_STENCIL_THREEPOINT = 2, LBM_STENCIL_KEYS = 3 };
enum { LBM_WALL_BOUNCEBACK = 0, LBM_WALL_REGULARIZED = 1 };
enum { LBM_FACE_XMIN = 0, LBM_FACE_XMAX = 1, LBM_FACE_YMIN = 2, LBM_FACE_YMAX = 3, LBM_FACE_ZMIN = 4, LBM_FACE_ZMAX = 5 };
enum { LBM_BOUNDARY_PERIODIC = 0, LBM_BOUNDARY_VELOCITY = 1, LBM_BOUNDARY_DENSITY = 2, LBM_BOUNDARY_DENSITY_VELOCITY = 3 };

/* Storage type of the population deviations f_q - w_q in device memory.  The collision computes in
   double for LBM_STORAGE_F64 and in float for the others. */
enum { LBM_STORAGE_F64 = 0, LBM_STORAGE_F32 = 1, LBM_STORAGE_F16 = 2, LBM_STORAGE_BF16 = 3 };

/* Where the particle arrays of a call live. */
enum { LBM_MEMORY_HOST = 0, LBM_MEMORY_DEVICE = 1 };

/*
 * The lattice parameters in lattice units and the conversion factors, as LBMLatticeParameters
 * (LBMKernels.h:30-92) for one domain (procs = 1,1,1; the MPI fields are absent).  particles and
 * solidNodes are passed separately to lbm_create().
 */
typedef struct LbmLatticeParameters {
    int nx, ny, nz;
    double dx, dt, density;              /* nm, ps, Da/nm^3 */
    double tau, omega;                   /* omega = 1/tau */
    double initial_velocity[3];          /* lattice units */
    double body_acceleration[3];         /* lattice units */
    double friction;                     /* 1/ps */
    double kT;                           /* kJ/mol, 0 without random force (NVE) */
    int drag_scheme;                     /* LBM_DRAG_* */
    int interpolation_stencil;           /* LBM_STENCIL_* */
    int fluid_fluctuations;              /* 0 or 1 */
    double fluid_kT;                     /* kJ/mol, 0 without fluctuations */
    int random_number_seed;
    int momentum_removal_frequency;      /* 0 = never */
    int mach_check_frequency;            /* 0 = never */
    double mach_number_limit;
    int wall_scheme;                     /* LBM_WALL_* */
    int face_boundary[6];                /* LBM_BOUNDARY_* per LBM_FACE_* */
    double face_velocity[6][3];          /* lattice units */
    double face_density[6];              /* lattice units, 1 = fluid at rest */
} LbmLatticeParameters;

/* Options of this implementation that have no counterpart in the reference. */
typedef struct LbmOptions {
    int storage;            /* LBM_STORAGE_* (the reference stores FP64 on its Reference platform) */
    int device;             /* CUDA device ordinal */
    void* stream;           /* cudaStream_t to launch on; NULL = a stream owned by the handle */
} LbmOptions;

/*
 * The coupled particles seen by one call, in coupling order (index i of LBMForce::addParticle()):
 * positions (nm), velocities (nm/ps) and forces (kJ/mol/nm), 3 doubles per particle, either all in
 * host memory or all in device memory of the handle's device.  lbm_begin_step() may reverse
 * velocities (reflection at walls); lbm_execute() adds the coupling forces to forces, and with the
 * centred drag reads the other forces already accumulated there (LBMForce must be the last force).
 */
typedef struct LbmParticleArrays {
    double* positions;
    double* velocities;
    double* forces;
    int memory;             /* LBM_MEMORY_* */
} LbmParticleArrays;

/*
 * The parameters of an LBMForce in OpenMM units, as set with its setters (LBMForce.h:162-666) and with
 * the defaults of its constructor (LBMForce.cpp:19-29, see lbm_default_force_description()).
 */
typedef struct LbmForceDescription {
    int nx, ny, nz;                      /* setGridSize */
    double fluid_density;                /* Da/nm^3, setFluidDensity */
    double kinematic_viscosity;          /* nm^2/ps, setKinematicViscosity */
    double friction;                     /* 1/ps, setFriction */
    double temperature;                  /* K, setTemperature */
    int coupling_scheme;                 /* 0 EulerMaruyama, 1 NVE (setCouplingScheme) */
    int drag_scheme;                     /* LBM_DRAG_* */
    int interpolation_stencil;           /* LBM_STENCIL_* */
    int fluid_fluctuations;              /* setFluidFluctuations */
    int wall_scheme;                     /* LBM_WALL_* */
    int face_boundary[6];                /* LBM_BOUNDARY_* */
    double face_velocity[6][3];          /* nm/ps */
    double face_density[6];              /* Da/nm^3, 0 = the fluid density */
    int random_number_seed;
    double body_acceleration[3];         /* nm/ps^2 */
    double initial_velocity[3];          /* nm/ps */
    int momentum_removal_frequency;
    int mach_check_frequency;
    double mach_number_limit;
} LbmForceDescription;

typedef struct LbmKernel LbmKernel;

/* Message of the last failed call on this thread (empty if none). */
const char* lbm_last_error(void);

/* The defaults of LBMForce's constructor (LBMForce.cpp:19-29). */
void lbm_default_force_description(LbmForceDescription* force);

/*
 * LBMForceImpl::computeLatticeParameters (openmmapi/src/LBMForceImpl.cpp:44-214): checks the setup and
 * converts it to lattice units, for a rectangular periodic box (box[3], nm), the integrator step size
 * (ps), the masses of the System's particles (Da) and the indices of the coupled ones.  The same error
 * messages as the reference.  Needs no GPU.
 */
LbmStatus lbm_compute_lattice_parameters(const LbmForceDescription* force, const double box[3], double step_size,
                                         int num_system_particles, const double* system_masses,
                                         int num_coupled, const int* coupled_particles,
                                         int num_solid_nodes, const int* solid_nodes,
                                         LbmLatticeParameters* lattice);

/* CalcLBMForceKernel::initialize (LBMKernels.h:111); masses in Da, solid node indices sorted or not. */
LbmStatus lbm_create(const LbmLatticeParameters* lattice, const LbmOptions* options,
                     int num_particles, const double* particle_masses,
                     int num_solid_nodes, const int* solid_nodes, LbmKernel** kernel);

void lbm_destroy(LbmKernel* kernel);

/* CalcLBMForceKernel::beginStep (LBMKernels.h:119). */
LbmStatus lbm_begin_step(LbmKernel* kernel, long long step_count, const LbmParticleArrays* particles);

/* CalcLBMForceKernel::execute (LBMKernels.h:128); the energy is always 0 (the coupling is dissipative). */
LbmStatus lbm_execute(LbmKernel* kernel, long long step_count, const LbmParticleArrays* particles,
                      int include_forces, int include_energy, double* energy);

/* CalcLBMForceKernel::copyParametersToContext (LBMKernels.h:135). */
LbmStatus lbm_copy_parameters(LbmKernel* kernel, const LbmLatticeParameters* lattice);

/* CalcLBMForceKernel::getFluidFields (LBMKernels.h:144), one domain, no halo: density[N] in Da/nm^3 and
   velocity[3N] in nm/ps (x, y, z per node), node index order; zero at solid nodes. */
LbmStatus lbm_get_fluid_fields(LbmKernel* kernel, double* density, double* velocity);

/* CalcLBMForceKernel::getFluidMachNumber (LBMKernels.h:149). */
LbmStatus lbm_get_fluid_mach_number(LbmKernel* kernel, double* mach);

/* CalcLBMForceKernel::getWallForce (LBMKernels.h:154): kJ/mol/nm. */
LbmStatus lbm_get_wall_force(LbmKernel* kernel, double force[3]);

/* CalcLBMForceKernel::getFluidState / setFluidState (LBMKernels.h:159-164): deviations f_q - w_q as
   double, [q*N + node]. */
LbmStatus lbm_get_fluid_state(LbmKernel* kernel, double* state);
LbmStatus lbm_set_fluid_state(LbmKernel* kernel, const double* state);

/* CalcLBMForceKernel::createCheckpoint / loadCheckpoint (LBMKernels.h:170-174).  The checkpoint is the kernel
   stream of the reference's GPU platforms (CommonCalcLBMForceKernel::createCheckpoint, CommonLBMKernels.cpp:
   2019-2058), which the reference's CUDA kernel reads, followed by a trailer of this kernel that the reference
   ignores:
     int element size E (8 for double and mixed precision, 4 for single); int flags[2] = {numbers drawn for the
     next step, fluid advanced}; the populations f_q - w_q, 19*N values of E bytes, [q*N + node]; with coupled
     particles P > 0, P float4 of drawn numbers and 3*P values of E bytes of particle wall momentum (SoA); 3*max(1,
     solid nodes) values of E bytes of wall momentum (SoA); with boundary nodes B > 0 (regularized walls, open
     faces), 3*B values of E bytes (SoA);
     the trailer: the tag "B200LBM1", the exact step statistics, the evaluation state and the random seed in use,
     and, when the populations of FP64 storage were written with E = 4, their raw storage bytes.
   This kernel writes no drawn numbers (flags[0] = 0: its random numbers are a function of the seed, the step and
   the particle or node) and puts the wall momentum of the last step, less the static part that a reader adds, into
   the first wall entry.  A checkpoint with its trailer restarts this kernel bit for bit (with the seed of the run
   that wrote it, as the reference restores its generator state); one without it (written
   by the reference's CUDA kernel) restores the populations, the wall momentum and the flag "fluid advanced", and
   the next step draws new random numbers.  A checkpoint of another element size is rejected with "LBMForce: the
   checkpoint was written with a different precision". */
LbmStatus lbm_checkpoint_size(LbmKernel* kernel, size_t* bytes);
LbmStatus lbm_create_checkpoint(LbmKernel* kernel, void* buffer, size_t bytes);
LbmStatus lbm_load_checkpoint(LbmKernel* kernel, const void* buffer, size_t bytes);
/* The element size E of the checkpoint stream (4 or 8), as the platform's precision gives it: 8 for double and
   mixed, 4 for single.  The default is 8 with FP64 storage and 4 otherwise. */
LbmStatus lbm_set_checkpoint_element_size(LbmKernel* kernel, int element_size);
/* The sizes of the two parts of the checkpoint: the reference's stream and the trailer. */
LbmStatus lbm_checkpoint_layout(LbmKernel* kernel, size_t* stream_bytes, size_t* trailer_bytes);

/* Number of device nodes N = nx*ny*nz and the storage type actually used. */
LbmStatus lbm_get_info(LbmKernel* kernel, long long* num_nodes, int* storage);

/* The CUDA stream that the handle launches on (cudaStream_t), for callers that order work with it. */
void* lbm_get_stream(LbmKernel* kernel);

/* Timing of the dense stream-collide kernel with CUDA events recorded on the handle's stream around each of its
   launches, while enabled (enable = 1 also clears the record).  lbm_dense_kernel_time synchronizes the stream
   and returns the number of timed launches and their total duration in milliseconds. */
LbmStatus lbm_profile_dense_kernel(LbmKernel* kernel, int enable);
LbmStatus lbm_dense_kernel_time(LbmKernel* kernel, long long* launches, double* total_ms);

/* Number of CUDA kernels this handle has launched since it was created. */
LbmStatus lbm_kernel_launches(LbmKernel* kernel, long long* launches);

/* Conjugate-gradient iterations of the last centred stencil drag solve (0 for the other coupling schemes). */
LbmStatus lbm_solver_iterations(LbmKernel* kernel, int* iterations);

/* Steps, since creation, whose centred stencil drag was solved by spreading and gathering on the lattice nodes
   instead of through the explicit coupling matrix (a cell of the particle cell list or a row of the matrix over its
   capacity, or LBM_B200_SPREAD_CG=1 in the environment).  No counterpart in the reference, whose solve is always the
   spread-and-gather one (platforms/reference/src/ReferenceLBMKernels.cpp:726-901). */
LbmStatus lbm_solver_fallback_steps(LbmKernel* kernel, long long* steps);

/*
 * The particle buffers of an OpenMM CUDA-platform Context (OpenMM's CudaContext: getPosq(), getPosqCorrection(),
 * getVelm(), getLongForceBuffer(), getAtomIndexArray()), on the handle's device, for an OpenMM platform kernel that
 * drives this library without copying the particles through host memory.  They are what the reference's CUDA kernels
 * read and write (platforms/common/src/kernels/lbmCoupling.cc:12-16, 47-54, 148-171, 2043-2053).  Atoms are in the
 * platform's storage order, which OpenMM changes when it reorders them: atom_index[j] is the System index of the atom
 * stored at slot j.
 */
enum { LBM_OPENMM_SINGLE = 0, LBM_OPENMM_MIXED = 1, LBM_OPENMM_DOUBLE = 2 };   /* the Context's "Precision" */
typedef struct LbmOpenMMBuffers {
    const void* posq;              /* float4 (single, mixed) or double4 (double): x, y, z (nm) and the charge */
    const void* posq_correction;   /* mixed: float4 added to posq for the full position; NULL otherwise */
    void* velm;                    /* float4 (single) or double4 (mixed, double): v (nm/ps) and 1/mass */
    long long* force;              /* fixed-point forces in units of 2^-32 kJ/mol/nm, [k*padded_num_atoms + j] */
    const int* atom_index;         /* [num_atoms] */
    int num_atoms, padded_num_atoms;
    int precision;                 /* LBM_OPENMM_* */
} LbmOpenMMBuffers;

/* The coupled particles as System indices, in coupling order (LBMLatticeParameters::particles, LBMKernels.h:61), and
   the number of atoms of the System; once, before the first lbm_begin_step_openmm / lbm_execute_openmm.  No
   counterpart call in the reference, whose CUDA kernel builds the same index (couplingIndex, lbmCoupling.cc:12-16). */
LbmStatus lbm_set_coupled_atoms(LbmKernel* kernel, int num_atoms, int num_coupled, const int* particles);

/* CalcLBMForceKernel::beginStep (LBMKernels.h:119) on the buffers of an OpenMM Context: the reflection at the walls
   reverses the velocities of the coupled atoms in velm (reflectParticles, lbmCoupling.cc:148-171). */
LbmStatus lbm_begin_step_openmm(LbmKernel* kernel, long long step_count, const LbmOpenMMBuffers* buffers);

/* CalcLBMForceKernel::execute (LBMKernels.h:128) on the buffers of an OpenMM Context: the coupling forces are added
   to the fixed-point force buffer as (long long) (F 2^32) (applyCouplingForces, lbmCoupling.cc:2043-2053).  With the
   centred drag the other forces of the coupled atoms are read from that buffer first (times 2^-32), so the call must
   come after every other force of the step, as the reference's post-computation (CommonLBMKernels.cpp:115-126). */
LbmStatus lbm_execute_openmm(LbmKernel* kernel, long long step_count, const LbmOpenMMBuffers* buffers,
                             int include_forces, int include_energy, double* energy);

/* Limits of the centred stencil drag's conjugate gradients, for tests of their failure paths: at most max_iterations
   iterations (then LBM_ERR_CG_NOT_CONVERGED, as ReferenceLBMKernels.cpp:864-866 after 1000), and barrier_polls polls
   of a block waiting at a grid barrier of the cooperative solve (then LBM_ERR_DEVICE_TIMEOUT).  A failed solve leaves
   no reaction on the fluid and the step can be evaluated again.  0 restores a default (1000 iterations, 2^26 polls).
   No counterpart in the reference, whose cap is fixed and whose solve has no device-side wait. */
LbmStatus lbm_set_solver_limits(LbmKernel* kernel, int max_iterations, long long barrier_polls);

/* The steady-state residual r = max_nodes |u - u_prev| / (interval max_nodes |u|) over the fluid nodes, in FP64 on the
   device, with u = j/rho of the current (post-stream) state and u_prev the velocities recorded by the previous call,
   which this call replaces; the first call records them and returns infinity.  Called every `interval` steps it is the
   convergence test of a steady solve (r <= 1e-6).  No counterpart in the reference, which defines no residual. */
LbmStatus lbm_steady_residual(LbmKernel* kernel, int interval, double* residual);

/* Advances a fluid without coupled particles from step first_step until the steady residual (lbm_steady_residual,
   checked every `interval` steps, first against the state at the start) is at most `tolerance`, or for max_steps
   steps; returns the steps taken and the last residual.  The plain solve of a steady flow, cold or warm started.
   No counterpart in the reference. */
LbmStatus lbm_steady_solve(LbmKernel* kernel, long long first_step, int interval, double tolerance, long long max_steps,
                           long long* steps_taken, double* residual);

/* Sets the fluid to the populations of the given fields, density [N] and velocity [N][3] in the units of
   lbm_get_fluid_fields, in host (memory = LBM_MEMORY_HOST) or device memory (LBM_MEMORY_DEVICE): the equilibrium, plus
   with strain != 0 the Chapman-Enskog non-equilibrium part of the strain rate (central differences of the velocity),
   which a steady flow has; the warm start of a steady solve from predicted fields.  Solid nodes are left at rest.
   No counterpart in the reference. */
LbmStatus lbm_set_fluid_equilibrium(LbmKernel* kernel, const double* density, const double* velocity, int memory,
                                    int strain);

/*
 * Fluid moments of a state that the caller owns, without allocating any memory.  It has no counterpart in the
 * reference: it is for callers that cannot call cudaMalloc -- a plugin whose host program owns the device memory
 * through its own allocator (an MD engine's context, a framework's caching allocator that holds the pool), or a
 * time-critical loop that cannot take the device synchronization cudaMalloc and cudaFree may imply.
 *
 * state: device array of 19*num_nodes doubles in the layout of lbm_get_fluid_state ([q*N + node], f_q - w_q);
 * is_fluid: device array of num_nodes bytes, nonzero for fluid nodes, or NULL when every node is fluid;
 * moments: device array of 5 doubles that receives the sum of the deviations over the fluid nodes (the fluid's mass
 * minus the number of fluid nodes), the fluid's momentum (x, y, z) and the Mach number sqrt(3 max |j/rho|^2) that
 * lbm_get_fluid_mach_number gives.  Launched on `stream` (a cudaStream_t, NULL for the default stream).
 *
 * The partial sums live in a fixed device array of the library (128 KB on every GPU that loads it, kept until the
 * process exits): at most 67,108,864 nodes (2048 chunks of 32,768); larger lattices are rejected with
 * LBM_ERR_INVALID_ARGUMENT.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress), so make it before any stream capture.  All calls share the array: calls that overlap on the
 * GPU race, and must be ordered (one stream, or events).
 */
LbmStatus lbm_fluid_moments_noalloc(const double* state, long long num_nodes, const unsigned char* is_fluid,
                                    double* moments, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H_ */
