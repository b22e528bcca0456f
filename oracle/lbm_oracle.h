/*
 * lbm_oracle.h -- TEST INFRASTRUCTURE: the CPU oracle of the B200 LBM force kernel.
 *
 * A plain-C restatement of the reference's Reference-platform kernel
 * (platforms/reference/src/ReferenceLBMKernels.cpp) in double precision, one domain.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load it; the product never
 * does.  Its entry points mirror include/lbm_b200.h with the prefix oracle_ and host arrays only.
 *
 * Random numbers come from one of two sources:
 *   ORACLE_RANDOM_SEQUENTIAL: the splitmix64 stream of the oracle's OpenMM shim (oracle/shim/sfmt/SFMT.h)
 *     turned into normals by the Box-Muller transform of ReferenceLBMKernels.cpp:1052-1064 and drawn in
 *     the reference's order (particles, then the nodes of the collision, then the boundary nodes), so
 *     that the oracle and the shimmed reference agree bit for bit also with noise;
 *   ORACLE_RANDOM_PHILOX: the counter-based Philox4x32-7 normals of the CUDA kernels (lbm_device.cuh),
 *     one counter per (purpose, node or particle, step), so that the oracle and the GPU agree to
 *     rounding also with noise.
 */
#ifndef LBM_ORACLE_H_
#define LBM_ORACLE_H_

#include "lbm_b200.h"
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_RANDOM_SEQUENTIAL = 0, ORACLE_RANDOM_PHILOX = 1 };

typedef struct OracleKernel OracleKernel;

const char* oracle_last_error(void);
LbmStatus oracle_create(const LbmLatticeParameters* lattice, int random_mode, int num_particles,
                        const double* particle_masses, int num_solid_nodes, const int* solid_nodes,
                        OracleKernel** kernel);
void oracle_destroy(OracleKernel* kernel);
LbmStatus oracle_begin_step(OracleKernel* kernel, long long step_count, const LbmParticleArrays* particles);
LbmStatus oracle_execute(OracleKernel* kernel, long long step_count, const LbmParticleArrays* particles,
                         int include_forces, int include_energy, double* energy);
LbmStatus oracle_copy_parameters(OracleKernel* kernel, const LbmLatticeParameters* lattice);
LbmStatus oracle_get_fluid_fields(OracleKernel* kernel, double* density, double* velocity);
LbmStatus oracle_get_fluid_mach_number(OracleKernel* kernel, double* mach);
LbmStatus oracle_get_wall_force(OracleKernel* kernel, double force[3]);
LbmStatus oracle_get_fluid_state(OracleKernel* kernel, double* state);
LbmStatus oracle_set_fluid_state(OracleKernel* kernel, const double* state);

/* Building blocks exposed for the tests. */
void oracle_philox4x32(const uint32_t counter[4], const uint32_t key[2], int rounds, uint32_t out[4]);
void oracle_philox4x32_10(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]);
/* Normal number m (0-based) of a purpose/index/step, in double (the Philox scheme of the kernels). */
double oracle_philox_normal(uint32_t seed, int purpose, long long index, long long step, int m);
void oracle_axis_weights(int stencil, double s, int n, int open, int* index, double* weight);
double oracle_stencil_kernel(int stencil, double r);
void oracle_fluctuation(const double r[15], double stress_amplitude, double ghost_amplitude, double xi[19]);
/* Boundary classification (LBMBoundaries::find): returns the number of boundary nodes, and fills the arrays
   when they are not NULL (each of size >= the count). */
int oracle_find_boundaries(const LbmLatticeParameters* lattice, int num_solid, const int* solid,
                           int* nodes, int* unknown, int* solid_bits, int* kind, int* face);

/* Bead forces (bonds, WCA or Lennard-Jones pairs) by brute force, the CPU counterpart of lbm_md_compute_forces. */
void oracle_md_forces(int n, const double* pos, const double box[3], int num_bonds, const int* bonds, double k, double r0,
                      int pair_type, double sigma, double eps, double cutoff, double* forces);

#ifdef __cplusplus
}
#endif

#endif
