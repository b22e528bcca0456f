/* Replica batches of the B200 LBM force kernel: many independent periodic lattices of uneven sizes, each with its own
 * coupled particles, advanced together on one device.
 *
 * No counterpart in the reference: its examples run seed ensembles as one OpenMM Context per replica, looping in
 * Python (examples/cocomo).  Here a run of steps of all replicas (bead pair forces, stencil and explicit drag, the
 * dense stream-collide step, the per-replica sums, the reaction clear and the leapfrog of the beads) is one
 * persistent cooperative launch, captured once in a CUDA graph and replayed (lbm_batch_set_persistent).  Each
 * replica follows the step of a kernel created by lbm_create with the same lattice parameters, driven as an OpenMM
 * VerletIntegrator step would drive it: beginStep, the bead forces, execute (explicit drag and the fluid step), and
 * the leapfrog v += dt F/m, x += dt v with the lattice time step.
 *
 * Replicas: periodic lattices (no solid nodes, every face periodic), explicit drag, one interpolation stencil and
 * one storage type (FP64 or FP32) for the batch; fluctuations, momentum removal and the body force per replica.
 * Bead pair forces (WCA or truncated Lennard-Jones) are summed over all pairs of a replica.  No Mach check.
 */
#ifndef LBM_B200_BATCH_H
#define LBM_B200_BATCH_H

#include "lbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct LbmBatch LbmBatch;

/* Pair force between the beads of a replica: pair_type LBM_PAIR_NONE, LBM_PAIR_WCA or LBM_PAIR_LJ
 * (include/lbm_b200_md.h), sigma and cutoff in nm, epsilon in kJ/mol. */
typedef struct LbmBatchPairForce {
    int pair_type;
    double sigma, epsilon, cutoff;
} LbmBatchPairForce;

/* Creates a batch of num_replicas replicas.  lattices[r]: the lattice parameters of replica r (as from
 * lbm_compute_lattice_parameters); num_particles[r]: its beads; masses and positions: all beads, replica by replica
 * (Da; nm, 3 per bead).  The fluids start at rest, the beads with zero velocity.  options: storage (LBM_STORAGE_F64
 * or LBM_STORAGE_F32), device and stream (NULL: the batch creates its own).  A replica seed of 0 asks for a random
 * one.  Status LBM_ERR_NOT_SUPPORTED for a replica outside the scope above. */
LbmStatus lbm_batch_create(int num_replicas, const LbmLatticeParameters* lattices, const int* num_particles,
                           const double* masses, const double* positions, const LbmBatchPairForce* pair,
                           const LbmOptions* options, LbmBatch** batch);
void lbm_batch_destroy(LbmBatch* batch);

/* Advances every replica by `steps` lattice steps: whole graphs of graph_steps steps are replayed, the rest launched
 * directly.  Asynchronous on the batch's stream. */
LbmStatus lbm_batch_step(LbmBatch* batch, int steps);

/* Chooses the block size of the batched dense kernel (128, 256 or 512 threads) by timing each on the current state,
 * without advancing it, and sets the number of steps per CUDA graph (graph_steps > 0; 0 keeps the current value).
 * Returns the block size chosen and its time per launch (ms, CUDA events over 5 launches). */
LbmStatus lbm_batch_autotune(LbmBatch* batch, int graph_steps, int* threads_per_block, double* dense_ms);

/* Bead positions and velocities of all replicas (host arrays of 3 doubles per bead, replica by replica). */
LbmStatus lbm_batch_get_particles(LbmBatch* batch, double* positions, double* velocities);
LbmStatus lbm_batch_set_velocities(LbmBatch* batch, const double* velocities);

/* Populations of replica r as deviations [q*N + node] (19 N doubles), the layout of lbm_get_fluid_state. */
LbmStatus lbm_batch_get_fluid_state(LbmBatch* batch, int replica, double* state);

/* Per replica (num_replicas values each, kJ/mol): the fluid temperature sum rho (u - <u>)^2/(3 N) over the nodes, with
 * u = j/rho + g/2 and <u> the mass-weighted mean, and the bead temperature sum m v^2/(3 n) of the current velocities. */
LbmStatus lbm_batch_temperatures(LbmBatch* batch, double* fluid_kT, double* bead_kT);

/* The form of a step: enable != 0 (the default) runs graph_steps steps in one persistent cooperative launch, captured
 * once in a CUDA graph and replayed -- the phases of a step (bead pair forces, stencil slots and the clear of the
 * previous reactions; explicit drag, reaction and leapfrog; the dense step with the per-replica sums) separated by
 * bounded grid barriers; enable = 0 launches the seven phase kernels of a step one after another (each replica then
 * computes the same step; the form exists for comparisons).  A grid barrier that waits more than the poll limit
 * gives up: that launch stops incomplete and the next call that synchronizes (lbm_batch_get_particles,
 * lbm_batch_get_fluid_state, lbm_batch_temperatures) returns LBM_ERR_DEVICE_TIMEOUT.
 * lbm_batch_set_barrier_polls sets that limit (0: the default 2^26 polls; a low value makes the timeout reachable in
 * tests). */
LbmStatus lbm_batch_set_persistent(LbmBatch* batch, int enable);
LbmStatus lbm_batch_set_barrier_polls(LbmBatch* batch, long long polls);

/* Total nodes of all replicas, lattice steps taken, kernels launched so far, the block size of the dense kernel and
 * the steps per CUDA graph (one launch per graph_steps steps in the persistent form). */
LbmStatus lbm_batch_info(LbmBatch* batch, long long* total_nodes, long long* steps, long long* launches,
                         int* threads_per_block, int* graph_steps);

#ifdef __cplusplus
}
#endif

#endif
