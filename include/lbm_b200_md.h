/*
 * lbm_b200_md.h -- C ABI of the bead dynamics that stand in for OpenMM around the LBM force kernel.
 *
 * The reference couples particles that OpenMM integrates: OpenMM computes their other forces and advances
 * them with its VerletIntegrator (leapfrog), calling the LBM kernel's beginStep/execute in between
 * (ContextImpl::updateContextState, calcForcesAndEnergy).  OpenMM is not part of this build, so these
 * entry points provide, on the device, the forces and the integrator of the benchmark configurations:
 * harmonic bonds U = k/2 (r - r0)^2, and Weeks-Chandler-Andersen or truncated Lennard-Jones pair forces
 * U = 4 eps [(sigma/r)^12 - (sigma/r)^6] within a cutoff (bonded pairs excluded), with minimum-image
 * periodic distances and a device cell list; and the leapfrog v += dt F/m, x += dt v.  They have no
 * counterpart in the reference's plugin.
 *
 * Arrays are device pointers of 3 doubles per particle (nm, nm/ps, kJ/mol/nm), launched on `stream`.
 */
#ifndef LBM_B200_MD_H_
#define LBM_B200_MD_H_

#include "lbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { LBM_PAIR_NONE = 0, LBM_PAIR_WCA = 1, LBM_PAIR_LJ = 2 };

typedef struct LbmMd LbmMd;

/* n particles with masses (Da), a rectangular periodic box (nm), num_bonds bonds (pairs of particle indices,
   2*num_bonds ints) with constant k (kJ/mol/nm^2) and length r0 (nm), and a pair force of type LBM_PAIR_* with
   sigma (nm), epsilon (kJ/mol) and cutoff (nm; the WCA cutoff is 2^(1/6) sigma whatever is given). */
LbmStatus lbm_md_create(int n, const double* masses, const double box[3], int num_bonds, const int* bonds, double k,
                        double r0, int pair_type, double sigma, double epsilon, double cutoff, int device, LbmMd** md);
void lbm_md_destroy(LbmMd* md);

/* forces = bond and pair forces at positions (both device arrays), overwriting forces. */
LbmStatus lbm_md_compute_forces(LbmMd* md, const double* positions, double* forces, void* stream);

/* Leapfrog step of OpenMM's VerletIntegrator: v += dt F/m; x += dt v (device arrays). */
LbmStatus lbm_md_integrate(LbmMd* md, double dt, double* positions, double* velocities, const double* forces,
                           void* stream);

/* Sum over particles of m v^2 (Da nm^2/ps^2) of the velocities (device array), for temperatures (synchronizes). */
LbmStatus lbm_md_kinetic(LbmMd* md, const double* velocities, double* twice_kinetic, void* stream);

/* Number of CUDA kernels this object has launched since it was created. */
LbmStatus lbm_md_kernel_launches(LbmMd* md, long long* launches);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_MD_H_ */
