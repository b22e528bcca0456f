/*
 * lbm_oracle.c -- TEST INFRASTRUCTURE: plain-C restatement of the reference's Reference-platform
 * LBM force kernel (platforms/reference/src/ReferenceLBMKernels.cpp), double precision, one domain.
 *
 * This file is the checker of the CUDA kernels, never the product: only tests/, the smoke check and
 * the CPU-baseline leg of bench.py load it.  Every function cites the reference lines it restates.
 * The D3Q19 algebra follows openmmapi/include/internal/D3Q19.h, the stencils LBMStencils.h and the
 * boundary classification LBMBoundaries.h.  Expressions keep the reference's order of operations,
 * so that (with -ffp-contract=off) the two agree to the last bit.
 *
 * Parity pins: tests/test_oracle.py compares this restatement with the reference kernel compiled
 * unmodified (oracle/_ref) on the reference's own cross-platform cases (python/tests/TestLBMForce.py:
 * 505-635) and with the analytic known answers of tests/TestLBMFluid.h and TestLBMCoupling.h.
 */
#include "lbm_oracle.h"
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define Q 19

/* D3Q19 velocity set, opposite directions and weights (D3Q19.h:29-37). */
static const int CX[Q] = {0, 1, -1, 0,  0, 0,  0, 1, -1,  1, -1, 0,  0,  0,  0, 1, -1, -1,  1};
static const int CY[Q] = {0, 0,  0, 1, -1, 0,  0, 1, -1, -1,  1, 1, -1,  1, -1, 0,  0,  0,  0};
static const int CZ[Q] = {0, 0,  0, 0,  0, 1, -1, 0,  0,  0,  0, 1, -1, -1,  1, 1, -1,  1, -1};
static const int OPP[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const double W[Q] = {1.0/3.0,
        1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0,
        1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0,
        1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0};
/* Norms b_k of the orthogonal basis (D3Q19.h:136-137). */
static const double MODE_NORM[Q] = {1.0, 1.0/3.0, 1.0/3.0, 1.0/3.0, 2.0/9.0, 2.0/9.0, 2.0/9.0, 1.0/9.0, 1.0/9.0,
        1.0/9.0, 2.0/27.0, 2.0/27.0, 2.0/27.0, 1.0/18.0, 1.0/18.0, 1.0/18.0, 7.0/162.0, 5.0/126.0, 1.0/30.0};

/* Boundary node kinds (LBMBoundaries.h:30). */
enum { KIND_WALL = 0, KIND_VELOCITY = 1, KIND_DENSITY = 2, KIND_DENSITY_AT_REST = 3, KIND_DENSITY_VELOCITY = 4 };

/* Purposes of the Philox counters. */
enum { PURPOSE_FLUID = 0, PURPOSE_BOUNDARY = 1, PURPOSE_PARTICLE = 2 };

static _Thread_local char last_error[512];

static LbmStatus set_error(LbmStatus status, const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    vsnprintf(last_error, sizeof(last_error), fmt, args);
    va_end(args);
    return status;
}

const char* oracle_last_error(void) {
    return last_error;
}

typedef struct { double v[3]; } vec3;

struct OracleKernel {
    LbmLatticeParameters L;
    int nx, ny, nz;
    long n;                          /* number of nodes */
    int random_mode;
    uint32_t seed;
    /* fluid state and per-step moments (ReferenceLBMKernels.h:133-141) */
    double *pop, *rho, *drho, *mom, *pi, *fd, *reaction;
    char* fluid;                     /* NULL without solid nodes */
    int nsolid;
    int* solid;
    int nwall;
    int *wall_nodes, *wall_links;
    int nbnd;
    int *bnd_node, *bnd_unknown, *bnd_solid, *bnd_kind, *bnd_face;
    int* bnd_of_node;                /* with fluctuations and equilibrium-noise kinds, else NULL */
    double* bnd_stress;
    /* evaluation state machine (ReferenceLBMKernels.h:158-164) */
    int step_pending, step_forces_current;
    long long step_index;
    /* particles, in lattice units of mass (m/m_c) */
    int np;
    double* pmass;
    double* pforce;                  /* coupling forces in kJ/mol/nm, 3 per particle */
    double* noise;                   /* 3 per particle */
    int noise_drawn;
    long long noise_step;
    vec3 wall_momentum;
    /* sequential generator (oracle/shim/sfmt/SFMT.h) and Box-Muller spare */
    uint64_t rng_state;
    int has_stored;
    double stored;
};

/* ------------------------------------------------------------------------------------------------ */
/* Random numbers                                                                                    */
/* ------------------------------------------------------------------------------------------------ */

/* The stream of the shim's SFMT stand-in: splitmix64, (z >> 11) * 2^-53 in [0, 1). */
static double seq_uniform(OracleKernel* k) {
    k->rng_state += 0x9E3779B97F4A7C15ULL;
    uint64_t z = k->rng_state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double) (z >> 11) * (1.0/9007199254740992.0);
}

/* Box-Muller with the spare kept for the next call (ReferenceLBMKernels.cpp:1052-1064). */
static double seq_gaussian(OracleKernel* k) {
    if (k->has_stored) {
        k->has_stored = 0;
        return k->stored;
    }
    const double twoPi = 6.283185307179586476925287;
    double r = sqrt(-2.0*log(1.0 - seq_uniform(k)));
    double angle = twoPi*seq_uniform(k);
    k->stored = r*sin(angle);
    k->has_stored = 1;
    return r*cos(angle);
}

/* Philox4x32 (Salmon, Moraes, Dror, Shaw, SC'11) with `rounds` rounds of two 32x32->64 multiplications with the
   published multipliers and Weyl key increments; 10 rounds is the published Philox4x32-10 (its known answers pin this
   function), 7 the round count of the normal numbers below. */
void oracle_philox4x32(const uint32_t counter[4], const uint32_t key[2], int rounds, uint32_t out[4]) {
    uint32_t c0 = counter[0], c1 = counter[1], c2 = counter[2], c3 = counter[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < rounds; round++) {
        uint64_t p0 = (uint64_t) 0xD2511F53u*c0;
        uint64_t p1 = (uint64_t) 0xCD9E8D57u*c2;
        uint32_t hi0 = (uint32_t) (p0 >> 32), lo0 = (uint32_t) p0;
        uint32_t hi1 = (uint32_t) (p1 >> 32), lo1 = (uint32_t) p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void oracle_philox4x32_10(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]) {
    oracle_philox4x32(counter, key, 10, out);
}

#define ORACLE_PHILOX_ROUNDS 7

/* Word k of the draw of (purpose, index, step): lane k%4 of Philox4x32-7 of the counter (index, step low, step high,
   purpose*256 + k/4) under the key (seed, 0x4C424D32). */
static uint32_t philox_word(uint32_t seed, int purpose, long long index, long long step, int k) {
    uint32_t counter[4] = {(uint32_t) index, (uint32_t) step, (uint32_t) ((unsigned long long) step >> 32),
                           (uint32_t) (purpose*256 + k/4)};
    uint32_t key[2] = {seed, 0x4C424D32u};
    uint32_t x[4];
    oracle_philox4x32(counter, key, ORACLE_PHILOX_ROUNDS, x);
    return x[k%4];
}

/* Normal number m of (purpose, index, step).  Box-Muller pairs i = m/2, two pairs per three words: the radius word
   a = 3(m/4) + i%2 gives u = (w_a + 1/2) 2^-32 and r = sqrt(-2 ln u); the 16-bit half h of word 3(m/4) + 2 (low half
   for even i, high half for odd i) gives the angle t = 2 pi ((h + 1/2) 2^-16 - 1/2); normal m is r cos t for even m,
   r sin t for odd m. */
double oracle_philox_normal(uint32_t seed, int purpose, long long index, long long step, int m) {
    int pair = m/2, group = m/4;
    uint32_t a = philox_word(seed, purpose, index, step, 3*group + pair%2);
    uint32_t angles = philox_word(seed, purpose, index, step, 3*group + 2);
    uint32_t h = (pair%2) ? (angles >> 16) : (angles & 0xFFFFu);
    double u = ((double) a + 0.5)*(1.0/4294967296.0);
    double v = ((double) h + 0.5)*(1.0/65536.0);
    double r = sqrt(-2.0*log(u));
    double angle = 6.283185307179586476925287*(v - 0.5);
    return (m%2 == 0 ? r*cos(angle) : r*sin(angle));
}

/* ------------------------------------------------------------------------------------------------ */
/* D3Q19 algebra (D3Q19.h)                                                                           */
/* ------------------------------------------------------------------------------------------------ */

/* D3Q19::equilibriumDeviation (D3Q19.h:55-62). */
static void eq_deviation(double drho, double ux, double uy, double uz, double dfeq[Q]) {
    double rho = 1.0 + drho;
    double uu = ux*ux + uy*uy + uz*uz;
    for (int q = 0; q < Q; q++) {
        double cu = CX[q]*ux + CY[q]*uy + CZ[q]*uz;
        dfeq[q] = W[q]*(drho + rho*(3.0*cu + 4.5*cu*cu - 1.5*uu));
    }
}

/* D3Q19::hermite2 (D3Q19.h:67-74). */
static void hermite2(int q, double h[6]) {
    h[0] = CX[q]*CX[q] - 1.0/3.0;
    h[1] = CY[q]*CY[q] - 1.0/3.0;
    h[2] = CZ[q]*CZ[q] - 1.0/3.0;
    h[3] = CX[q]*CY[q];
    h[4] = CX[q]*CZ[q];
    h[5] = CY[q]*CZ[q];
}

/* D3Q19::nonEquilibriumMomentFromDeviation (D3Q19.h:98-110). */
static void pi_neq_from_deviation(const double df[Q], double drho, double jx, double jy, double jz, double pi[6]) {
    double rho = 1.0 + drho;
    double dfeq[Q], h[6];
    eq_deviation(drho, jx/rho, jy/rho, jz/rho, dfeq);
    for (int k = 0; k < 6; k++)
        pi[k] = 0.0;
    for (int q = 0; q < Q; q++) {
        hermite2(q, h);
        double fneq = df[q]-dfeq[q];
        for (int k = 0; k < 6; k++)
            pi[k] += h[k]*fneq;
    }
}

/* D3Q19::regularizedNonEquilibrium (D3Q19.h:116-121). */
static void regularized_fneq(const double pi[6], double fneq[Q]) {
    double h[6];
    for (int q = 0; q < Q; q++) {
        hermite2(q, h);
        fneq[q] = 4.5*W[q]*(h[0]*pi[0] + h[1]*pi[1] + h[2]*pi[2] + 2.0*(h[3]*pi[3] + h[4]*pi[4] + h[5]*pi[5]));
    }
}

/* D3Q19::guoForcing (D3Q19.h:127-134). */
static void guo_forcing(double ux, double uy, double uz, double fx, double fy, double fz, double s[Q]) {
    double uf = ux*fx + uy*fy + uz*fz;
    for (int q = 0; q < Q; q++) {
        double cu = CX[q]*ux + CY[q]*uy + CZ[q]*uz;
        double cf = CX[q]*fx + CY[q]*fy + CZ[q]*fz;
        s[q] = W[q]*(3.0*(cf - uf) + 9.0*cu*cf);
    }
}

/* D3Q19::mode, the Lulli et al. orthogonal basis e_k(c_q) (D3Q19.h:145-169). */
static double mode(int k, int q) {
    double x = CX[q], y = CY[q], z = CZ[q];
    double x2 = x*x, y2 = y*y, z2 = z*z;
    switch (k) {
    case 0: return 1.0;
    case 1: return x;
    case 2: return y;
    case 3: return z;
    case 4: return x2 - 1.0/3.0;
    case 5: return y2 - 1.0/3.0;
    case 6: return z2 - 1.0/3.0;
    case 7: return x*y;
    case 8: return x*z;
    case 9: return y*z;
    case 10: return y*(x2 - 1.0/3.0);
    case 11: return z*(x2 - 1.0/3.0);
    case 12: return x*(y2 - 1.0/3.0);
    case 13: return 0.5*x*(y2 + 2.0*z2 - 1.0);
    case 14: return 0.5*y*(x2 + 2.0*z2 - 1.0);
    case 15: return 0.5*z*(x2 + 2.0*y2 - 1.0);
    case 16: return x2*y2 - x2/3.0 - y2/3.0 + z2/6.0 + 1.0/18.0;
    case 17: return (2.0/7.0)*x2*y2 + x2*z2 - (3.0/7.0)*x2 + y2/14.0 - (2.0/7.0)*z2 + 1.0/14.0;
    default: return 0.4*x2*y2 + 0.4*x2*z2 + y2*z2 - 0.1*x2 - 0.4*y2 - 0.4*z2 + 0.1;
    }
}

/* D3Q19::fluctuation (D3Q19.h:179-190): xi_q = w_q sum_{k=4..18} e_k(c_q)/sqrt(b_k) phi_k r_{k-4}. */
void oracle_fluctuation(const double r[15], double stress, double ghost, double xi[Q]) {
    for (int q = 0; q < Q; q++) {
        double sum = 0;
        for (int k = 4; k < Q; k++)
            sum += mode(k, q)/sqrt(MODE_NORM[k])*(k < 10 ? stress : ghost)*r[k-4];
        xi[q] = W[q]*sum;
    }
}

/* D3Q19::equilibriumFluctuation (D3Q19.h:194-199). */
static void equilibrium_fluctuation(const double r[Q], double conserved, double stress, double ghost, double xi[Q]) {
    oracle_fluctuation(r, stress, ghost, xi);
    for (int q = 0; q < Q; q++)
        xi[q] += W[q]*conserved*(r[15] + sqrt(3.0)*(CX[q]*r[16] + CY[q]*r[17] + CZ[q]*r[18]));
}

/* D3Q19::boundaryStressWeight (D3Q19.h:206-208). */
static double boundary_stress_weight(double omega) {
    return (1.0-omega)*(1.0-omega)/(omega*(2.0-omega));
}

/* ------------------------------------------------------------------------------------------------ */
/* Stencils (LBMStencils.h)                                                                          */
/* ------------------------------------------------------------------------------------------------ */

static int stencil_width(int stencil) {
    switch (stencil) {
    case LBM_STENCIL_TRILINEAR: return 2;
    case LBM_STENCIL_THREEPOINT: return 3;
    case LBM_STENCIL_KEYS: return 4;
    default: return 1;
    }
}

/* LBMStencils::kernel (LBMStencils.h:42-62). */
double oracle_stencil_kernel(int stencil, double r) {
    double s = fabs(r);
    switch (stencil) {
    case LBM_STENCIL_TRILINEAR:
        return (s < 1.0 ? 1.0-s : 0.0);
    case LBM_STENCIL_THREEPOINT:
        if (s <= 0.5)
            return (1.0 + sqrt(1.0-3.0*s*s))/3.0;
        if (s < 1.5) {
            double t = 1.0-3.0*(1.0-s)*(1.0-s);
            return (5.0 - 3.0*s - sqrt(t > 0.0 ? t : 0.0))/6.0;
        }
        return 0.0;
    case LBM_STENCIL_KEYS:
        if (s <= 1.0)
            return 1.0 - 2.5*s*s + 1.5*s*s*s;
        if (s < 2.0)
            return 2.0 - 4.0*s + 2.5*s*s - 0.5*s*s*s;
        return 0.0;
    default:
        return (r >= -0.5 && r < 0.5 ? 1.0 : 0.0);
    }
}

/* LBMStencils::axisWeights (LBMStencils.h:73-95): nodes and weights along one axis, clamped at open faces,
   repeated nodes merged into their first slot. */
void oracle_axis_weights(int stencil, double s, int n, int open, int* index, double* weight) {
    int w = stencil_width(stencil);
    int first;
    if (stencil == LBM_STENCIL_THREEPOINT)
        first = (int) floor(s + 0.5) - 1;
    else if (stencil == LBM_STENCIL_KEYS)
        first = (int) floor(s) - 1;
    else if (stencil == LBM_STENCIL_TRILINEAR)
        first = (int) floor(s);
    else
        first = (int) floor(s + 0.5);
    for (int i = 0; i < w; i++) {
        weight[i] = oracle_stencil_kernel(stencil, s - (first + i));
        int idx = first + i;
        if (open)
            index[i] = (idx < 0 ? 0 : (idx > n-1 ? n-1 : idx));
        else
            index[i] = ((idx%n) + n)%n;
    }
    for (int i = 1; i < w; i++)
        for (int j = 0; j < i; j++)
            if (index[j] == index[i]) {
                weight[j] += weight[i];
                weight[i] = 0.0;
                break;
            }
}

/* ------------------------------------------------------------------------------------------------ */
/* Setup                                                                                             */
/* ------------------------------------------------------------------------------------------------ */

static int is_open_axis(const LbmLatticeParameters* L, int axis) {
    return L->face_boundary[2*axis] != LBM_BOUNDARY_PERIODIC;
}

static int has_open_faces(const LbmLatticeParameters* L) {
    return is_open_axis(L, 0) || is_open_axis(L, 1) || is_open_axis(L, 2);
}

static int has_equilibrium_noise(int kind) {
    return kind == KIND_WALL || kind == KIND_DENSITY_VELOCITY;   /* LBMBoundaries.h:34-36 */
}

/* LBMBoundaries::find (LBMBoundaries.h:46-109).  fluid is NULL without solid nodes. */
static int find_boundaries(const LbmLatticeParameters* L, int nsolid, const char* fluid,
                           int* nodes, int* unknown, int* solid, int* kind, int* face) {
    int regularized = (nsolid > 0 && L->wall_scheme == LBM_WALL_REGULARIZED);
    if (!regularized && !has_open_faces(L))
        return 0;
    int size[3] = {L->nx, L->ny, L->nz};
    int nx = size[0], ny = size[1];
    long n = (long) L->nx*L->ny*L->nz;
    int count = 0;
    for (long node = 0; node < n; node++) {
        if (fluid != NULL && !fluid[node])
            continue;
        int index[3] = {(int) (node%nx), (int) ((node/nx)%ny), (int) (node/((long) nx*ny))};
        int solidBits = 0, outsideBits = 0;
        for (int q = 1; q < Q; q++) {
            int c[3] = {CX[q], CY[q], CZ[q]}, source[3];
            int beyond = 0;
            for (int a = 0; a < 3; a++) {
                source[a] = index[a] - c[a];
                if (source[a] < 0 || source[a] >= size[a]) {
                    beyond = beyond || is_open_axis(L, a);
                    source[a] = (source[a] + size[a])%size[a];
                }
            }
            if (beyond)
                outsideBits |= 1<<q;
            else if (regularized && !fluid[source[0] + (long) nx*(source[1] + (long) ny*source[2])])
                solidBits |= 1<<q;
        }
        if (solidBits == 0 && outsideBits == 0)
            continue;
        int nodeKind = KIND_WALL, nodeFace = -1;
        if (solidBits == 0) {
            int velocityFace = -1, densityFace = -1, numDensityFaces = 0;
            for (int f = 0; f < 6; f++) {
                int a = f/2;
                if (!is_open_axis(L, a) || index[a] != (f%2 == 0 ? 0 : size[a]-1))
                    continue;
                int type = L->face_boundary[f];
                if ((type == LBM_BOUNDARY_VELOCITY || type == LBM_BOUNDARY_DENSITY_VELOCITY) && velocityFace < 0)
                    velocityFace = f;
                if (type == LBM_BOUNDARY_DENSITY && numDensityFaces++ == 0)
                    densityFace = f;
            }
            if (velocityFace >= 0) {
                int both = (L->face_boundary[velocityFace] == LBM_BOUNDARY_DENSITY_VELOCITY);
                nodeKind = (both ? KIND_DENSITY_VELOCITY : KIND_VELOCITY);
                nodeFace = velocityFace;
            }
            else {
                nodeKind = (numDensityFaces == 1 ? KIND_DENSITY : KIND_DENSITY_AT_REST);
                nodeFace = densityFace;
            }
        }
        if (nodes) {
            nodes[count] = (int) node;
            unknown[count] = solidBits | outsideBits;
            solid[count] = solidBits;
            kind[count] = nodeKind;
            face[count] = nodeFace;
        }
        count++;
    }
    return count;
}

static char* make_fluid_mask(const LbmLatticeParameters* L, int nsolid, const int* solid) {
    if (nsolid == 0)
        return NULL;
    long n = (long) L->nx*L->ny*L->nz;
    char* fluid = (char*) malloc(n);
    memset(fluid, 1, n);
    for (int i = 0; i < nsolid; i++)
        fluid[solid[i]] = 0;
    return fluid;
}

int oracle_find_boundaries(const LbmLatticeParameters* L, int nsolid, const int* solid,
                           int* nodes, int* unknown, int* solid_bits, int* kind, int* face) {
    char* fluid = make_fluid_mask(L, nsolid, solid);
    int count = find_boundaries(L, nsolid, fluid, nodes, unknown, solid_bits, kind, face);
    free(fluid);
    return count;
}

/* LBMBoundaries::findWallLinks (LBMBoundaries.h:118-148). */
static int find_wall_links(const LbmLatticeParameters* L, int nsolid, const char* fluid, int* nodes, int* links) {
    if (nsolid == 0 || L->wall_scheme != LBM_WALL_BOUNCEBACK)
        return 0;
    int size[3] = {L->nx, L->ny, L->nz};
    int nx = size[0], ny = size[1];
    long n = (long) L->nx*L->ny*L->nz;
    int count = 0;
    for (long node = 0; node < n; node++) {
        if (!fluid[node])
            continue;
        int index[3] = {(int) (node%nx), (int) ((node/nx)%ny), (int) (node/((long) nx*ny))};
        int bits = 0;
        for (int q = 1; q < Q; q++) {
            int c[3] = {CX[q], CY[q], CZ[q]}, target[3];
            int crosses = 0;
            for (int a = 0; a < 3; a++) {
                target[a] = index[a] + c[a];
                crosses = crosses || (is_open_axis(L, a) && (target[a] < 0 || target[a] >= size[a]));
                target[a] = (target[a] + size[a])%size[a];
            }
            if (!crosses && !fluid[target[0] + (long) nx*(target[1] + (long) ny*target[2])])
                bits |= 1<<q;
        }
        if (bits != 0) {
            if (nodes) {
                nodes[count] = (int) node;
                links[count] = bits;
            }
            count++;
        }
    }
    return count;
}

static int cmp_int(const void* a, const void* b) {
    int x = *(const int*) a, y = *(const int*) b;
    return (x > y) - (x < y);
}

void oracle_destroy(OracleKernel* k) {
    if (!k)
        return;
    free(k->pop); free(k->rho); free(k->drho); free(k->mom); free(k->pi); free(k->fd); free(k->reaction);
    free(k->fluid); free(k->solid); free(k->wall_nodes); free(k->wall_links);
    free(k->bnd_node); free(k->bnd_unknown); free(k->bnd_solid); free(k->bnd_kind); free(k->bnd_face);
    free(k->bnd_of_node); free(k->bnd_stress);
    free(k->pmass); free(k->pforce); free(k->noise);
    free(k);
}

/* ReferenceCalcLBMForceKernel::initialize (ReferenceLBMKernels.cpp:43-306), one domain. */
LbmStatus oracle_create(const LbmLatticeParameters* L, int random_mode, int np, const double* masses,
                        int nsolid, const int* solid, OracleKernel** out) {
    if (L == NULL || out == NULL || L->nx <= 0 || L->ny <= 0 || L->nz <= 0 || np < 0 || nsolid < 0)
        return set_error(LBM_ERR_INVALID_ARGUMENT, "oracle_create: invalid arguments");
    OracleKernel* k = (OracleKernel*) calloc(1, sizeof(OracleKernel));
    k->L = *L;
    k->nx = L->nx; k->ny = L->ny; k->nz = L->nz;
    k->n = (long) L->nx*L->ny*L->nz;
    k->random_mode = random_mode;
    long n = k->n;
    k->pop = (double*) malloc(sizeof(double)*Q*n);
    double dfeq[Q];
    eq_deviation(0.0, L->initial_velocity[0], L->initial_velocity[1], L->initial_velocity[2], dfeq);
    for (int q = 0; q < Q; q++)
        for (long node = 0; node < n; node++)
            k->pop[q*n+node] = dfeq[q];
    k->rho = (double*) calloc(n, sizeof(double));
    k->drho = (double*) calloc(n, sizeof(double));
    k->mom = (double*) calloc(3*n, sizeof(double));
    k->pi = (double*) calloc(6*n, sizeof(double));
    k->fd = (double*) calloc(3*n, sizeof(double));
    k->reaction = (double*) calloc(3*n, sizeof(double));

    /* Solid nodes: sorted, start at the deviation -w_q (:69-79). */
    k->nsolid = nsolid;
    k->solid = (int*) malloc(sizeof(int)*(nsolid > 0 ? nsolid : 1));
    if (nsolid > 0)
        memcpy(k->solid, solid, sizeof(int)*nsolid);
    qsort(k->solid, nsolid, sizeof(int), cmp_int);
    for (int i = 0; i < nsolid; i++)
        if (k->solid[i] < 0 || k->solid[i] >= n || (i > 0 && k->solid[i] == k->solid[i-1])) {
            oracle_destroy(k);
            return set_error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: invalid or repeated solid node index");
        }
    k->fluid = make_fluid_mask(L, nsolid, k->solid);
    for (int i = 0; i < nsolid; i++)
        for (int q = 0; q < Q; q++)
            k->pop[q*n + k->solid[i]] = -W[q];
    k->nwall = find_wall_links(L, nsolid, k->fluid, NULL, NULL);
    k->wall_nodes = (int*) malloc(sizeof(int)*(k->nwall + 1));
    k->wall_links = (int*) malloc(sizeof(int)*(k->nwall + 1));
    find_wall_links(L, nsolid, k->fluid, k->wall_nodes, k->wall_links);

    /* Boundary nodes (:82-94). */
    k->nbnd = find_boundaries(L, nsolid, k->fluid, NULL, NULL, NULL, NULL, NULL);
    int nb = k->nbnd + 1;
    k->bnd_node = (int*) malloc(sizeof(int)*nb);
    k->bnd_unknown = (int*) malloc(sizeof(int)*nb);
    k->bnd_solid = (int*) malloc(sizeof(int)*nb);
    k->bnd_kind = (int*) malloc(sizeof(int)*nb);
    k->bnd_face = (int*) malloc(sizeof(int)*nb);
    find_boundaries(L, nsolid, k->fluid, k->bnd_node, k->bnd_unknown, k->bnd_solid, k->bnd_kind, k->bnd_face);

    /* Stress part of the collision noise of the boundary nodes with equilibrium noise (:264-277). */
    int equilibriumNoise = 0;
    for (int b = 0; b < k->nbnd; b++)
        equilibriumNoise = equilibriumNoise || has_equilibrium_noise(k->bnd_kind[b]);
    if (L->fluid_fluctuations && equilibriumNoise) {
        k->bnd_of_node = (int*) malloc(sizeof(int)*n);
        for (long node = 0; node < n; node++)
            k->bnd_of_node[node] = -1;
        for (int b = 0; b < k->nbnd; b++)
            k->bnd_of_node[k->bnd_node[b]] = b;
        k->bnd_stress = (double*) calloc((size_t) Q*nb, sizeof(double));
    }

    /* Particles (:279-303). */
    double cellMass = L->density*L->dx*L->dx*L->dx;
    k->np = np;
    k->pmass = (double*) malloc(sizeof(double)*(np + 1));
    for (int i = 0; i < np; i++) {
        if (!(masses[i] > 0)) {
            oracle_destroy(k);
            return set_error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: coupled particles must have a positive mass");
        }
        k->pmass[i] = masses[i]/cellMass;
    }
    k->pforce = (double*) calloc(3*(size_t) (np + 1), sizeof(double));
    k->noise = (double*) calloc(3*(size_t) (np + 1), sizeof(double));
    k->noise_drawn = 0;
    k->noise_step = -1;
    int seed = L->random_number_seed;
    if (seed == 0)
        seed = 20260101;                      /* the shim's osrngseed() */
    k->seed = (uint32_t) seed;
    k->rng_state = (uint64_t) (uint32_t) seed;
    k->has_stored = 0;
    *out = k;
    return LBM_OK;
}

/* ------------------------------------------------------------------------------------------------ */
/* One lattice step                                                                                  */
/* ------------------------------------------------------------------------------------------------ */

/* ReferenceCalcLBMForceKernel::computeMoments (ReferenceLBMKernels.cpp:430-469). */
static void compute_moments(OracleKernel* k) {
    long n = k->n;
    const double* g = k->L.body_acceleration;
    double f[Q];
    for (long node = 0; node < n; node++) {
        if (k->fluid && !k->fluid[node]) {
            k->rho[node] = k->drho[node] = 0;
            for (int a = 0; a < 3; a++)
                k->mom[3*node+a] = k->fd[3*node+a] = 0;
            for (int a = 0; a < 6; a++)
                k->pi[6*node+a] = 0;
            continue;
        }
        double dr = 0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < Q; q++) {
            f[q] = k->pop[q*n+node];
            dr += f[q];
            jx += CX[q]*f[q];
            jy += CY[q]*f[q];
            jz += CZ[q]*f[q];
        }
        double r = 1.0 + dr;
        k->rho[node] = r;
        k->drho[node] = dr;
        k->mom[3*node] = jx;
        k->mom[3*node+1] = jy;
        k->mom[3*node+2] = jz;
        pi_neq_from_deviation(f, dr, jx, jy, jz, &k->pi[6*node]);
        k->fd[3*node] = r*g[0];
        k->fd[3*node+1] = r*g[1];
        k->fd[3*node+2] = r*g[2];
    }
}

/* ReferenceCalcLBMForceKernel::removeFluidMomentum (ReferenceLBMKernels.cpp:471-501). */
static void remove_fluid_momentum(OracleKernel* k) {
    long n = k->n;
    double mass = 0, px = 0, py = 0, pz = 0;
    for (long node = 0; node < n; node++) {
        mass += k->rho[node];
        px += k->mom[3*node];
        py += k->mom[3*node+1];
        pz += k->mom[3*node+2];
    }
    double ux = px/mass, uy = py/mass, uz = pz/mass;
    for (long node = 0; node < n; node++) {
        k->mom[3*node] -= k->rho[node]*ux;
        k->mom[3*node+1] -= k->rho[node]*uy;
        k->mom[3*node+2] -= k->rho[node]*uz;
    }
}

/* Wrapped lattice coordinate of a position along one axis (ReferenceLBMKernels.cpp:978-979). */
static double lattice_coordinate(const OracleKernel* k, double x, int axis) {
    int size[3] = {k->nx, k->ny, k->nz};
    double s = x/k->L.dx;
    s -= floor(s/size[axis])*size[axis];
    return s;
}

/* nearestNode (ReferenceLBMKernels.cpp:973-983). */
static long nearest_node(const OracleKernel* k, const double* x) {
    int size[3] = {k->nx, k->ny, k->nz};
    int index[3];
    for (int a = 0; a < 3; a++) {
        double s = lattice_coordinate(k, x[a], a);
        index[a] = ((int) floor(s + 0.5))%size[a];
    }
    return index[0] + (long) k->nx*(index[1] + (long) k->ny*index[2]);
}

/* stencilOwnerNode (ReferenceLBMKernels.cpp:985-996) decides which MPI rank couples a particle; with one domain
   every particle is coupled, so the restatement needs no owner. */

/* stencilNodes (ReferenceLBMKernels.cpp:998-1018): x fastest, then y, then z.  Returns the count. */
static int stencil_nodes(const OracleKernel* k, const double* x, long* nodes, double* weights) {
    int size[3] = {k->nx, k->ny, k->nz};
    int index[3][4];
    double weight[3][4];
    int stencil = k->L.interpolation_stencil;
    for (int a = 0; a < 3; a++)
        oracle_axis_weights(stencil, lattice_coordinate(k, x[a], a), size[a], is_open_axis(&k->L, a),
                            index[a], weight[a]);
    int w = stencil_width(stencil), count = 0;
    for (int c = 0; c < w; c++)
        for (int b = 0; b < w; b++)
            for (int a = 0; a < w; a++) {
                nodes[count] = index[0][a] + (long) k->nx*(index[1][b] + (long) k->ny*index[2][c]);
                weights[count] = weight[0][a]*weight[1][b]*weight[2][c];
                count++;
            }
    return count;
}

/* wallNormal (ReferenceLBMKernels.cpp:1020-1050). */
static void wall_normal(const OracleKernel* k, const double* x, double* gradient) {
    int size[3] = {k->nx, k->ny, k->nz};
    int index[3][2];
    double weight[3][2];
    for (int a = 0; a < 3; a++) {
        double s = lattice_coordinate(k, x[a], a);
        double lower = floor(s);
        index[a][0] = ((int) lower)%size[a];
        index[a][1] = (index[a][0]+1)%size[a];
        weight[a][1] = s-lower;
        weight[a][0] = 1.0-weight[a][1];
    }
    double solid[2][2][2];
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int c = 0; c < 2; c++)
                solid[a][b][c] = (k->fluid[index[0][a] + (long) k->nx*(index[1][b] + (long) k->ny*index[2][c])] ? 0.0 : 1.0);
    gradient[0] = gradient[1] = gradient[2] = 0;
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
            gradient[0] += weight[1][a]*weight[2][b]*(solid[1][a][b]-solid[0][a][b]);
            gradient[1] += weight[0][a]*weight[2][b]*(solid[a][1][b]-solid[a][0][b]);
            gradient[2] += weight[0][a]*weight[1][b]*(solid[a][b][1]-solid[a][b][0]);
        }
}

/* drawNoise (ReferenceLBMKernels.cpp:945-957); in Philox mode the numbers of step s are a function of s. */
static void draw_noise(OracleKernel* k, long long step) {
    if (k->random_mode == ORACLE_RANDOM_PHILOX) {
        for (int i = 0; i < k->np; i++)
            for (int a = 0; a < 3; a++)
                k->noise[3*i+a] = oracle_philox_normal(k->seed, PURPOSE_PARTICLE, i, step, a);
        return;
    }
    if (k->noise_drawn)
        return;
    for (int i = 0; i < k->np; i++) {
        double xi0 = seq_gaussian(k);
        double xi1 = seq_gaussian(k);
        double xi2 = seq_gaussian(k);
        k->noise[3*i] = xi0;
        k->noise[3*i+1] = xi1;
        k->noise[3*i+2] = xi2;
    }
    k->noise_drawn = 1;
}

/* applyReaction (ReferenceLBMKernels.cpp:959-971). */
static void apply_reaction(OracleKernel* k) {
    long n = k->n;
    k->noise_drawn = 0;
    for (long node = 0; node < n; node++)
        for (int a = 0; a < 3; a++)
            k->fd[3*node+a] += k->reaction[3*node+a];
    double cellMass = k->L.density*k->L.dx*k->L.dx*k->L.dx;
    double momentumScale = cellMass*k->L.dx/k->L.dt;
    for (int i = 0; i < k->nsolid; i++) {
        long node = k->solid[i];
        for (int a = 0; a < 3; a++)
            k->wall_momentum.v[a] += k->reaction[3*node+a]*momentumScale;
    }
}

typedef struct {
    double gamma, kT, velocityScale, forceScale;
    int randomForce;
} CouplingScales;

static CouplingScales coupling_scales(const OracleKernel* k) {
    CouplingScales c;
    const LbmLatticeParameters* L = &k->L;
    double cellMass = L->density*L->dx*L->dx*L->dx;
    c.gamma = L->friction*L->dt;
    c.kT = L->kT*L->dt*L->dt/(cellMass*L->dx*L->dx);
    c.velocityScale = L->dx/L->dt;
    c.forceScale = cellMass*L->dx/(L->dt*L->dt);
    c.randomForce = (c.kT > 0 && c.gamma > 0);
    return c;
}

/* coupleParticles, nearest node, explicit (ReferenceLBMKernels.cpp:503-553). */
static void couple_nearest(OracleKernel* k, const LbmParticleArrays* p, int isStep, long long step) {
    CouplingScales c = coupling_scales(k);
    if (c.randomForce)
        draw_noise(k, step);
    if (isStep)
        memset(k->reaction, 0, sizeof(double)*3*k->n);
    for (int i = 0; i < k->np; i++) {
        long node = nearest_node(k, &p->positions[3*i]);
        double u[3] = {0, 0, 0};
        if (k->rho[node] > 0)
            for (int a = 0; a < 3; a++)
                u[a] = k->mom[3*node+a]*(1.0/k->rho[node]);
        double m = k->pmass[i];
        for (int a = 0; a < 3; a++) {
            double v = p->velocities[3*i+a]*(1.0/c.velocityScale);
            double f = (v-u[a])*(-c.gamma*m);
            if (c.randomForce)
                f += k->noise[3*i+a]*sqrt(2.0*c.gamma*m*c.kT);
            k->pforce[3*i+a] = f*c.forceScale;
            if (isStep)
                k->reaction[3*node+a] -= f;
        }
    }
    if (isStep)
        apply_reaction(k);
}

typedef struct { long long key; } SortKey;

static int cmp_ll(const void* a, const void* b) {
    long long x = *(const long long*) a, y = *(const long long*) b;
    return (x > y) - (x < y);
}

/* coupleParticlesCentered, nearest node (ReferenceLBMKernels.cpp:555-641). */
static void couple_centered(OracleKernel* k, const LbmParticleArrays* p, int isStep, long long step) {
    CouplingScales c = coupling_scales(k);
    int np = k->np;
    double h = 0.5, a = c.gamma*h;
    if (c.randomForce)
        draw_noise(k, step);
    long long* keys = (long long*) malloc(sizeof(long long)*np);
    double* known = (double*) malloc(sizeof(double)*3*np);
    double* random = (double*) calloc(3*(size_t) np, sizeof(double));
    for (int i = 0; i < np; i++) {
        double m = k->pmass[i];
        for (int d = 0; d < 3; d++) {
            known[3*i+d] = p->velocities[3*i+d]*(1.0/c.velocityScale) + p->forces[3*i+d]*(h/(m*c.forceScale));
            if (c.randomForce)
                random[3*i+d] = k->noise[3*i+d]*sqrt(2.0*c.gamma*m*c.kT);
        }
        keys[i] = nearest_node(k, &p->positions[3*i])*(long long) np + i;
    }
    qsort(keys, np, sizeof(long long), cmp_ll);
    if (isStep)
        memset(k->reaction, 0, sizeof(double)*3*k->n);
    for (int first = 0; first < np; ) {
        long node = (long) (keys[first]/np);
        int end = first;
        double mass = 0, pm[3] = {0, 0, 0}, rs[3] = {0, 0, 0};
        for (; end < np && keys[end]/np == node; end++) {
            int i = (int) (keys[end]%np);
            mass += k->pmass[i];
            for (int d = 0; d < 3; d++) {
                pm[d] += known[3*i+d]*k->pmass[i];
                rs[d] += random[3*i+d];
            }
        }
        double u[3] = {0, 0, 0}, sum[3];
        if (k->rho[node] > 0) {
            const double* j = &k->mom[3*node];
            const double* F = &k->fd[3*node];
            double kn[3];
            for (int d = 0; d < 3; d++)
                kn[d] = (j[d] + h*F[d])*(1.0/k->rho[node]);
            for (int d = 0; d < 3; d++)
                sum[d] = ((pm[d] - kn[d]*mass)*(-c.gamma) + rs[d])*(1.0/(1.0 + a + a*mass/k->rho[node]));
            for (int d = 0; d < 3; d++)
                u[d] = kn[d] - sum[d]*(h/k->rho[node]);
        }
        else
            for (int d = 0; d < 3; d++)
                sum[d] = ((pm[d] - u[d]*mass)*(-c.gamma) + rs[d])*(1.0/(1.0 + a));
        for (int e = first; e < end; e++) {
            int i = (int) (keys[e]%np);
            for (int d = 0; d < 3; d++) {
                double f = ((known[3*i+d] - u[d])*(-c.gamma*k->pmass[i]) + random[3*i+d])*(1.0/(1.0 + a));
                k->pforce[3*i+d] = f*c.forceScale;
            }
        }
        if (isStep)
            for (int d = 0; d < 3; d++)
                k->reaction[3*node+d] = -sum[d];
        first = end;
    }
    free(keys);
    free(known);
    free(random);
    if (isStep)
        apply_reaction(k);
}

/* coupleParticlesStencil, explicit (ReferenceLBMKernels.cpp:643-697). */
static void couple_stencil(OracleKernel* k, const LbmParticleArrays* p, int isStep, long long step) {
    CouplingScales c = coupling_scales(k);
    int np = k->np;
    if (c.randomForce)
        draw_noise(k, step);
    int S = 64;
    long* nodes = (long*) malloc(sizeof(long)*S*(np + 1));
    double* weights = (double*) malloc(sizeof(double)*S*(np + 1));
    int* count = (int*) malloc(sizeof(int)*(np + 1));
    double* lf = (double*) calloc(3*(size_t) (np + 1), sizeof(double));
    for (int i = 0; i < np; i++) {
        count[i] = stencil_nodes(k, &p->positions[3*i], &nodes[S*i], &weights[S*i]);
        double u[3] = {0, 0, 0};
        for (int s = 0; s < count[i]; s++) {
            long node = nodes[S*i+s];
            if (k->rho[node] > 0)
                for (int d = 0; d < 3; d++)
                    u[d] += k->mom[3*node+d]*(weights[S*i+s]/k->rho[node]);
        }
        double m = k->pmass[i];
        for (int d = 0; d < 3; d++) {
            double v = p->velocities[3*i+d]*(1.0/c.velocityScale);
            double f = (v-u[d])*(-c.gamma*m);
            if (c.randomForce)
                f += k->noise[3*i+d]*sqrt(2.0*c.gamma*m*c.kT);
            lf[3*i+d] = f;
        }
    }
    if (isStep)
        memset(k->reaction, 0, sizeof(double)*3*k->n);
    for (int i = 0; i < np; i++) {
        for (int d = 0; d < 3; d++)
            k->pforce[3*i+d] = lf[3*i+d]*c.forceScale;
        if (isStep)
            for (int s = 0; s < count[i]; s++)
                for (int d = 0; d < 3; d++)
                    k->reaction[3*nodes[S*i+s]+d] -= weights[S*i+s]*lf[3*i+d];
    }
    free(nodes); free(weights); free(count); free(lf);
    if (isStep)
        apply_reaction(k);
}

/* coupleParticlesCenteredStencil: Jacobi-preconditioned CG (ReferenceLBMKernels.cpp:726-901). */
static LbmStatus couple_centered_stencil(OracleKernel* k, const LbmParticleArrays* p, int isStep, long long step) {
    CouplingScales c = coupling_scales(k);
    int np = k->np;
    double h = 0.5, a = c.gamma*h;
    if (c.randomForce)
        draw_noise(k, step);
    int S = 64;
    long* nodes = (long*) malloc(sizeof(long)*S*(np + 1));
    double* weights = (double*) malloc(sizeof(double)*S*(np + 1));
    int* count = (int*) malloc(sizeof(int)*(np + 1));
    size_t v3 = 3*(size_t) (np + 1);
    double *rhs = calloc(v3, sizeof(double)), *diag = calloc(np + 1, sizeof(double));
    for (int i = 0; i < np; i++) {
        double m = k->pmass[i];
        count[i] = stencil_nodes(k, &p->positions[3*i], &nodes[S*i], &weights[S*i]);
        double known[3], u[3] = {0, 0, 0}, self = 0;
        for (int d = 0; d < 3; d++)
            known[d] = p->velocities[3*i+d]*(1.0/c.velocityScale) + p->forces[3*i+d]*(h/(m*c.forceScale));
        for (int s = 0; s < count[i]; s++) {
            long node = nodes[S*i+s];
            double wgt = weights[S*i+s];
            if (k->rho[node] > 0) {
                const double* j = &k->mom[3*node];
                const double* F = &k->fd[3*node];
                for (int d = 0; d < 3; d++)
                    u[d] += (j[d] + h*F[d])*(wgt/k->rho[node]);
                self += wgt*wgt/k->rho[node];
            }
        }
        for (int d = 0; d < 3; d++) {
            double b = (known[d]-u[d])*(-c.gamma*m);
            if (c.randomForce)
                b += k->noise[3*i+d]*sqrt(2.0*c.gamma*m*c.kT);
            rhs[3*i+d] = b*(1.0/m);
        }
        diag[i] = (1.0+a)/m + a*self;
    }
    double* spread = (double*) calloc(3*(size_t) k->n, sizeof(double));
    double *F = calloc(v3, sizeof(double)), *r = calloc(v3, sizeof(double)), *z = calloc(v3, sizeof(double));
    double *pv = calloc(v3, sizeof(double)), *Ap = calloc(v3, sizeof(double));
#define MULTIPLY(P, RESULT) do { \
        for (int i = 0; i < np; i++) \
            for (int s = 0; s < count[i]; s++) \
                for (int d = 0; d < 3; d++) \
                    spread[3*nodes[S*i+s]+d] += weights[S*i+s]*(P)[3*i+d]; \
        for (int i = 0; i < np; i++) { \
            double sm[3] = {0, 0, 0}; \
            for (int s = 0; s < count[i]; s++) { \
                long node = nodes[S*i+s]; \
                if (k->rho[node] > 0) \
                    for (int d = 0; d < 3; d++) \
                        sm[d] += spread[3*node+d]*(weights[S*i+s]/k->rho[node]); \
            } \
            for (int d = 0; d < 3; d++) \
                (RESULT)[3*i+d] = (P)[3*i+d]*((1.0+a)/k->pmass[i]) + sm[d]*a; \
        } \
        for (int i = 0; i < np; i++) \
            for (int s = 0; s < count[i]; s++) \
                for (int d = 0; d < 3; d++) \
                    spread[3*nodes[S*i+s]+d] = 0.0; \
    } while (0)
    double rz[3] = {0, 0, 0}, norm[3] = {0, 0, 0};
    for (int i = 0; i < np; i++)
        for (int d = 0; d < 3; d++)
            F[3*i+d] = rhs[3*i+d]*(1.0/diag[i]);
    MULTIPLY(F, Ap);
    for (int i = 0; i < np; i++)
        for (int d = 0; d < 3; d++) {
            r[3*i+d] = rhs[3*i+d]-Ap[3*i+d];
            z[3*i+d] = r[3*i+d]*(1.0/diag[i]);
            pv[3*i+d] = z[3*i+d];
            rz[d] += r[3*i+d]*z[3*i+d];
            norm[d] += rhs[3*i+d]*rhs[3*i+d];
        }
    const double tolerance = 1e-13;
    const int maxIterations = 1000;
    LbmStatus status = LBM_OK;
    for (int iteration = 0; ; iteration++) {
        double residual[3] = {0, 0, 0};
        for (int i = 0; i < np; i++)
            for (int d = 0; d < 3; d++)
                residual[d] += r[3*i+d]*r[3*i+d];
        int converged = 1;
        for (int d = 0; d < 3; d++)
            if (residual[d] > tolerance*tolerance*norm[d])
                converged = 0;
        if (converged)
            break;
        if (iteration == maxIterations) {
            status = set_error(LBM_ERR_CG_NOT_CONVERGED, "LBMForce: the centred drag with the interpolation stencil did "
                               "not converge in 1000 iterations of the conjugate gradients");
            break;
        }
        MULTIPLY(pv, Ap);
        double pAp[3] = {0, 0, 0}, rzNew[3] = {0, 0, 0}, alpha[3];
        for (int i = 0; i < np; i++)
            for (int d = 0; d < 3; d++)
                pAp[d] += pv[3*i+d]*Ap[3*i+d];
        for (int d = 0; d < 3; d++)
            alpha[d] = (pAp[d] > 0 ? rz[d]/pAp[d] : 0.0);
        for (int i = 0; i < np; i++) {
            for (int d = 0; d < 3; d++) {
                F[3*i+d] += alpha[d]*pv[3*i+d];
                r[3*i+d] -= alpha[d]*Ap[3*i+d];
            }
            for (int d = 0; d < 3; d++)
                z[3*i+d] = r[3*i+d]*(1.0/diag[i]);
            for (int d = 0; d < 3; d++)
                rzNew[d] += r[3*i+d]*z[3*i+d];
        }
        for (int i = 0; i < np; i++)
            for (int d = 0; d < 3; d++)
                pv[3*i+d] = z[3*i+d] + (rz[d] > 0 ? rzNew[d]/rz[d] : 0.0)*pv[3*i+d];
        for (int d = 0; d < 3; d++)
            rz[d] = rzNew[d];
    }
#undef MULTIPLY
    if (status == LBM_OK) {
        if (isStep)
            memset(k->reaction, 0, sizeof(double)*3*k->n);
        for (int i = 0; i < np; i++) {
            for (int d = 0; d < 3; d++)
                k->pforce[3*i+d] = F[3*i+d]*c.forceScale;
            if (isStep)
                for (int s = 0; s < count[i]; s++)
                    for (int d = 0; d < 3; d++)
                        k->reaction[3*nodes[S*i+s]+d] -= weights[S*i+s]*F[3*i+d];
        }
        if (isStep)
            apply_reaction(k);
    }
    free(nodes); free(weights); free(count); free(rhs); free(diag); free(spread);
    free(F); free(r); free(z); free(pv); free(Ap);
    return status;
}

/* couple (ReferenceLBMKernels.cpp:403-410). */
static LbmStatus couple(OracleKernel* k, const LbmParticleArrays* p, int isStep, long long step) {
    int stencil = k->L.interpolation_stencil != LBM_STENCIL_NEAREST;
    if (k->L.drag_scheme == LBM_DRAG_CENTERED) {
        if (stencil)
            return couple_centered_stencil(k, p, isStep, step);
        couple_centered(k, p, isStep, step);
    }
    else if (stencil)
        couple_stencil(k, p, isStep, step);
    else
        couple_nearest(k, p, isStep, step);
    return LBM_OK;
}

/* collideNode (ReferenceLBMKernels.cpp:1090-1120): push-stream one node. */
static void collide_node(OracleKernel* k, long node, double mu, const double* normal) {
    int nx = k->nx, ny = k->ny, nz = k->nz;
    long n = k->n;
    int i = (int) (node%nx), j = (int) ((node/nx)%ny), kk = (int) (node/((long) nx*ny));
    double omega = k->L.omega;
    double dfeq[Q], fneq[Q], s[Q], xi[Q];
    double r = k->rho[node];
    const double* F = &k->fd[3*node];
    double ux = (k->mom[3*node] + 0.5*F[0])/r;
    double uy = (k->mom[3*node+1] + 0.5*F[1])/r;
    double uz = (k->mom[3*node+2] + 0.5*F[2])/r;
    eq_deviation(k->drho[node], ux, uy, uz, dfeq);
    regularized_fneq(&k->pi[6*node], fneq);
    guo_forcing(ux, uy, uz, F[0], F[1], F[2], s);
    if (normal != NULL) {
        oracle_fluctuation(normal, sqrt(mu*r*omega*(2.0-omega)), sqrt(mu*r), xi);
        if (k->bnd_of_node != NULL && k->bnd_of_node[node] >= 0)
            oracle_fluctuation(normal, sqrt(mu*r*omega*(2.0-omega)), 0.0, &k->bnd_stress[(size_t) Q*k->bnd_of_node[node]]);
    }
    for (int q = 0; q < Q; q++) {
        int di = (i + CX[q] + nx)%nx;
        int dj = (j + CY[q] + ny)%ny;
        int dk = (kk + CZ[q] + nz)%nz;
        double value = dfeq[q] + (1.0-omega)*fneq[q] + 0.5*s[q];
        if (normal != NULL)
            value += xi[q];
        k->pop[q*n + di + (long) nx*(dj + (long) ny*dk)] = value;
    }
}

static double fluid_mu(const OracleKernel* k) {
    const LbmLatticeParameters* L = &k->L;
    double cellMass = L->density*L->dx*L->dx*L->dx;
    return 3.0*L->fluid_kT*L->dt*L->dt/(cellMass*L->dx*L->dx);
}

/* collideAndStream (ReferenceLBMKernels.cpp:1066-1088). */
static void collide_and_stream(OracleKernel* k, long long step) {
    int fluctuate = (k->L.fluid_fluctuations && k->L.fluid_kT > 0);
    double mu = fluid_mu(k);
    double normal[15];
    for (long node = 0; node < k->n; node++) {
        if (k->fluid && !k->fluid[node])
            continue;
        if (fluctuate)
            for (int m = 0; m < 15; m++)
                normal[m] = (k->random_mode == ORACLE_RANDOM_PHILOX ?
                             oracle_philox_normal(k->seed, PURPOSE_FLUID, node, step, m) : seq_gaussian(k));
        collide_node(k, node, mu, fluctuate ? normal : NULL);
    }
}

/* bounceBack (ReferenceLBMKernels.cpp:1156-1174). */
static void bounce_back(OracleKernel* k) {
    int nx = k->nx, ny = k->ny, nz = k->nz;
    long n = k->n;
    for (int b = 0; b < k->nwall; b++) {
        long node = k->wall_nodes[b];
        int i = (int) (node%nx), j = (int) ((node/nx)%ny), kk = (int) (node/((long) nx*ny));
        for (int q = 1; q < Q; q++) {
            if (!(k->wall_links[b] & (1<<q)))
                continue;
            long solid = (i + CX[q] + nx)%nx + (long) nx*((j + CY[q] + ny)%ny + (long) ny*((kk + CZ[q] + nz)%nz));
            k->pop[OPP[q]*n + node] = k->pop[q*n + solid];
        }
    }
}

/* computeWallMomentum (ReferenceLBMKernels.cpp:1176-1205). */
static void compute_wall_momentum(OracleKernel* k) {
    int nx = k->nx, ny = k->ny, nz = k->nz;
    long n = k->n;
    double ex[3] = {0, 0, 0};
    for (int s = 0; s < k->nsolid; s++) {
        long node = k->solid[s];
        int i = (int) (node%nx), j = (int) ((node/nx)%ny), kk = (int) (node/((long) nx*ny));
        for (int q = 1; q < Q; q++) {
            int di = i + CX[q], dj = j + CY[q], dk = kk + CZ[q];
            if ((is_open_axis(&k->L, 0) && (di < 0 || di >= nx)) || (is_open_axis(&k->L, 1) && (dj < 0 || dj >= ny)) ||
                    (is_open_axis(&k->L, 2) && (dk < 0 || dk >= nz)))
                continue;
            di = (di + nx)%nx;
            dj = (dj + ny)%ny;
            dk = (dk + nz)%nz;
            long target = di + (long) nx*(dj + (long) ny*dk);
            if (!k->fluid[target])
                continue;
            double df = k->pop[OPP[q]*n + node];
            ex[0] -= CX[q]*(2.0*(df + W[q]));
            ex[1] -= CY[q]*(2.0*(df + W[q]));
            ex[2] -= CZ[q]*(2.0*(df + W[q]));
        }
    }
    double cellMass = k->L.density*k->L.dx*k->L.dx*k->L.dx;
    for (int a = 0; a < 3; a++)
        k->wall_momentum.v[a] += ex[a]*(cellMass*k->L.dx/k->L.dt);
}

/* applyBoundaries (ReferenceLBMKernels.cpp:1207-1343). */
static void apply_boundaries(OracleKernel* k, long long step) {
    const LbmLatticeParameters* L = &k->L;
    int nx = k->nx, ny = k->ny, nz = k->nz;
    long n = k->n;
    const double* g = L->body_acceleration;
    double omega = L->omega;
    int fluctuate = (L->fluid_fluctuations && L->fluid_kT > 0);
    double cellMass = L->density*L->dx*L->dx*L->dx;
    double mu = fluid_mu(k);
    double dfeq[Q], fneq[Q], s[Q], xi[Q], normal[Q];
    double c = boundary_stress_weight(omega);
    double ex[3] = {0, 0, 0};
    for (int b = 0; b < k->nbnd; b++) {
        long node = k->bnd_node[b];
        int unknown = k->bnd_unknown[b], solid = k->bnd_solid[b];
        int kind = k->bnd_kind[b], face = k->bnd_face[b];
        int i = (int) (node%nx), j = (int) ((node/nx)%ny), kk = (int) (node/((long) nx*ny));
        double rb = k->rho[node], dr = k->drho[node];
        double ub[3] = {(k->mom[3*node] + 0.5*(rb*g[0]))/rb, (k->mom[3*node+1] + 0.5*(rb*g[1]))/rb,
                        (k->mom[3*node+2] + 0.5*(rb*g[2]))/rb};
        if (kind == KIND_WALL || kind == KIND_DENSITY_AT_REST)
            ub[0] = ub[1] = ub[2] = 0;
        if (kind == KIND_VELOCITY || kind == KIND_DENSITY_VELOCITY)
            for (int a = 0; a < 3; a++)
                ub[a] = L->face_velocity[face][a];
        if (kind == KIND_DENSITY || kind == KIND_DENSITY_AT_REST || kind == KIND_DENSITY_VELOCITY) {
            dr = L->face_density[face]-1.0;
            rb = L->face_density[face];
        }
        if (kind == KIND_DENSITY) {
            int axis = face/2;
            double inward = (face%2 == 0 ? 1.0 : -1.0), sum = 0;
            for (int q = 0; q < Q; q++)
                sum += k->pop[(unknown & (1<<q) ? OPP[q] : q)*n+node];
            ub[axis] = 0.5*(inward*(dr-sum)/rb + ub[axis]);
        }
        double Fb[3] = {g[0]*rb, g[1]*rb, g[2]*rb};
        eq_deviation(dr, ub[0], ub[1], ub[2], dfeq);
        regularized_fneq(&k->pi[6*node], fneq);
        guo_forcing(ub[0], ub[1], ub[2], Fb[0], Fb[1], Fb[2], s);
        if (fluctuate && has_equilibrium_noise(kind)) {
            for (int m = 0; m < Q; m++)
                normal[m] = (k->random_mode == ORACLE_RANDOM_PHILOX ?
                             oracle_philox_normal(k->seed, PURPOSE_BOUNDARY, node, step, m) : seq_gaussian(k));
            double oneMinusC = 1.0-c;
            equilibrium_fluctuation(normal, sqrt(mu*rb), sqrt(mu*rb*(oneMinusC > 0.0 ? oneMinusC : 0.0)), sqrt(mu*rb), xi);
            for (int q = 0; q < Q; q++)
                xi[q] -= c*k->bnd_stress[(size_t) Q*b+q];
        }
        else if (fluctuate) {
            for (int m = 0; m < 15; m++)
                normal[m] = (k->random_mode == ORACLE_RANDOM_PHILOX ?
                             oracle_philox_normal(k->seed, PURPOSE_BOUNDARY, node, step, m) : seq_gaussian(k));
            oracle_fluctuation(normal, sqrt(mu*rb*omega*(2.0-omega)), sqrt(mu*rb), xi);
        }
        if (kind == KIND_WALL || kind == KIND_VELOCITY) {
            double e0[Q], sg[Q];
            eq_deviation(0.0, ub[0], ub[1], ub[2], e0);
            guo_forcing(ub[0], ub[1], ub[2], g[0], g[1], g[2], sg);
            double numerator = 0, denominator = 0;
            for (int q = 1; q < Q; q++) {
                if (!(unknown & (1<<q)))
                    continue;
                double arriving, flux = 0;
                if (solid & (1<<q)) {
                    long source = (i - CX[q] + nx)%nx + (long) nx*((j - CY[q] + ny)%ny + (long) ny*((kk - CZ[q] + nz)%nz));
                    arriving = k->pop[OPP[q]*n + source];
                }
                else if (!(unknown & (1<<OPP[q]))) {
                    arriving = k->pop[OPP[q]*n + node];
                    flux = 6.0*W[q]*(CX[q]*ub[0] + CY[q]*ub[1] + CZ[q]*ub[2]);
                }
                else
                    continue;
                double rest = (1.0-omega)*fneq[q] + (fluctuate ? xi[q] : 0.0);
                numerator += arriving - rest - e0[q] - 0.5*sg[q] + flux;
                denominator += W[q] + e0[q] + 0.5*sg[q] - flux;
            }
            if (denominator != 0) {
                dr = numerator/denominator;
                rb = 1.0 + dr;
                Fb[0] = g[0]*rb; Fb[1] = g[1]*rb; Fb[2] = g[2]*rb;
                eq_deviation(dr, ub[0], ub[1], ub[2], dfeq);
                guo_forcing(ub[0], ub[1], ub[2], Fb[0], Fb[1], Fb[2], s);
            }
        }
        for (int q = 1; q < Q; q++) {
            if (!(unknown & (1<<q)))
                continue;
            double value = dfeq[q] + (1.0-omega)*fneq[q] + 0.5*s[q];
            if (fluctuate)
                value += xi[q];
            if (solid & (1<<q)) {
                long source = (i - CX[q] + nx)%nx + (long) nx*((j - CY[q] + ny)%ny + (long) ny*((kk - CZ[q] + nz)%nz));
                double sent = k->pop[OPP[q]*n + source];
                ex[0] -= CX[q]*(sent + value + 2.0*W[q]);
                ex[1] -= CY[q]*(sent + value + 2.0*W[q]);
                ex[2] -= CZ[q]*(sent + value + 2.0*W[q]);
            }
            k->pop[q*n+node] = value;
        }
    }
    for (int a = 0; a < 3; a++)
        k->wall_momentum.v[a] += ex[a]*(cellMass*L->dx/L->dt);
}

/* computeMachNumber (ReferenceLBMKernels.cpp:1449-1468). */
static double compute_mach(const OracleKernel* k) {
    long n = k->n;
    double maxSpeed2 = 0;
    for (long node = 0; node < n; node++) {
        if (k->fluid && !k->fluid[node])
            continue;
        double r = 1.0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < Q; q++) {
            double f = k->pop[q*n+node];
            r += f;
            jx += CX[q]*f;
            jy += CY[q]*f;
            jz += CZ[q]*f;
        }
        double s2 = (jx*jx + jy*jy + jz*jz)/(r*r);
        if (s2 > maxSpeed2)
            maxSpeed2 = s2;
    }
    return sqrt(3.0*maxSpeed2);
}

/* advanceFluid (ReferenceLBMKernels.cpp:367-389). */
static LbmStatus advance_fluid(OracleKernel* k, const LbmParticleArrays* p) {
    const LbmLatticeParameters* L = &k->L;
    long long step = k->step_index;
    compute_moments(k);
    if (L->momentum_removal_frequency > 0 && k->step_index%L->momentum_removal_frequency == 0)
        remove_fluid_momentum(k);
    if (k->np > 0) {
        LbmStatus status = couple(k, p, 1, step);
        if (status != LBM_OK)
            return status;
    }
    collide_and_stream(k, step);
    if (k->nwall > 0) {
        bounce_back(k);
        compute_wall_momentum(k);
    }
    if (k->nbnd > 0)
        apply_boundaries(k, step);
    k->step_forces_current = 1;
    k->step_index++;
    if (L->mach_check_frequency > 0 && k->step_index%L->mach_check_frequency == 0) {
        double mach = compute_mach(k);
        if (mach > L->mach_number_limit)
            return set_error(LBM_ERR_MACH_LIMIT, "LBMForce: the Mach number of the fluid is %g after %lld lattice steps, "
                             "above the limit %g", mach, k->step_index, L->mach_number_limit);
    }
    return LBM_OK;
}

/* computeNextStepForces (ReferenceLBMKernels.cpp:391-401). */
static LbmStatus compute_next_step_forces(OracleKernel* k, long long stepCount, const LbmParticleArrays* p) {
    k->step_forces_current = 0;
    compute_moments(k);
    if (k->L.momentum_removal_frequency > 0 && stepCount%k->L.momentum_removal_frequency == 0)
        remove_fluid_momentum(k);
    return couple(k, p, 0, stepCount);
}

/* beginStep (ReferenceLBMKernels.cpp:308-339). */
LbmStatus oracle_begin_step(OracleKernel* k, long long stepCount, const LbmParticleArrays* p) {
    k->step_index = stepCount;
    k->step_pending = 1;
    k->wall_momentum.v[0] = k->wall_momentum.v[1] = k->wall_momentum.v[2] = 0;
    if (k->fluid != NULL && k->np > 0) {
        double cellMass = k->L.density*k->L.dx*k->L.dx*k->L.dx;
        for (int i = 0; i < k->np; i++) {
            double* v = &p->velocities[3*i];
            double normal[3];
            long node = nearest_node(k, &p->positions[3*i]);
            wall_normal(k, &p->positions[3*i], normal);
            if (!k->fluid[node] && v[0]*normal[0] + v[1]*normal[1] + v[2]*normal[2] > 0) {
                for (int a = 0; a < 3; a++) {
                    k->wall_momentum.v[a] += v[a]*(2.0*k->pmass[i]*cellMass);
                    v[a] = -v[a];
                }
            }
        }
    }
    return LBM_OK;
}

/* execute (ReferenceLBMKernels.cpp:341-365). */
LbmStatus oracle_execute(OracleKernel* k, long long stepCount, const LbmParticleArrays* p, int includeForces,
                         int includeEnergy, double* energy) {
    int repeatedStep = (k->step_forces_current && stepCount == k->step_index-1);
    LbmStatus status = LBM_OK;
    if (k->step_pending) {
        k->step_pending = 0;
        status = advance_fluid(k, p);
    }
    else if (includeForces && k->np > 0 && stepCount > 0 && !repeatedStep)
        status = compute_next_step_forces(k, stepCount, p);
    if (status != LBM_OK)
        return status;
    if (includeForces)
        for (int i = 0; i < 3*k->np; i++)
            p->forces[i] += k->pforce[i];
    if (energy)
        *energy = 0.0;
    return status;
}

LbmStatus oracle_copy_parameters(OracleKernel* k, const LbmLatticeParameters* L) {
    k->L = *L;
    return LBM_OK;
}

/* getFluidFields / nodeFields (ReferenceLBMKernels.cpp:1349-1368, 1403-1436), one domain. */
LbmStatus oracle_get_fluid_fields(OracleKernel* k, double* density, double* velocity) {
    long n = k->n;
    double vs = k->L.dx/k->L.dt;
    for (long node = 0; node < n; node++) {
        if (k->fluid && !k->fluid[node]) {
            density[node] = 0;
            velocity[3*node] = velocity[3*node+1] = velocity[3*node+2] = 0;
            continue;
        }
        double r = 1.0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < Q; q++) {
            double f = k->pop[q*n+node];
            r += f;
            jx += CX[q]*f;
            jy += CY[q]*f;
            jz += CZ[q]*f;
        }
        density[node] = r*k->L.density;
        velocity[3*node] = (jx*(1.0/r) + k->L.body_acceleration[0]*0.5)*vs;
        velocity[3*node+1] = (jy*(1.0/r) + k->L.body_acceleration[1]*0.5)*vs;
        velocity[3*node+2] = (jz*(1.0/r) + k->L.body_acceleration[2]*0.5)*vs;
    }
    return LBM_OK;
}

LbmStatus oracle_get_fluid_mach_number(OracleKernel* k, double* mach) {
    *mach = compute_mach(k);
    return LBM_OK;
}

/* getWallForce (ReferenceLBMKernels.cpp:1438-1443). */
LbmStatus oracle_get_wall_force(OracleKernel* k, double force[3]) {
    for (int a = 0; a < 3; a++)
        force[a] = k->wall_momentum.v[a]*(1.0/k->L.dt);
    return LBM_OK;
}

LbmStatus oracle_get_fluid_state(OracleKernel* k, double* state) {
    memcpy(state, k->pop, sizeof(double)*Q*k->n);
    return LBM_OK;
}

/* setFluidState (ReferenceLBMKernels.cpp:1488-1505). */
LbmStatus oracle_set_fluid_state(OracleKernel* k, const double* state) {
    memcpy(k->pop, state, sizeof(double)*Q*k->n);
    k->step_forces_current = 0;
    return LBM_OK;
}

/* ------------------------------------------------------------------------------------------------ */
/* Bead forces on the CPU (the stand-in for OpenMM's forces in the benchmark configurations)          */
/* ------------------------------------------------------------------------------------------------ */

/* Harmonic bonds k/2 (r - r0)^2 and WCA (pair_type 1) or truncated Lennard-Jones (2) pairs within the cutoff, bonded
   pairs excluded, minimum image; brute force over pairs.  forces is overwritten. */
void oracle_md_forces(int n, const double* pos, const double box[3], int num_bonds, const int* bonds, double k, double r0,
                      int pair_type, double sigma, double eps, double cutoff, double* forces) {
    memset(forces, 0, sizeof(double)*3*(size_t) n);
    for (int b = 0; b < num_bonds; b++) {
        int i = bonds[2*b], j = bonds[2*b+1];
        double d[3];
        for (int a = 0; a < 3; a++) {
            d[a] = pos[3*i+a] - pos[3*j+a];
            d[a] -= box[a]*nearbyint(d[a]/box[a]);
        }
        double r = sqrt(d[0]*d[0] + d[1]*d[1] + d[2]*d[2]);
        if (r == 0.0)
            continue;
        double s = -k*(r - r0)/r;
        for (int a = 0; a < 3; a++) {
            forces[3*i+a] += s*d[a];
            forces[3*j+a] -= s*d[a];
        }
    }
    if (pair_type == 0)
        return;
    double rc = (pair_type == 1 ? pow(2.0, 1.0/6.0)*sigma : cutoff), rc2 = rc*rc, s2 = sigma*sigma;
    /* bonded partners for the exclusions */
    int* count = (int*) calloc(n + 1, sizeof(int));
    for (int b = 0; b < num_bonds; b++) {
        count[bonds[2*b]+1]++;
        count[bonds[2*b+1]+1]++;
    }
    for (int i = 0; i < n; i++)
        count[i+1] += count[i];
    int* partner = (int*) malloc(sizeof(int)*(2*(size_t) num_bonds + 1));
    int* fill = (int*) malloc(sizeof(int)*(n + 1));
    memcpy(fill, count, sizeof(int)*(n + 1));
    for (int b = 0; b < num_bonds; b++) {
        partner[fill[bonds[2*b]]++] = bonds[2*b+1];
        partner[fill[bonds[2*b+1]]++] = bonds[2*b];
    }
    for (int i = 0; i < n; i++)
        for (int j = i+1; j < n; j++) {
            double d[3];
            for (int a = 0; a < 3; a++) {
                d[a] = pos[3*i+a] - pos[3*j+a];
                d[a] -= box[a]*nearbyint(d[a]/box[a]);
            }
            double r2 = d[0]*d[0] + d[1]*d[1] + d[2]*d[2];
            if (r2 >= rc2 || r2 == 0.0)
                continue;
            int excluded = 0;
            for (int p = count[i]; p < count[i+1]; p++)
                if (partner[p] == j)
                    excluded = 1;
            if (excluded)
                continue;
            double q = s2/r2, q6 = q*q*q;
            double s = 24.0*eps*q6*(2.0*q6 - 1.0)/r2;
            for (int a = 0; a < 3; a++) {
                forces[3*i+a] += s*d[a];
                forces[3*j+a] -= s*d[a];
            }
        }
    free(count);
    free(partner);
    free(fill);
}
