// Device functions of the particle coupling, shared by the kernels of one lattice (coupling.cu) and of the replica
// batch (batch.cu): stencil weights and slots, the pulled moments of a node, the explicit drag of a particle and the
// reaction on the fluid, after the reference (platforms/reference/src/ReferenceLBMKernels.cpp:503-1018,
// openmmapi/include/internal/LBMStencils.h).
#pragma once

#include "fluid.cuh"
#include "lbm_device.cuh"
#include <cstring>
#include <type_traits>

namespace lbm {

// The coupling parameters in lattice units, by value to the kernels.
struct CouplingView {
    int np, width, slots, stencil;
    int nx, ny, nz;
    int open[3];
    long long n;
    int wordsPerRow;
    double dx, velocityScale, forceScale;
    double gamma, kT, h, a;
    double g[3];
    uint32_t seed;
    int randomForce;
    const uint32_t* solidMask;
    const double* mass;          // m/m_c per particle
};

// The coupling parameters in lattice units (ReferenceLBMKernels.cpp:520-525).
inline CouplingView makeCouplingView(const LbmLatticeParameters& l, const FluidView& f, int np, int width, const double* mass) {
    CouplingView c;
    std::memset(&c, 0, sizeof(c));
    c.np = np;
    c.width = width;
    c.slots = width*width*width;
    c.stencil = l.interpolation_stencil;
    c.nx = l.nx; c.ny = l.ny; c.nz = l.nz;
    for (int a = 0; a < 3; a++)
        c.open[a] = l.face_boundary[2*a] != LBM_BOUNDARY_PERIODIC;
    c.n = f.n;
    c.wordsPerRow = f.wordsPerRow;
    double cellMass = l.density*l.dx*l.dx*l.dx;
    c.dx = l.dx;
    c.velocityScale = l.dx/l.dt;
    c.forceScale = cellMass*l.dx/(l.dt*l.dt);
    c.gamma = l.friction*l.dt;
    c.kT = l.kT*l.dt*l.dt/(cellMass*l.dx*l.dx);
    c.h = 0.5;
    c.a = c.gamma*c.h;
    for (int a = 0; a < 3; a++)
        c.g[a] = l.body_acceleration[a];
    c.seed = (uint32_t) l.random_number_seed;
    c.randomForce = (c.kT > 0 && c.gamma > 0) ? 1 : 0;
    c.solidMask = f.solidMask;
    c.mass = mass;
    return c;
}

namespace {

template <typename R> struct Vec4;
template <> struct Vec4<float> {
    typedef float4 type;
    static __device__ __forceinline__ float4 make(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
};
template <> struct Vec4<double> {
    typedef double4 type;
    static __device__ __forceinline__ double4 make(double a, double b, double c, double d) { return make_double4(a, b, c, d); }
};

// Loads of a slot's 4-vector through the read-only path (data of an earlier launch) or through L2 (data written by the
// same launch); double4 as two double2.
__device__ __forceinline__ float4 loadReadOnly(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 loadReadOnly(const double4* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 loadCoherent(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ double4 loadCoherent(const double4* p) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p)), b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// r[0..2] += (x, y, z): one vector atomic for float (sm_90 and later), three for double.
__device__ __forceinline__ void atomicAdd3(float* r, double x, double y, double z) {
    atomicAdd(reinterpret_cast<float4*>(r), make_float4((float) x, (float) y, (float) z, 0.0f));
}
__device__ __forceinline__ void atomicAdd3(double* r, double x, double y, double z) {
    atomicAdd(&r[0], x);
    atomicAdd(&r[1], y);
    atomicAdd(&r[2], z);
}

// Node indices are below 2^32 (the fluid checks it), so 32-bit division finds their rows.
__device__ __forceinline__ bool isSolid(const uint32_t* mask, int wordsPerRow, int nx, long long node) {
    if (mask == nullptr)
        return false;
    const unsigned row = (unsigned) node/(unsigned) nx;
    const int x = (int) ((unsigned) node - row*(unsigned) nx);
    return (__ldg(&mask[(size_t) row*wordsPerRow + x/32]) >> (x%32)) & 1u;
}

// Lattice coordinate of a position along an axis, wrapped into [0, n) (ReferenceLBMKernels.cpp:978-979).
__device__ __forceinline__ double latticeCoordinate(double x, double dx, int n) {
    double s = x/dx;
    s -= floor(s/n)*n;
    return s;
}

// LBMStencils::kernel (LBMStencils.h:42-62).
__device__ double stencilKernel1(int stencil, double r) {
    double s = fabs(r);
    switch (stencil) {
    case LBM_STENCIL_TRILINEAR:
        return (s < 1.0 ? 1.0-s : 0.0);
    case LBM_STENCIL_THREEPOINT:
        if (s <= 0.5)
            return (1.0 + sqrt(1.0-3.0*s*s))/3.0;
        if (s < 1.5)
            return (5.0 - 3.0*s - sqrt(fmax(0.0, 1.0-3.0*(1.0-s)*(1.0-s))))/6.0;
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

// LBMStencils::axisWeights (LBMStencils.h:73-95): the nodes of the stencil along one axis and their weights,
// clamped at open faces, with repeated nodes merged into their first slot.
__device__ void axisWeights(int stencil, int width, double s, int n, bool open, int* index, double* weight) {
    int first;
    if (stencil == LBM_STENCIL_THREEPOINT)
        first = (int) floor(s + 0.5) - 1;
    else if (stencil == LBM_STENCIL_KEYS)
        first = (int) floor(s) - 1;
    else if (stencil == LBM_STENCIL_TRILINEAR)
        first = (int) floor(s);
    else
        first = (int) floor(s + 0.5);
    for (int i = 0; i < width; i++) {
        weight[i] = stencilKernel1(stencil, s - (first + i));
        int idx = first + i;
        index[i] = open ? min(max(idx, 0), n - 1) : ((idx%n) + n)%n;
    }
    for (int i = 1; i < width; i++)
        for (int j = 0; j < i; j++)
            if (index[j] == index[i]) {
                weight[j] += weight[i];
                weight[i] = 0.0;
                break;
            }
}

// Density deviation and momentum of the post-stream populations of a node (pulled from the input array).
template <typename T>
__device__ void pullMomentsAt(const T* A, const FluidView& f, int x, int y, int z, double& dr, double& jx, double& jy,
                              double& jz) {
    typedef typename std::conditional<std::is_same<T, double>::value, double, float>::type R;
    int xs[3] = {x == 0 ? f.nx-1 : x-1, x, x == f.nx-1 ? 0 : x+1};
    int ys[3] = {y == 0 ? f.ny-1 : y-1, y, y == f.ny-1 ? 0 : y+1};
    int zs[3] = {z == 0 ? f.nz-1 : z-1, z, z == f.nz-1 ? 0 : z+1};
    R d = 0, a = 0, b = 0, c = 0;
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
        long long src = xs[1-cx] + (long long) f.nx*(ys[1-cy] + (long long) f.ny*zs[1-cz]);
        R v = loadq<T, R>(A + (long long) q*f.n + src, q);
        d += v;
        a += cx*v;
        b += cy*v;
        c += cz*v;
    }
    dr = d; jx = a; jy = b; jz = c;
}

template <typename T>
__device__ void pullMoments(const T* A, const FluidView& f, long long node, double& dr, double& jx, double& jy, double& jz) {
    long long r = node/f.nx;
    pullMomentsAt<T>(A, f, (int) (node%f.nx), (int) (r%f.ny), (int) (r/f.ny), dr, jx, jy, jz);
}

// The node indices and weights of particle i's stencil on each axis (entries past the width: index -1, weight 0).
__device__ __forceinline__ void stencilAxes(const CouplingView& c, const double* __restrict__ pos, int i, int index[3][4],
                                            double weight[3][4]) {
    const int size[3] = {c.nx, c.ny, c.nz};
    for (int a = 0; a < 3; a++) {
        for (int k = 0; k < 4; k++) {
            index[a][k] = -1;
            weight[a][k] = 0.0;
        }
        double sc = latticeCoordinate(pos[3*i+a], c.dx, size[a]);
        if (c.stencil == LBM_STENCIL_NEAREST) {
            // nearestNode (ReferenceLBMKernels.cpp:973-983): periodic wrap on every axis.
            index[a][0] = ((int) floor(sc + 0.5))%size[a];
            weight[a][0] = 1.0;
        }
        else
            axisWeights(c.stencil, c.width, sc, size[a], c.open[a] != 0, index[a], weight[a]);
    }
}

// The node, weight and fluid velocity of stencil slot t = i*slots + s (particle i, slot s): the node and weight of
// the slot (LBMStencils::axisWeights, LBMStencils.h:73-95) and the moments of the node pulled from the populations
// (density, momentum after the momentum removal; a solid node has rho = 0).  centred: the velocity is
// u~ = (j + h rho g)/rho (ReferenceLBMKernels.cpp:622, 773); explicit: u = j/rho (:539, :672).
template <typename T, typename R, bool COHERENT = false>
__device__ __forceinline__ void stencilSlot(const T* __restrict__ A, const FluidView& f, const CouplingView& c,
                                            const double* __restrict__ posIn, long long t, int remove, int centred,
                                            int* slotNode, R* slotWeight, typename Vec4<R>::type* slotU) {
    // COHERENT: the positions were written by the same launch (a persistent kernel): read them through L2.  The slots
    // of all particles are fewer than 2^31: 32-bit division.
    const int i = (int) t/c.slots, s = (int) t - i*c.slots;
    double pos[3];
    for (int a = 0; a < 3; a++)
        pos[a] = COHERENT ? __ldcg(&posIn[3*i+a]) : posIn[3*i+a];
    int size[3] = {c.nx, c.ny, c.nz};
    int idx[3];
    double w = 1.0;
    if (c.stencil == LBM_STENCIL_NEAREST) {
        // nearestNode (ReferenceLBMKernels.cpp:973-983): periodic wrap on every axis.
        for (int a = 0; a < 3; a++) {
            double sc = latticeCoordinate(pos[a], c.dx, size[a]);
            idx[a] = ((int) floor(sc + 0.5))%size[a];
        }
    }
    else {
        int sub[3] = {s%c.width, (s/c.width)%c.width, s/(c.width*c.width)};
        for (int a = 0; a < 3; a++) {
            int index[4];
            double weight[4];
            axisWeights(c.stencil, c.width, latticeCoordinate(pos[a], c.dx, size[a]), size[a], c.open[a] != 0,
                        index, weight);
            idx[a] = index[sub[a]];
            w *= weight[sub[a]];
        }
    }
    long long node = idx[0] + (long long) c.nx*(idx[1] + (long long) c.ny*idx[2]);
    slotNode[t] = (int) node;
    slotWeight[t] = (R) w;
    double ux = 0, uy = 0, uz = 0, rho = 0;
    if (w != 0.0 && !isSolid(c.solidMask, c.wordsPerRow, c.nx, node)) {
        double dr, jx, jy, jz;
        pullMoments<T>(A, f, node, dr, jx, jy, jz);
        rho = 1.0 + dr;
        if (remove) {
            jx -= rho*f.stats->ucm[0];
            jy -= rho*f.stats->ucm[1];
            jz -= rho*f.stats->ucm[2];
        }
        if (centred) {
            jx += c.h*rho*c.g[0];
            jy += c.h*rho*c.g[1];
            jz += c.h*rho*c.g[2];
        }
        ux = jx*(1.0/rho);
        uy = jy*(1.0/rho);
        uz = jz*(1.0/rho);
    }
    slotU[t] = Vec4<R>::make((R) ux, (R) uy, (R) uz, (R) rho);
}

// The node and weight of stencil slot t, as stencilSlot (from the particle's axis indices and weights, computed once
// per particle by stencilAxes), with the moments computed once per node: the first slot of a fluid node to claim it in
// this pass (nodeStamp[node] set to `stamp`) pulls the node's moments into nodeU[node]; stencilGatherSlot then copies
// them to every slot of the node.  The moments of a node are the same for all its slots, and overlapping stencils
// share most of their nodes.  With `mark` (the fluid's reaction mask, for the pass of a step) the claiming slot also
// flags the node and zeroes its reaction, once per node: every fluid node of a slot with a nonzero weight receives a
// reaction in this step, so the reactions are then added without touching the mask, and the end of a step clears the
// mask alone.
// W: the stencil width when it is known at compile time (the slot's particle and axis entries then come from
// divisions by constants), 0 for c.width.  The slots of all particles are fewer than 2^31.
template <typename T, typename R, int W = 0>
__device__ __forceinline__ void stencilClaimSlot(const T* __restrict__ A, const FluidView& f, const CouplingView& c,
                                                 const int4* __restrict__ axisIndex,
                                                 const double2* __restrict__ axisWeight, long long t, int remove,
                                                 int centred, int* slotNode, R* slotWeight, unsigned* nodeStamp,
                                                 unsigned stamp, typename Vec4<R>::type* nodeU, uint32_t* mark,
                                                 R* reaction) {
    const int width = W > 0 ? W : c.width, slots = W > 0 ? W*W*W : c.slots;
    const int i = (int) t/slots, s = (int) t - i*slots;
    const int sub[3] = {s%width, (s/width)%width, s/(width*width)};
    int idx[3];
    double w = 1.0;
    for (int a = 0; a < 3; a++) {
        const int4 ia = axisIndex[3*i + a];
        const double2 wa = axisWeight[6*i + 2*a + sub[a]/2];
        idx[a] = sub[a] == 0 ? ia.x : sub[a] == 1 ? ia.y : sub[a] == 2 ? ia.z : ia.w;
        w *= (sub[a] & 1) ? wa.y : wa.x;
    }
    long long node = idx[0] + (long long) c.nx*(idx[1] + (long long) c.ny*idx[2]);
    slotNode[t] = (int) node;
    slotWeight[t] = (R) w;
    if (w == 0.0)
        return;
    if (c.solidMask != nullptr) {
        const long long row = idx[1] + (long long) c.ny*idx[2];
        if ((__ldg(&c.solidMask[row*c.wordsPerRow + idx[0]/32]) >> (idx[0]%32)) & 1u)
            return;
    }
    if (atomicExch(&nodeStamp[node], stamp) != stamp) {
        double dr, jx, jy, jz;
        pullMomentsAt<T>(A, f, idx[0], idx[1], idx[2], dr, jx, jy, jz);
        double rho = 1.0 + dr;
        if (remove) {
            jx -= rho*f.stats->ucm[0];
            jy -= rho*f.stats->ucm[1];
            jz -= rho*f.stats->ucm[2];
        }
        if (centred) {
            jx += c.h*rho*c.g[0];
            jy += c.h*rho*c.g[1];
            jz += c.h*rho*c.g[2];
        }
        nodeU[node] = Vec4<R>::make((R) (jx*(1.0/rho)), (R) (jy*(1.0/rho)), (R) (jz*(1.0/rho)), (R) rho);
        if (mark != nullptr) {
            const size_t row = (size_t) idx[1] + (size_t) c.ny*idx[2];
            atomicOr(&mark[row*f.wordsPerRow + idx[0]/32], 1u << (idx[0]%32));
            // The node's reaction starts from zero (the last step's were left in place; only their flags were cleared).
            *reinterpret_cast<typename Vec4<R>::type*>(reaction + 4*node) = Vec4<R>::make(0, 0, 0, 0);
        }
    }
}

template <typename R>
// With `coef` (the coupling matrix's solve) it also stores w/rho of the slot (0 where rho is 0).
__device__ __forceinline__ void stencilGatherSlot(long long t, const int* __restrict__ slotNode,
                                                  const R* __restrict__ slotWeight, const unsigned* __restrict__ nodeStamp,
                                                  unsigned stamp, const typename Vec4<R>::type* __restrict__ nodeU,
                                                  typename Vec4<R>::type* slotU, R* coef) {
    const long long node = slotNode[t];
    const R weight = slotWeight[t];
    typename Vec4<R>::type u = Vec4<R>::make(0, 0, 0, 0);
    if (weight != (R) 0 && nodeStamp[node] == stamp)
        u = nodeU[node];
    slotU[t] = u;
    if (coef != nullptr) {
        const double w = (double) weight, rho = (double) u.w;
        coef[t] = (R) (rho > 0 ? w/rho : 0.0);
    }
}

// Reaction (fx, fy, fz) on a node: added into the fluid's reaction buffer and the node flagged in `mask` (nullptr: the
// stencil pass flagged it), or for a solid node counted as momentum given to the wall (applyReaction,
// ReferenceLBMKernels.cpp:959-971).
template <typename R>
__device__ void addReaction(const FluidView& f, const CouplingView& c, R* reaction, uint32_t* mask, double* wall,
                            long long node, double fx, double fy, double fz) {
    if (isSolid(c.solidMask, c.wordsPerRow, c.nx, node)) {
        atomicAdd(&wall[0], fx);
        atomicAdd(&wall[1], fy);
        atomicAdd(&wall[2], fz);
        return;
    }
    atomicAdd3(reaction + 4*node, fx, fy, fz);
    if (mask == nullptr)
        return;
    const unsigned row = (unsigned) node/(unsigned) f.nx;
    const int x = (int) ((unsigned) node - row*(unsigned) f.nx);
    uint32_t bit = 1u << (x%32);
    uint32_t* word = &mask[(size_t) row*f.wordsPerRow + x/32];
    if (!(*((volatile uint32_t*) word) & bit))
        atomicOr(word, bit);
}

// Three normals of particle i for step `step` (Philox, purpose 2), in double.
__device__ __forceinline__ void particleNoise(uint32_t seed, int i, long long step, double xi[3]) {
    philoxNormals<double, 3>(seed, PurposeParticle, i, step, xi);
}

__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Explicit drag of particle i, nearest node or stencil (ReferenceLBMKernels.cpp:503-553, 643-697), by one warp (the
// lanes over the stencil slots): F = -gamma m (v - u) + sqrt(2 gamma m kT) xi with u interpolated over the stencil,
// written to fout; on a lattice step the reaction -w F goes to the stencil nodes.
template <typename R, bool COHERENT = false>
__device__ __forceinline__ void explicitParticle(const FluidView& f, const CouplingView& c, const double* vel,
                                                 const int* slotNode, const R* slotWeight,
                                                 const typename Vec4<R>::type* slotU, int i, int lane,
                                                 long long step, int isStep, double* fout, R* reaction, uint32_t* mask,
                                                 double* wall, const double* removal = nullptr) {
    // COHERENT: the slots and velocities were written by the same launch (a persistent kernel): loads through L2.
    // removal: the velocity that this step's momentum removal subtracts from every node, where the slots hold the
    // nodes' j/rho before the removal (the persistent batch step); (j - rho ucm)/rho = j/rho - ucm, so the fluid
    // velocity at the particle is sum w j/rho - ucm sum w over the fluid slots.
    typedef typename Vec4<R>::type V;
    auto slotU_ = [&](long long t) { if constexpr (COHERENT) return loadCoherent(slotU + t); else return loadReadOnly(slotU + t); };
    auto weight_ = [&](long long t) { if constexpr (COHERENT) return __ldcg(slotWeight + t); else return __ldg(slotWeight + t); };
    auto node_ = [&](long long t) { if constexpr (COHERENT) return __ldcg(slotNode + t); else return __ldg(slotNode + t); };
    auto vel_ = [&](int k) { if constexpr (COHERENT) return __ldcg(vel + k); else return __ldg(vel + k); };
    double u[3] = {0, 0, 0}, wsum = 0;
    for (int s = lane; s < c.slots; s += 32) {
        long long t = (long long) i*c.slots + s;
        V su = slotU_(t);
        if (su.w > 0) {
            double w = (double) weight_(t);
            u[0] += (double) su.x*w;
            u[1] += (double) su.y*w;
            u[2] += (double) su.z*w;
            wsum += w;
        }
    }
    for (int a = 0; a < 3; a++)
        u[a] = warpSum(u[a]);
    if (removal != nullptr) {
        wsum = warpSum(wsum);
        for (int a = 0; a < 3; a++)
            u[a] -= __ldcg(&removal[a])*wsum;
    }
    double m = c.mass[i];
    double xi[3] = {0, 0, 0};
    if (c.randomForce)
        particleNoise(c.seed, i, step, xi);
    double F[3];
    for (int a = 0; a < 3; a++) {
        double v = vel_(3*i+a)*(1.0/c.velocityScale);
        F[a] = (v - u[a])*(-c.gamma*m);
        if (c.randomForce)
            F[a] += xi[a]*sqrt(2.0*c.gamma*m*c.kT);
    }
    if (lane == 0)
        for (int a = 0; a < 3; a++)
            fout[3*i+a] = F[a]*c.forceScale;
    if (isStep)
        for (int s = lane; s < c.slots; s += 32) {
            long long t = (long long) i*c.slots + s;
            double w = (double) weight_(t);
            if (w != 0.0)
                addReaction<R>(f, c, reaction, mask, wall, node_(t), -w*F[0], -w*F[1], -w*F[2]);
        }
}

} // namespace
} // namespace lbm
