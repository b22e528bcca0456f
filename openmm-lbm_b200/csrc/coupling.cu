// Particle coupling kernels of the B200 LBM force kernel (sm_100a).
//
// The coupling of the reference (platforms/reference/src/ReferenceLBMKernels.cpp:503-1018), on the device:
//   stencilClaimKernel    one thread per (particle, stencil slot): the node and weight of the slot
//                         (LBMStencils::axisWeights, LBMStencils.h:73-95); the first slot of each fluid node pulls the
//                         node's moments from the populations (density, momentum after the momentum removal)
//   stencilGatherKernel   the moments of every slot from its node (a solid node has rho = 0)
//   explicitKernel        one warp per particle: explicit drag F = -gamma m (v - u) + sqrt(2 gamma m kT) xi with u
//                         interpolated over the stencil (:503-553, :643-697), reaction -w F on the stencil nodes
//   centeredNearestKernel the closed form of the centred drag per node (:555-641), after a stable radix sort of the
//                         particles by node; the particles of a node summed in particle order
//   centeredStencilKernel the centred drag with a stencil: Jacobi-preconditioned conjugate gradients for
//                         (1 + a) F_k + a m_k sum_l K_kl F_l = b_k (:726-901), the whole solve in one cooperative
//                         launch, one warp per particle, with a bounded grid barrier and no host round trip
//   reflectKernel         reversal of the particles that move into a wall (:315-338, wallNormal :1020-1050)
// Slot data, reactions and the spread vectors are kept in the precision of the fluid's arithmetic (double with FP64
// storage, float otherwise); particle quantities and all reductions are double.  Reactions are added with (vector)
// atomics into the fluid's node reaction buffer and their nodes flagged in its bitmask, so the dense kernel reads a
// reaction only where there is one.
#include "coupling.cuh"
#include "coupling_device.cuh"
#include "grid_barrier.cuh"
#include "lbm_device.cuh"
#include "radix_sort.cuh"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

namespace lbm {

#define CUDA_CHECK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    throw Error(LBM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

namespace {

const int kThreads = 256;

// The stencil pass: the axis indices and weights of each particle, then one thread per (particle, stencil slot) in
// two passes: nodes, weights and the moments of each node once, then the moments of every slot.
// One thread per particle: the node indices and weights of its stencil on each axis, and the first index on each.
__global__ void stencilAxesKernel(CouplingView c, const double* __restrict__ pos, int4* axisIndex, double2* axisWeight,
                                  int4* firstIndex) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < c.np; i += gridDim.x*blockDim.x) {
        int index[3][4];
        double weight[3][4];
        stencilAxes(c, pos, i, index, weight);
        for (int a = 0; a < 3; a++) {
            axisIndex[3*i + a] = make_int4(index[a][0], index[a][1], index[a][2], index[a][3]);
            axisWeight[6*i + 2*a] = make_double2(weight[a][0], weight[a][1]);
            axisWeight[6*i + 2*a + 1] = make_double2(weight[a][2], weight[a][3]);
        }
        firstIndex[i] = make_int4(index[0][0], index[1][0], index[2][0], 0);
    }
}

template <typename T, typename R, int W>
__global__ void stencilClaimKernel(const T* __restrict__ A, FluidView f, CouplingView c, const int4* __restrict__ axisIndex,
                                   const double2* __restrict__ axisWeight, int remove, int centred, int* slotNode,
                                   R* slotWeight, unsigned* nodeStamp, unsigned stamp, typename Vec4<R>::type* nodeU,
                                   uint32_t* mark, R* reaction) {
    const int total = c.np*c.slots;     // below 2^31 (the coupling's constructor checks it)
    for (int t = blockIdx.x*blockDim.x + threadIdx.x; t < total; t += gridDim.x*blockDim.x)
        stencilClaimSlot<T, R, W>(A, f, c, axisIndex, axisWeight, t, remove, centred, slotNode, slotWeight, nodeStamp,
                                  stamp, nodeU, mark, reaction);
}

template <typename R>
__global__ void stencilGatherKernel(CouplingView c, const int* __restrict__ slotNode, const R* __restrict__ slotWeight,
                                    const unsigned* __restrict__ nodeStamp, unsigned stamp,
                                    const typename Vec4<R>::type* __restrict__ nodeU, typename Vec4<R>::type* slotU,
                                    R* coef) {
    long long total = (long long) c.np*c.slots;
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < total; t += (long long) gridDim.x*blockDim.x)
        stencilGatherSlot<R>(t, slotNode, slotWeight, nodeStamp, stamp, nodeU, slotU, coef);
}

// One warp per particle.
template <typename R>
__global__ void explicitKernel(FluidView f, CouplingView c, const double* __restrict__ vel, const int* __restrict__ slotNode,
                               const R* __restrict__ slotWeight, const typename Vec4<R>::type* __restrict__ slotU,
                               long long step, int isStep, double* fout, R* reaction, uint32_t* mask, double* wall) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x*blockDim.x) >> 5;
    for (int i = (blockIdx.x*blockDim.x + threadIdx.x) >> 5; i < c.np; i += warps)
        explicitParticle<R>(f, c, vel, slotNode, slotWeight, slotU, i, lane, step, isStep, fout, reaction, mask, wall);
}

// Keys: nearest node of each particle (ReferenceLBMKernels.cpp:596, the key node*N + k sorted).
__global__ void nodeKeysKernel(const int* slotNode, int np, unsigned* keys, int* values) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < np; i += gridDim.x*blockDim.x) {
        keys[i] = (unsigned) slotNode[i];
        values[i] = i;
    }
}

// Centred drag at the nearest node (ReferenceLBMKernels.cpp:555-641): one thread per run of particles with the same
// node in the sorted order; sums in particle order.
template <typename R>
__global__ void centeredNearestKernel(FluidView f, CouplingView c, const unsigned* keys, const int* order,
                                      const double* __restrict__ vel, const double* __restrict__ fin,
                                      const typename Vec4<R>::type* __restrict__ slotU, long long step, int isStep,
                                      double* fout, R* reaction, uint32_t* mask, double* wall) {
    for (int k = blockIdx.x*blockDim.x + threadIdx.x; k < c.np; k += gridDim.x*blockDim.x) {
        if (k > 0 && keys[k-1] == keys[k])
            continue;
        int end = k;
        while (end < c.np && keys[end] == keys[k])
            end++;
        long long node = keys[k];
        double mass = 0, pm[3] = {0, 0, 0}, rs[3] = {0, 0, 0};
        for (int e = k; e < end; e++) {
            int i = order[e];
            double m = c.mass[i];
            double xi[3] = {0, 0, 0};
            if (c.randomForce)
                particleNoise(c.seed, i, step, xi);
            mass += m;
            for (int a = 0; a < 3; a++) {
                double known = vel[3*i+a]*(1.0/c.velocityScale) + fin[3*i+a]*(c.h/(m*c.forceScale));
                pm[a] += known*m;
                rs[a] += c.randomForce ? xi[a]*sqrt(2.0*c.gamma*m*c.kT) : 0.0;
            }
        }
        typename Vec4<R>::type su = slotU[order[k]];
        double u[3] = {0, 0, 0}, sum[3];
        if (su.w > 0) {
            double rho = su.w, kn[3] = {(double) su.x, (double) su.y, (double) su.z};
            for (int a = 0; a < 3; a++)
                sum[a] = ((pm[a] - kn[a]*mass)*(-c.gamma) + rs[a])*(1.0/(1.0 + c.a + c.a*mass/rho));
            for (int a = 0; a < 3; a++)
                u[a] = kn[a] - sum[a]*(c.h/rho);
        }
        else
            for (int a = 0; a < 3; a++)
                sum[a] = ((pm[a] - u[a]*mass)*(-c.gamma) + rs[a])*(1.0/(1.0 + c.a));
        for (int e = k; e < end; e++) {
            int i = order[e];
            double m = c.mass[i];
            double xi[3] = {0, 0, 0};
            if (c.randomForce)
                particleNoise(c.seed, i, step, xi);
            for (int a = 0; a < 3; a++) {
                double known = vel[3*i+a]*(1.0/c.velocityScale) + fin[3*i+a]*(c.h/(m*c.forceScale));
                double random = c.randomForce ? xi[a]*sqrt(2.0*c.gamma*m*c.kT) : 0.0;
                fout[3*i+a] = ((known - u[a])*(-c.gamma*m) + random)*(1.0/(1.0 + c.a))*c.forceScale;
            }
        }
        if (isStep)
            addReaction<R>(f, c, reaction, mask, wall, node, -sum[0], -sum[1], -sum[2]);
    }
}

// ------------------------------------------------------------------------------------------------------
// Centred drag with a stencil: conjugate gradients in one cooperative launch.
// ------------------------------------------------------------------------------------------------------

constexpr int kPartial = 12;   // doubles per block record

struct CgBuffers {
    double* rhs;           // 3 per particle (b/m)
    double* diag;          // 1 per particle
    double* F;             // solution
    double* r;
    double* z;             // holds A p between the product and the update
    double* p;
    double* partials[2];   // kPartial doubles per block, two buffers used alternately
    unsigned* barrier;     // arrivals at the grid barriers of the launch (cleared before it, with the status words)
    int* status;           // 0 ok, LBM_ERR_CG_NOT_CONVERGED, LBM_ERR_DEVICE_TIMEOUT
    int* iterations;
    long long pollLimit;   // polls of a waiting block before it gives up (kDefaultBarrierPolls)
};

// Block sum of a record (thread values v) into partials[block]; after a grid barrier (by the caller) every block adds
// the records of all blocks in block order, so every block gets the same result, bit for bit.
__device__ void blockSumStore(double v[kPartial], double* partials) {
    __shared__ double red[32][kPartial];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < kPartial; k++)
        v[k] = warpSum(v[k]);
    if (lane == 0)
        for (int k = 0; k < kPartial; k++)
            red[warp][k] = v[k];
    __syncthreads();
    if (threadIdx.x < kPartial) {
        double s = 0;
        for (int w = 0; w < (int) blockDim.x/32; w++)
            s += red[w][threadIdx.x];
        partials[kPartial*blockIdx.x + threadIdx.x] = s;
    }
    __syncthreads();
}

__device__ void reducePartials(const double* partials, int count, double out[kPartial]) {
    // Warp k sums component k over the blocks (lanes strided over the records, then a fixed tree), so every block
    // gets the same result, bit for bit.  The records were written by other blocks before a grid barrier: loads bypass
    // L1.
    __shared__ double total[kPartial];
    const int lane = threadIdx.x & 31;
    for (int k = threadIdx.x >> 5; k < kPartial; k += blockDim.x >> 5) {
        double s = 0;
        for (int r = lane; r < count; r += 32)
            s += __ldcg(partials + kPartial*r + k);
        s = warpSum(s);
        if (lane == 0)
            total[k] = s;
    }
    __syncthreads();
    for (int k = 0; k < kPartial; k++)
        out[k] = total[k];
    __syncthreads();
}

// The barriers of one iteration: after the spread of A p (products complete), after the partial sums of p.Ap
// (alpha), and after the partial sums of r.z and r.r (beta, convergence).  The two partial buffers alternate, so a
// buffer is never written while another block may still read it.
template <typename R>
__global__ void __launch_bounds__(kThreads)
centeredStencilKernel(FluidView f, CouplingView c, const double* __restrict__ vel, const double* __restrict__ fin,
                      const int* __restrict__ slotNode, const R* __restrict__ slotWeight,
                      const typename Vec4<R>::type* __restrict__ slotU, R* coef, long long step, int isStep,
                      double tolerance, int maxIterations, CgBuffers b, R* spread, double* fout, R* reaction,
                      uint32_t* mask, double* wall) {
    typedef typename Vec4<R>::type V;
    const int lane = threadIdx.x & 31;
    const int firstWarp = (blockIdx.x*blockDim.x + threadIdx.x) >> 5;
    const int warps = (gridDim.x*blockDim.x) >> 5;
    const int S = c.slots;
    const double a = c.a;
    // spread(n) += w p_i on the stencil nodes of particle i.
    auto spreadP = [&](int i, const double* p) {
        double p0 = p[3*i], p1 = p[3*i+1], p2 = p[3*i+2];
        for (int s = lane; s < S; s += 32) {
            long long t = (long long) i*S + s;
            double w = (double) slotWeight[t];
            if (w != 0.0)
                atomicAdd3(spread + 4*(long long) slotNode[t], w*p0, w*p1, w*p2);
        }
    };
    // sum_s (w_s/rho_s) spread(n_s), in every lane.
    auto gather = [&](int i, double g[3]) {
        g[0] = g[1] = g[2] = 0;
        for (int s = lane; s < S; s += 32) {
            long long t = (long long) i*S + s;
            double k = (double) coef[t];
            if (k != 0.0) {
                V v = *reinterpret_cast<const V*>(spread + 4*(long long) slotNode[t]);
                g[0] += k*(double) v.x;
                g[1] += k*(double) v.y;
                g[2] += k*(double) v.z;
            }
        }
        for (int d = 0; d < 3; d++)
            g[d] = warpSum(g[d]);
    };
    auto clearSpread = [&](int i) {
        for (int s = lane; s < S; s += 32) {
            long long t = (long long) i*S + s;
            if (slotWeight[t] != (R) 0)
                *reinterpret_cast<V*>(spread + 4*(long long) slotNode[t]) = Vec4<R>::make(0, 0, 0, 0);
        }
    };
    // Right-hand side, diagonal and the start F = rhs/diag (ReferenceLBMKernels.cpp:758-782, 839-840); coef = w/rho.
    for (int i = firstWarp; i < c.np; i += warps) {
        double m = c.mass[i];
        double u[3] = {0, 0, 0}, self = 0;
        for (int s = lane; s < S; s += 32) {
            long long t = (long long) i*S + s;
            V su = slotU[t];
            double w = (double) slotWeight[t];
            double k = 0;
            if (su.w > 0) {
                u[0] += (double) su.x*w;
                u[1] += (double) su.y*w;
                u[2] += (double) su.z*w;
                self += w*w/(double) su.w;
                k = w/(double) su.w;
            }
            coef[t] = (R) k;
        }
        for (int d = 0; d < 3; d++)
            u[d] = warpSum(u[d]);
        self = warpSum(self);
        double xi[3] = {0, 0, 0};
        if (c.randomForce)
            particleNoise(c.seed, i, step, xi);
        double diag = (1.0 + a)/m + a*self;
        double F[3];
        for (int d = 0; d < 3; d++) {
            double known = vel[3*i+d]*(1.0/c.velocityScale) + fin[3*i+d]*(c.h/(m*c.forceScale));
            double v = (known - u[d])*(-c.gamma*m);
            if (c.randomForce)
                v += xi[d]*sqrt(2.0*c.gamma*m*c.kT);
            double rhs = v*(1.0/m);
            F[d] = rhs*(1.0/diag);
            if (lane == 0) {
                b.rhs[3*i+d] = rhs;
                b.F[3*i+d] = F[d];
            }
        }
        if (lane == 0)
            b.diag[i] = diag;
        for (int s = lane; s < S; s += 32) {
            long long t = (long long) i*S + s;
            double w = (double) slotWeight[t];
            if (w != 0.0)
                atomicAdd3(spread + 4*(long long) slotNode[t], w*F[0], w*F[1], w*F[2]);
        }
    }
    if (!gridSync(b.barrier, b.status, b.pollLimit))
        return;
    // r = rhs - A F, z = r/diag, p = z; r.z, the norm of the right-hand side and r.r per component.
    double acc[kPartial] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = firstWarp; i < c.np; i += warps) {
        double g[3];
        gather(i, g);
        double m = c.mass[i], diag = b.diag[i];
        for (int d = 0; d < 3; d++) {
            double Ap = b.F[3*i+d]*((1.0 + a)/m) + g[d]*a;
            double rhs = b.rhs[3*i+d];
            double r = rhs - Ap;
            double z = r*(1.0/diag);
            if (lane == 0) {
                b.r[3*i+d] = r;
                b.z[3*i+d] = z;
                b.p[3*i+d] = z;
                acc[d] += r*z;
                acc[3+d] += rhs*rhs;
                acc[6+d] += r*r;
            }
        }
    }
    blockSumStore(acc, b.partials[1]);
    if (!gridSync(b.barrier, b.status, b.pollLimit))
        return;
    for (int i = firstWarp; i < c.np; i += warps)
        clearSpread(i);
    double tot[kPartial];
    reducePartials(b.partials[1], gridDim.x, tot);
    double rz[3] = {tot[0], tot[1], tot[2]}, norm[3] = {tot[3], tot[4], tot[5]}, residual[3] = {tot[6], tot[7], tot[8]};
    int iteration = 0;
    bool failed = false;       // the same in every block: every decision comes from the same reduced sums
    bool clearBeforeSpread = true;
    for (;; iteration++) {
        bool converged = true;
        for (int d = 0; d < 3; d++)
            if (residual[d] > tolerance*tolerance*norm[d])
                converged = false;
        if (converged)
            break;
        if (iteration == maxIterations) {
            if (firstWarp == 0 && lane == 0)
                atomicExch(b.status, LBM_ERR_CG_NOT_CONVERGED);
            failed = true;
            break;
        }
        // The spread buffer was cleared by every block before the last barrier (the clearing of the start comes
        // before the barrier at the top of the first iteration's spread below).
        if (clearBeforeSpread) {
            if (!gridSync(b.barrier, b.status, b.pollLimit))
                return;
            clearBeforeSpread = false;
        }
        for (int i = firstWarp; i < c.np; i += warps)
            spreadP(i, b.p);
        if (!gridSync(b.barrier, b.status, b.pollLimit))
            return;
        double acc3[kPartial] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = firstWarp; i < c.np; i += warps) {
            double g[3];
            gather(i, g);
            double m = c.mass[i];
            for (int d = 0; d < 3; d++) {
                double p = b.p[3*i+d];
                double Ap = p*((1.0 + a)/m) + g[d]*a;
                if (lane == 0) {
                    acc3[d] += p*Ap;
                    b.z[3*i+d] = Ap;
                }
            }
        }
        blockSumStore(acc3, b.partials[0]);
        if (!gridSync(b.barrier, b.status, b.pollLimit))
            return;
        reducePartials(b.partials[0], gridDim.x, tot);
        double alpha[3];
        for (int d = 0; d < 3; d++)
            alpha[d] = (tot[d] > 0 ? rz[d]/tot[d] : 0.0);
        double acc4[kPartial] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = firstWarp; i < c.np; i += warps) {
            clearSpread(i);
            if (lane == 0) {
                double diag = b.diag[i];
                for (int d = 0; d < 3; d++) {
                    b.F[3*i+d] += alpha[d]*b.p[3*i+d];
                    double r = b.r[3*i+d] - alpha[d]*b.z[3*i+d];
                    b.r[3*i+d] = r;
                    double z = r*(1.0/diag);
                    b.z[3*i+d] = z;
                    acc4[d] += r*z;
                    acc4[3+d] += r*r;
                }
            }
        }
        blockSumStore(acc4, b.partials[1]);
        if (!gridSync(b.barrier, b.status, b.pollLimit))
            return;
        reducePartials(b.partials[1], gridDim.x, tot);
        double beta[3];
        for (int d = 0; d < 3; d++) {
            beta[d] = (rz[d] > 0 ? tot[d]/rz[d] : 0.0);
            rz[d] = tot[d];
            residual[d] = tot[3+d];
        }
        if (lane == 0)
            for (int i = firstWarp; i < c.np; i += warps)
                for (int d = 0; d < 3; d++)
                    b.p[3*i+d] = b.z[3*i+d] + beta[d]*b.p[3*i+d];
        __syncwarp();
    }
    if (firstWarp == 0 && lane == 0)
        *b.iterations = iteration;
    if (failed)
        return;
    // Forces and reactions (ReferenceLBMKernels.cpp:889-900).
    for (int i = firstWarp; i < c.np; i += warps) {
        double F0 = b.F[3*i], F1 = b.F[3*i+1], F2 = b.F[3*i+2];
        if (lane == 0) {
            fout[3*i] = F0*c.forceScale;
            fout[3*i+1] = F1*c.forceScale;
            fout[3*i+2] = F2*c.forceScale;
        }
        if (isStep)
            for (int s = lane; s < S; s += 32) {
                long long t = (long long) i*S + s;
                double w = (double) slotWeight[t];
                if (w != 0.0)
                    addReaction<R>(f, c, reaction, mask, wall, slotNode[t], -w*F0, -w*F1, -w*F2);
            }
    }
}

// ------------------------------------------------------------------------------------------------------
// Centred drag with a stencil through the explicit coupling matrix.
//
// The operator of the conjugate gradients, (1 + a) F_k/m_k + a sum_l K_kl F_l with K_kl = sum_n w_k(n) w_l(n)/rho(n)
// over the fluid nodes n that the stencils of k and l share, is the same as the spread-and-gather of the kernel above
// (spread w_l F_l onto the nodes, gather with w_k/rho).  K is sparse (a particle's stencil overlaps those of the
// particles within one stencil width), so it is built once per step and every iteration is a sparse product over a few
// dozen entries per particle instead of a pass over the lattice nodes of all stencils.
//   cgBinKernel     per particle: its cell (cells of kCgCellEdge nodes, on the first stencil index of the stencil
//                   pass), inserted into a fixed-capacity cell list (w/rho of every slot comes from the stencil
//                   pass's slot copy)
//   cgRowsKernel    one warp per particle k: the particles of the neighbouring cells whose first stencil indices are
//                   within a stencil width of k's on every axis, sorted by index (so that every row, and every sum
//                   over it, has one order), and K_kl for each, a lane per entry
//   centeredSparseKernel  the conjugate gradients (same start, preconditioner, stopping rule and per-component
//                   iteration as the kernel above) in one cooperative launch, two grid barriers per iteration
// Rows are stored row-major (entry e of row k at k kCgRowCapacity + e), so that the kProductLanes threads that share a
// row in the products read its entries coalesced.  A cell or a row over its capacity sets a flag; the host then
// runs the spread-and-gather kernel for that step.
// ------------------------------------------------------------------------------------------------------

constexpr int kCgCellEdge = 4;      // nodes per cell edge (no less than the widest stencil)
constexpr int kCgCellCapacity = 64; // particles per cell
constexpr int kCgRowCapacity = 128; // entries per row of K
constexpr int kSolveThreads = 1024; // threads per block of the solve (one block per SM: few barrier arrivals)

struct SparseCg {
    int4* axisIndex;       // 3 per particle: the stencil's node indices on each axis (-1 past the width)
    double2* axisWeight;   // 6 per particle: the stencil's weights on each axis, [2 axis + 0/1] = entries 0-1 / 2-3
    int4* firstIndex;      // the first stencil index on each axis
    int* cellOf;           // cell of each particle
    unsigned* cellCount;   // particles per cell (cleared by the solve kernel)
    int4* cellList;        // kCgCellCapacity per cell: the particle and its first stencil index on each axis
    int* rowCount;         // entries per row
    int* rowIndex;         // entry e of row k at k kCgRowCapacity + e: the column particle
    double* rowValue;      // K_kl, same layout
    double* Ap;            // A p, 3 per particle
    double* slotSums;      // per particle: sum w u over its fluid slots (3) and sum w^2/rho (written by the rows)
    int* overflow;         // nonzero: a cell or a row over its capacity
    int cells[3];          // cells per axis
};

__global__ void __launch_bounds__(kThreads)
cgBinKernel(CouplingView c, SparseCg g) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < c.np; i += gridDim.x*blockDim.x) {
        const int4 first = g.firstIndex[i];
        const int cell[3] = {min(first.x/kCgCellEdge, g.cells[0] - 1), min(first.y/kCgCellEdge, g.cells[1] - 1),
                             min(first.z/kCgCellEdge, g.cells[2] - 1)};
        int key = cell[0] + g.cells[0]*(cell[1] + g.cells[1]*cell[2]);
        g.cellOf[i] = key;
        unsigned slot = atomicAdd(&g.cellCount[key], 1u);
        if (slot < (unsigned) kCgCellCapacity)
            g.cellList[(long long) key*kCgCellCapacity + slot] = make_int4(i, first.x, first.y, first.z);
        else
            atomicExch(g.overflow, 1);
    }
}

// Periodic distance of two lattice indices on an axis of n nodes.
__device__ __forceinline__ int periodicDistance(int a, int b, int n) {
    int d = abs(a - b);
    return min(d, n - d);
}

// W: the stencil width when known at compile time (0: c.width).  With W = 4 in single precision a row of k's w/rho
// (4 x-adjacent slots) is one 16-byte shared-memory load in the values' loop.
template <typename R, int W>
__global__ void __launch_bounds__(kThreads, 4)
cgRowsKernel(CouplingView c, const int* __restrict__ slotNode, const R* __restrict__ slotWeight,
             const unsigned* __restrict__ nodeStamp, unsigned stamp, const typename Vec4<R>::type* __restrict__ nodeU,
             SparseCg g) {
    __shared__ int candidates[kThreads/32][kCgRowCapacity];
    __shared__ int sorted[kThreads/32][kCgRowCapacity];
    __shared__ __align__(16) R rowCoef[kThreads/32][64];
    __shared__ int cellEnd[kThreads/32][32], cellStart[kThreads/32][32], cellId[kThreads/32][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int* list = candidates[warp];
    const int firstWarp = (blockIdx.x*blockDim.x + threadIdx.x) >> 5;
    const int warps = (gridDim.x*blockDim.x) >> 5;
    const int size[3] = {c.nx, c.ny, c.nz};
    const int w = W > 0 ? W : c.width, S = W > 0 ? W*W*W : c.slots;
    for (int k = firstWarp; k < c.np; k += warps) {
        // The particle's sums over its slots for the solve's right-hand side and diagonal (ReferenceLBMKernels.cpp:
        // 758-782): u = sum w u_node over the fluid slots and sum w^2/rho; they need no velocities or forces.
        // The slot's moments are its node's from the stencil pass (a node that no slot claimed in the pass, a solid
        // one, has none: rho = 0), and (w/rho)_k, the row's factor for K, goes to shared memory.
        double su[4] = {0, 0, 0, 0};
        for (int s = lane; s < S; s += 32) {
            const long long t = (long long) k*S + s;
            const R weight = slotWeight[t];
            const long long node = slotNode[t];
            typename Vec4<R>::type u = Vec4<R>::make(0, 0, 0, 0);
            if (weight != (R) 0 && nodeStamp[node] == stamp)
                u = nodeU[node];
            const double wt = (double) weight, rho = (double) u.w;
            rowCoef[warp][s] = (R) (rho > 0 ? wt/rho : 0.0);
            if (u.w > 0) {
                su[0] += (double) u.x*wt;
                su[1] += (double) u.y*wt;
                su[2] += (double) u.z*wt;
                su[3] += wt*wt/(double) u.w;
            }
        }
        for (int d = 0; d < 4; d++)
            su[d] = warpSum(su[d]);
        if (lane == 0)
            reinterpret_cast<double4*>(g.slotSums)[k] = make_double4(su[0], su[1], su[2], su[3]);
        const int4 fk = g.firstIndex[k];
        const int key = g.cellOf[k];
        const int keyYZ = key/g.cells[0];
        const int home[3] = {key - keyYZ*g.cells[0], keyYZ%g.cells[1], keyYZ/g.cells[1]};
        // Lane j < 27 takes the neighbouring cell (j%3 - 1, j/3%3 - 1, j/9 - 1); a cell that an axis with fewer than
        // 3 cells reaches twice is taken once (by its first offset).  The offsets are -1, 0 or 1, so one conditional
        // wrap replaces the modulo (whose integer divisions by the runtime cell counts were a quarter of the kernel's
        // instructions).
        int cell = -1, members = 0;
        if (lane < 27) {
            const int off[3] = {lane%3 - 1, (lane/3)%3 - 1, lane/9 - 1};
            bool first = true;
            int cc[3];
            for (int a = 0; a < 3; a++) {
                const int n = g.cells[a];
                const int v = home[a] + off[a];
                cc[a] = v < 0 ? v + n : (v >= n ? v - n : v);
                if (n < 3)
                    for (int d = -1; d < off[a]; d++) {
                        const int u = home[a] + d;
                        first &= (u < 0 ? u + n : (u >= n ? u - n : u)) != cc[a];
                    }
            }
            if (first) {
                cell = cc[0] + g.cells[0]*(cc[1] + g.cells[1]*cc[2]);
                members = min((int) g.cellCount[cell], kCgCellCapacity);
            }
        }
        // Exclusive scan of the member counts over the lanes.
        int start = members;
        for (int d = 1; d < 32; d *= 2) {
            const int v = __shfl_up_sync(0xFFFFFFFFu, start, d);
            if (lane >= d)
                start += v;
        }
        const int total = __shfl_sync(0xFFFFFFFFu, start, 31);
        cellEnd[warp][lane] = lane < 27 ? start : 0x7FFFFFFF;
        cellStart[warp][lane] = start - members;
        cellId[warp][lane] = cell;
        __syncwarp();
        int found = 0;     // the same in every lane
        // Four rounds of 32 members at a time, their loads issued together.
        for (int base = 0; base < total; base += 128) {
            int lq[4];
            bool nq[4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int e = base + 32*r + lane;
                lq[r] = -1;
                nq[r] = false;
                if (e < total) {
                    // The cell holding member e: the first of the 27 whose running end exceeds e.
                    int lo = 0, hi = 26;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (cellEnd[warp][mid] > e)
                            hi = mid;
                        else
                            lo = mid + 1;
                    }
                    const int4 m = g.cellList[(long long) cellId[warp][lo]*kCgCellCapacity + (e - cellStart[warp][lo])];
                    lq[r] = m.x;
                    nq[r] = periodicDistance(m.y, fk.x, size[0]) < c.width &&
                            periodicDistance(m.z, fk.y, size[1]) < c.width &&
                            periodicDistance(m.w, fk.z, size[2]) < c.width;
                }
            }
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const unsigned ballot = __ballot_sync(0xFFFFFFFFu, nq[r]);
                const int at = found + __popc(ballot & ((1u << lane) - 1u));
                if (nq[r] && at < kCgRowCapacity)
                    list[at] = lq[r];
                found += __popc(ballot);
            }
        }
        __syncwarp();
        if (found > kCgRowCapacity) {
            if (lane == 0)
                atomicExch(g.overflow, 1);
            found = kCgRowCapacity;
        }
        // Rank sort (particle indices are distinct).
        for (int j = lane; j < found; j += 32) {
            const int v = list[j];
            int rank = 0;
            for (int i = 0; i < found; i++)
                rank += list[i] < v;
            sorted[warp][rank] = v;
        }
        __syncwarp();
        // K_kl = sum over k's slots (ix, iy, iz) of (w/rho)_k times l's weight at the same node, the product of l's
        // axis weights at the entries with k's indices (on each axis the first such entry: later duplicates, at
        // clamped open faces, have weight zero).  Lanes over the row's entries.
        const int4 ik[3] = {g.axisIndex[3*k], g.axisIndex[3*k + 1], g.axisIndex[3*k + 2]};
        for (int j = lane; j < found; j += 32) {
            const int l = sorted[warp][j];
            // In the precision of the fluid's arithmetic (the slots' w/rho are stored in it).
            R shifted[3][4];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const int4 il = g.axisIndex[3*l + a];
                const double2 w01 = g.axisWeight[6*l + 2*a], w23 = g.axisWeight[6*l + 2*a + 1];
                const int mine[4] = {ik[a].x, ik[a].y, ik[a].z, ik[a].w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    double v = 0.0;
                    if (mine[i] >= 0) {
                        if (il.w == mine[i]) v = w23.y;
                        if (il.z == mine[i]) v = w23.x;
                        if (il.y == mine[i]) v = w01.y;
                        if (il.x == mine[i]) v = w01.x;
                    }
                    shifted[a][i] = (R) v;
                }
            }
            R K = 0;
#pragma unroll
            for (int iz = 0; iz < 4; iz++) {
                if (iz >= w || shifted[2][iz] == (R) 0)
                    continue;
#pragma unroll
                for (int iy = 0; iy < 4; iy++) {
                    if (iy >= w || shifted[1][iy] == (R) 0)
                        continue;
                    const R wyz = shifted[1][iy]*shifted[2][iz];
                    if constexpr (W == 4 && std::is_same<R, float>::value) {
                        const float4 cf = *reinterpret_cast<const float4*>(&rowCoef[warp][4*(iy + 4*iz)]);
                        K += cf.x*(shifted[0][0]*wyz);
                        K += cf.y*(shifted[0][1]*wyz);
                        K += cf.z*(shifted[0][2]*wyz);
                        K += cf.w*(shifted[0][3]*wyz);
                    }
                    else {
#pragma unroll
                        for (int ix = 0; ix < 4; ix++)
                            if (ix < w)
                                K += rowCoef[warp][ix + w*(iy + w*iz)]*(shifted[0][ix]*wyz);
                    }
                }
            }
            g.rowIndex[(long long) k*kCgRowCapacity + j] = l;
            g.rowValue[(long long) k*kCgRowCapacity + j] = (double) K;
        }
        if (lane == 0)
            g.rowCount[k] = found;
        __syncwarp();
    }
}

// (K v)_k for the three components of v, by the kProductLanes threads of a row (entries sub, sub + kProductLanes, ...,
// then the sum over the lanes), in all of them; k < 0: no row (the threads still take part in the exchange).  Called
// by every thread of the warp.
constexpr int kProductLanes = 4;

__device__ __forceinline__ void rowProduct(const SparseCg& g, int k, const double* v, double out[3]) {
    double s0 = 0, s1 = 0, s2 = 0;
    if (k >= 0) {
        const int n = g.rowCount[k];
        const int* index = g.rowIndex + (long long) k*kCgRowCapacity;
        const double* value = g.rowValue + (long long) k*kCgRowCapacity;
#pragma unroll 4
        for (int e = threadIdx.x%kProductLanes; e < n; e += kProductLanes) {
            const int l = index[e];
            const double K = value[e];
            s0 += K*v[3*l];
            s1 += K*v[3*l+1];
            s2 += K*v[3*l+2];
        }
    }
#pragma unroll
    for (int o = 1; o < kProductLanes; o <<= 1) {
        s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, o);
        s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, o);
        s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, o);
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
}

template <typename R>
__global__ void __launch_bounds__(kSolveThreads, 1)
centeredSparseKernel(FluidView f, CouplingView c, const double* __restrict__ vel, const double* __restrict__ fin,
                     const int* __restrict__ slotNode, const R* __restrict__ slotWeight,
                     const typename Vec4<R>::type* __restrict__ slotU, long long step, int isStep, double tolerance,
                     int maxIterations, CgBuffers b, SparseCg g, double* fout, R* reaction, uint32_t* mask,
                     double* wall) {
    const int lane = threadIdx.x & 31;
    const int firstWarp = (blockIdx.x*blockDim.x + threadIdx.x) >> 5;
    const int firstThread = blockIdx.x*blockDim.x + threadIdx.x, threads = gridDim.x*blockDim.x;
    // The rows of this block (a contiguous range).
    const int rowBegin = (int) ((long long) c.np*blockIdx.x/gridDim.x);
    const int rowEnd = (int) ((long long) c.np*(blockIdx.x + 1)/gridDim.x);
    const int S = c.slots;
    const double a = c.a;
    // The cell list has been read (by the rows kernel): empty it for the next step.
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < c.np; i += gridDim.x*blockDim.x)
        g.cellCount[g.cellOf[i]] = 0u;
    if (*((volatile int*) g.overflow) != 0)
        return;
    // Right-hand side, diagonal and the start F = rhs/diag (ReferenceLBMKernels.cpp:758-782, 839-840), a thread per
    // particle, from the sums over its slots that the rows kernel formed.
    for (int i = firstThread; i < c.np; i += threads) {
        const double4 su = reinterpret_cast<const double4*>(g.slotSums)[i];
        const double u[3] = {su.x, su.y, su.z}, self = su.w;
        double m = c.mass[i];
        double xi[3] = {0, 0, 0};
        if (c.randomForce)
            particleNoise(c.seed, i, step, xi);
        double diag = (1.0 + a)/m + a*self;
        for (int d = 0; d < 3; d++) {
            double known = vel[3*i+d]*(1.0/c.velocityScale) + fin[3*i+d]*(c.h/(m*c.forceScale));
            double v = (known - u[d])*(-c.gamma*m);
            if (c.randomForce)
                v += xi[d]*sqrt(2.0*c.gamma*m*c.kT);
            double rhs = v*(1.0/m);
            b.rhs[3*i+d] = rhs;
            b.F[3*i+d] = rhs*(1.0/diag);
        }
        b.diag[i] = diag;
    }
    if (!gridSync(b.barrier, b.status, b.pollLimit))
        return;
    // r = rhs - A F, z = r/diag, p = z; r.z, the norm of the right-hand side and r.r per component.
    double acc[kPartial] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int base = rowBegin; base < rowEnd; base += blockDim.x/kProductLanes) {
        const int i = base + threadIdx.x/kProductLanes;
        double g3[3];
        rowProduct(g, i < rowEnd ? i : -1, b.F, g3);
        if (i >= rowEnd || threadIdx.x%kProductLanes != 0)
            continue;
        double m = c.mass[i], diag = b.diag[i];
        for (int d = 0; d < 3; d++) {
            double AF = b.F[3*i+d]*((1.0 + a)/m) + g3[d]*a;
            double rhs = b.rhs[3*i+d];
            double r = rhs - AF;
            double z = r*(1.0/diag);
            b.r[3*i+d] = r;
            b.z[3*i+d] = z;
            b.p[3*i+d] = z;
            acc[d] += r*z;
            acc[3+d] += rhs*rhs;
            acc[6+d] += r*r;
        }
    }
    blockSumStore(acc, b.partials[1]);
    if (!gridSync(b.barrier, b.status, b.pollLimit))
        return;
    double tot[kPartial];
    reducePartials(b.partials[1], gridDim.x, tot);
    double rz[3] = {tot[0], tot[1], tot[2]}, norm[3] = {tot[3], tot[4], tot[5]}, residual[3] = {tot[6], tot[7], tot[8]};
    double beta[3] = {0, 0, 0};
    int iteration = 0;
    bool failed = false;       // the same in every block: every decision comes from the same reduced sums
    for (;; iteration++) {
        bool converged = true;
        for (int d = 0; d < 3; d++)
            if (residual[d] > tolerance*tolerance*norm[d])
                converged = false;
        if (converged)
            break;
        if (iteration == maxIterations) {
            if (firstWarp == 0 && lane == 0)
                atomicExch(b.status, LBM_ERR_CG_NOT_CONVERGED);
            failed = true;
            break;
        }
        // p = z + beta p and A p = A z + beta A p (p = z at the first iteration), with p.Ap.
        double acc3[kPartial] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int base = rowBegin; base < rowEnd; base += blockDim.x/kProductLanes) {
            const int i = base + threadIdx.x/kProductLanes;
            double g3[3];
            rowProduct(g, i < rowEnd ? i : -1, b.z, g3);
            if (i >= rowEnd || threadIdx.x%kProductLanes != 0)
                continue;
            double m = c.mass[i];
            for (int d = 0; d < 3; d++) {
                double z = b.z[3*i+d];
                double Az = z*((1.0 + a)/m) + g3[d]*a;
                double p = z, Ap = Az;
                if (iteration > 0) {
                    p = z + beta[d]*b.p[3*i+d];
                    Ap = Az + beta[d]*g.Ap[3*i+d];
                }
                b.p[3*i+d] = p;
                g.Ap[3*i+d] = Ap;
                acc3[d] += p*Ap;
            }
        }
        blockSumStore(acc3, b.partials[0]);
        if (!gridSync(b.barrier, b.status, b.pollLimit))
            return;
        reducePartials(b.partials[0], gridDim.x, tot);
        double alpha[3];
        for (int d = 0; d < 3; d++)
            alpha[d] = (tot[d] > 0 ? rz[d]/tot[d] : 0.0);
        double acc4[kPartial] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = rowBegin + threadIdx.x; i < rowEnd; i += blockDim.x) {
            double diag = b.diag[i];
            for (int d = 0; d < 3; d++) {
                b.F[3*i+d] += alpha[d]*b.p[3*i+d];
                double r = b.r[3*i+d] - alpha[d]*g.Ap[3*i+d];
                b.r[3*i+d] = r;
                double z = r*(1.0/diag);
                b.z[3*i+d] = z;
                acc4[d] += r*z;
                acc4[3+d] += r*r;
            }
        }
        blockSumStore(acc4, b.partials[1]);
        if (!gridSync(b.barrier, b.status, b.pollLimit))
            return;
        reducePartials(b.partials[1], gridDim.x, tot);
        for (int d = 0; d < 3; d++) {
            beta[d] = (rz[d] > 0 ? tot[d]/rz[d] : 0.0);
            rz[d] = tot[d];
            residual[d] = tot[3+d];
        }
    }
    if (firstWarp == 0 && lane == 0)
        *b.iterations = iteration;
    if (failed)
        return;
    // Forces and reactions (ReferenceLBMKernels.cpp:889-900): a thread per particle, then a thread per slot.
    for (int i = firstThread; i < c.np; i += threads)
        for (int d = 0; d < 3; d++)
            fout[3*i+d] = b.F[3*i+d]*c.forceScale;
    // (np S < 2^31, which the constructor checks: the slots are indexed by int.)
    if (isStep) {
        const int total = c.np*S;
        for (int t = firstThread; t < total; t += threads) {
            const int i = t/S;
            const double w = (double) slotWeight[t];
            if (w != 0.0)
                addReaction<R>(f, c, reaction, mask, wall, slotNode[t], -w*b.F[3*i], -w*b.F[3*i+1], -w*b.F[3*i+2]);
        }
    }
}

// Clear the reaction of the slots of the last step (and their mask words).
template <typename R>
__global__ void clearReactionKernel(FluidView f, const int* slotNode, long long total, R* reaction, uint32_t* mask) {
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < total; t += (long long) gridDim.x*blockDim.x) {
        const unsigned node = (unsigned) slotNode[t];
        *reinterpret_cast<typename Vec4<R>::type*>(reaction + 4*(size_t) node) = Vec4<R>::make(0, 0, 0, 0);
        const unsigned row = node/(unsigned) f.nx;
        const int x = (int) (node - row*(unsigned) f.nx);
        mask[(size_t) row*f.wordsPerRow + x/32] = 0u;
    }
}

// Reflection at the walls (beginStep, ReferenceLBMKernels.cpp:315-338).
__global__ void reflectKernel(CouplingView c, const double* pos, double* vel, double cellMass, double* wall) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < c.np; i += gridDim.x*blockDim.x) {
        int size[3] = {c.nx, c.ny, c.nz};
        int near[3], index[3][2];
        double weight[3][2];
        for (int a = 0; a < 3; a++) {
            double s = latticeCoordinate(pos[3*i+a], c.dx, size[a]);
            near[a] = ((int) floor(s + 0.5))%size[a];
            double lower = floor(s);
            index[a][0] = ((int) lower)%size[a];
            index[a][1] = (index[a][0] + 1)%size[a];
            weight[a][1] = s - lower;
            weight[a][0] = 1.0 - weight[a][1];
        }
        long long node = near[0] + (long long) c.nx*(near[1] + (long long) c.ny*near[2]);
        if (!isSolid(c.solidMask, c.wordsPerRow, c.nx, node))
            continue;
        double solid[2][2][2];
        for (int x = 0; x < 2; x++)
            for (int y = 0; y < 2; y++)
                for (int z = 0; z < 2; z++)
                    solid[x][y][z] = isSolid(c.solidMask, c.wordsPerRow, c.nx,
                                             index[0][x] + (long long) c.nx*(index[1][y] + (long long) c.ny*index[2][z])) ? 1.0 : 0.0;
        double n[3] = {0, 0, 0};
        for (int p = 0; p < 2; p++)
            for (int q = 0; q < 2; q++) {
                n[0] += weight[1][p]*weight[2][q]*(solid[1][p][q] - solid[0][p][q]);
                n[1] += weight[0][p]*weight[2][q]*(solid[p][1][q] - solid[p][0][q]);
                n[2] += weight[0][p]*weight[1][q]*(solid[p][q][1] - solid[p][q][0]);
            }
        double* v = &vel[3*i];
        if (v[0]*n[0] + v[1]*n[1] + v[2]*n[2] > 0) {
            for (int a = 0; a < 3; a++) {
                atomicAdd(&wall[a], v[a]*(2.0*c.mass[i]*cellMass));
                v[a] = -v[a];
            }
        }
    }
}

__global__ void addForcesKernel(const double* fout, double* forces, int count) {
    for (int i = blockIdx.x*blockDim.x + threadIdx.x; i < count; i += gridDim.x*blockDim.x)
        forces[i] += fout[i];
}

int widthOf(int stencil) {
    return stencil == LBM_STENCIL_TRILINEAR ? 2 : stencil == LBM_STENCIL_THREEPOINT ? 3 : stencil == LBM_STENCIL_KEYS ? 4 : 1;
}

// Blocks for one warp per particle.
int warpGrid(long long particles) {
    return (int) std::max(1LL, std::min(4736LL, (particles*32 + kThreads - 1)/kThreads));
}

} // namespace

// ------------------------------------------------------------------------------------------------------
// Host side.
// ------------------------------------------------------------------------------------------------------

struct CouplingEngine::Device {
    int* slotNode = nullptr;
    void* slotWeight = nullptr;   // R per slot
    void* slotU = nullptr;        // 4 R per slot
    void* coef = nullptr;         // R per slot (centred stencil)
    unsigned* keys[2] = {nullptr, nullptr};
    int* values[2] = {nullptr, nullptr};
    unsigned* hist = nullptr;
    CgBuffers cg;
    SparseCg sparse;
    int sparseGrid = 0;
    void* spread = nullptr;
    int4* axisIndex = nullptr;      // per particle: 3, the stencil's node indices on each axis
    double2* axisWeight = nullptr;  // per particle: 6, the stencil's weights on each axis
    int4* firstIndex = nullptr;     // per particle: the first stencil index on each axis
    unsigned* nodeStamp = nullptr;  // per node: the stamp of the last stencil pass that computed its moments
    void* nodeU = nullptr;          // per node: 4 R, the moments of that pass
    unsigned stamp = 0;
    double* reflectWall = nullptr;
    int cgGrid = 0;
    size_t histCount = 0;
};

CouplingEngine::CouplingEngine(const LbmLatticeParameters& l, FluidEngine& f, const Geometry& g, int n,
                               const double* masses, cudaStream_t s)
        : lattice(l), fluid(f), stream(s), np(n), storageType(f.storage()), posDev(nullptr), velDev(nullptr),
          forceInDev(nullptr), forceOutDev(nullptr), massDev(nullptr), wallDev(nullptr), statusDev(nullptr),
          pinned(nullptr), dev(new Device()) {
    (void) g;
    std::memset(&dev->cg, 0, sizeof(CgBuffers));
    std::memset(&dev->sparse, 0, sizeof(SparseCg));
    stencilSlots = widthOf(l.interpolation_stencil);
    stencilSlots = stencilSlots*stencilSlots*stencilSlots;
    bool f64 = storageType == LBM_STORAGE_F64;
    size_t r = f64 ? 8 : 4;
    try {
        // The stencil slots of all particles are indexed by int in the solves.
        if ((long long) np*stencilSlots >= (1LL << 31))
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: too many coupled particles for the interpolation stencil "
                        "(particles x stencil nodes must stay below 2^31)");
        size_t v3 = sizeof(double)*3*(size_t) np;
        CUDA_CHECK(cudaMalloc(&posDev, v3));
        CUDA_CHECK(cudaMalloc(&velDev, v3));
        CUDA_CHECK(cudaMalloc(&forceInDev, v3));
        CUDA_CHECK(cudaMalloc(&forceOutDev, v3));
        CUDA_CHECK(cudaMemsetAsync(forceOutDev, 0, v3, stream));
        CUDA_CHECK(cudaMemsetAsync(forceInDev, 0, v3, stream));
        CUDA_CHECK(cudaMalloc(&massDev, sizeof(double)*np));
        double cellMass = l.density*l.dx*l.dx*l.dx;
        std::vector<double> m(np);
        for (int i = 0; i < np; i++)
            m[i] = masses[i]/cellMass;
        CUDA_CHECK(cudaMemcpy(massDev, m.data(), sizeof(double)*np, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMalloc(&wallDev, sizeof(double)*8));
        CUDA_CHECK(cudaMemsetAsync(wallDev, 0, sizeof(double)*8, stream));
        dev->reflectWall = wallDev + 4;
        CUDA_CHECK(cudaMalloc(&statusDev, sizeof(int)*4));
        CUDA_CHECK(cudaMemsetAsync(statusDev, 0, sizeof(int)*4, stream));
        size_t slots = (size_t) np*stencilSlots;
        CUDA_CHECK(cudaMalloc(&dev->slotNode, sizeof(int)*slots));
        CUDA_CHECK(cudaMalloc(&dev->slotWeight, r*slots));
        CUDA_CHECK(cudaMalloc(&dev->slotU, 4*r*slots));
        CUDA_CHECK(cudaMemsetAsync(dev->slotNode, 0, sizeof(int)*slots, stream));
        CUDA_CHECK(cudaMemsetAsync(dev->slotWeight, 0, r*slots, stream));
        CUDA_CHECK(cudaMalloc(&dev->axisIndex, sizeof(int4)*3*(size_t) np));
        CUDA_CHECK(cudaMalloc(&dev->axisWeight, sizeof(double2)*6*(size_t) np));
        CUDA_CHECK(cudaMalloc(&dev->firstIndex, sizeof(int4)*(size_t) np));
        CUDA_CHECK(cudaMalloc(&dev->nodeStamp, sizeof(unsigned)*(size_t) f.numNodes()));
        CUDA_CHECK(cudaMemsetAsync(dev->nodeStamp, 0, sizeof(unsigned)*(size_t) f.numNodes(), stream));
        CUDA_CHECK(cudaMalloc(&dev->nodeU, 4*r*(size_t) f.numNodes()));
        if (l.drag_scheme == LBM_DRAG_CENTERED && l.interpolation_stencil == LBM_STENCIL_NEAREST) {
            int blocks = (np + kSortItems - 1)/kSortItems;
            dev->histCount = (size_t) 256*blocks;
            CUDA_CHECK(cudaMalloc(&dev->hist, sizeof(unsigned)*dev->histCount));
            for (int k = 0; k < 2; k++) {
                CUDA_CHECK(cudaMalloc(&dev->keys[k], sizeof(unsigned)*np));
                CUDA_CHECK(cudaMalloc(&dev->values[k], sizeof(int)*np));
            }
        }
        if (l.drag_scheme == LBM_DRAG_CENTERED && l.interpolation_stencil != LBM_STENCIL_NEAREST) {
            CgBuffers& b = dev->cg;
            CUDA_CHECK(cudaMalloc(&b.rhs, v3));
            CUDA_CHECK(cudaMalloc(&b.diag, sizeof(double)*np));
            CUDA_CHECK(cudaMalloc(&b.F, v3));
            CUDA_CHECK(cudaMalloc(&b.r, v3));
            CUDA_CHECK(cudaMalloc(&b.z, v3));
            CUDA_CHECK(cudaMalloc(&b.p, v3));
            CUDA_CHECK(cudaMalloc(&dev->coef, r*slots));
            b.status = statusDev;
            b.iterations = statusDev + 1;
            b.pollLimit = kDefaultBarrierPolls;
            // The arrival counter of the grid barriers is statusDev[3]: the memset of the status words before every
            // cooperative launch clears it too.
            b.barrier = reinterpret_cast<unsigned*>(statusDev + 3);
            int device = 0, sms = 0, perSM = 0;
            CUDA_CHECK(cudaGetDevice(&device));
            CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
            if (f64)
                CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, centeredStencilKernel<double>, kThreads, 0));
            else
                CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, centeredStencilKernel<float>, kThreads, 0));
            long long wanted = ((long long) np*32 + kThreads - 1)/kThreads;     // one warp per particle
            dev->cgGrid = (int) std::max(1LL, std::min(wanted, (long long) std::max(1, perSM)*sms));
            for (int k = 0; k < 2; k++)
                CUDA_CHECK(cudaMalloc(&b.partials[k], sizeof(double)*kPartial*(size_t) dev->cgGrid));
            CUDA_CHECK(cudaMalloc(&dev->spread, 4*r*(size_t) f.numNodes()));
            CUDA_CHECK(cudaMemsetAsync(dev->spread, 0, 4*r*(size_t) f.numNodes(), stream));
            // The explicit coupling matrix (centeredSparseKernel) and its cell list.
            SparseCg& g = dev->sparse;
            int size[3] = {l.nx, l.ny, l.nz};
            long long cells = 1;
            for (int a = 0; a < 3; a++) {
                g.cells[a] = std::max(1, size[a]/kCgCellEdge);
                cells *= g.cells[a];
            }
            g.axisIndex = dev->axisIndex;
            g.axisWeight = dev->axisWeight;
            g.firstIndex = dev->firstIndex;
            CUDA_CHECK(cudaMalloc(&g.cellOf, sizeof(int)*(size_t) np));
            CUDA_CHECK(cudaMalloc(&g.cellCount, sizeof(unsigned)*(size_t) cells));
            CUDA_CHECK(cudaMemsetAsync(g.cellCount, 0, sizeof(unsigned)*(size_t) cells, stream));
            CUDA_CHECK(cudaMalloc(&g.cellList, sizeof(int4)*kCgCellCapacity*(size_t) cells));
            CUDA_CHECK(cudaMalloc(&g.rowCount, sizeof(int)*(size_t) np));
            CUDA_CHECK(cudaMalloc(&g.rowIndex, sizeof(int)*kCgRowCapacity*(size_t) np));
            CUDA_CHECK(cudaMalloc(&g.rowValue, sizeof(double)*kCgRowCapacity*(size_t) np));
            CUDA_CHECK(cudaMalloc(&g.Ap, v3));
            CUDA_CHECK(cudaMalloc(&g.slotSums, sizeof(double)*4*(size_t) np));
            g.overflow = statusDev + 2;
            if (f64)
                CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, centeredSparseKernel<double>, kSolveThreads, 0));
            else
                CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, centeredSparseKernel<float>, kSolveThreads, 0));
            long long wantedSolve = ((long long) np*32 + kSolveThreads - 1)/kSolveThreads;
            // No more blocks than the partial records hold (cgGrid of the 256-thread solve).
            dev->sparseGrid = (int) std::max(1LL, std::min(std::min(wantedSolve, (long long) std::max(1, perSM)*sms),
                                                          (long long) dev->cgGrid));
        }
        CUDA_CHECK(cudaMallocHost(&pinned, v3));
        CUDA_CHECK(cudaStreamSynchronize(stream));
    }
    catch (...) {
        release();
        throw;
    }
    setParameters(l);
}

void CouplingEngine::release() {
    if (side != nullptr) {
        cudaStreamSynchronize(side);
        cudaEventDestroy(begun);
        cudaEventDestroy(ready);
        cudaStreamDestroy(side);
        side = nullptr;
    }
    cudaFree(posDev); cudaFree(velDev); cudaFree(forceInDev); cudaFree(forceOutDev); cudaFree(massDev);
    cudaFree(wallDev); cudaFree(statusDev);
    posDev = velDev = forceInDev = forceOutDev = massDev = wallDev = nullptr;
    statusDev = nullptr;
    if (pinned)
        cudaFreeHost(pinned);
    pinned = nullptr;
    if (dev) {
        cudaFree(dev->slotNode); cudaFree(dev->slotWeight); cudaFree(dev->slotU); cudaFree(dev->coef);
        cudaFree(dev->nodeStamp); cudaFree(dev->nodeU);
        cudaFree(dev->axisIndex); cudaFree(dev->axisWeight); cudaFree(dev->firstIndex);
        for (int k = 0; k < 2; k++) {
            cudaFree(dev->keys[k]);
            cudaFree(dev->values[k]);
        }
        cudaFree(dev->hist);
        CgBuffers& b = dev->cg;
        cudaFree(b.rhs); cudaFree(b.diag); cudaFree(b.F); cudaFree(b.r); cudaFree(b.z); cudaFree(b.p);
        cudaFree(b.partials[0]); cudaFree(b.partials[1]);
        cudaFree(dev->spread);
        SparseCg& g = dev->sparse;
        cudaFree(g.cellOf); cudaFree(g.cellCount); cudaFree(g.cellList);
        cudaFree(g.rowCount); cudaFree(g.rowIndex); cudaFree(g.rowValue); cudaFree(g.Ap); cudaFree(g.slotSums);
        delete dev;
        dev = nullptr;
    }
}

CouplingEngine::~CouplingEngine() {
    release();
}

void CouplingEngine::setParameters(const LbmLatticeParameters& l) {
    lattice = l;
}

void CouplingEngine::load(const LbmParticleArrays* p, bool withForces) {
    size_t v3 = sizeof(double)*3*(size_t) np;
    cudaMemcpyKind kind = p->memory == LBM_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CUDA_CHECK(cudaMemcpyAsync(posDev, p->positions, v3, kind, stream));
    CUDA_CHECK(cudaMemcpyAsync(velDev, p->velocities, v3, kind, stream));
    if (withForces)
        CUDA_CHECK(cudaMemcpyAsync(forceInDev, p->forces, v3, kind, stream));
}

void CouplingEngine::reflect(const LbmParticleArrays* p, double wallMomentum[3]) {
    load(p, false);
    const FluidView& f = fluid.deviceView();
    CouplingView c = makeCouplingView(lattice, f, np, 1, massDev);
    CUDA_CHECK(cudaMemsetAsync(dev->reflectWall, 0, sizeof(double)*3, stream));
    double cellMass = lattice.density*lattice.dx*lattice.dx*lattice.dx;
    reflectKernel<<<std::max(1, std::min(1184, (np + kThreads - 1)/kThreads)), kThreads, 0, stream>>>(c, posDev, velDev, cellMass, dev->reflectWall);
    CUDA_CHECK(cudaGetLastError());
    fluid.launches++;
    size_t v3 = sizeof(double)*3*(size_t) np;
    cudaMemcpyKind kind = p->memory == LBM_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CUDA_CHECK(cudaMemcpyAsync(p->velocities, velDev, v3, kind, stream));
    CUDA_CHECK(cudaMemcpyAsync(wallMomentum, dev->reflectWall, sizeof(double)*3, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

template <typename T, typename R>
static void launchStencil(const void* A, const FluidView& f, const CouplingView& c, const double* pos, int remove, int centred,
                          int* slotNode, void* slotWeight, void* slotU, unsigned* nodeStamp, unsigned stamp,
                          void* nodeU, int4* axisIndex, double2* axisWeight, int4* firstIndex, uint32_t* mark,
                          void* reaction, void* coef, cudaStream_t s) {
    typedef typename Vec4<R>::type V;
    long long total = (long long) c.np*c.slots;
    int grid = (int) std::max(1LL, std::min(4736LL, (total + kThreads - 1)/kThreads));
    stencilAxesKernel<<<std::max(1, (c.np + kThreads - 1)/kThreads), kThreads, 0, s>>>(c, pos, axisIndex, axisWeight,
                                                                                      firstIndex);
    // The stencil widths: 1 (nearest node), 2 (trilinear), 3 (three-point), 4 (Keys).
    auto claim = [&](auto w) {
        stencilClaimKernel<T, R, decltype(w)::value><<<grid, kThreads, 0, s>>>(
            (const T*) A, f, c, axisIndex, axisWeight, remove, centred, slotNode, (R*) slotWeight, nodeStamp, stamp,
            (V*) nodeU, mark, (R*) reaction);
    };
    switch (c.width) {
    case 1: claim(std::integral_constant<int, 1>()); break;
    case 2: claim(std::integral_constant<int, 2>()); break;
    case 3: claim(std::integral_constant<int, 3>()); break;
    case 4: claim(std::integral_constant<int, 4>()); break;
    default: claim(std::integral_constant<int, 0>()); break;
    }
    if (slotU != nullptr)
        stencilGatherKernel<R><<<grid, kThreads, 0, s>>>(c, slotNode, (const R*) slotWeight, nodeStamp, stamp,
                                                         (const V*) nodeU, (V*) slotU, (R*) coef);
}

// The moments of every slot from its node (the slot copy of the stencil pass), for the kernels that read them per slot.
template <typename R>
static void launchSlotMoments(const CouplingView& c, const int* slotNode, const void* slotWeight,
                              const unsigned* nodeStamp, unsigned stamp, const void* nodeU, void* slotU, cudaStream_t s) {
    typedef typename Vec4<R>::type V;
    long long total = (long long) c.np*c.slots;
    int grid = (int) std::max(1LL, std::min(4736LL, (total + kThreads - 1)/kThreads));
    stencilGatherKernel<R><<<grid, kThreads, 0, s>>>(c, slotNode, (const R*) slotWeight, nodeStamp, stamp,
                                                     (const V*) nodeU, (V*) slotU, (R*) nullptr);
}

// The cell list and the rows of the coupling matrix, after the status words are cleared (their overflow flag).
template <typename R>
void CouplingEngine::launchMatrix(const CouplingView* cv, cudaStream_t s) {
    const CouplingView& c = *cv;
    CUDA_CHECK(cudaMemsetAsync(statusDev, 0, sizeof(int)*4, s));
    cgBinKernel<<<std::max(1, std::min(1184, (np + kThreads - 1)/kThreads)), kThreads, 0, s>>>(c, dev->sparse);
    CUDA_CHECK(cudaGetLastError());
    auto rows = [&](auto w) {
        cgRowsKernel<R, decltype(w)::value><<<warpGrid(np), kThreads, 0, s>>>(
            c, dev->slotNode, (const R*) dev->slotWeight, dev->nodeStamp, dev->stamp,
            (const typename Vec4<R>::type*) dev->nodeU, dev->sparse);
    };
    switch (c.width) {
    case 2: rows(std::integral_constant<int, 2>()); break;
    case 3: rows(std::integral_constant<int, 3>()); break;
    case 4: rows(std::integral_constant<int, 4>()); break;
    default: rows(std::integral_constant<int, 0>()); break;
    }
    CUDA_CHECK(cudaGetLastError());
    fluid.launches += 2;
}

template <typename R>
void CouplingEngine::coupleWith(long long step, bool isStep, const CouplingView* cv, bool matrixReady) {
    const CouplingView& c = *cv;
    const FluidView& f = fluid.deviceView();
    bool centred = lattice.drag_scheme == LBM_DRAG_CENTERED;
    R* reaction = (R*) fluid.reactionBuffer();
    uint32_t* mask = nullptr;        // the stencil pass of the step flagged the nodes of its reactions
    const R* sw = (const R*) dev->slotWeight;
    const typename Vec4<R>::type* su = (const typename Vec4<R>::type*) dev->slotU;
    if (!centred) {
        explicitKernel<R><<<warpGrid(np), kThreads, 0, stream>>>(f, c, velDev, dev->slotNode, sw, su, step, isStep,
                                                                 forceOutDev, reaction, mask, wallDev);
        CUDA_CHECK(cudaGetLastError());
        fluid.launches++;
        return;
    }
    int gridP = std::max(1, std::min(1184, (np + kThreads - 1)/kThreads));
    if (lattice.interpolation_stencil == LBM_STENCIL_NEAREST) {
        // Sort the particles by node, stably (particle order within a node).
        nodeKeysKernel<<<gridP, kThreads, 0, stream>>>(dev->slotNode, np, dev->keys[0], dev->values[0]);
        CUDA_CHECK(cudaGetLastError());
        fluid.launches++;
        int bits = 1;
        while (bits < 32 && (1LL << bits) < f.n)
            bits++;
        int cur = radixSortByKey(dev->keys, dev->values, dev->hist, np, bits, stream);
        fluid.launches += 3*((bits + 7)/8);
        centeredNearestKernel<R><<<gridP, kThreads, 0, stream>>>(f, c, dev->keys[cur], dev->values[cur], velDev, forceInDev,
                                                                  su, step, isStep, forceOutDev, reaction, mask, wallDev);
        CUDA_CHECK(cudaGetLastError());
        fluid.launches++;
        return;
    }
    // Centred drag with a stencil: the conjugate gradients on the device (ReferenceLBMKernels.cpp:834-888, tolerance
    // 1e-13 in double; 1e-5 with single-precision arithmetic, as the reference's GPU platforms in single precision),
    // through the explicit coupling matrix; the spread-and-gather kernel serves a step whose cell list or matrix rows
    // overflow their capacity (and every step with LBM_B200_SPREAD_CG=1 in the environment, for comparisons).
    // The status words are cleared with the matrix (launchMatrix), or before the spread-and-gather solve below.
    CgBuffers b = dev->cg;
    SparseCg g = dev->sparse;
    double tolerance = std::is_same<R, double>::value ? 1e-13 : 1e-5;
    int maxIterations = cgMaxIterations;
    b.pollLimit = barrierPollLimit;
    long long stepArg = step;
    int isStepArg = isStep ? 1 : 0;
    R* spread = (R*) dev->spread;
    R* coef = (R*) dev->coef;
    double* fout = forceOutDev;
    double* wall = wallDev;
    double* fin = forceInDev;
    double* vel = velDev;
    int* sn = dev->slotNode;
    FluidView fv = f;
    CouplingView cc = c;
    int status[3] = {0, 0, 0};
    const bool spreadOnly = !matrixSolve();
    if (!spreadOnly) {
        if (!matrixReady)
            launchMatrix<R>(&c, stream);
        void* sparseArgs[] = {&fv, &cc, &vel, &fin, &sn, &sw, &su, &stepArg, &isStepArg, &tolerance, &maxIterations, &b,
                              &g, &fout, &reaction, &mask, &wall};
        CUDA_CHECK(cudaLaunchCooperativeKernel((const void*) centeredSparseKernel<R>, dev->sparseGrid, kSolveThreads,
                                               sparseArgs, 0, stream));
        fluid.launches++;
        CUDA_CHECK(cudaMemcpyAsync(status, statusDev, sizeof(int)*3, cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
    }
    if (spreadOnly || status[2] != 0) {
        launchSlotMomentsNow();
        CUDA_CHECK(cudaMemsetAsync(statusDev, 0, sizeof(int)*4, stream));
        void* args[] = {&fv, &cc, &vel, &fin, &sn, &sw, &su, &coef, &stepArg, &isStepArg, &tolerance, &maxIterations, &b,
                        &spread, &fout, &reaction, &mask, &wall};
        CUDA_CHECK(cudaLaunchCooperativeKernel((const void*) centeredStencilKernel<R>, dev->cgGrid, kThreads, args, 0, stream));
        fluid.launches++;
        CUDA_CHECK(cudaMemcpyAsync(status, statusDev, sizeof(int)*2, cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
        spreadSteps++;
    }
    lastIterations = status[1];
    if (status[0] == LBM_ERR_CG_NOT_CONVERGED)
        throw Error(LBM_ERR_CG_NOT_CONVERGED, "LBMForce: the centred drag with the interpolation stencil did not converge "
                    "in " + std::to_string(maxIterations) + " iterations of the conjugate gradients");
    if (status[0] == LBM_ERR_DEVICE_TIMEOUT)
        // The blocks left the solve at different barriers; the arrival counter holds a partial count, which the
        // memset before the next cooperative launch clears.
        throw Error(LBM_ERR_DEVICE_TIMEOUT, "LBMForce: a grid barrier of the conjugate gradients timed out");
}

void CouplingEngine::setSolverLimits(int maxIterations, long long barrierPolls) {
    if (maxIterations < 0 || barrierPolls < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_set_solver_limits: the limits must not be negative");
    cgMaxIterations = maxIterations > 0 ? maxIterations : kDefaultCgIterations;
    barrierPollLimit = barrierPolls > 0 ? barrierPolls : kDefaultBarrierPolls;
}

void CouplingEngine::launchStencilPass(const CouplingView& c, bool remove, bool mark, cudaStream_t s) {
    const FluidView& f = fluid.deviceView();
    uint32_t* m = mark ? fluid.reactMask() : nullptr;
    // The coupling matrix's rows read the node moments of their slots themselves; the per-slot copy then waits for
    // a step that falls back to the spread-and-gather solve (launchSlotMomentsNow).
    void* su = matrixSolve() ? nullptr : dev->slotU;
    slotMomentsPending = su == nullptr;
    void* cf = nullptr;
    bool centred = lattice.drag_scheme == LBM_DRAG_CENTERED;
    const void* A = fluid.inputArray();
    if (++dev->stamp == 0u) {     // the stamps wrapped around: no node may carry a stale stamp
        CUDA_CHECK(cudaMemsetAsync(dev->nodeStamp, 0, sizeof(unsigned)*(size_t) f.n, s));
        dev->stamp = 1u;
    }
    unsigned* ns = dev->nodeStamp;
    void* nu = dev->nodeU;
    unsigned st = dev->stamp;
    switch (storageType) {
    case LBM_STORAGE_F64: launchStencil<double, double>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, su, ns, st, nu, dev->axisIndex, dev->axisWeight, dev->firstIndex, m, m != nullptr ? fluid.reactionBuffer() : nullptr, cf, s); break;
    case LBM_STORAGE_F32: launchStencil<float, float>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, su, ns, st, nu, dev->axisIndex, dev->axisWeight, dev->firstIndex, m, m != nullptr ? fluid.reactionBuffer() : nullptr, cf, s); break;
    case LBM_STORAGE_F16: launchStencil<__half, float>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, su, ns, st, nu, dev->axisIndex, dev->axisWeight, dev->firstIndex, m, m != nullptr ? fluid.reactionBuffer() : nullptr, cf, s); break;
    default: launchStencil<__nv_bfloat16, float>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, su, ns, st, nu, dev->axisIndex, dev->axisWeight, dev->firstIndex, m, m != nullptr ? fluid.reactionBuffer() : nullptr, cf, s); break;
    }
    CUDA_CHECK(cudaGetLastError());
    fluid.launches += su != nullptr ? 3 : 2;
}

// The per-slot moments of the last stencil pass, if it left them out.
void CouplingEngine::launchSlotMomentsNow() {
    if (!slotMomentsPending)
        return;
    const CouplingView c = makeCouplingView(lattice, fluid.deviceView(), np, widthOf(lattice.interpolation_stencil), massDev);
    if (storageType == LBM_STORAGE_F64)
        launchSlotMoments<double>(c, dev->slotNode, dev->slotWeight, dev->nodeStamp, dev->stamp, dev->nodeU, dev->slotU, stream);
    else
        launchSlotMoments<float>(c, dev->slotNode, dev->slotWeight, dev->nodeStamp, dev->stamp, dev->nodeU, dev->slotU, stream);
    CUDA_CHECK(cudaGetLastError());
    fluid.launches++;
    slotMomentsPending = false;
}

// The centred stencil drag through the explicit coupling matrix (not the spread-and-gather solve of every step).
bool CouplingEngine::matrixSolve() const {
    static const bool spreadOnly = [] {
        const char* e = std::getenv("LBM_B200_SPREAD_CG");
        return e != nullptr && e[0] == '1';
    }();
    return lattice.drag_scheme == LBM_DRAG_CENTERED && lattice.interpolation_stencil != LBM_STENCIL_NEAREST &&
           !spreadOnly;
}

void CouplingEngine::prepare(const LbmParticleArrays* p, long long step, bool remove) {
    discardPrepared();
    size_t v3 = sizeof(double)*3*(size_t) np;
    cudaMemcpyKind kind = p->memory == LBM_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CUDA_CHECK(cudaMemcpyAsync(posDev, p->positions, v3, kind, stream));
    if (side == nullptr) {
        // The prepared work is the step's critical path (the caller's forces run beside it): its blocks go first.
        int least = 0, greatest = 0;
        CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUDA_CHECK(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, greatest));
        CUDA_CHECK(cudaEventCreateWithFlags(&begun, cudaEventDisableTiming));
        CUDA_CHECK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    }
    CUDA_CHECK(cudaEventRecord(begun, stream));
    CUDA_CHECK(cudaStreamWaitEvent(side, begun, 0));
    const FluidView& f = fluid.deviceView();
    CouplingView c = makeCouplingView(lattice, f, np, widthOf(lattice.interpolation_stencil), massDev);
    launchStencilPass(c, remove, true, side);
    if (matrixSolve()) {
        if (storageType == LBM_STORAGE_F64)
            launchMatrix<double>(&c, side);
        else
            launchMatrix<float>(&c, side);
    }
    CUDA_CHECK(cudaEventRecord(ready, side));
    prepared = true;
    preparedStep = step;
    preparedRemove = remove;
}

void CouplingEngine::joinPrepared() {
    if (prepared)
        CUDA_CHECK(cudaStreamWaitEvent(stream, ready, 0));
}

void CouplingEngine::discardPrepared() {
    joinPrepared();
    prepared = false;
}

void CouplingEngine::couple(long long step, bool isStep, bool remove) {
    const FluidView& f = fluid.deviceView();
    CouplingView c = makeCouplingView(lattice, f, np, widthOf(lattice.interpolation_stencil), massDev);
    const bool usePrepared = prepared && isStep && step == preparedStep && remove == preparedRemove;
    discardPrepared();
    if (!usePrepared)
        launchStencilPass(c, remove, isStep, stream);
    if (isStep)
        CUDA_CHECK(cudaMemsetAsync(wallDev, 0, sizeof(double)*3, stream));
    if (storageType == LBM_STORAGE_F64)
        coupleWith<double>(step, isStep, &c, usePrepared);
    else
        coupleWith<float>(step, isStep, &c, usePrepared);
}

void CouplingEngine::addForces(const LbmParticleArrays* p) {
    size_t count = 3*(size_t) np;
    if (p->memory == LBM_MEMORY_DEVICE) {
        addForcesKernel<<<std::max(1, std::min(1184, (int) ((count + kThreads - 1)/kThreads))), kThreads, 0, stream>>>(
            forceOutDev, p->forces, (int) count);
        CUDA_CHECK(cudaGetLastError());
        fluid.launches++;
        return;
    }
    CUDA_CHECK(cudaMemcpyAsync(pinned, forceOutDev, sizeof(double)*count, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    for (size_t i = 0; i < count; i++)
        p->forces[i] += pinned[i];
}

void CouplingEngine::clearReactionFlags() {
    fluid.clearReactMask(stream);
}

void CouplingEngine::clearReaction() {
    const FluidView& f = fluid.deviceView();
    long long total = (long long) np*stencilSlots;
    int grid = (int) std::max(1LL, std::min(4736LL, (total + kThreads - 1)/kThreads));
    if (storageType == LBM_STORAGE_F64)
        clearReactionKernel<double><<<grid, kThreads, 0, stream>>>(f, dev->slotNode, total, (double*) fluid.reactionBuffer(), fluid.reactMask());
    else
        clearReactionKernel<float><<<grid, kThreads, 0, stream>>>(f, dev->slotNode, total, (float*) fluid.reactionBuffer(), fluid.reactMask());
    CUDA_CHECK(cudaGetLastError());
    fluid.launches++;
}

void CouplingEngine::reactionWallMomentum(double out[3]) {
    CUDA_CHECK(cudaMemcpyAsync(out, wallDev, sizeof(double)*3, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

} // namespace lbm
