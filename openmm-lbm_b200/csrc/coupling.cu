// Particle coupling kernels of the B200 LBM force kernel (sm_100a).
//
// The coupling of the reference (platforms/reference/src/ReferenceLBMKernels.cpp:503-1018), on the device:
//   stencilKernel         one thread per (particle, stencil slot): the node and weight of the slot
//                         (LBMStencils::axisWeights, LBMStencils.h:73-95) and the moments of the node pulled from the
//                         populations (density, momentum after the momentum removal; a solid node has rho = 0)
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
#include "lbm_device.cuh"
#include "radix_sort.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

namespace lbm {

#define CUDA_CHECK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    throw Error(LBM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

namespace {

const int kThreads = 256;

// One thread per (particle, slot).
template <typename T, typename R>
__global__ void stencilKernel(const T* __restrict__ A, FluidView f, CouplingView c, const double* __restrict__ pos,
                              int remove, int centred, int* slotNode, R* slotWeight, typename Vec4<R>::type* slotU) {
    long long total = (long long) c.np*c.slots;
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < total; t += (long long) gridDim.x*blockDim.x)
        stencilSlot<T, R>(A, f, c, pos, t, remove, centred, slotNode, slotWeight, slotU);
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
    unsigned* barrier;     // [0] arrival count, [1] generation
    int* status;           // 0 ok, LBM_ERR_CG_NOT_CONVERGED, LBM_ERR_DEVICE_TIMEOUT
    int* iterations;
};

// Grid barrier for a cooperative launch (all blocks resident), with a bounded spin: after about 2^26 polls the
// waiting block gives up, records a timeout in the status word and returns false; every block then leaves the
// solve at its next barrier.
__device__ bool gridBarrier(unsigned* bar, int* status, unsigned& generation) {
    __syncthreads();
    bool ok = true;
    if (threadIdx.x == 0) {
        unsigned target = generation + 1;
        __threadfence();
        unsigned arrived = atomicAdd(&bar[0], 1u);
        if (arrived == gridDim.x - 1) {
            bar[0] = 0;
            __threadfence();
            atomicExch(&bar[1], target);
        }
        else {
            long long polls = 0;
            while (atomicAdd(&bar[1], 0u) != target) {
                if (++polls > (1LL << 26) || atomicAdd(status, 0) == LBM_ERR_DEVICE_TIMEOUT) {
                    atomicExch(status, LBM_ERR_DEVICE_TIMEOUT);
                    ok = false;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        generation = target;
    }
    __shared__ int okShared;
    if (threadIdx.x == 0)
        okShared = ok;
    __syncthreads();
    return okShared != 0 && *((volatile int*) status) != LBM_ERR_DEVICE_TIMEOUT;
}

// Block sum of a record (thread values v) into partials[block]; after a grid barrier (by the caller) every block adds
// the records of all blocks in block order, so every block gets the same result, bit for bit.
__device__ void blockSumStore(double v[kPartial], double* partials) {
    __shared__ double red[kThreads/32][kPartial];
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
    __shared__ double total[kPartial];
    if (threadIdx.x < kPartial) {
        double s = 0;
        for (int b = 0; b < count; b++)
            s += ((volatile const double*) partials)[kPartial*b + threadIdx.x];
        total[threadIdx.x] = s;
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
    unsigned generation = 0;
    if (threadIdx.x == 0)
        generation = *((volatile unsigned*) &b.barrier[1]);
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
    if (!gridBarrier(b.barrier, b.status, generation))
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
    if (!gridBarrier(b.barrier, b.status, generation))
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
            if (!gridBarrier(b.barrier, b.status, generation))
                return;
            clearBeforeSpread = false;
        }
        for (int i = firstWarp; i < c.np; i += warps)
            spreadP(i, b.p);
        if (!gridBarrier(b.barrier, b.status, generation))
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
        if (!gridBarrier(b.barrier, b.status, generation))
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
        if (!gridBarrier(b.barrier, b.status, generation))
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

// Clear the reaction of the slots of the last step (and their mask words).
template <typename R>
__global__ void clearReactionKernel(FluidView f, const int* slotNode, long long total, R* reaction, uint32_t* mask) {
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < total; t += (long long) gridDim.x*blockDim.x) {
        long long node = slotNode[t];
        *reinterpret_cast<typename Vec4<R>::type*>(reaction + 4*node) = Vec4<R>::make(0, 0, 0, 0);
        long long row = node/f.nx;
        int x = (int) (node - row*f.nx);
        mask[row*f.wordsPerRow + x/32] = 0u;
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
    void* spread = nullptr;
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
    stencilSlots = widthOf(l.interpolation_stencil);
    stencilSlots = stencilSlots*stencilSlots*stencilSlots;
    bool f64 = storageType == LBM_STORAGE_F64;
    size_t r = f64 ? 8 : 4;
    try {
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
            CUDA_CHECK(cudaMalloc(&b.barrier, sizeof(unsigned)*2));
            CUDA_CHECK(cudaMemsetAsync(b.barrier, 0, sizeof(unsigned)*2, stream));
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
    cudaFree(posDev); cudaFree(velDev); cudaFree(forceInDev); cudaFree(forceOutDev); cudaFree(massDev);
    cudaFree(wallDev); cudaFree(statusDev);
    posDev = velDev = forceInDev = forceOutDev = massDev = wallDev = nullptr;
    statusDev = nullptr;
    if (pinned)
        cudaFreeHost(pinned);
    pinned = nullptr;
    if (dev) {
        cudaFree(dev->slotNode); cudaFree(dev->slotWeight); cudaFree(dev->slotU); cudaFree(dev->coef);
        for (int k = 0; k < 2; k++) {
            cudaFree(dev->keys[k]);
            cudaFree(dev->values[k]);
        }
        cudaFree(dev->hist);
        CgBuffers& b = dev->cg;
        cudaFree(b.rhs); cudaFree(b.diag); cudaFree(b.F); cudaFree(b.r); cudaFree(b.z); cudaFree(b.p);
        cudaFree(b.partials[0]); cudaFree(b.partials[1]); cudaFree(b.barrier);
        cudaFree(dev->spread);
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
                          int* slotNode, void* slotWeight, void* slotU, cudaStream_t s) {
    long long total = (long long) c.np*c.slots;
    int grid = (int) std::max(1LL, std::min(4736LL, (total + kThreads - 1)/kThreads));
    stencilKernel<T, R><<<grid, kThreads, 0, s>>>((const T*) A, f, c, pos, remove, centred, slotNode, (R*) slotWeight,
                                                   (typename Vec4<R>::type*) slotU);
}

template <typename R>
void CouplingEngine::coupleWith(long long step, bool isStep, const CouplingView* cv) {
    const CouplingView& c = *cv;
    const FluidView& f = fluid.deviceView();
    bool centred = lattice.drag_scheme == LBM_DRAG_CENTERED;
    R* reaction = (R*) fluid.reactionBuffer();
    uint32_t* mask = fluid.reactMask();
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
    // 1e-13 in double; 1e-5 with single-precision arithmetic, as the reference's GPU platforms in single precision).
    CgBuffers b = dev->cg;
    CUDA_CHECK(cudaMemsetAsync(statusDev, 0, sizeof(int)*2, stream));
    double tolerance = std::is_same<R, double>::value ? 1e-13 : 1e-5;
    int maxIterations = 1000;
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
    void* args[] = {&fv, &cc, &vel, &fin, &sn, &sw, &su, &coef, &stepArg, &isStepArg, &tolerance, &maxIterations, &b,
                    &spread, &fout, &reaction, &mask, &wall};
    CUDA_CHECK(cudaLaunchCooperativeKernel((const void*) centeredStencilKernel<R>, dev->cgGrid, kThreads, args, 0, stream));
    fluid.launches++;
    int status[2] = {0, 0};
    CUDA_CHECK(cudaMemcpyAsync(status, statusDev, sizeof(int)*2, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    lastIterations = status[1];
    if (status[0] == LBM_ERR_CG_NOT_CONVERGED)
        throw Error(LBM_ERR_CG_NOT_CONVERGED, "LBMForce: the centred drag with the interpolation stencil did not converge "
                    "in 1000 iterations of the conjugate gradients");
    if (status[0] == LBM_ERR_DEVICE_TIMEOUT)
        throw Error(LBM_ERR_DEVICE_TIMEOUT, "LBMForce: a grid barrier of the conjugate gradients timed out");
}

void CouplingEngine::couple(long long step, bool isStep, bool remove) {
    const FluidView& f = fluid.deviceView();
    CouplingView c = makeCouplingView(lattice, f, np, widthOf(lattice.interpolation_stencil), massDev);
    bool centred = lattice.drag_scheme == LBM_DRAG_CENTERED;
    const void* A = fluid.inputArray();
    switch (storageType) {
    case LBM_STORAGE_F64: launchStencil<double, double>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, dev->slotU, stream); break;
    case LBM_STORAGE_F32: launchStencil<float, float>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, dev->slotU, stream); break;
    case LBM_STORAGE_F16: launchStencil<__half, float>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, dev->slotU, stream); break;
    default: launchStencil<__nv_bfloat16, float>(A, f, c, posDev, remove, centred, dev->slotNode, dev->slotWeight, dev->slotU, stream); break;
    }
    CUDA_CHECK(cudaGetLastError());
    fluid.launches++;
    if (isStep)
        CUDA_CHECK(cudaMemsetAsync(wallDev, 0, sizeof(double)*3, stream));
    if (storageType == LBM_STORAGE_F64)
        coupleWith<double>(step, isStep, &c);
    else
        coupleWith<float>(step, isStep, &c);
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
