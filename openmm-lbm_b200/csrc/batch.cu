// Replica batches (include/lbm_b200_batch.h): independent periodic lattices of uneven sizes, each with its own beads,
// advanced together.  Every phase of a step is one persistent launch over all replicas:
//
//  batchPairKernel            bead pair forces, one block per replica, all pairs (WCA / truncated Lennard-Jones)
//  batchStencilKernel         stencil slots of every bead (node, weight, pulled fluid velocity), one thread per slot
//  batchExplicitKernel        explicit drag of every bead and its reaction on the fluid, one warp per bead
//  batchStreamCollideKernel   the dense step of every replica: work items of BT consecutive nodes of one replica,
//                             the node body of the single-lattice kernel (collide.cuh), per-warp partial sums
//  batchFinishKernel          per-replica mass and momentum (momentum removal of the next step), deterministic
//  batchClearKernel           reaction buffers and masks back to zero at the stencil nodes
//  batchLeapfrogKernel        v += dt F/m, x += dt v for every bead
//
// The step index lives on the device (a clock the finish kernel advances), so that a run of steps captured once in a
// CUDA graph replays with the right random numbers and removal schedule.  The node and slot bodies are the device
// functions of the single-lattice kernels (collide.cuh, coupling_device.cuh), with each replica's FluidView and
// CouplingView, so a replica computes what a kernel of lbm_create with its parameters computes.
#include "lbm_b200_batch.h"
#include "lbm_b200_md.h"
#include "collide.cuh"
#include "collide_pair.cuh"
#include "coupling_device.cuh"
#include "grid_barrier.cuh"
#include "lbm_internal.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

namespace lbm {

#define CUDA_CHECK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    throw Error(LBM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

namespace {

struct BatchClock {
    long long step;
    long long pad;
};

// Per replica, on the device.
struct ReplicaTable {
    unsigned nodeOffset;     // first node of the replica in the concatenated populations (19 arrays of N_r each; even)
    unsigned numNodes;
    int firstItem, numItems; // work items of the dense kernel
    int paired;              // FP32 storage, two x-adjacent nodes per thread: 1 for an even nx (aligned pairs of the
                             // replica's node order), 2 for an odd nx (pairs within each row); 0: one node per thread
    unsigned units;          // threads of the dense step: nodes, pairs, or pairs and row ends
    int firstParticle, numParticles;
    int removeFrequency;
    double dt;               // ps
    double box[3];           // nm
};

struct PairParams {
    int type;
    double sigma2, eps, rc2;
};

constexpr int kBatchThreads = 256;     // blocks of the particle kernels

template <typename R, int BT>
constexpr int batchMinBlocks() { return sizeof(R) == 4 ? 768/BT : 512/BT; }

__device__ __forceinline__ double warpReduceSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Where the paired body puts a pair's values: as one aligned float2 per direction (an even nx: the replica's arrays
// start at an even node and its planes hold an even number of nodes), or as single floats (an odd nx, whose rows
// start at nodes of either parity), the copy of a row's last node (`single`) discarded.  Planes are N floats apart.
struct UnitStore {
    float* out;         // the pair's first node in plane 0
    unsigned N;
    bool aligned, single;
    template <int q> __device__ __forceinline__ void put(F2 value, uint32_t) {
        float* p = out + (size_t) q*N;
        if (aligned) {
            *reinterpret_cast<float2*>(p) = value.v;
            return;
        }
        p[0] = value.v.x;
        if (!single)
            p[1] = value.v.y;
    }
};

// Unit `unit` of a replica with FP32 storage, by the paired body of the single-lattice kernel (collide_pair.cuh) with
// the replica's view.  paired == 1 (an even nx): nodes 2 unit and 2 unit + 1, pulled as aligned float2 words.
// paired == 2 (an odd nx): a row holds (nx + 1)/2 units, unit u the nodes 2u and 2u + 1 of its row, the last one
// (2u = nx - 1) its row's last node alone, collided as a pair with itself and the copy discarded (its sums left out);
// the pulls are single floats.  The random numbers of a node are those of the one-node body.  COHERENT: the inputs
// were written by other blocks of the same launch, so they are read through L2.  One instantiation of the collision
// serves both forms.
template <bool REACT, bool FLUCT, bool COHERENT>
__device__ __forceinline__ void pairedUnit(const float* __restrict__ A, float* __restrict__ B, const FluidView& v,
                                           unsigned N, unsigned unit, int paired, int remove, const double ucm[3],
                                           long long step, float (&sums)[4]) {
    const int nx = v.nx, ny = v.ny, nz = v.nz;
    unsigned row, node;
    int x0;
    bool single = false;
    if (paired == 1) {
        node = 2*unit;
        if (node >= N)
            return;
        row = node/(unsigned) nx;
        x0 = (int) (node - row*(unsigned) nx);
    }
    else {
        const unsigned perRow = (unsigned) (nx + 1)/2;
        row = unit/perRow;
        if (row >= (unsigned) ny*(unsigned) nz)
            return;
        x0 = 2*(int) (unit - row*perRow);
        single = x0 + 1 == nx;
        node = row*(unsigned) nx + (unsigned) x0;
    }
    const int x1 = single ? x0 : x0 + 1;
    const int y = (int) (row%(unsigned) ny), z = (int) (row/(unsigned) ny);
    const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
    const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
    F2 r[19];
    if (paired == 1) {
        const float2* aw = reinterpret_cast<const float2*>(A);
        const unsigned halfN = N/2;
        const int xl = x0 == 0 ? nx - 2 : x0 - 2, xr = x0 + 2 == nx ? 0 : x0 + 2;
        auto load = [&](const float2* p) { return COHERENT ? __ldcg(p) : __ldg(p); };
        staticFor<19>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
            const unsigned base = ((unsigned) zs[1-cz]*ny + ys[1-cy])*nx;
            const float2* plane = aw + (size_t) q*halfN;
            float2 w;
            if (cx == 0)
                w = load(plane + (base + x0)/2);
            else if (cx == 1)
                w = PairIO<float>::left(load(plane + (base + xl)/2), load(plane + (base + x0)/2));
            else
                w = PairIO<float>::right(load(plane + (base + x0)/2), load(plane + (base + xr)/2));
            r[q] = PairIO<float>::decode(w);
        });
    }
    else {
        auto load = [&](const float* p) { return COHERENT ? __ldcg(p) : __ldg(p); };
        auto wrapX = [&](int x) { return x < 0 ? x + nx : (x >= nx ? x - nx : x); };
        staticFor<19>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
            const float* plane = A + (size_t) q*N + ((unsigned) zs[1-cz]*ny + ys[1-cy])*nx;
            r[q] = F2{make_float2(load(plane + wrapX(x0 - cx)), load(plane + wrapX(x1 - cx)))};
        });
    }
    bool reactA = false, reactB = false;
    if (REACT) {
        const uint32_t* mp = &v.reactMask[(size_t) row*v.wordsPerRow];
        const uint32_t wordA = COHERENT ? __ldcg(mp + (x0 >> 5)) : __ldg(mp + (x0 >> 5));
        const uint32_t wordB = COHERENT ? __ldcg(mp + (x1 >> 5)) : __ldg(mp + (x1 >> 5));
        reactA = (wordA >> (x0 & 31)) & 1u;
        reactB = !single && ((wordB >> (x1 & 31)) & 1u);
    }
    const PairConstants c = pairConstants(v, remove, step, ucm);
    UnitStore out{B + node, N, paired == 1, single};
    collidePair<float, false, REACT, FLUCT, COHERENT>(r, v, c, remove, step, node, false, single, reactA, reactB, out,
                                                      sums);
}

template <typename T, typename R, bool REACT, bool FLUCT, int BT>
__global__ void __launch_bounds__(BT, batchMinBlocks<R, BT>())
batchStreamCollideKernel(const T* __restrict__ A, T* __restrict__ B, const FluidView* __restrict__ views,
                         const ReplicaTable* __restrict__ table, const int* __restrict__ itemReplica, int numItems,
                         const BatchClock* clock, double* partials) {
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    const long long step = clock->step;
    for (int w = blockIdx.x; w < numItems; w += gridDim.x) {
        const int r = itemReplica[w];
        const FluidView& v = views[r];
        const ReplicaTable& rt = table[r];
        const int remove = rt.removeFrequency > 0 && step%rt.removeFrequency == 0;
        const unsigned N = rt.numNodes;
        const size_t base = (size_t) 19*rt.nodeOffset;
        if constexpr (std::is_same<T, float>::value) {
            if (rt.paired) {
                float sums[4] = {0, 0, 0, 0};
                const unsigned unit = (unsigned) (w - rt.firstItem)*BT + threadIdx.x;
                pairedUnit<REACT, FLUCT, false>(A + base, B + base, v, N, unit, rt.paired, remove, v.stats->ucm, step,
                                                sums);
                double s0 = warpReduceSum((double) sums[0]), s1 = warpReduceSum((double) sums[1]);
                double s2 = warpReduceSum((double) sums[2]), s3 = warpReduceSum((double) sums[3]);
                if (lane == 0) {
                    double* out = partials + 4*((size_t) w*(BT/32) + warp);
                    out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
                }
                continue;
            }
        }
        const CollideConstants<R> k = collideConstants<R>(v.omega, v.g, v.stats->ucm, remove, v.mu, v.seed);
        const unsigned local = (unsigned) (w - rt.firstItem)*BT + threadIdx.x;
        R sm = 0, sx = 0, sy = 0, sz = 0;
        if (local < N) {
            const int nx = v.nx, ny = v.ny, nz = v.nz;
            const unsigned row = local/(unsigned) nx;
            const int x = (int) (local - row*nx);
            const int y = (int) (row%ny), z = (int) (row/ny);
            R ex = 0, ey = 0, ez = 0;
            if (REACT) {
                uint32_t word = __ldg(&v.reactMask[(size_t) row*v.wordsPerRow + x/32]);
                if ((word >> (x%32)) & 1u) {
                    const R* rp = reinterpret_cast<const R*>(v.reaction) + 4*(size_t) local;
                    ex = rp[0];
                    ey = rp[1];
                    ez = rp[2];
                }
            }
            collideNode<T, R, FLUCT>(A + base, B + base, N, local, x, y, z, nx, ny, nz, k, ex, ey, ez, step, sm, sx, sy, sz);
        }
        double s0 = warpReduceSum((double) sm), s1 = warpReduceSum((double) sx);
        double s2 = warpReduceSum((double) sy), s3 = warpReduceSum((double) sz);
        if (lane == 0) {
            double* out = partials + 4*((size_t) w*(BT/32) + warp);
            out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
        }
    }
}

// Sums of a step per replica (one block each, fixed order): mass deviation, momentum and the velocity that the next
// momentum removal subtracts (the single-lattice finishKernel, mode 0).  Block 0 advances the clock.
__global__ void __launch_bounds__(kBatchThreads)
batchFinishKernel(const double* __restrict__ partials, const ReplicaTable* __restrict__ table, const FluidView* views,
                  int numReplicas, int warpsPerItem, BatchClock* clock) {
    __shared__ double red[kBatchThreads/32][4];
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    for (int r = blockIdx.x; r < numReplicas; r += gridDim.x) {
        const ReplicaTable& rt = table[r];
        size_t begin = (size_t) rt.firstItem*warpsPerItem, count = (size_t) rt.numItems*warpsPerItem;
        double acc[4] = {0, 0, 0, 0};
        for (size_t i = threadIdx.x; i < count; i += blockDim.x)
            for (int k = 0; k < 4; k++)
                acc[k] += partials[4*(begin + i) + k];
        for (int k = 0; k < 4; k++)
            acc[k] = warpReduceSum(acc[k]);
        if (lane == 0)
            for (int k = 0; k < 4; k++)
                red[warp][k] = acc[k];
        __syncthreads();
        if (threadIdx.x == 0) {
            double total[4] = {0, 0, 0, 0};
            for (int w = 0; w < (int) blockDim.x/32; w++)
                for (int k = 0; k < 4; k++)
                    total[k] += red[w][k];
            StepStats* s = views[r].stats;
            s->mass = total[0];
            double mass = views[r].numFluid + total[0];
            for (int a = 0; a < 3; a++) {
                s->momentum[a] = total[1+a];
                s->ucm[a] = total[1+a]/mass;
            }
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        clock->step++;
}

template <typename T, typename R>
__global__ void __launch_bounds__(kBatchThreads)
batchStencilKernel(const T* __restrict__ A, const FluidView* __restrict__ views, const CouplingView* __restrict__ cviews,
                   const ReplicaTable* __restrict__ table, const int* __restrict__ particleReplica, long long totalSlots,
                   int slots, const double* __restrict__ pos, const BatchClock* clock, int* slotNode, R* slotWeight,
                   typename Vec4<R>::type* slotU) {
    const long long step = clock->step;
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < totalSlots; t += (long long) gridDim.x*blockDim.x) {
        int p = (int) (t/slots), s = (int) (t - (long long) p*slots);
        int r = particleReplica[p];
        const ReplicaTable& rt = table[r];
        int p0 = rt.firstParticle, i = p - p0;
        int remove = rt.removeFrequency > 0 && step%rt.removeFrequency == 0;
        size_t so = (size_t) p0*slots;
        stencilSlot<T, R>(A + (size_t) 19*rt.nodeOffset, views[r], cviews[r], pos + 3*(size_t) p0,
                          (long long) i*slots + s, remove, 0, slotNode + so, slotWeight + so, slotU + so);
    }
}

template <typename R>
__global__ void __launch_bounds__(kBatchThreads)
batchExplicitKernel(const FluidView* __restrict__ views, const CouplingView* __restrict__ cviews,
                    const ReplicaTable* __restrict__ table, const int* __restrict__ particleReplica, int totalParticles,
                    int slots, const double* __restrict__ vel, const int* __restrict__ slotNode,
                    const R* __restrict__ slotWeight, const typename Vec4<R>::type* __restrict__ slotU,
                    const BatchClock* clock, double* fout, double* wall) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x*blockDim.x) >> 5;
    const long long step = clock->step;
    for (int p = (blockIdx.x*blockDim.x + threadIdx.x) >> 5; p < totalParticles; p += warps) {
        int r = particleReplica[p];
        const ReplicaTable& rt = table[r];
        const FluidView& f = views[r];
        int p0 = rt.firstParticle;
        size_t so = (size_t) p0*slots;
        explicitParticle<R>(f, cviews[r], vel + 3*(size_t) p0, slotNode + so, slotWeight + so, slotU + so, p - p0, lane,
                            step, 1, fout + 3*(size_t) p0, (R*) const_cast<void*>(f.reaction),
                            const_cast<uint32_t*>(f.reactMask), wall);
    }
}

template <typename R>
__global__ void __launch_bounds__(kBatchThreads)
batchClearKernel(const FluidView* __restrict__ views, const int* __restrict__ particleReplica, long long totalSlots,
                 int slots, const int* __restrict__ slotNode) {
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < totalSlots; t += (long long) gridDim.x*blockDim.x) {
        const FluidView& f = views[particleReplica[t/slots]];
        long long node = slotNode[t];
        R* reaction = (R*) const_cast<void*>(f.reaction);
        *reinterpret_cast<typename Vec4<R>::type*>(reaction + 4*node) = Vec4<R>::make(0, 0, 0, 0);
        long long row = node/f.nx;
        int x = (int) (node - row*f.nx);
        const_cast<uint32_t*>(f.reactMask)[row*f.wordsPerRow + x/32] = 0u;
    }
}

// Pair force on bead i of a replica from all others, minimum image (the pair force of the bead dynamics, md.cu).
__global__ void __launch_bounds__(kBatchThreads)
batchPairKernel(const ReplicaTable* __restrict__ table, int numReplicas, PairParams pp, const double* __restrict__ pos,
                double* fpair) {
    for (int r = blockIdx.x; r < numReplicas; r += gridDim.x) {
        const ReplicaTable& rt = table[r];
        const double* x = pos + 3*(size_t) rt.firstParticle;
        double* out = fpair + 3*(size_t) rt.firstParticle;
        for (int i = threadIdx.x; i < rt.numParticles; i += blockDim.x) {
            double f[3] = {0, 0, 0};
            if (pp.type != LBM_PAIR_NONE)
                for (int j = 0; j < rt.numParticles; j++) {
                    if (j == i)
                        continue;
                    double d[3];
                    for (int a = 0; a < 3; a++) {
                        d[a] = x[3*i+a] - x[3*j+a];
                        d[a] -= rt.box[a]*rint(d[a]/rt.box[a]);
                    }
                    double r2 = d[0]*d[0] + d[1]*d[1] + d[2]*d[2];
                    if (r2 >= pp.rc2 || r2 == 0.0)
                        continue;
                    double s2 = pp.sigma2/r2, s6 = s2*s2*s2;
                    double scale = 24.0*pp.eps*s6*(2.0*s6 - 1.0)/r2;
                    for (int a = 0; a < 3; a++)
                        f[a] += scale*d[a];
                }
            for (int a = 0; a < 3; a++)
                out[3*i+a] = f[a];
        }
    }
}

// Leapfrog of every bead with the bead forces plus the drag: v += dt F/m, x += dt v (the bead dynamics' integrator).
__global__ void __launch_bounds__(kBatchThreads)
batchLeapfrogKernel(const ReplicaTable* __restrict__ table, const int* __restrict__ particleReplica, int totalParticles,
                    const double* __restrict__ invMass, const double* __restrict__ fpair, const double* __restrict__ fdrag,
                    double* pos, double* vel) {
    for (int t = blockIdx.x*blockDim.x + threadIdx.x; t < 3*totalParticles; t += gridDim.x*blockDim.x) {
        int p = t/3;
        double dt = table[particleReplica[p]].dt;
        double f = fpair[t];
        f += fdrag[t];
        double v = vel[t] + dt*f*invMass[p];
        vel[t] = v;
        pos[t] += dt*v;
    }
}

// Fluid and bead temperatures of every replica (one block each).
template <typename T>
__global__ void __launch_bounds__(kBatchThreads)
batchTemperatureKernel(const T* __restrict__ pop, const FluidView* __restrict__ views, const ReplicaTable* __restrict__ table,
                       int numReplicas, const double* cellEnergy, const double* __restrict__ vel,
                       const double* __restrict__ masses, double* out) {
    __shared__ double red[kBatchThreads/32][8];
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    for (int r = blockIdx.x; r < numReplicas; r += gridDim.x) {
        const FluidView& f = views[r];
        const ReplicaTable& rt = table[r];
        const T* A = pop + (size_t) 19*rt.nodeOffset;
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (unsigned node = threadIdx.x; node < rt.numNodes; node += blockDim.x) {
            double dr, jx, jy, jz;
            pullMoments<T>(A, f, node, dr, jx, jy, jz);
            double rho = 1.0 + dr;
            double p[3] = {jx + 0.5*rho*f.g[0], jy + 0.5*rho*f.g[1], jz + 0.5*rho*f.g[2]};
            acc[0] += rho;
            for (int a = 0; a < 3; a++) {
                acc[1+a] += p[a];
                acc[4] += p[a]*p[a]/rho;
            }
        }
        for (int i = threadIdx.x; i < rt.numParticles; i += blockDim.x) {
            const double* v = vel + 3*(size_t) (rt.firstParticle + i);
            acc[5] += masses[rt.firstParticle + i]*(v[0]*v[0] + v[1]*v[1] + v[2]*v[2]);
        }
        for (int k = 0; k < 6; k++)
            acc[k] = warpReduceSum(acc[k]);
        if (lane == 0)
            for (int k = 0; k < 6; k++)
                red[warp][k] = acc[k];
        __syncthreads();
        if (threadIdx.x == 0) {
            double t[6] = {0, 0, 0, 0, 0, 0};
            for (int w = 0; w < (int) blockDim.x/32; w++)
                for (int k = 0; k < 6; k++)
                    t[k] += red[w][k];
            double mean2 = (t[1]*t[1] + t[2]*t[2] + t[3]*t[3])/t[0];
            out[2*r] = (t[4] - mean2)/(3.0*rt.numNodes)*cellEnergy[r];
            out[2*r+1] = rt.numParticles > 0 ? t[5]/(3.0*rt.numParticles) : 0.0;
        }
        __syncthreads();
    }
}

// Post-stream populations of one replica in the reference's state layout: out[q*N + node] = the value the node pulls.
template <typename T>
__global__ void batchGatherKernel(const T* __restrict__ A, FluidView f, double* out) {
    typedef typename std::conditional<std::is_same<T, double>::value, double, float>::type R;
    long long total = 19*f.n;
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < total; t += (long long) gridDim.x*blockDim.x) {
        int q = (int) (t/f.n);
        long long node = t - q*f.n;
        int x = (int) (node%f.nx);
        long long rr = node/f.nx;
        int y = (int) (rr%f.ny), z = (int) (rr/f.ny);
        int xs = (x - cxOf(q) + f.nx)%f.nx, ys = (y - cyOf(q) + f.ny)%f.ny, zs = (z - czOf(q) + f.nz)%f.nz;
        long long src = xs + (long long) f.nx*(ys + (long long) f.ny*zs);
        out[t] = (double) loadq<T, R>(A + q*f.n + src, q);
    }
}

// ------------------------------------------------------------------------------------------------------------------
// The persistent step: `steps` lattice steps of every replica in one cooperative launch (every block resident), the
// phases of a step separated by bounded grid barriers (grid_barrier.cuh):
//
//   phase 1  the sums of the previous step per replica (blocks over replicas: mass, momentum and the velocity that this
//            step's momentum removal subtracts), bead pair forces (blocks over replicas), stencil slots of every bead
//            (threads over slots) with the nodes' j/rho before the removal, and the clear of the previous step's
//            reactions (their slot nodes are kept in the other half of slotNode)
//   phase 2  explicit drag of every bead (the removal applied to the interpolated velocity: sum w (j/rho - ucm) =
//            sum w j/rho - ucm sum w) and its reaction on the fluid (warps over beads), then the bead's leapfrog
//   phase 3  the dense step of every replica (work items of BT nodes), per-warp partial sums
//
// After the last step a final phase forms the last step's sums, so that the statistics are complete between launches.
// The reaction buffers and slot nodes alternate between steps (buffer step & 1), so that the clear of step s - 1 and
// the slots of step s share phase 1.  A replica computes what the seven-kernel step computes, up to the rounding of
// the removal's form.  A barrier that times out sets LBM_ERR_DEVICE_TIMEOUT in the status word and every block leaves
// the launch.
// ------------------------------------------------------------------------------------------------------------------

struct PersistentArgs {
    const FluidView* views[2];     // the replicas' views with reaction buffer 0 / 1
    const CouplingView* cviews;
    const ReplicaTable* table;
    const int* itemReplica;
    const int* particleReplica;
    int numReplicas, numItems, totalParticles, slots, coupled, steps;
    PairParams pair;
    void* pop[2];                  // populations: the launch starts from pop[cur]
    int cur;
    double* partials;              // 4 per warp of every item
    BatchClock* clock;
    double *pos, *vel, *fpair, *fdrag, *invMass, *wall;
    int* slotNode[2];
    void* slotWeight;
    void* slotU;
    unsigned* barrier;
    int* status;
    long long pollLimit;
};

// Sums of replica r's items (the body of batchFinishKernel for one replica, by the whole block), in the same order.
__device__ __forceinline__ void finishReplica(const PersistentArgs& a, int r, int warpsPerItem) {
    __shared__ double red[16][4];
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    const ReplicaTable& rt = a.table[r];
    size_t begin = (size_t) rt.firstItem*warpsPerItem, count = (size_t) rt.numItems*warpsPerItem;
    double acc[4] = {0, 0, 0, 0};
    for (size_t i = threadIdx.x; i < count; i += blockDim.x)
        for (int k = 0; k < 4; k++)
            acc[k] += __ldcg(&a.partials[4*(begin + i) + k]);
    for (int k = 0; k < 4; k++)
        acc[k] = warpReduceSum(acc[k]);
    if (lane == 0)
        for (int k = 0; k < 4; k++)
            red[warp][k] = acc[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        double total[4] = {0, 0, 0, 0};
        for (int w = 0; w < (int) blockDim.x/32; w++)
            for (int k = 0; k < 4; k++)
                total[k] += red[w][k];
        StepStats* st = a.views[0][r].stats;
        st->mass = total[0];
        double mass = a.views[0][r].numFluid + total[0];
        for (int k = 0; k < 3; k++) {
            st->momentum[k] = total[1+k];
            st->ucm[k] = total[1+k]/mass;
        }
    }
    __syncthreads();
}

constexpr int kPairTile = 256;     // beads per shared-memory tile of the pair forces

template <typename T, typename R, bool FLUCT, int BT>
__global__ void __launch_bounds__(BT, batchMinBlocks<R, BT>())
batchPersistentKernel(PersistentArgs a) {
    typedef typename Vec4<R>::type V;
    __shared__ double pairTile[3*kPairTile];
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    const long long step0 = a.clock->step;
    const long long totalSlots = (long long) a.totalParticles*a.slots;
    const int threads = gridDim.x*blockDim.x, firstThread = blockIdx.x*blockDim.x + threadIdx.x;
    const int warps = threads >> 5, firstWarp = firstThread >> 5;
    R* slotWeight = (R*) a.slotWeight;
    V* slotU = (V*) a.slotU;
    for (int s = 0; s < a.steps; s++) {
        const long long step = step0 + s;
        const int buf = (int) (step & 1);
        const FluidView* views = a.views[buf];
        const T* A = (const T*) a.pop[(a.cur + s) & 1];
        T* B = (T*) a.pop[(a.cur + s + 1) & 1];
        // Phase 1.  The sums of the previous step (those of the launch's first step are complete already).
        if (s > 0)
            for (int r = blockIdx.x; r < a.numReplicas; r += gridDim.x)
                finishReplica(a, r, BT/32);
        if (a.coupled) {
            // Pair forces, all pairs of each replica in bead order (as batchPairKernel).  The positions were written in
            // this launch by other blocks: they are read once through L2 into shared-memory tiles, which every bead of
            // the block then reads.
            for (int r = blockIdx.x; r < a.numReplicas; r += gridDim.x) {
                const ReplicaTable& rt = a.table[r];
                const double* x = a.pos + 3*(size_t) rt.firstParticle;
                double* out = a.fpair + 3*(size_t) rt.firstParticle;
                const int n = rt.numParticles;
                for (int i0 = 0; i0 < n; i0 += blockDim.x) {
                    const int i = i0 + threadIdx.x;
                    double xi[3] = {0, 0, 0}, f[3] = {0, 0, 0};
                    if (i < n)
                        for (int k = 0; k < 3; k++)
                            xi[k] = __ldcg(&x[3*i+k]);
                    for (int j0 = 0; j0 < n && a.pair.type != LBM_PAIR_NONE; j0 += kPairTile) {
                        const int count = min(kPairTile, n - j0);
                        __syncthreads();
                        for (int e = threadIdx.x; e < 3*count; e += blockDim.x)
                            pairTile[e] = __ldcg(&x[3*j0 + e]);
                        __syncthreads();
                        if (i >= n)
                            continue;
                        for (int jj = 0; jj < count; jj++) {
                            if (j0 + jj == i)
                                continue;
                            double d[3];
                            for (int k = 0; k < 3; k++) {
                                d[k] = xi[k] - pairTile[3*jj+k];
                                d[k] -= rt.box[k]*rint(d[k]/rt.box[k]);
                            }
                            double r2 = d[0]*d[0] + d[1]*d[1] + d[2]*d[2];
                            if (r2 >= a.pair.rc2 || r2 == 0.0)
                                continue;
                            double s2 = a.pair.sigma2/r2, s6 = s2*s2*s2;
                            double scale = 24.0*a.pair.eps*s6*(2.0*s6 - 1.0)/r2;
                            for (int k = 0; k < 3; k++)
                                f[k] += scale*d[k];
                        }
                    }
                    if (i < n)
                        for (int k = 0; k < 3; k++)
                            out[3*i+k] = f[k];
                }
            }
            int* nodes = a.slotNode[buf];
            const int* oldNodes = a.slotNode[1 - buf];
            const FluidView* oldViews = a.views[1 - buf];
            for (long long t = firstThread; t < totalSlots; t += threads) {
                const int p = (int) (t/a.slots), sl = (int) (t - (long long) p*a.slots);
                const int r = a.particleReplica[p];
                const ReplicaTable& rt = a.table[r];
                const int p0 = rt.firstParticle, i = p - p0;
                const size_t so = (size_t) p0*a.slots;
                // The clear of slot t of the previous step (reaction buffer 1 - buf).
                const FluidView& of = oldViews[r];
                const long long node = __ldcg(&oldNodes[t]);
                R* reaction = (R*) const_cast<void*>(of.reaction);
                *reinterpret_cast<V*>(reaction + 4*node) = Vec4<R>::make(0, 0, 0, 0);
                const long long row = node/of.nx;
                const int xx = (int) (node - row*of.nx);
                const_cast<uint32_t*>(of.reactMask)[row*of.wordsPerRow + xx/32] = 0u;
                // The slot with the nodes' j/rho before the removal (applied in phase 2).
                stencilSlot<T, R, true>(A + (size_t) 19*rt.nodeOffset, views[r], a.cviews[r], a.pos + 3*(size_t) p0,
                                        (long long) i*a.slots + sl, 0, 0, nodes + so, slotWeight + so, slotU + so);
            }
        }
        if (!gridSync(a.barrier, a.status, a.pollLimit))
            return;
        if (a.coupled) {
            // Phase 2: explicit drag and reaction, then the leapfrog of the bead (v += dt F/m, x += dt v).
            int* nodes = a.slotNode[buf];
            for (int p = firstWarp; p < a.totalParticles; p += warps) {
                const int r = a.particleReplica[p];
                const ReplicaTable& rt = a.table[r];
                const FluidView& f = views[r];
                const int p0 = rt.firstParticle;
                const size_t so = (size_t) p0*a.slots;
                const bool remove = rt.removeFrequency > 0 && step%rt.removeFrequency == 0;
                explicitParticle<R, true>(f, a.cviews[r], a.vel + 3*(size_t) p0, nodes + so, slotWeight + so, slotU + so,
                                          p - p0, lane, step, 1, a.fdrag + 3*(size_t) p0,
                                          (R*) const_cast<void*>(f.reaction), const_cast<uint32_t*>(f.reactMask), a.wall,
                                          remove ? f.stats->ucm : nullptr);
                __syncwarp();
                if (lane < 3) {
                    const size_t k = 3*(size_t) p + lane;
                    const double force = __ldcg(&a.fpair[k]) + a.fdrag[k];
                    const double v = a.vel[k] + rt.dt*force*a.invMass[p];
                    a.vel[k] = v;
                    a.pos[k] += rt.dt*v;
                }
            }
            if (!gridSync(a.barrier, a.status, a.pollLimit))
                return;
        }
        // Phase 3: the dense step, per-warp partial sums (formed into the replica's sums in the next phase 1).
        for (int w = blockIdx.x; w < a.numItems; w += gridDim.x) {
            const int r = a.itemReplica[w];
            const FluidView& v = views[r];
            const ReplicaTable& rt = a.table[r];
            const int remove = rt.removeFrequency > 0 && step%rt.removeFrequency == 0;
            // The removal velocity of this step, written by phase 1 of this launch: read through L2.
            const double ucm[3] = {__ldcg(&v.stats->ucm[0]), __ldcg(&v.stats->ucm[1]), __ldcg(&v.stats->ucm[2])};
            const unsigned N = rt.numNodes;
            if constexpr (std::is_same<T, float>::value) {
                if (rt.paired) {
                    float sums[4] = {0, 0, 0, 0};
                    const size_t base = (size_t) 19*rt.nodeOffset;
                    const unsigned unit = (unsigned) (w - rt.firstItem)*BT + threadIdx.x;
                    if (a.coupled)
                        pairedUnit<true, FLUCT, true>(A + base, B + base, v, N, unit, rt.paired, remove, ucm, step, sums);
                    else
                        pairedUnit<false, FLUCT, true>(A + base, B + base, v, N, unit, rt.paired, remove, ucm, step, sums);
                    double s0 = warpReduceSum((double) sums[0]), s1 = warpReduceSum((double) sums[1]);
                    double s2 = warpReduceSum((double) sums[2]), s3 = warpReduceSum((double) sums[3]);
                    if (lane == 0) {
                        double* out = a.partials + 4*((size_t) w*(BT/32) + warp);
                        out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
                    }
                    continue;
                }
            }
            const CollideConstants<R> k = collideConstants<R>(v.omega, v.g, ucm, remove, v.mu, v.seed);
            const unsigned local = (unsigned) (w - rt.firstItem)*BT + threadIdx.x;
            R sm = 0, sx = 0, sy = 0, sz = 0;
            if (local < N) {
                const int nx = v.nx, ny = v.ny, nz = v.nz;
                const unsigned row = local/(unsigned) nx;
                const int x = (int) (local - row*nx);
                const int y = (int) (row%ny), z = (int) (row/ny);
                R ex = 0, ey = 0, ez = 0;
                if (a.coupled) {
                    uint32_t word = __ldcg(&v.reactMask[(size_t) row*v.wordsPerRow + x/32]);
                    if ((word >> (x%32)) & 1u) {
                        const R* rp = reinterpret_cast<const R*>(v.reaction) + 4*(size_t) local;
                        ex = __ldcg(rp);
                        ey = __ldcg(rp + 1);
                        ez = __ldcg(rp + 2);
                    }
                }
                const size_t base = (size_t) 19*rt.nodeOffset;
                collideNode<T, R, FLUCT, true>(A + base, B + base, N, local, x, y, z, nx, ny, nz, k, ex, ey, ez, step, sm,
                                               sx, sy, sz);
            }
            double s0 = warpReduceSum((double) sm), s1 = warpReduceSum((double) sx);
            double s2 = warpReduceSum((double) sy), s3 = warpReduceSum((double) sz);
            if (lane == 0) {
                double* out = a.partials + 4*((size_t) w*(BT/32) + warp);
                out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
            }
        }
        if (!gridSync(a.barrier, a.status, a.pollLimit))
            return;
    }
    // The sums of the last step.
    for (int r = blockIdx.x; r < a.numReplicas; r += gridDim.x)
        finishReplica(a, r, BT/32);
    if (blockIdx.x == 0 && threadIdx.x == 0)
        a.clock->step = step0 + a.steps;
}

int stencilWidth(int stencil) {
    switch (stencil) {
    case LBM_STENCIL_TRILINEAR: return 2;
    case LBM_STENCIL_THREEPOINT: return 3;
    case LBM_STENCIL_KEYS: return 4;
    default: return 1;
    }
}

} // namespace

class BatchEngine {
public:
    BatchEngine(int numReplicas, const LbmLatticeParameters* lattices, const int* numParticles, const double* masses,
                const double* positions, const LbmBatchPairForce* pair, const LbmOptions* options);
    ~BatchEngine();
    void step(int steps);
    int autotune(int graphSteps, double* denseMs);
    void getParticles(double* positions, double* velocities);
    void setVelocities(const double* velocities);
    void getFluidState(int replica, double* state);
    void temperatures(double* fluidKT, double* beadKT);
    void info(long long* totalNodes, long long* steps, long long* launchCount, int* threads, int* graphSteps);
    void setPersistent(bool enable);
    void setBarrierPolls(long long polls);
private:
    template <typename T> void launchStep();
    template <typename T, int BT> void launchPersistent(int steps);
    void launchPersistentAny(int steps);
    void checkStatus();
    template <typename T, int BT> void launchDense(const void* A, void* B);
    void launchDenseAny(const void* A, void* B);
    template <typename T, int BT> int denseGrid();
    void buildItems(int threads);
    void releaseGraph();
    void release();

    int numReplicas, storage, device, slots, totalParticles;
    bool ownStream, fluctuate, coupled;
    cudaStream_t stream;
    long long totalNodes, stepsTaken, launches;
    int threads, graphSteps, numItems, sms;
    std::vector<LbmLatticeParameters> lattices;
    std::vector<ReplicaTable> tableHost;
    std::vector<FluidView> viewsHost;
    std::vector<double> cellEnergyHost;
    PairParams pairParams;
    void* pop[2];
    int cur;
    FluidView* viewsDev;
    CouplingView* cviewsDev;
    ReplicaTable* tableDev;
    StepStats* statsDev;
    BatchClock* clockDev;
    int* itemReplicaDev;
    double* partialsDev;
    void* reactionDev;
    uint32_t* maskDev;
    int* particleReplicaDev;
    double *posDev, *velDev, *fpairDev, *fdragDev, *invMassDev, *massDev, *cellMassDev, *wallDev, *cellEnergyDev;
    int* slotNodeDev;
    void *slotWeightDev, *slotUDev;
    cudaGraphExec_t graphExec;
    int graphCur;
    // The persistent step (batchPersistentKernel): the reaction buffers, masks and slot nodes come in two halves
    // (buffer step & 1), viewsDev holds the replicas' views for both, and the grid barrier its counter and status.
    bool persistent;
    unsigned maskWordsTotal;
    unsigned* barrierDev;
    int* statusDev;
    long long barrierPolls;
};

BatchEngine::BatchEngine(int nr, const LbmLatticeParameters* ls, const int* np, const double* masses,
                         const double* positions, const LbmBatchPairForce* pair, const LbmOptions* options)
        : numReplicas(nr), storage(options->storage), device(options->device), slots(1), totalParticles(0),
          ownStream(false), fluctuate(false), coupled(false), stream(nullptr), totalNodes(0), stepsTaken(0), launches(0),
          threads(256), graphSteps(20), numItems(0), sms(0), cur(0), viewsDev(nullptr), cviewsDev(nullptr),
          tableDev(nullptr), statsDev(nullptr), clockDev(nullptr), itemReplicaDev(nullptr), partialsDev(nullptr),
          reactionDev(nullptr), maskDev(nullptr), particleReplicaDev(nullptr), posDev(nullptr), velDev(nullptr),
          fpairDev(nullptr), fdragDev(nullptr), invMassDev(nullptr), massDev(nullptr), cellMassDev(nullptr),
          wallDev(nullptr), cellEnergyDev(nullptr), slotNodeDev(nullptr), slotWeightDev(nullptr), slotUDev(nullptr),
          graphExec(nullptr), graphCur(0), persistent(true), maskWordsTotal(0), barrierDev(nullptr), statusDev(nullptr), barrierPolls(1LL << 26) {
    pop[0] = pop[1] = nullptr;
    if (nr <= 0 || ls == nullptr || np == nullptr)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_create: no replicas");
    if (storage != LBM_STORAGE_F64 && storage != LBM_STORAGE_F32)
        throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_batch_create: a batch stores its populations in FP64 or FP32");
    lattices.assign(ls, ls + nr);
    int stencil = lattices[0].interpolation_stencil;
    std::random_device rd;
    unsigned maskWords = 0;
    for (int r = 0; r < nr; r++) {
        LbmLatticeParameters& l = lattices[r];
        if (l.nx <= 0 || l.ny <= 0 || l.nz <= 0 || !(l.tau > 0.5) || np[r] < 0)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_create: invalid lattice or particle count of a replica");
        for (int f = 0; f < 6; f++)
            if (l.face_boundary[f] != LBM_BOUNDARY_PERIODIC)
                throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_batch_create: the replicas of a batch are periodic lattices");
        if (np[r] > 0 && l.drag_scheme != LBM_DRAG_EXPLICIT)
            throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_batch_create: the replicas of a batch use the explicit drag");
        if (l.interpolation_stencil != stencil)
            throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_batch_create: the replicas of a batch share one interpolation stencil");
        if (l.initial_velocity[0] != 0 || l.initial_velocity[1] != 0 || l.initial_velocity[2] != 0)
            throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_batch_create: the fluids of a batch start at rest");
        if (l.random_number_seed == 0)
            do
                l.random_number_seed = (int) (rd() & 0x7fffffffu);
            while (l.random_number_seed == 0);
        ReplicaTable t;
        std::memset(&t, 0, sizeof(t));
        long long n = (long long) l.nx*l.ny*l.nz;
        t.nodeOffset = (unsigned) totalNodes;
        t.numNodes = (unsigned) n;
        t.paired = storage != LBM_STORAGE_F32 ? 0 : (l.nx%2 == 0 ? 1 : 2);
        t.units = t.paired == 0 ? (unsigned) n : t.paired == 1 ? (unsigned) (n/2)
                                                               : (unsigned) (((l.nx + 1)/2)*(long long) l.ny*l.nz);
        t.firstParticle = totalParticles;
        t.numParticles = np[r];
        t.removeFrequency = l.momentum_removal_frequency;
        t.dt = l.dt;
        t.box[0] = l.nx*l.dx; t.box[1] = l.ny*l.dx; t.box[2] = l.nz*l.dx;
        tableHost.push_back(t);
        totalNodes += n + (n & 1);       // every replica starts at an even node (aligned float2 words)
        totalParticles += np[r];
        maskWords += (unsigned) (((l.nx + 31)/32)*l.ny*l.nz);
        if (totalNodes >= (1LL << 32) - 1024)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_create: the replicas have too many nodes together (2^32)");
        if (l.fluid_fluctuations && l.fluid_kT > 0)
            fluctuate = true;
    }
    coupled = totalParticles > 0;
    slots = stencilWidth(stencil);
    slots = slots*slots*slots;
    if ((long long) totalParticles*slots >= (1LL << 31))
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_create: too many particles for the interpolation stencil "
                    "(particles x stencil nodes must stay below 2^31)");
    if (pair != nullptr) {
        pairParams.type = pair->pair_type;
        pairParams.sigma2 = pair->sigma*pair->sigma;
        pairParams.eps = pair->epsilon;
        double rc = pair->pair_type == LBM_PAIR_WCA ? std::pow(2.0, 1.0/6.0)*pair->sigma : pair->cutoff;
        pairParams.rc2 = rc*rc;
    }
    else
        pairParams = PairParams{LBM_PAIR_NONE, 0, 0, 0};
    try {
        CUDA_CHECK(cudaSetDevice(device));
        CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        if (options->stream != nullptr)
            stream = (cudaStream_t) options->stream;
        else {
            CUDA_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            ownStream = true;
        }
        size_t e = storage == LBM_STORAGE_F64 ? 8 : 4;
        for (int k = 0; k < 2; k++) {
            CUDA_CHECK(cudaMalloc(&pop[k], (size_t) 19*totalNodes*e));
            CUDA_CHECK(cudaMemsetAsync(pop[k], 0, (size_t) 19*totalNodes*e, stream));
        }
        CUDA_CHECK(cudaMalloc(&statsDev, sizeof(StepStats)*nr));
        CUDA_CHECK(cudaMemsetAsync(statsDev, 0, sizeof(StepStats)*nr, stream));
        CUDA_CHECK(cudaMalloc(&clockDev, sizeof(BatchClock)));
        CUDA_CHECK(cudaMemsetAsync(clockDev, 0, sizeof(BatchClock), stream));
        CUDA_CHECK(cudaMalloc(&wallDev, sizeof(double)*4));
        CUDA_CHECK(cudaMemsetAsync(wallDev, 0, sizeof(double)*4, stream));
        maskWordsTotal = maskWords;
        if (coupled) {
            // Two halves (the reactions of even and odd steps in the persistent step).
            CUDA_CHECK(cudaMalloc(&reactionDev, 2*4*e*(size_t) totalNodes));
            CUDA_CHECK(cudaMemsetAsync(reactionDev, 0, 2*4*e*(size_t) totalNodes, stream));
            CUDA_CHECK(cudaMalloc(&maskDev, 2*sizeof(uint32_t)*(size_t) maskWords));
            CUDA_CHECK(cudaMemsetAsync(maskDev, 0, 2*sizeof(uint32_t)*(size_t) maskWords, stream));
        }
        CUDA_CHECK(cudaMalloc(&statusDev, sizeof(int)*2));
        CUDA_CHECK(cudaMemsetAsync(statusDev, 0, sizeof(int)*2, stream));
        barrierDev = reinterpret_cast<unsigned*>(statusDev + 1);
        // Views of the replicas.
        std::vector<CouplingView> cviews(nr);
        std::vector<double> cellMass(nr);
        unsigned maskOffset = 0;
        size_t v3 = sizeof(double)*3*(size_t) std::max(1, totalParticles);
        CUDA_CHECK(cudaMalloc(&posDev, v3));
        CUDA_CHECK(cudaMalloc(&velDev, v3));
        CUDA_CHECK(cudaMalloc(&fpairDev, v3));
        CUDA_CHECK(cudaMalloc(&fdragDev, v3));
        CUDA_CHECK(cudaMemsetAsync(velDev, 0, v3, stream));
        CUDA_CHECK(cudaMemsetAsync(fpairDev, 0, v3, stream));
        CUDA_CHECK(cudaMemsetAsync(fdragDev, 0, v3, stream));
        size_t s1 = sizeof(double)*(size_t) std::max(1, totalParticles);
        CUDA_CHECK(cudaMalloc(&invMassDev, s1));
        CUDA_CHECK(cudaMalloc(&massDev, s1));
        CUDA_CHECK(cudaMalloc(&cellMassDev, s1));
        std::vector<double> invMass(std::max(1, totalParticles), 0.0), massRel(std::max(1, totalParticles), 0.0);
        std::vector<int> particleReplica(std::max(1, totalParticles), 0);
        for (int r = 0; r < nr; r++) {
            const LbmLatticeParameters& l = lattices[r];
            ReplicaTable& t = tableHost[r];
            FluidView v;
            std::memset(&v, 0, sizeof(v));
            v.nx = l.nx; v.ny = l.ny; v.nz = l.nz;
            v.n = t.numNodes;
            v.wordsPerRow = (l.nx + 31)/32;
            v.omega = l.omega;
            for (int a = 0; a < 3; a++)
                v.g[a] = l.body_acceleration[a];
            v.numFluid = (double) t.numNodes;
            v.seed = (uint32_t) l.random_number_seed;
            cellMass[r] = l.density*l.dx*l.dx*l.dx;
            bool fl = l.fluid_fluctuations && l.fluid_kT > 0;
            v.mu = fl ? 3.0*l.fluid_kT*l.dt*l.dt/(cellMass[r]*l.dx*l.dx) : 0.0;
            v.stats = statsDev + r;
            if (coupled) {
                v.reactMask = maskDev + maskOffset;
                v.reaction = (const char*) reactionDev + 4*e*(size_t) t.nodeOffset;
            }
            maskOffset += (unsigned) (v.wordsPerRow*l.ny*l.nz);
            viewsHost.push_back(v);
            cviews[r] = makeCouplingView(l, v, t.numParticles, stencilWidth(stencil), massDev + t.firstParticle);
            cellEnergyHost.push_back(cellMass[r]*(l.dx/l.dt)*(l.dx/l.dt));
            for (int i = 0; i < t.numParticles; i++) {
                int p = t.firstParticle + i;
                if (!(masses[p] > 0))
                    throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_create: coupled particles must have a positive mass");
                invMass[p] = 1.0/masses[p];
                massRel[p] = masses[p]/cellMass[r];
                particleReplica[p] = r;
            }
        }
        // The views of the second half of the reaction buffers follow those of the first.
        std::vector<FluidView> views2 = viewsHost;
        for (int r = 0; r < nr; r++)
            if (coupled) {
                views2[r].reaction = (const char*) viewsHost[r].reaction + 4*e*(size_t) totalNodes;
                views2[r].reactMask = viewsHost[r].reactMask + maskWords;
            }
        views2.insert(views2.begin(), viewsHost.begin(), viewsHost.end());
        CUDA_CHECK(cudaMalloc(&viewsDev, sizeof(FluidView)*2*nr));
        CUDA_CHECK(cudaMemcpy(viewsDev, views2.data(), sizeof(FluidView)*2*nr, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMalloc(&cviewsDev, sizeof(CouplingView)*nr));
        CUDA_CHECK(cudaMemcpy(cviewsDev, cviews.data(), sizeof(CouplingView)*nr, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMalloc(&cellEnergyDev, sizeof(double)*nr));
        CUDA_CHECK(cudaMemcpy(cellEnergyDev, cellEnergyHost.data(), sizeof(double)*nr, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(invMassDev, invMass.data(), s1, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(massDev, massRel.data(), s1, cudaMemcpyHostToDevice));
        std::vector<double> m(std::max(1, totalParticles), 0.0);
        for (int p = 0; p < totalParticles; p++)
            m[p] = masses[p];
        CUDA_CHECK(cudaMemcpy(cellMassDev, m.data(), s1, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMalloc(&particleReplicaDev, sizeof(int)*particleReplica.size()));
        CUDA_CHECK(cudaMemcpy(particleReplicaDev, particleReplica.data(), sizeof(int)*particleReplica.size(), cudaMemcpyHostToDevice));
        if (totalParticles > 0)
            CUDA_CHECK(cudaMemcpy(posDev, positions, sizeof(double)*3*(size_t) totalParticles, cudaMemcpyHostToDevice));
        size_t ns = (size_t) std::max(1, totalParticles)*slots;
        CUDA_CHECK(cudaMalloc(&slotNodeDev, 2*sizeof(int)*ns));
        CUDA_CHECK(cudaMemsetAsync(slotNodeDev, 0, 2*sizeof(int)*ns, stream));
        CUDA_CHECK(cudaMalloc(&slotWeightDev, e*ns));
        CUDA_CHECK(cudaMalloc(&slotUDev, 4*e*ns));
        CUDA_CHECK(cudaMalloc(&tableDev, sizeof(ReplicaTable)*nr));
        buildItems(threads);
        CUDA_CHECK(cudaStreamSynchronize(stream));
    }
    catch (...) {
        release();
        throw;
    }
}

BatchEngine::~BatchEngine() {
    release();
}

void BatchEngine::releaseGraph() {
    if (graphExec)
        cudaGraphExecDestroy(graphExec);
    graphExec = nullptr;
}

void BatchEngine::release() {
    if (stream)
        cudaStreamSynchronize(stream);
    releaseGraph();
    void* ptrs[] = {pop[0], pop[1], viewsDev, cviewsDev, tableDev, statsDev, clockDev, itemReplicaDev, partialsDev,
                    reactionDev, maskDev, particleReplicaDev, posDev, velDev, fpairDev, fdragDev, invMassDev, massDev,
                    cellMassDev, wallDev, cellEnergyDev, slotNodeDev, slotWeightDev, slotUDev, statusDev};
    for (void* p : ptrs)
        cudaFree(p);
    pop[0] = pop[1] = nullptr;
    viewsDev = nullptr; cviewsDev = nullptr; tableDev = nullptr; statsDev = nullptr; clockDev = nullptr;
    itemReplicaDev = nullptr; partialsDev = nullptr; reactionDev = nullptr; maskDev = nullptr; particleReplicaDev = nullptr;
    posDev = velDev = fpairDev = fdragDev = invMassDev = massDev = cellMassDev = wallDev = cellEnergyDev = nullptr;
    slotNodeDev = nullptr; slotWeightDev = slotUDev = nullptr;
    statusDev = nullptr; barrierDev = nullptr;
    if (ownStream && stream)
        cudaStreamDestroy(stream);
    stream = nullptr;
}

// Work items of `bt` consecutive units of one replica (nodes, or pairs of a paired replica), and the per-warp partial
// sums they write.
void BatchEngine::buildItems(int bt) {
    std::vector<int> itemReplica;
    for (int r = 0; r < numReplicas; r++) {
        ReplicaTable& t = tableHost[r];
        t.firstItem = (int) itemReplica.size();
        t.numItems = (int) ((t.units + bt - 1)/bt);
        itemReplica.insert(itemReplica.end(), t.numItems, r);
    }
    numItems = (int) itemReplica.size();
    threads = bt;
    cudaFree(itemReplicaDev);
    cudaFree(partialsDev);
    itemReplicaDev = nullptr;
    partialsDev = nullptr;
    CUDA_CHECK(cudaMalloc(&itemReplicaDev, sizeof(int)*itemReplica.size()));
    CUDA_CHECK(cudaMemcpyAsync(itemReplicaDev, itemReplica.data(), sizeof(int)*itemReplica.size(), cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaMalloc(&partialsDev, sizeof(double)*4*(size_t) numItems*(bt/32)));
    CUDA_CHECK(cudaMemcpyAsync(tableDev, tableHost.data(), sizeof(ReplicaTable)*numReplicas, cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

template <typename T, int BT>
int BatchEngine::denseGrid() {
    int perSM = 0;
    if (fluctuate && coupled)
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, batchStreamCollideKernel<T, T, true, true, BT>, BT, 0));
    else if (fluctuate)
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, batchStreamCollideKernel<T, T, false, true, BT>, BT, 0));
    else if (coupled)
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, batchStreamCollideKernel<T, T, true, false, BT>, BT, 0));
    else
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, batchStreamCollideKernel<T, T, false, false, BT>, BT, 0));
    return std::max(1, std::min(numItems, std::max(1, perSM)*sms));
}

template <typename T, int BT>
void BatchEngine::launchDense(const void* A, void* B) {
    int grid = denseGrid<T, BT>();
    const T* a = (const T*) A;
    T* b = (T*) B;
    if (fluctuate && coupled)
        batchStreamCollideKernel<T, T, true, true, BT><<<grid, BT, 0, stream>>>(a, b, viewsDev, tableDev, itemReplicaDev, numItems, clockDev, partialsDev);
    else if (fluctuate)
        batchStreamCollideKernel<T, T, false, true, BT><<<grid, BT, 0, stream>>>(a, b, viewsDev, tableDev, itemReplicaDev, numItems, clockDev, partialsDev);
    else if (coupled)
        batchStreamCollideKernel<T, T, true, false, BT><<<grid, BT, 0, stream>>>(a, b, viewsDev, tableDev, itemReplicaDev, numItems, clockDev, partialsDev);
    else
        batchStreamCollideKernel<T, T, false, false, BT><<<grid, BT, 0, stream>>>(a, b, viewsDev, tableDev, itemReplicaDev, numItems, clockDev, partialsDev);
    CUDA_CHECK(cudaGetLastError());
    launches++;
}

void BatchEngine::launchDenseAny(const void* A, void* B) {
    bool f64 = storage == LBM_STORAGE_F64;
    switch (threads) {
    case 128: f64 ? launchDense<double, 128>(A, B) : launchDense<float, 128>(A, B); break;
    case 512: f64 ? launchDense<double, 512>(A, B) : launchDense<float, 512>(A, B); break;
    default: f64 ? launchDense<double, 256>(A, B) : launchDense<float, 256>(A, B); break;
    }
}

// One lattice step of every replica.
template <typename T>
void BatchEngine::launchStep() {
    typedef T R;
    int gridP = std::max(1, std::min(sms*8, (totalParticles*32 + kBatchThreads - 1)/kBatchThreads));
    long long totalSlots = (long long) totalParticles*slots;
    int gridS = (int) std::max(1LL, std::min((long long) sms*16, (totalSlots + kBatchThreads - 1)/kBatchThreads));
    const T* A = (const T*) pop[cur];
    T* B = (T*) pop[1 - cur];
    if (coupled) {
        batchPairKernel<<<std::min(numReplicas, sms*8), kBatchThreads, 0, stream>>>(tableDev, numReplicas, pairParams, posDev, fpairDev);
        batchStencilKernel<T, R><<<gridS, kBatchThreads, 0, stream>>>(A, viewsDev, cviewsDev, tableDev, particleReplicaDev,
                                                                      totalSlots, slots, posDev, clockDev, slotNodeDev,
                                                                      (R*) slotWeightDev, (typename Vec4<R>::type*) slotUDev);
        batchExplicitKernel<R><<<gridP, kBatchThreads, 0, stream>>>(viewsDev, cviewsDev, tableDev, particleReplicaDev,
                                                                    totalParticles, slots, velDev, slotNodeDev,
                                                                    (const R*) slotWeightDev,
                                                                    (const typename Vec4<R>::type*) slotUDev, clockDev,
                                                                    fdragDev, wallDev);
        launches += 3;
    }
    launchDenseAny(A, B);
    batchFinishKernel<<<std::min(numReplicas, sms*8), kBatchThreads, 0, stream>>>(partialsDev, tableDev, viewsDev,
                                                                                 numReplicas, threads/32, clockDev);
    launches++;
    if (coupled) {
        batchClearKernel<R><<<gridS, kBatchThreads, 0, stream>>>(viewsDev, particleReplicaDev, totalSlots, slots, slotNodeDev);
        int gridL = std::max(1, std::min(sms*8, (3*totalParticles + kBatchThreads - 1)/kBatchThreads));
        batchLeapfrogKernel<<<gridL, kBatchThreads, 0, stream>>>(tableDev, particleReplicaDev, totalParticles, invMassDev,
                                                                 fpairDev, fdragDev, posDev, velDev);
        launches += 2;
    }
    CUDA_CHECK(cudaGetLastError());
    cur = 1 - cur;
}

template <typename T, int BT>
void BatchEngine::launchPersistent(int steps) {
    typedef T R;
    // Every block must be resident (the grid barriers): the grid is the occupancy of this variant times the SMs.
    int perSM = 0;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &perSM, fluctuate ? batchPersistentKernel<T, R, true, BT> : batchPersistentKernel<T, R, false, BT>, BT, 0));
    if (perSM < 1)
        throw Error(LBM_ERR_NOT_SUPPORTED, "lbm_batch_step: the persistent step does not fit on a multiprocessor");
    PersistentArgs a;
    std::memset(&a, 0, sizeof(a));
    a.views[0] = viewsDev;
    a.views[1] = viewsDev + numReplicas;
    a.cviews = cviewsDev;
    a.table = tableDev;
    a.itemReplica = itemReplicaDev;
    a.particleReplica = particleReplicaDev;
    a.numReplicas = numReplicas;
    a.numItems = numItems;
    a.totalParticles = totalParticles;
    a.slots = slots;
    a.coupled = coupled ? 1 : 0;
    a.steps = steps;
    a.pair = pairParams;
    a.pop[0] = pop[0];
    a.pop[1] = pop[1];
    a.cur = cur;
    a.partials = partialsDev;
    a.clock = clockDev;
    a.pos = posDev; a.vel = velDev; a.fpair = fpairDev; a.fdrag = fdragDev; a.invMass = invMassDev; a.wall = wallDev;
    a.slotNode[0] = slotNodeDev;
    a.slotNode[1] = slotNodeDev + (size_t) std::max(1, totalParticles)*slots;
    a.slotWeight = slotWeightDev;
    a.slotU = slotUDev;
    a.barrier = barrierDev;
    a.status = statusDev;
    a.pollLimit = barrierPolls;
    int grid = perSM*sms;
    void* args[] = {&a};
    CUDA_CHECK(cudaMemsetAsync(barrierDev, 0, sizeof(unsigned), stream));
    CUDA_CHECK(cudaLaunchCooperativeKernel(fluctuate ? (const void*) batchPersistentKernel<T, R, true, BT> :
                                           (const void*) batchPersistentKernel<T, R, false, BT>,
                                           grid, BT, args, 0, stream));
    launches++;
    cur = (cur + steps) & 1;
}

void BatchEngine::launchPersistentAny(int steps) {
    bool f64 = storage == LBM_STORAGE_F64;
    switch (threads) {
    case 128: f64 ? launchPersistent<double, 128>(steps) : launchPersistent<float, 128>(steps); break;
    case 512: f64 ? launchPersistent<double, 512>(steps) : launchPersistent<float, 512>(steps); break;
    default: f64 ? launchPersistent<double, 256>(steps) : launchPersistent<float, 256>(steps); break;
    }
}

// A timed-out grid barrier of the persistent step leaves LBM_ERR_DEVICE_TIMEOUT in the status word: reported (and
// cleared) by the next call that synchronizes.
void BatchEngine::checkStatus() {
    int status = 0;
    CUDA_CHECK(cudaMemcpyAsync(&status, statusDev, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    if (status != 0) {
        // The blocks left the launch at different points: the reaction buffers may hold partial values.  Clear them,
        // so that later steps start from a consistent state.
        CUDA_CHECK(cudaMemsetAsync(statusDev, 0, sizeof(int), stream));
        if (coupled) {
            size_t e = storage == LBM_STORAGE_F64 ? 8 : 4;
            CUDA_CHECK(cudaMemsetAsync(reactionDev, 0, 2*4*e*(size_t) totalNodes, stream));
            CUDA_CHECK(cudaMemsetAsync(maskDev, 0, 2*sizeof(uint32_t)*(size_t) maskWordsTotal, stream));
        }
        CUDA_CHECK(cudaStreamSynchronize(stream));
        throw Error((LbmStatus) status, "lbm_batch: a grid barrier of the persistent step timed out; the steps of that "
                    "launch are incomplete");
    }
}

void BatchEngine::setPersistent(bool enable) {
    CUDA_CHECK(cudaSetDevice(device));
    if (enable == persistent)
        return;
    releaseGraph();
    // The two step forms keep the reactions of a step in different halves of the buffers: start from clean ones (a
    // step's reactions are not needed after it).
    size_t e = storage == LBM_STORAGE_F64 ? 8 : 4;
    if (coupled) {
        CUDA_CHECK(cudaMemsetAsync(reactionDev, 0, 2*4*e*(size_t) totalNodes, stream));
        CUDA_CHECK(cudaMemsetAsync(maskDev, 0, 2*sizeof(uint32_t)*(size_t) maskWordsTotal, stream));
    }
    persistent = enable;
}

void BatchEngine::setBarrierPolls(long long polls) {
    if (polls < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_set_barrier_polls: the limit must not be negative");
    barrierPolls = polls > 0 ? polls : (1LL << 26);
    releaseGraph();
}

void BatchEngine::step(int steps) {
    CUDA_CHECK(cudaSetDevice(device));
    if (steps < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_step: negative step count");
    if (persistent) {
        // graphSteps steps per launch, captured once into a graph (the launch and the clear of its barrier) and
        // replayed; the rest in one direct launch.  graphSteps is even, so a replay leaves the populations in the
        // buffer where it found them.
        int s = 0;
        if (steps >= graphSteps && graphExec == nullptr) {
            int start = cur;
            long long launches0 = launches;
            cudaGraph_t graph = nullptr;
            CUDA_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try {
                launchPersistentAny(graphSteps);
            }
            catch (...) {
                cudaStreamEndCapture(stream, &graph);
                if (graph)
                    cudaGraphDestroy(graph);
                cur = start;
                throw;
            }
            CUDA_CHECK(cudaStreamEndCapture(stream, &graph));
            cudaError_t e = cudaGraphInstantiate(&graphExec, graph, 0);
            cudaGraphDestroy(graph);
            CUDA_CHECK(e);
            cur = start;
            graphCur = start;
            launches = launches0;
        }
        if (graphExec != nullptr && cur == graphCur)
            for (; s + graphSteps <= steps; s += graphSteps) {
                CUDA_CHECK(cudaGraphLaunch(graphExec, stream));
                launches++;
            }
        if (s < steps)
            launchPersistentAny(steps - s);
        stepsTaken += steps;
        return;
    }
    long long perStep = coupled ? 7 : 2;
    if (steps >= graphSteps && graphExec == nullptr) {
        // Capture graphSteps steps (an even number, so that the populations end in the buffer they started in).
        int start = cur;
        long long launches0 = launches;
        cudaGraph_t graph = nullptr;
        CUDA_CHECK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            for (int s = 0; s < graphSteps; s++)
                storage == LBM_STORAGE_F64 ? launchStep<double>() : launchStep<float>();
        }
        catch (...) {
            cudaStreamEndCapture(stream, &graph);
            if (graph)
                cudaGraphDestroy(graph);
            cur = start;
            throw;
        }
        CUDA_CHECK(cudaStreamEndCapture(stream, &graph));
        cudaError_t e = cudaGraphInstantiate(&graphExec, graph, 0);
        cudaGraphDestroy(graph);
        CUDA_CHECK(e);
        cur = start;
        graphCur = start;
        launches = launches0;
    }
    int s = 0;
    if (graphExec != nullptr && cur != graphCur && steps > graphSteps) {
        // An odd number of steps was launched directly: one more realigns the buffers with the graph's.
        storage == LBM_STORAGE_F64 ? launchStep<double>() : launchStep<float>();
        s = 1;
    }
    if (graphExec != nullptr && cur == graphCur)
        for (; s + graphSteps <= steps; s += graphSteps) {
            CUDA_CHECK(cudaGraphLaunch(graphExec, stream));
            launches += perStep*graphSteps;
        }
    for (; s < steps; s++)
        storage == LBM_STORAGE_F64 ? launchStep<double>() : launchStep<float>();
    stepsTaken += steps;
}

int BatchEngine::autotune(int newGraphSteps, double* denseMs) {
    CUDA_CHECK(cudaSetDevice(device));
    if (newGraphSteps > 0) {
        releaseGraph();
        graphSteps = newGraphSteps + (newGraphSteps & 1);
    }
    const int candidates[3] = {128, 256, 512};
    float best = 1e30f;
    int bestThreads = threads;
    cudaEvent_t start, stop;
    CUDA_CHECK(cudaEventCreate(&start));
    CUDA_CHECK(cudaEventCreate(&stop));
    // The dense kernel reads pop[cur] and writes pop[1 - cur] and the partial sums, which the next step overwrites:
    // timing it does not advance the state.
    for (int c : candidates) {
        buildItems(c);
        for (int i = 0; i < 2; i++)
            launchDenseAny(pop[cur], pop[1 - cur]);
        CUDA_CHECK(cudaEventRecord(start, stream));
        for (int i = 0; i < 5; i++)
            launchDenseAny(pop[cur], pop[1 - cur]);
        CUDA_CHECK(cudaEventRecord(stop, stream));
        CUDA_CHECK(cudaEventSynchronize(stop));
        float ms = 0;
        CUDA_CHECK(cudaEventElapsedTime(&ms, start, stop));
        if (ms < best) {
            best = ms;
            bestThreads = c;
        }
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    releaseGraph();
    buildItems(bestThreads);
    if (denseMs)
        *denseMs = best/5.0;
    return bestThreads;
}

void BatchEngine::getParticles(double* positions, double* velocities) {
    CUDA_CHECK(cudaSetDevice(device));
    checkStatus();
    size_t v3 = sizeof(double)*3*(size_t) totalParticles;
    if (positions && totalParticles)
        CUDA_CHECK(cudaMemcpyAsync(positions, posDev, v3, cudaMemcpyDeviceToHost, stream));
    if (velocities && totalParticles)
        CUDA_CHECK(cudaMemcpyAsync(velocities, velDev, v3, cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

void BatchEngine::setVelocities(const double* velocities) {
    CUDA_CHECK(cudaSetDevice(device));
    if (totalParticles)
        CUDA_CHECK(cudaMemcpyAsync(velDev, velocities, sizeof(double)*3*(size_t) totalParticles, cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

void BatchEngine::getFluidState(int r, double* state) {
    CUDA_CHECK(cudaSetDevice(device));
    checkStatus();
    CUDA_CHECK(cudaSetDevice(device));
    if (r < 0 || r >= numReplicas)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "lbm_batch_get_fluid_state: no such replica");
    const ReplicaTable& t = tableHost[r];
    double* out = nullptr;
    CUDA_CHECK(cudaMalloc(&out, sizeof(double)*19*(size_t) t.numNodes));
    int grid = (int) std::min(4096LL, (19LL*t.numNodes + 255)/256);
    size_t e = storage == LBM_STORAGE_F64 ? 8 : 4;
    const char* A = (const char*) pop[cur] + e*19*(size_t) t.nodeOffset;
    if (storage == LBM_STORAGE_F64)
        batchGatherKernel<double><<<grid, 256, 0, stream>>>((const double*) A, viewsHost[r], out);
    else
        batchGatherKernel<float><<<grid, 256, 0, stream>>>((const float*) A, viewsHost[r], out);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(state, out, sizeof(double)*19*(size_t) t.numNodes, cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess)
        err = cudaStreamSynchronize(stream);
    cudaFree(out);
    CUDA_CHECK(err);
}

void BatchEngine::temperatures(double* fluidKT, double* beadKT) {
    CUDA_CHECK(cudaSetDevice(device));
    checkStatus();
    CUDA_CHECK(cudaSetDevice(device));
    double* out = nullptr;
    CUDA_CHECK(cudaMalloc(&out, sizeof(double)*2*numReplicas));
    int grid = std::min(numReplicas, sms*8);
    if (storage == LBM_STORAGE_F64)
        batchTemperatureKernel<double><<<grid, kBatchThreads, 0, stream>>>((const double*) pop[cur], viewsDev, tableDev,
                                                                           numReplicas, cellEnergyDev, velDev, cellMassDev, out);
    else
        batchTemperatureKernel<float><<<grid, kBatchThreads, 0, stream>>>((const float*) pop[cur], viewsDev, tableDev,
                                                                          numReplicas, cellEnergyDev, velDev, cellMassDev, out);
    std::vector<double> host(2*numReplicas);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(host.data(), out, sizeof(double)*2*numReplicas, cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess)
        err = cudaStreamSynchronize(stream);
    cudaFree(out);
    CUDA_CHECK(err);
    for (int r = 0; r < numReplicas; r++) {
        if (fluidKT)
            fluidKT[r] = host[2*r];
        if (beadKT)
            beadKT[r] = host[2*r+1];
    }
}

void BatchEngine::info(long long* nodes, long long* steps, long long* launchCount, int* t, int* g) {
    if (nodes) *nodes = totalNodes;
    if (steps) *steps = stepsTaken;
    if (launchCount) *launchCount = launches;
    if (t) *t = threads;
    if (g) *g = graphSteps;
}

} // namespace lbm

struct LbmBatch {
    lbm::BatchEngine* impl;
};

namespace {

template <typename F>
LbmStatus batchGuard(F&& f) {
    try {
        lbm::setLastError("");
        f();
        return LBM_OK;
    }
    catch (const lbm::Error& e) {
        lbm::setLastError(e.what());
        return e.status;
    }
    catch (const std::bad_alloc&) {
        lbm::setLastError("out of host memory");
        return LBM_ERR_OUT_OF_MEMORY;
    }
    catch (const std::exception& e) {
        lbm::setLastError(e.what());
        return LBM_ERR_INVALID_ARGUMENT;
    }
}

LbmStatus nullBatch() {
    lbm::setLastError("lbm_batch: null batch");
    return LBM_ERR_INVALID_ARGUMENT;
}

} // namespace

extern "C" {

LbmStatus lbm_batch_create(int num_replicas, const LbmLatticeParameters* lattices, const int* num_particles,
                           const double* masses, const double* positions, const LbmBatchPairForce* pair,
                           const LbmOptions* options, LbmBatch** batch) {
    if (!batch || !options) {
        lbm::setLastError("lbm_batch_create: null argument");
        return LBM_ERR_INVALID_ARGUMENT;
    }
    *batch = nullptr;
    return batchGuard([&] {
        LbmBatch* b = new LbmBatch;
        try {
            b->impl = new lbm::BatchEngine(num_replicas, lattices, num_particles, masses, positions, pair, options);
        }
        catch (...) {
            delete b;
            throw;
        }
        *batch = b;
    });
}

void lbm_batch_destroy(LbmBatch* batch) {
    if (batch) {
        delete batch->impl;
        delete batch;
    }
}

LbmStatus lbm_batch_step(LbmBatch* batch, int steps) {
    if (!batch) return nullBatch();
    return batchGuard([&] { batch->impl->step(steps); });
}

LbmStatus lbm_batch_autotune(LbmBatch* batch, int graph_steps, int* threads_per_block, double* dense_ms) {
    if (!batch) return nullBatch();
    return batchGuard([&] {
        int t = batch->impl->autotune(graph_steps, dense_ms);
        if (threads_per_block)
            *threads_per_block = t;
    });
}

LbmStatus lbm_batch_get_particles(LbmBatch* batch, double* positions, double* velocities) {
    if (!batch) return nullBatch();
    return batchGuard([&] { batch->impl->getParticles(positions, velocities); });
}

LbmStatus lbm_batch_set_velocities(LbmBatch* batch, const double* velocities) {
    if (!batch || !velocities) return nullBatch();
    return batchGuard([&] { batch->impl->setVelocities(velocities); });
}

LbmStatus lbm_batch_get_fluid_state(LbmBatch* batch, int replica, double* state) {
    if (!batch || !state) return nullBatch();
    return batchGuard([&] { batch->impl->getFluidState(replica, state); });
}

LbmStatus lbm_batch_temperatures(LbmBatch* batch, double* fluid_kT, double* bead_kT) {
    if (!batch) return nullBatch();
    return batchGuard([&] { batch->impl->temperatures(fluid_kT, bead_kT); });
}

LbmStatus lbm_batch_set_persistent(LbmBatch* batch, int enable) {
    if (!batch)
        return nullBatch();
    return batchGuard([&] { batch->impl->setPersistent(enable != 0); });
}

LbmStatus lbm_batch_set_barrier_polls(LbmBatch* batch, long long polls) {
    if (!batch)
        return nullBatch();
    return batchGuard([&] { batch->impl->setBarrierPolls(polls); });
}

LbmStatus lbm_batch_info(LbmBatch* batch, long long* total_nodes, long long* steps, long long* launches,
                         int* threads_per_block, int* graph_steps) {
    if (!batch) return nullBatch();
    return batchGuard([&] { batch->impl->info(total_nodes, steps, launches, threads_per_block, graph_steps); });
}

} // extern "C"
