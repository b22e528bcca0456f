// Fluid kernels of the B200 LBM force kernel (sm_100a).
//
//  streamCollideKernel   the dense, fused step: pull streaming, moments, momentum removal, regularized
//                        collision with Guo forcing (+ particle reaction, + Philox fluctuations), store;
//                        HBM-bound, 2*19 population transfers per fluid node.  Restates, fused, the
//                        reference's computeMoments, removeFluidMomentum and collideAndStream
//                        (platforms/reference/src/ReferenceLBMKernels.cpp:430-501, 1066-1120).
//  bounceBackKernel      halfway bounce-back and wall momentum exchange over the wall links
//                        (ReferenceLBMKernels.cpp:1156-1205), writing into the slots of solid nodes.
//  boundaryKernel        regularized walls and open faces (ReferenceLBMKernels.cpp:1207-1343), writing
//                        into the slots that the boundary node pulls.
//  finishKernel          deterministic reduction of the per-block partial sums of a step.
//  momentsKernel         mass, momentum and largest speed of the current state (Mach check, start-up).
//  gather/scatter        conversion between the pull layout and the reference's state layout.
#include "fluid.cuh"
#include "collide.cuh"
#include "collide_pair.cuh"
#include "lbm_device.cuh"
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>

namespace lbm {

#define CUDA_CHECK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    throw Error(LBM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

namespace {

constexpr int TX = 32, TY = 8, THREADS = TX*TY;
constexpr int NPART = 8;           // doubles per partial record: mass, momentum[3], wall[3], maxSpeed2

// Block reduction of a partial record (sums, and max for the last entry) into partials[slot], deterministic.
__device__ void blockReduceStore(double v[NPART], double* out) {
    __shared__ double red[THREADS/32][NPART];
    int lane = threadIdx.x%32, warp = threadIdx.x/32, warps = blockDim.x/32;
#pragma unroll
    for (int i = 0; i < NPART; i++)
        for (int offset = 16; offset > 0; offset >>= 1) {
            double o = __shfl_down_sync(0xffffffffu, v[i], offset);
            v[i] = (i == NPART-1 ? fmax(v[i], o) : v[i] + o);
        }
    if (lane == 0)
        for (int i = 0; i < NPART; i++)
            red[warp][i] = v[i];
    __syncthreads();
    if (threadIdx.x < NPART) {
        int i = threadIdx.x;
        double s = red[0][i];
        for (int w = 1; w < warps; w++)
            s = (i == NPART-1 ? fmax(s, red[w][i]) : s + red[w][i]);
        out[i] = s;
    }
}

struct Coords {
    int x, y, z;
};

__device__ __forceinline__ Coords nodeCoords(long long node, int nx, int ny) {
    Coords c;
    c.x = (int) (node%nx);
    long long r = node/nx;
    c.y = (int) (r%ny);
    c.z = (int) (r/ny);
    return c;
}

__device__ __forceinline__ int wrap(int i, int n) {
    return (i < 0 ? i + n : (i >= n ? i - n : i));
}

// Index of node (x + dx, y + dy, z + dz), periodic.
__device__ __forceinline__ long long shifted(const FluidView& v, int x, int y, int z, int dx, int dy, int dz) {
    return wrap(x + dx, v.nx) + (long long) v.nx*(wrap(y + dy, v.ny) + (long long) v.ny*wrap(z + dz, v.nz));
}

__device__ __forceinline__ int cxr(int q) { return cxOf(q); }
__device__ __forceinline__ int cyr(int q) { return cyOf(q); }
__device__ __forceinline__ int czr(int q) { return czOf(q); }

// Runtime-q fluctuation (slow paths): xi_q = w_q sum_k e_k(c_q) a_k.
template <typename R>
__device__ R fluctuationAt(int q, const R a[15]) {
    R sum = 0;
    R x = cxr(q), y = cyr(q), z = czr(q);
    R x2 = x*x, y2 = y*y, z2 = z*z;
    R e[15] = {x2 - R(1.0/3.0), y2 - R(1.0/3.0), z2 - R(1.0/3.0), x*y, x*z, y*z, y*(x2 - R(1.0/3.0)),
               z*(x2 - R(1.0/3.0)), x*(y2 - R(1.0/3.0)), R(0.5)*x*(y2 + R(2)*z2 - R(1)), R(0.5)*y*(x2 + R(2)*z2 - R(1)),
               R(0.5)*z*(x2 + R(2)*y2 - R(1)), x2*y2 - x2/R(3) - y2/R(3) + z2/R(6) + R(1.0/18.0),
               R(2.0/7.0)*x2*y2 + x2*z2 - R(3.0/7.0)*x2 + y2/R(14) - R(2.0/7.0)*z2 + R(1.0/14.0),
               R(0.4)*x2*y2 + R(0.4)*x2*z2 + y2*z2 - R(0.1)*x2 - R(0.4)*y2 - R(0.4)*z2 + R(0.1)};
#pragma unroll
    for (int k = 0; k < 15; k++)
        sum += e[k]*a[k];
    R w = (q == 0 ? R(1.0/3.0) : (q <= 6 ? R(1.0/18.0) : R(1.0/36.0)));
    return w*sum;
}

template <typename R>
__device__ __forceinline__ R weightOf(int q) {
    return (q == 0 ? R(1.0/3.0) : (q <= 6 ? R(1.0/18.0) : R(1.0/36.0)));
}

// ---------------------------------------------------------------------------------------------------
// The dense step.
// ---------------------------------------------------------------------------------------------------

// Resident blocks of 256 threads per SM that the register allocation of the dense kernel must allow: 3 for float
// arithmetic (85 registers, 24 warps per SM) and 2 for double.  Measured on B200 at 256^3 (FP32, plain): 0.479 ms
// per launch with 3 blocks, 0.549 ms with 4 (64 registers: the loads of a node are no longer all in flight).
#ifdef LBM_DENSE_MIN_BLOCKS
template <typename R> constexpr int denseMinBlocks() { return LBM_DENSE_MIN_BLOCKS; }
#else
template <typename R> constexpr int denseMinBlocks() { return sizeof(R) == 4 ? 3 : 2; }
#endif

// The dense step over 32 x 8 node tiles (lane = x, warp = y), persistent blocks striding over the tiles.  Node
// indices are 32-bit (the host limits the lattice to 2^32 nodes); the tile coordinates advance by the grid
// stride without divisions.  Solid nodes are skipped by their bit in the solid mask; nodes with a particle
// reaction add it to the body force.
template <typename T, typename R, bool SOLID, bool REACT, bool FLUCT>
__global__ void __launch_bounds__(THREADS, denseMinBlocks<R>())
streamCollideKernel(const T* __restrict__ A, T* __restrict__ B, FluidView v, int remove, long long step) {
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    const unsigned N = (unsigned) v.n;
    const int nx = v.nx, ny = v.ny, nz = v.nz;
    const CollideConstants<R> k = collideConstants<R>(v.omega, v.g, v.stats->ucm, remove, v.mu, v.seed);
    R sumMass = 0, sumX = 0, sumY = 0, sumZ = 0;
    const unsigned numTiles = (unsigned) v.numTiles, stride = gridDim.x;
    const int tilesX = v.tilesX, tilesY = v.tilesY;
    int tx = (int) (blockIdx.x%tilesX), ty = (int) ((blockIdx.x/tilesX)%tilesY), tz = (int) (blockIdx.x/tilesX/tilesY);
    const int dtx = (int) (stride%tilesX), dty = (int) ((stride/tilesX)%tilesY), dtz = (int) (stride/tilesX/tilesY);
    for (unsigned t = blockIdx.x; t < numTiles; t += stride) {
        const int x = tx*TX + lane, y = ty*TY + warp, z = tz, tileX = tx;
        tx += dtx;
        int carry = tx >= tilesX;
        tx -= carry ? tilesX : 0;
        ty += dty + carry;
        carry = ty >= tilesY;
        ty -= carry ? tilesY : 0;
        tz += dtz + carry;
        if (x >= nx || y >= ny)
            continue;
        const unsigned row = (unsigned) z*ny + y;
        if (SOLID) {
            uint32_t word = __ldg(&v.solidMask[(size_t) row*v.wordsPerRow + tileX]);
            if ((word >> lane) & 1u)
                continue;
        }
        const unsigned node = row*nx + x;
        R ex = 0, ey = 0, ez = 0;
        if (REACT) {
            uint32_t word = __ldg(&v.reactMask[(size_t) row*v.wordsPerRow + tileX]);
            if ((word >> lane) & 1u) {
                const R* rp = reinterpret_cast<const R*>(v.reaction) + 4*(size_t) node;
                ex = rp[0];
                ey = rp[1];
                ez = rp[2];
            }
        }
        collideNode<T, R, FLUCT>(A, B, N, node, x, y, z, nx, ny, nz, k, ex, ey, ez, step, sumMass, sumX, sumY, sumZ);
    }
    double acc[NPART] = {(double) sumMass, (double) sumX, (double) sumY, (double) sumZ, 0, 0, 0, 0};
    blockReduceStore(acc, v.partials + NPART*(long long) blockIdx.x);
}


// The dense step with two x-adjacent nodes per thread (nx even), the arithmetic of both in packed FP32 pairs; each
// thread loads its pulled words from global memory.
template <typename T, bool SOLID, bool REACT, bool FLUCT>
__global__ void __launch_bounds__(THREADS, (sizeof(T) == 2 && !FLUCT) ? LBM_PAIR_MIN_BLOCKS_16BIT : LBM_PAIR_MIN_BLOCKS)
streamCollidePairKernel(const T* __restrict__ A, T* __restrict__ B, FluidView v, int remove, long long step) {
    typedef typename PairIO<T>::Word Word;
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    const unsigned N = (unsigned) v.n;
    const int nx = v.nx, ny = v.ny, nz = v.nz;
    const Word* __restrict__ aw = reinterpret_cast<const Word*>(A);
    Word* __restrict__ bw = reinterpret_cast<Word*>(B);
    const unsigned halfN = N/2;                       // words per direction plane (N is even)
    const PairConstants c = pairConstants(v, remove, step);
    float sums[4] = {0, 0, 0, 0};
    const int tilesX = (nx + PAIR_TX - 1)/PAIR_TX, tilesY = v.tilesY;
    const unsigned numTiles = (unsigned) tilesX*tilesY*nz, stride = gridDim.x;
    for (unsigned t = blockIdx.x; t < numTiles; t += stride) {
        const int tx = (int) (t%tilesX);
        const unsigned rr = t/tilesX;
        const int y = (int) (rr%tilesY)*TY + warp, z = (int) (rr/tilesY);
        const int x0 = tx*PAIR_TX + 2*lane;
        if (x0 >= nx || y >= ny)
            continue;
        const unsigned row = (unsigned) z*ny + y;
        bool solidA = false, solidB = false;
        if (SOLID) {
            uint32_t word = __ldg(&v.solidMask[(size_t) row*v.wordsPerRow + (x0 >> 5)]);
            solidA = (word >> (x0 & 31)) & 1u;
            solidB = (word >> ((x0 + 1) & 31)) & 1u;
            if (solidA && solidB)
                continue;
        }
        const unsigned node = row*nx + x0;
        // Rows of the pull sources: index [1 - cy][1 - cz] (periodic in y and z).
        const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
        const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
        const int xl = x0 == 0 ? nx - 2 : x0 - 2, xr = x0 + 2 == nx ? 0 : x0 + 2;
        F2 r[19];
        staticFor<19>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
            const unsigned base = ((unsigned) zs[1-cz]*ny + ys[1-cy])*nx;
            const Word* plane = aw + (size_t) q*halfN;
            Word w;
            if (cx == 0)
                w = __ldg(plane + (base + x0)/2);
            else if (cx == 1)
                w = PairIO<T>::left(__ldg(plane + (base + xl)/2), __ldg(plane + (base + x0)/2));
            else
                w = PairIO<T>::right(__ldg(plane + (base + x0)/2), __ldg(plane + (base + xr)/2));
            r[q] = PairIO<T>::decode(w);
        });
        bool reactA = false, reactB = false;
        if (REACT) {
            uint32_t word = __ldg(&v.reactMask[(size_t) row*v.wordsPerRow + (x0 >> 5)]);
            reactA = (word >> (x0 & 31)) & 1u;
            reactB = (word >> ((x0 + 1) & 31)) & 1u;
        }
        PairStore<T, SOLID> out{bw + node/2, halfN, solidA, solidB};
        collidePair<T, SOLID, REACT, FLUCT>(r, v, c, remove, step, node, solidA, solidB, reactA, reactB, out, sums);
    }
    double acc[NPART] = {(double) sums[0], (double) sums[1], (double) sums[2], (double) sums[3], 0, 0, 0, 0};
    blockReduceStore(acc, v.partials + NPART*(long long) blockIdx.x);
}

// The dense step for 16-bit storage without fluctuations, four x-adjacent nodes per thread (nx a multiple of 4):
// each direction's four sources are one aligned 64-bit word of the source row, with c_x = +1 the high half of the
// 32-bit word to the left in front of its first three, with c_x = -1 the low half of the word to the right after its
// last three; the four post-collision values of a direction go out as one 64-bit word.  The nodes are collided as two
// pairs (collidePulled, the same arithmetic and dither bits as the paired kernel, so the results are the paired
// kernel's bit for bit); the first pair's packed words wait in registers for the second's.  A warp takes a row tile
// of QUAD_TX nodes.  Against the paired kernel this halves the loads, stores and address arithmetic per node (29 loads
// and 19 stores per 4 nodes) and doubles the bytes in flight per warp: FP16 channel step 0.578 -> 0.511 ms, BF16
// 0.571 -> 0.503 ms.  Measured slower: 4 or 6 blocks per SM (0.527 / 0.548 ms FP16), the first pair's words held in
// shared memory (0.592 ms at 6 blocks), and each pair storing its own 32-bit words (0.599 ms).
constexpr int QUAD_TX = 128;        // nodes per warp row tile: 4 per lane
#ifndef LBM_QUAD_THREADS
#define LBM_QUAD_THREADS 128
#endif
#ifndef LBM_QUAD_MIN_BLOCKS
#define LBM_QUAD_MIN_BLOCKS 5
#endif

// The first pair of a quad: its packed words, held until the second pair's are ready.
template <typename T>
struct QuadHold {
    uint32_t word[19];
    template <int q> __device__ __forceinline__ void put(F2 value, uint32_t dither) {
        word[q] = PairIO<T>::pack(value.v.x, value.v.y, dither);
    }
};

// The second pair: stores both pairs' words of direction q as one 64-bit word (word halves per node when a node of
// the quad is solid).
template <typename T, bool SOLID>
struct QuadStore {
    uint2* out;                   // the quad's word in plane 0
    unsigned quarterN;            // 64-bit words per plane
    const QuadHold<T>& first;
    uint32_t solidBits;           // bit i: node x0 + i is solid
    template <int q> __device__ __forceinline__ void put(F2 value, uint32_t dither) {
        const uint32_t second = PairIO<T>::pack(value.v.x, value.v.y, dither);
        uint2* p = out + (size_t) q*quarterN;
        if (SOLID && solidBits != 0) {
            uint32_t* w = reinterpret_cast<uint32_t*>(p);
            storeWord16<SOLID>(w, first.word[q], solidBits & 1u, solidBits & 2u);
            storeWord16<SOLID>(w + 1, second, solidBits & 4u, solidBits & 8u);
            return;
        }
        *p = make_uint2(first.word[q], second);
    }
};

template <typename T, bool SOLID, bool REACT>
__global__ void __launch_bounds__(LBM_QUAD_THREADS, LBM_QUAD_MIN_BLOCKS)
streamCollideQuadKernel(const T* __restrict__ A, T* __restrict__ B, FluidView v, int remove, long long step) {
    static_assert(sizeof(T) == 2, "the quad kernel is for 16-bit storage");
    const int lane = threadIdx.x%32;
    const unsigned N = (unsigned) v.n;
    const int nx = v.nx, ny = v.ny, nz = v.nz;
    const uint32_t* __restrict__ a32 = reinterpret_cast<const uint32_t*>(A);
    const uint2* __restrict__ a64 = reinterpret_cast<const uint2*>(A);
    uint2* __restrict__ b64 = reinterpret_cast<uint2*>(B);
    const unsigned halfN = N/2, quarterN = N/4;     // 32-bit and 64-bit words per direction plane (N % 4 == 0)
    const PairConstants c = pairConstants(v, remove, step);
    float sums[4] = {0, 0, 0, 0};
    const int tilesX = (nx + QUAD_TX - 1)/QUAD_TX;
    const unsigned numTiles = (unsigned) tilesX*ny*nz, warps = blockDim.x/32;
    for (unsigned t = blockIdx.x*warps + threadIdx.x/32; t < numTiles; t += gridDim.x*warps) {
        const int tx = (int) (t%tilesX);
        const unsigned row = t/tilesX;
        const int y = (int) (row%(unsigned) ny), z = (int) (row/(unsigned) ny);
        const int x0 = tx*QUAD_TX + 4*lane;
        if (x0 >= nx)
            continue;
        uint32_t solidBits = 0;
        if (SOLID) {
            // x0 % 4 == 0: the quad's four bits sit in one mask word.
            solidBits = (__ldg(&v.solidMask[(size_t) row*v.wordsPerRow + (x0 >> 5)]) >> (x0 & 31)) & 0xFu;
            if (solidBits == 0xFu)
                continue;
        }
        const unsigned node = row*nx + x0;
        const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
        const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
        const int xl = x0 == 0 ? nx - 2 : x0 - 2, xr = x0 + 4 == nx ? 0 : x0 + 4;
        uint32_t wa[19], wb[19];
        staticFor<19>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
            const unsigned base = ((unsigned) zs[1-cz]*ny + ys[1-cy])*nx;
            const uint2 w = __ldg(a64 + (size_t) q*quarterN + (base + x0)/4);
            if (cx == 0) {
                wa[q] = w.x;
                wb[q] = w.y;
            }
            else if (cx == 1) {
                wa[q] = __byte_perm(__ldg(a32 + (size_t) q*halfN + (base + xl)/2), w.x, 0x5432);
                wb[q] = __byte_perm(w.x, w.y, 0x5432);
            }
            else {
                wa[q] = __byte_perm(w.x, w.y, 0x5432);
                wb[q] = __byte_perm(w.y, __ldg(a32 + (size_t) q*halfN + (base + xr)/2), 0x5432);
            }
        });
        uint32_t reactBits = 0;
        if (REACT)
            reactBits = (__ldg(&v.reactMask[(size_t) row*v.wordsPerRow + (x0 >> 5)]) >> (x0 & 31)) & 0xFu;
        QuadHold<T> first;
        collidePulled<T, SOLID, REACT, false>(PulledWords<T>{wa}, v, c, remove, step, node, solidBits & 1u,
                                              solidBits & 2u, reactBits & 1u, reactBits & 2u, first, sums);
        QuadStore<T, SOLID> out{b64 + node/4, quarterN, first, solidBits};
        collidePulled<T, SOLID, REACT, false>(PulledWords<T>{wb}, v, c, remove, step, node + 2, solidBits & 4u,
                                              solidBits & 8u, reactBits & 4u, reactBits & 8u, out, sums);
    }
    double acc[NPART] = {(double) sums[0], (double) sums[1], (double) sums[2], (double) sums[3], 0, 0, 0, 0};
    blockReduceStore(acc, v.partials + NPART*(long long) blockIdx.x);
}

// ---------------------------------------------------------------------------------------------------
// Bounce-back over the wall links (after the dense step, on the output array).
// ---------------------------------------------------------------------------------------------------

// One wall node per thread (a grid of up to kGridWall blocks covers the channel's wall planes in one pass): the
// node's wall links are known at compile time per direction, so the loads of all its links are issued before any of
// the stores (a store may alias a later load as far as the compiler knows) and do not wait on one another.
template <typename T, typename R>
__global__ void __launch_bounds__(THREADS)
bounceBackKernel(T* __restrict__ B, const int* __restrict__ wall, int numWall, FluidView v, double* partials) {
    double acc[NPART] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = blockIdx.x*blockDim.x + threadIdx.x; b < numWall; b += gridDim.x*blockDim.x) {
        const int2 entry = __ldg(reinterpret_cast<const int2*>(wall) + b);
        const long long node = (unsigned) entry.x;
        const int links = entry.y;
        const Coords c = nodeCoords(node, v.nx, v.ny);
        T raw[19];
        staticFor<18>([&](auto qc) {
            constexpr int q = decltype(qc)::value + 1;
            if (links & (1 << q))
                raw[q] = B[(long long) q*v.n + node];
        });
        staticFor<18>([&](auto qc) {
            constexpr int q = decltype(qc)::value + 1;
            if (links & (1 << q)) {
                // The population x built for q streamed into the solid node s = x + c_q; x takes it back along
                // -c_q, so it goes into the slot of s that x pulls for opp(q).  Opposite directions have the same
                // weight, so the stored element is copied as it is.
                const long long s = shifted(v, c.x, c.y, c.z, cxOf(q), cyOf(q), czOf(q));
                B[(long long) oppOf(q)*v.n + s] = raw[q];
                const double value = (double) loadq<T, R>(&raw[q], q);
                const double w = weightOf<double>(q);
                // The fluid momentum of the population is reversed; the wall receives 2 c_q (f + w)
                // (ReferenceLBMKernels.cpp:1176-1205, momentum exchange of Ladd 1994).
                acc[1] -= 2.0*cxOf(q)*value;
                acc[2] -= 2.0*cyOf(q)*value;
                acc[3] -= 2.0*czOf(q)*value;
                acc[4] += 2.0*cxOf(q)*(value + w);
                acc[5] += 2.0*cyOf(q)*(value + w);
                acc[6] += 2.0*czOf(q)*(value + w);
            }
        });
    }
    blockReduceStore(acc, partials + NPART*(long long) blockIdx.x);
}

// ---------------------------------------------------------------------------------------------------
// Regularized walls and open faces (applyBoundaries, ReferenceLBMKernels.cpp:1207-1343), on the boundary
// node list, after the dense step: A is the input of the step (its moments are recomputed from it) and B
// its output.
// ---------------------------------------------------------------------------------------------------

template <typename R>
__device__ void eqDeviation(R drho, R ux, R uy, R uz, int q, R& out) {
    R rho = R(1) + drho;
    R uu = ux*ux + uy*uy + uz*uz;
    R cu = cxr(q)*ux + cyr(q)*uy + czr(q)*uz;
    out = weightOf<R>(q)*(drho + rho*(R(3)*cu + R(4.5)*cu*cu - R(1.5)*uu));
}

template <typename R>
__device__ R guoAt(int q, R ux, R uy, R uz, R fx, R fy, R fz) {
    R uf = ux*fx + uy*fy + uz*fz;
    R cu = cxr(q)*ux + cyr(q)*uy + czr(q)*uz;
    R cf = cxr(q)*fx + cyr(q)*fy + czr(q)*fz;
    return weightOf<R>(q)*(R(3)*(cf - uf) + R(9)*cu*cf);
}

template <typename R>
__device__ R fneqAt(int q, const Moments<R>& m) {
    R cx = cxr(q), cy = cyr(q), cz = czr(q);
    R h0 = cx*cx - R(1.0/3.0), h1 = cy*cy - R(1.0/3.0), h2 = cz*cz - R(1.0/3.0);
    return R(4.5)*weightOf<R>(q)*(h0*m.pxx + h1*m.pyy + h2*m.pzz + R(2)*(cx*cy*m.pxy + cx*cz*m.pxz + cy*cz*m.pyz));
}

template <typename T, typename R, bool FLUCT>
__global__ void __launch_bounds__(128)
boundaryKernel(const T* __restrict__ A, T* __restrict__ B, const int* __restrict__ bnd, int numBoundary, FluidView v,
               int remove, long long step, double* partials, const double* faceData) {
    // faceData: per face (6): velocity[3], density, then boundary stress weight c, and the flags.
    double acc[NPART] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long long N = v.n;
    const R omega = R(v.omega);
    const R gx = R(v.g[0]), gy = R(v.g[1]), gz = R(v.g[2]);
    for (int b = blockIdx.x*blockDim.x + threadIdx.x; b < numBoundary; b += gridDim.x*blockDim.x) {
        long long node = bnd[4*b];
        int unknown = bnd[4*b+1], solid = bnd[4*b+2];
        int kind = bnd[4*b+3] & 255, face = (bnd[4*b+3] >> 8) - 1;
        Coords c = nodeCoords(node, v.nx, v.ny);
        // Moments of x at this step, from the input array, as in the dense kernel.
        R f[19];
        for (int q = 0; q < 19; q++)
            f[q] = loadq<T, R>(A + (long long) q*N + shifted(v, c.x, c.y, c.z, -cxr(q), -cyr(q), -czr(q)), q);
        Moments<R> m = momentsOf<R>(f);
        R rhoNode = R(1) + m.dr;
        R jx = m.jx, jy = m.jy, jz = m.jz;
        if (remove) {
            jx -= rhoNode*R(v.stats->ucm[0]);
            jy -= rhoNode*R(v.stats->ucm[1]);
            jz -= rhoNode*R(v.stats->ucm[2]);
        }
        // The post-stream value of x for direction p: B_p(x - c_p).
        auto arrived = [&](int p) -> R {
            return loadq<T, R>(B + (long long) p*N + shifted(v, c.x, c.y, c.z, -cxr(p), -cyr(p), -czr(p)), p);
        };
        R rb = rhoNode, dr = m.dr;
        R ub[3] = {(jx + R(0.5)*(rb*gx))/rb, (jy + R(0.5)*(rb*gy))/rb, (jz + R(0.5)*(rb*gz))/rb};
        if (kind == KindWall || kind == KindDensityAtRest)
            ub[0] = ub[1] = ub[2] = 0;
        if (kind == KindVelocity || kind == KindDensityVelocity)
            for (int a = 0; a < 3; a++)
                ub[a] = R(faceData[4*face + a]);
        if (kind == KindDensity || kind == KindDensityAtRest || kind == KindDensityVelocity) {
            dr = R(faceData[4*face + 3]) - R(1);
            rb = R(faceData[4*face + 3]);
        }
        if (kind == KindDensity) {
            int axis = face/2;
            R inward = (face%2 == 0 ? R(1) : R(-1)), sum = 0;
            for (int q = 0; q < 19; q++)
                sum += arrived((unknown & (1<<q)) ? oppOf(q) : q);
            ub[axis] = R(0.5)*(inward*(dr - sum)/rb + ub[axis]);
        }
        R xi[19];
        bool fluct = FLUCT;
        if (FLUCT) {
            R mu = R(v.mu);
            R cw = R(faceData[24]);
            if (hasEquilibriumNoise(kind)) {
                // Random part of a node at equilibrium (D3Q19::equilibriumFluctuation) minus c times the
                // stress part of the random part of the collision of x (ReferenceLBMKernels.cpp:1278-1284).
                R r[19], a[15], rc[15], ac[15];
                philoxNormals<R, 19>(v.seed, PurposeBoundary, node, step, r);
                R oneMinusC = R(1) - cw;
                modeAmplitudes<R>(r, sqrt(mu*rb*(oneMinusC > R(0) ? oneMinusC : R(0))), sqrt(mu*rb), a);
                philoxNormals<R, 15>(v.seed, PurposeFluid, node, step, rc);
                modeAmplitudes<R>(rc, sqrt(mu*rhoNode*omega*(R(2) - omega)), R(0), ac);
                R conserved = sqrt(mu*rb);
                for (int q = 0; q < 19; q++) {
                    xi[q] = fluctuationAt<R>(q, a)
                          + weightOf<R>(q)*conserved*(r[15] + R(1.7320508075688772)*(cxr(q)*r[16] + cyr(q)*r[17] + czr(q)*r[18]))
                          - cw*fluctuationAt<R>(q, ac);
                }
            }
            else {
                R r[15], a[15];
                philoxNormals<R, 15>(v.seed, PurposeBoundary, node, step, r);
                modeAmplitudes<R>(r, sqrt(mu*rb*omega*(R(2) - omega)), sqrt(mu*rb), a);
                for (int q = 0; q < 19; q++)
                    xi[q] = fluctuationAt<R>(q, a);
            }
        }
        R Fb[3] = {gx*rb, gy*rb, gz*rb};
        if (kind == KindWall || kind == KindVelocity) {
            // Mass balance (ReferenceLBMKernels.cpp:1290-1325), linear in rho_b = 1 + dr.
            R numerator = 0, denominator = 0;
            for (int q = 1; q < 19; q++) {
                if (!(unknown & (1<<q)))
                    continue;
                R arriving, flux = 0;
                if (solid & (1<<q))
                    arriving = loadq<T, R>(B + (long long) oppOf(q)*N + node, oppOf(q));
                else if (!(unknown & (1<<oppOf(q)))) {
                    arriving = arrived(oppOf(q));
                    flux = R(6)*weightOf<R>(q)*(cxr(q)*ub[0] + cyr(q)*ub[1] + czr(q)*ub[2]);
                }
                else
                    continue;
                R e0;
                eqDeviation<R>(R(0), ub[0], ub[1], ub[2], q, e0);
                R sg = guoAt<R>(q, ub[0], ub[1], ub[2], gx, gy, gz);
                R rest = (R(1) - omega)*fneqAt<R>(q, m) + (fluct ? xi[q] : R(0));
                numerator += arriving - rest - e0 - R(0.5)*sg + flux;
                denominator += weightOf<R>(q) + e0 + R(0.5)*sg - flux;
            }
            if (denominator != R(0)) {
                dr = numerator/denominator;
                rb = R(1) + dr;
                Fb[0] = gx*rb; Fb[1] = gy*rb; Fb[2] = gz*rb;
            }
        }
        for (int q = 1; q < 19; q++) {
            if (!(unknown & (1<<q)))
                continue;
            R dfeq;
            eqDeviation<R>(dr, ub[0], ub[1], ub[2], q, dfeq);
            R value = dfeq + (R(1) - omega)*fneqAt<R>(q, m) + R(0.5)*guoAt<R>(q, ub[0], ub[1], ub[2], Fb[0], Fb[1], Fb[2]);
            if (fluct)
                value += xi[q];
            long long src = shifted(v, c.x, c.y, c.z, -cxr(q), -cyr(q), -czr(q));
            T* slot = B + (long long) q*N + src;
            // Mass and momentum bookkeeping of the step sums: the value that would have arrived leaves, the rebuilt
            // one enters.  For a solid source the population that x sent into the wall leaves instead.
            double old = 0;
            if (solid & (1<<q)) {
                R sent = loadq<T, R>(B + (long long) oppOf(q)*N + node, oppOf(q));
                old = (double) sent;
                acc[1] += (double) sent*cxr(q);     // sent moves along -c_q
                acc[2] += (double) sent*cyr(q);
                acc[3] += (double) sent*czr(q);
                // The wall receives the momentum of the population sent along -c_q and gives that of the rebuilt
                // one along c_q (full populations, ReferenceLBMKernels.cpp:1332-1338).
                double w = weightOf<double>(q);
                acc[4] -= cxr(q)*((double) sent + (double) value + 2.0*w);
                acc[5] -= cyr(q)*((double) sent + (double) value + 2.0*w);
                acc[6] -= czr(q)*((double) sent + (double) value + 2.0*w);
                acc[0] -= old;
            }
            else if (v.solidMask != nullptr && ((v.solidMask[(src/v.nx)*v.wordsPerRow + (src%v.nx)/32] >> ((src%v.nx)%32)) & 1u)) {
                // The node across the face is solid: the dense step wrote nothing there.
            }
            else {
                old = (double) loadq<T, R>(slot, q);
                acc[0] -= old;
                acc[1] -= old*cxr(q);
                acc[2] -= old*cyr(q);
                acc[3] -= old*czr(q);
            }
            storeq<T, R>(slot, q, value);
            double stored = (double) loadq<T, R>(slot, q);
            acc[0] += stored;
            acc[1] += stored*cxr(q);
            acc[2] += stored*cyr(q);
            acc[3] += stored*czr(q);
        }
    }
    // Block of 128 threads: pad the reduction to the generic routine.
    blockReduceStore(acc, partials + NPART*(long long) blockIdx.x);
}

// ---------------------------------------------------------------------------------------------------
// Deterministic finish of the step sums: one block adds the partial records in a fixed order.
// ---------------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(THREADS) finishKernel(const double* partials, int count, FluidView v, int mode) {
    // mode 0: the sums of a step (mass, momentum, ucm, wall); 1: a moments pass that sets the sums and the largest
    // speed; 2: a moments pass for the largest speed only (the sums of the step are kept).
    double acc[NPART] = {0, 0, 0, 0, 0, 0, 0, 0};
    // Several records in flight per thread (the loads do not wait on the sums).
#pragma unroll 4
    for (int i = threadIdx.x; i < count; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NPART; k++)
            acc[k] = (k == NPART-1 ? fmax(acc[k], partials[NPART*(long long) i + k]) : acc[k] + partials[NPART*(long long) i + k]);
    __shared__ double total[NPART];
    blockReduceStore(acc, total);
    __syncthreads();
    if (threadIdx.x == 0) {
        StepStats* s = v.stats;
        if (mode != 2) {
            s->mass = total[0];
            double mass = v.numFluid + total[0];
            for (int a = 0; a < 3; a++) {
                s->momentum[a] = total[1+a];
                s->ucm[a] = total[1+a]/mass;
            }
        }
        if (mode == 0)
            for (int a = 0; a < 3; a++)
                s->wall[a] = total[4+a];
        if (mode != 0)
            s->maxSpeed2 = total[7];
    }
}

// ---------------------------------------------------------------------------------------------------
// Moments of the current state (post-stream values pulled from the input array).
// ---------------------------------------------------------------------------------------------------

template <typename T, typename R>
__global__ void __launch_bounds__(THREADS) momentsKernel(const T* __restrict__ A, FluidView v) {
    double acc[NPART] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    for (long long t = blockIdx.x; t < v.numTiles; t += gridDim.x) {
        int tx = (int) (t%v.tilesX);
        long long rr = t/v.tilesX;
        int ty = (int) (rr%v.tilesY);
        int z = (int) (rr/v.tilesY);
        int x = tx*TX + lane, y = ty*TY + warp;
        if (x >= v.nx || y >= v.ny)
            continue;
        long long row = (long long) z*v.ny + y;
        if (v.solidMask != nullptr && ((__ldg(&v.solidMask[row*v.wordsPerRow + tx]) >> lane) & 1u))
            continue;
        R dr = 0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 19; q++) {
            R fq = loadq<T, R>(A + (long long) q*v.n + shifted(v, x, y, z, -cxr(q), -cyr(q), -czr(q)), q);
            dr += fq;
            jx += cxr(q)*fq;
            jy += cyr(q)*fq;
            jz += czr(q)*fq;
        }
        double r = 1.0 + (double) dr;
        acc[0] += (double) dr;
        acc[1] += (double) jx;
        acc[2] += (double) jy;
        acc[3] += (double) jz;
        double s2 = ((double) jx*jx + (double) jy*jy + (double) jz*jz)/(r*r);
        acc[7] = fmax(acc[7], s2);
    }
    blockReduceStore(acc, v.partials + NPART*(long long) blockIdx.x);
}

// The steady-state residual of the build (the reference defines none): r = max over fluid nodes of |u - u_prev|,
// and max |u|, with u = j/rho of the post-stream state in FP64; u_prev (3N doubles, [a*N + node]) is replaced by u.
// Per block: partials[NPART*b] = max |u - u_prev|^2, partials[NPART*b + 7] = max |u|^2.
template <typename T, typename R>
__global__ void __launch_bounds__(THREADS) residualKernel(const T* __restrict__ A, FluidView v, double* prev, int first) {
    double maxDiff2 = 0, maxU2 = 0;
    const int lane = threadIdx.x%32, warp = threadIdx.x/32;
    for (long long t = blockIdx.x; t < v.numTiles; t += gridDim.x) {
        int tx = (int) (t%v.tilesX);
        long long rr = t/v.tilesX;
        int ty = (int) (rr%v.tilesY);
        int z = (int) (rr/v.tilesY);
        int x = tx*TX + lane, y = ty*TY + warp;
        if (x >= v.nx || y >= v.ny)
            continue;
        long long row = (long long) z*v.ny + y;
        if (v.solidMask != nullptr && ((__ldg(&v.solidMask[row*v.wordsPerRow + tx]) >> lane) & 1u))
            continue;
        double dr = 0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 19; q++) {
            double fq = (double) loadq<T, R>(A + (long long) q*v.n + shifted(v, x, y, z, -cxr(q), -cyr(q), -czr(q)), q);
            dr += fq;
            jx += cxr(q)*fq;
            jy += cyr(q)*fq;
            jz += czr(q)*fq;
        }
        double inv = 1.0/(1.0 + dr);
        double u[3] = {jx*inv, jy*inv, jz*inv};
        long long node = row*v.nx + x;
        double d2 = 0;
        for (int a = 0; a < 3; a++) {
            double* p = prev + a*v.n + node;
            double d = u[a] - *p;
            d2 += d*d;
            *p = u[a];
        }
        if (!first)
            maxDiff2 = fmax(maxDiff2, d2);
        maxU2 = fmax(maxU2, u[0]*u[0] + u[1]*u[1] + u[2]*u[2]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        maxDiff2 = fmax(maxDiff2, __shfl_down_sync(0xffffffffu, maxDiff2, o));
        maxU2 = fmax(maxU2, __shfl_down_sync(0xffffffffu, maxU2, o));
    }
    __shared__ double red[THREADS/32][2];
    if (lane == 0) {
        red[warp][0] = maxDiff2;
        red[warp][1] = maxU2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < THREADS/32; w++) {
            maxDiff2 = fmax(maxDiff2, red[w][0]);
            maxU2 = fmax(maxU2, red[w][1]);
        }
        v.partials[NPART*(long long) blockIdx.x] = maxDiff2;
        v.partials[NPART*(long long) blockIdx.x + 7] = maxU2;
    }
}

// ---------------------------------------------------------------------------------------------------
// Initial state and state transfer.
// ---------------------------------------------------------------------------------------------------

// Equilibrium at the initial velocity on fluid nodes and -w_q on solid nodes, in the pull layout:
// A_q(y) = f_q(y + c_q) (ReferenceLBMKernels.cpp:53-79).
template <typename T, typename R>
__global__ void initKernel(T* A, T* B, FluidView v, const char* fluid, double ux, double uy, double uz) {
    long long total = 19*v.n;
    for (long long i = blockIdx.x*(long long) blockDim.x + threadIdx.x; i < total; i += (long long) gridDim.x*blockDim.x) {
        int q = (int) (i/v.n);
        long long y = i%v.n;
        Coords c = nodeCoords(y, v.nx, v.ny);
        long long target = shifted(v, c.x, c.y, c.z, cxr(q), cyr(q), czr(q));
        double value;
        if (fluid != nullptr && !fluid[target])
            value = -weightOf<double>(q);
        else {
            double uu = ux*ux + uy*uy + uz*uz;
            double cu = cxr(q)*ux + cyr(q)*uy + czr(q)*uz;
            value = weightOf<double>(q)*(0.0 + 1.0*(3.0*cu + 4.5*cu*cu - 1.5*uu));
        }
        storeq<T, R>(A + i, q, (R) value);
        storeq<T, R>(B + i, q, (R) value);
    }
}

// Plane q of the state: out[x] = f_q(x) = A_q(x - c_q).
template <typename T, typename R>
__global__ void gatherKernel(const T* A, int q, FluidView v, double* out) {
    for (long long x = blockIdx.x*(long long) blockDim.x + threadIdx.x; x < v.n; x += (long long) gridDim.x*blockDim.x) {
        Coords c = nodeCoords(x, v.nx, v.ny);
        out[x] = (double) loadq<T, R>(A + (long long) q*v.n + shifted(v, c.x, c.y, c.z, -cxr(q), -cyr(q), -czr(q)), q);
    }
}

template <typename T>
__device__ __forceinline__ bool bitsEqual(const T& a, const T& b) {
    const unsigned char* pa = reinterpret_cast<const unsigned char*>(&a);
    const unsigned char* pb = reinterpret_cast<const unsigned char*>(&b);
    for (int i = 0; i < (int) sizeof(T); i++)
        if (pa[i] != pb[i])
            return false;
    return true;
}

// Plane q of a state into both arrays: A_q(y) = f_q(y + c_q).  *changed is set when a stored element of A
// changes, so that setting the state a kernel already holds keeps the sums of its last step (bitwise restarts).
template <typename T, typename R>
__global__ void scatterKernel(T* A, T* B, int q, FluidView v, const double* in, int* changed) {
    for (long long y = blockIdx.x*(long long) blockDim.x + threadIdx.x; y < v.n; y += (long long) gridDim.x*blockDim.x) {
        Coords c = nodeCoords(y, v.nx, v.ny);
        R value = (R) in[shifted(v, c.x, c.y, c.z, cxr(q), cyr(q), czr(q))];
        T before = A[(long long) q*v.n + y];
        storeq<T, R>(A + (long long) q*v.n + y, q, value);
        T after = A[(long long) q*v.n + y];
        if (!bitsEqual(before, after))
            *changed = 1;
        storeq<T, R>(B + (long long) q*v.n + y, q, value);
    }
}

// Velocity component a of node (x, y, z) in lattice units, 0 at solid nodes; out-of-lattice neighbours (open faces)
// take the value of the node itself.
__device__ __forceinline__ double velocityAt(const FluidView& v, const double* velocity, double scale, int x, int y,
                                            int z, int a, long long self) {
    long long node;
    if (x < 0 || x >= v.nx || y < 0 || y >= v.ny || z < 0 || z >= v.nz) {
        if (v.faceOpen)
            node = self;
        else
            node = wrap(x, v.nx) + (long long) v.nx*(wrap(y, v.ny) + (long long) v.ny*wrap(z, v.nz));
    }
    else
        node = x + (long long) v.nx*(y + (long long) v.ny*z);
    long long row = node/v.nx;
    int xx = (int) (node - row*v.nx);
    if (v.solidMask != nullptr && ((v.solidMask[row*v.wordsPerRow + xx/32] >> (xx%32)) & 1u))
        return 0.0;
    return velocity[3*node + a]/scale;
}

// Populations of given fields (density [N], velocity [N][3] in the units of the fields, divided by the scales into
// lattice units), written in the pull layout of both arrays: slot (q, y) holds the population that node x = y + c_q
// pulls, the equilibrium w_q (rho - 1 + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2)) of x plus, with `strain`, the
// Chapman-Enskog non-equilibrium part -3 tau w_q rho (c.S.c - tr S/3) of the strain rate S (central differences of
// the velocity, zero velocity at solid nodes), so that a steady flow starts without the transient of a stress-free
// state; solid nodes hold 0.
template <typename T, typename R>
__global__ void equilibriumKernel(T* A, T* B, FluidView v, const double* density, const double* velocity,
                                  double densityScale, double velocityScale, int strain) {
    for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x; t < 19*v.n; t += (long long) gridDim.x*blockDim.x) {
        int q = (int) (t/v.n);
        long long y = t - q*v.n;
        Coords c = nodeCoords(y, v.nx, v.ny);
        long long x = shifted(v, c.x, c.y, c.z, cxr(q), cyr(q), czr(q));
        Coords cx = nodeCoords(x, v.nx, v.ny);
        long long row = (long long) cx.z*v.ny + cx.y;
        double value = 0;
        if (v.solidMask == nullptr || !((v.solidMask[row*v.wordsPerRow + cx.x/32] >> (cx.x%32)) & 1u)) {
            double rho = density[x]/densityScale;
            double u[3] = {velocity[3*x]/velocityScale, velocity[3*x+1]/velocityScale, velocity[3*x+2]/velocityScale};
            double cu = cxr(q)*u[0] + cyr(q)*u[1] + czr(q)*u[2];
            double uu = u[0]*u[0] + u[1]*u[1] + u[2]*u[2];
            value = weightOf<double>(q)*(rho - 1.0 + rho*(3.0*cu + 4.5*cu*cu - 1.5*uu));
            if (strain) {
                // grad[a][b] = d u_b / d x_a
                double grad[3][3];
                int cxyz[3] = {cx.x, cx.y, cx.z};
                for (int a = 0; a < 3; a++) {
                    int p[3] = {cxyz[0], cxyz[1], cxyz[2]}, m[3] = {cxyz[0], cxyz[1], cxyz[2]};
                    p[a]++;
                    m[a]--;
                    for (int b = 0; b < 3; b++)
                        grad[a][b] = 0.5*(velocityAt(v, velocity, velocityScale, p[0], p[1], p[2], b, x)
                                          - velocityAt(v, velocity, velocityScale, m[0], m[1], m[2], b, x));
                }
                double c[3] = {(double) cxr(q), (double) cyr(q), (double) czr(q)};
                double cSc = 0, tr = grad[0][0] + grad[1][1] + grad[2][2];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        cSc += c[a]*c[b]*0.5*(grad[a][b] + grad[b][a]);
                value += -3.0*(1.0/v.omega)*weightOf<double>(q)*rho*(cSc - tr/3.0);
            }
        }
        storeq<T, R>(A + t, q, (R) value);
        storeq<T, R>(B + t, q, (R) value);
    }
}

// Density and velocity u = j/rho + g/2 of every node, zero at solid nodes (nodeFields,
// ReferenceLBMKernels.cpp:1349-1368).
template <typename T, typename R>
__global__ void fieldsKernel(const T* A, FluidView v, double* out, double densityScale, double velocityScale) {
    for (long long x = blockIdx.x*(long long) blockDim.x + threadIdx.x; x < v.n; x += (long long) gridDim.x*blockDim.x) {
        Coords c = nodeCoords(x, v.nx, v.ny);
        long long row = (long long) c.z*v.ny + c.y;
        if (v.solidMask != nullptr && ((v.solidMask[row*v.wordsPerRow + c.x/32] >> (c.x%32)) & 1u)) {
            for (int k = 0; k < 4; k++)
                out[4*x + k] = 0;
            continue;
        }
        double r = 1.0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 19; q++) {
            double fq = (double) loadq<T, R>(A + (long long) q*v.n + shifted(v, c.x, c.y, c.z, -cxr(q), -cyr(q), -czr(q)), q);
            r += fq;
            jx += cxr(q)*fq;
            jy += cyr(q)*fq;
            jz += czr(q)*fq;
        }
        out[4*x] = r*densityScale;
        out[4*x+1] = (jx*(1.0/r) + v.g[0]*0.5)*velocityScale;
        out[4*x+2] = (jy*(1.0/r) + v.g[1]*0.5)*velocityScale;
        out[4*x+3] = (jz*(1.0/r) + v.g[2]*0.5)*velocityScale;
    }
}

// ---------------------------------------------------------------------------------------------------
// Launch tables per storage type.
// ---------------------------------------------------------------------------------------------------

template <typename T> struct ComputeOf { typedef float type; };
template <> struct ComputeOf<double> { typedef double type; };

template <typename T>
struct Launcher {
    typedef typename ComputeOf<T>::type R;

    // The paired kernel serves FP32 and 16-bit storage on lattices with an even nx (measured at 256^3, FP32: 0.596
    // against 0.677 ms per launch with fluctuations, 0.464 against 0.482 ms without).  LBM_B200_PAIRED16 = 0 and
    // LBM_B200_PAIRED32 = 0 in the environment select the one-node kernel instead (for comparisons).
    static int pairChoice(const char* name) {
        const char* e = std::getenv(name);
        return e == nullptr ? -1 : (e[0] == '0' ? 0 : 1);
    }
    template <bool FL>
    static bool pairedKernels() {
        static int enabled = -2;
        if (enabled == -2) {
            if (sizeof(T) == 2) {
                int c = pairChoice("LBM_B200_PAIRED16");
                enabled = c == 0 ? 0 : 1;
            }
            else {
                int c = pairChoice("LBM_B200_PAIRED32");
                enabled = c == 0 ? 0 : 1;
            }
        }
        return enabled == 1;
    }

    // The quad kernel for 16-bit storage without fluctuations (nx % 4 == 0); LBM_B200_QUAD16 = 0 in the environment
    // selects the paired kernel instead (for comparisons).
    static bool quadKernels() {
        static int enabled = -2;
        if (enabled == -2)
            enabled = pairChoice("LBM_B200_QUAD16") == 0 ? 0 : 1;
        return enabled == 1;
    }

    // The persistent grid of a kernel variant: one wave of resident blocks (blocks per SM of this variant times
    // the SMs), so that every block processes the same number of tiles in one wave.
    template <bool S, bool RE, bool FL>
    static int residentGrid(const FluidView& v) {
        static int blocks = 0;
        if (blocks == 0) {
            int perSM = 0, device = 0, sms = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, streamCollideKernel<T, R, S, RE, FL>, THREADS, 0);
            cudaGetDevice(&device);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            blocks = std::max(1, perSM)*std::max(1, sms);
        }
        return (int) std::max(1LL, std::min((long long) blocks, v.numTiles));
    }
    template <bool S, bool RE, bool FL>
    static int pairGrid(const FluidView& v) {
        static int blocks = 0;
        if (blocks == 0) {
            int perSM = 0, device = 0, sms = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, streamCollidePairKernel<T, S, RE, FL>, THREADS, 0);
            cudaGetDevice(&device);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            blocks = std::max(1, perSM)*std::max(1, sms);
        }
        long long tiles = (long long) ((v.nx + PAIR_TX - 1)/PAIR_TX)*v.tilesY*v.nz;
        return (int) std::max(1LL, std::min((long long) blocks, tiles));
    }
    template <bool S, bool RE>
    static int quadGrid(const FluidView& v) {
        static int blocks = 0;
        if (blocks == 0) {
            int perSM = 0, device = 0, sms = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, streamCollideQuadKernel<T, S, RE>, LBM_QUAD_THREADS, 0);
            cudaGetDevice(&device);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            blocks = std::max(1, perSM)*std::max(1, sms);
        }
        const long long warps = LBM_QUAD_THREADS/32;
        long long tiles = (long long) ((v.nx + QUAD_TX - 1)/QUAD_TX)*v.ny*v.nz;
        return (int) std::max(1LL, std::min((long long) blocks, (tiles + warps - 1)/warps));
    }
    template <bool S, bool RE, bool FL>
    static int dense(const void* A, void* B, const FluidView& v, int remove, long long step, int maxGrid, cudaStream_t s) {
        if constexpr (sizeof(T) == 2 && !FL) {
            if (v.nx%4 == 0 && pairedKernels<FL>() && quadKernels()) {
                int grid = std::min(maxGrid, quadGrid<S, RE>(v));
                streamCollideQuadKernel<T, S, RE><<<grid, LBM_QUAD_THREADS, 0, s>>>((const T*) A, (T*) B, v, remove, step);
                return grid;
            }
        }
        if constexpr (sizeof(T) <= 4) {
            if (v.nx%2 == 0 && pairedKernels<FL>()) {
                int grid = std::min(maxGrid, pairGrid<S, RE, FL>(v));
                streamCollidePairKernel<T, S, RE, FL><<<grid, THREADS, 0, s>>>((const T*) A, (T*) B, v, remove, step);
                return grid;
            }
        }
        int grid = std::min(maxGrid, residentGrid<S, RE, FL>(v));
        streamCollideKernel<T, R, S, RE, FL><<<grid, THREADS, 0, s>>>((const T*) A, (T*) B, v, remove, step);
        return grid;
    }
    template <bool S, bool RE>
    static int denseF(bool fl, const void* A, void* B, const FluidView& v, int remove, long long step, int grid, cudaStream_t s) {
        return fl ? dense<S, RE, true>(A, B, v, remove, step, grid, s) : dense<S, RE, false>(A, B, v, remove, step, grid, s);
    }
    template <bool S>
    static int denseR(bool re, bool fl, const void* A, void* B, const FluidView& v, int remove, long long step, int grid, cudaStream_t s) {
        return re ? denseF<S, true>(fl, A, B, v, remove, step, grid, s) : denseF<S, false>(fl, A, B, v, remove, step, grid, s);
    }
    // Launch the dense step; returns the grid it used (one partial record per block).
    static int denseAny(bool so, bool re, bool fl, const void* A, void* B, const FluidView& v, int remove, long long step,
                        int grid, cudaStream_t s) {
        return so ? denseR<true>(re, fl, A, B, v, remove, step, grid, s) : denseR<false>(re, fl, A, B, v, remove, step, grid, s);
    }
    static int occupancy() {
        // The largest grid any variant uses (the partial sums are sized for it).
        int best = 1;
        auto probe = [&](auto kernel) {
            int blocks = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, THREADS, 0);
            best = std::max(best, blocks);
        };
        probe(streamCollideKernel<T, R, false, false, false>);
        probe(streamCollideKernel<T, R, false, false, true>);
        probe(streamCollideKernel<T, R, true, true, true>);
        probe(streamCollideKernel<T, R, true, false, false>);
        if constexpr (sizeof(T) <= 4) {
            probe(streamCollidePairKernel<T, false, false, false>);
            probe(streamCollidePairKernel<T, false, true, true>);
            probe(streamCollidePairKernel<T, true, true, true>);
        }
        if constexpr (sizeof(T) == 2) {
            auto probeQuad = [&](auto kernel) {
                int blocks = 0;
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, LBM_QUAD_THREADS, 0);
                best = std::max(best, blocks);
            };
            probeQuad(streamCollideQuadKernel<T, false, false>);
            probeQuad(streamCollideQuadKernel<T, true, true>);
        }
        return best;
    }
    static void bounceBack(void* B, const int* wall, int numWall, const FluidView& v, double* partials, int grid, cudaStream_t s) {
        bounceBackKernel<T, R><<<grid, THREADS, 0, s>>>((T*) B, wall, numWall, v, partials);
    }
    static void boundary(bool fl, const void* A, void* B, const int* bnd, int count, const FluidView& v, int remove, long long step,
                         double* partials, const double* faceData, int grid, cudaStream_t s) {
        if (fl) boundaryKernel<T, R, true><<<grid, 128, 0, s>>>((const T*) A, (T*) B, bnd, count, v, remove, step, partials, faceData);
        else boundaryKernel<T, R, false><<<grid, 128, 0, s>>>((const T*) A, (T*) B, bnd, count, v, remove, step, partials, faceData);
    }
    static void moments(const void* A, const FluidView& v, int grid, cudaStream_t s) {
        momentsKernel<T, R><<<grid, THREADS, 0, s>>>((const T*) A, v);
    }
    static void equilibrium(void* A, void* B, const FluidView& v, const double* rho, const double* u, double ds,
                            double vs, int strain, cudaStream_t s) {
        equilibriumKernel<T, R><<<1184, 256, 0, s>>>((T*) A, (T*) B, v, rho, u, ds, vs, strain);
    }
    static void residual(const void* A, const FluidView& v, double* prev, int first, int grid, cudaStream_t s) {
        residualKernel<T, R><<<grid, THREADS, 0, s>>>((const T*) A, v, prev, first);
    }
    static void init(void* A, void* B, const FluidView& v, const char* fluid, const double* u, cudaStream_t s) {
        initKernel<T, R><<<1184, 256, 0, s>>>((T*) A, (T*) B, v, fluid, u[0], u[1], u[2]);
    }
    static void gather(const void* A, int q, const FluidView& v, double* out, cudaStream_t s) {
        gatherKernel<T, R><<<1184, 256, 0, s>>>((const T*) A, q, v, out);
    }
    static void scatter(void* A, void* B, int q, const FluidView& v, const double* in, int* changed, cudaStream_t s) {
        scatterKernel<T, R><<<1184, 256, 0, s>>>((T*) A, (T*) B, q, v, in, changed);
    }
    static void fields(const void* A, const FluidView& v, double* out, double ds, double vs, cudaStream_t s) {
        fieldsKernel<T, R><<<1184, 256, 0, s>>>((const T*) A, v, out, ds, vs);
    }
};

template <typename F>
void dispatchStorage(int storage, F&& f) {
    switch (storage) {
    case LBM_STORAGE_F64: f(Launcher<double>()); break;
    case LBM_STORAGE_F32: f(Launcher<float>()); break;
    case LBM_STORAGE_F16: f(Launcher<__half>()); break;
    case LBM_STORAGE_BF16: f(Launcher<__nv_bfloat16>()); break;
    default: throw Error(LBM_ERR_NOT_SUPPORTED, "unknown storage type");
    }
}

size_t elementSizeOf(int storage) {
    switch (storage) {
    case LBM_STORAGE_F64: return 8;
    case LBM_STORAGE_F32: return 4;
    case LBM_STORAGE_F16: return 2;
    case LBM_STORAGE_BF16: return 2;
    default: throw Error(LBM_ERR_NOT_SUPPORTED, "unknown storage type");
    }
}

const int kGridSparse = 148;      // blocks of the sparse passes (one wave)
const int kGridWall = 4*148;      // blocks of the bounce-back pass (a wall node per thread on the largest lattices)

} // namespace

FluidEngine::FluidEngine(const LbmLatticeParameters& l, int storage, const Geometry& g, cudaStream_t s)
        : lattice(l), storageType(storage), elementSize(elementSizeOf(storage)), stream(s), cur(0), gridBlocks(0),
          solidMaskDev(nullptr), reactMaskDev(nullptr), reactionDev(nullptr), partialsDev(nullptr), statsDev(nullptr),
          numWall(0), numBoundary(0), wallDev(nullptr), boundaryDev(nullptr), equilibriumNoise(false),
          stagingDev(nullptr), extraBlocks(0), faceDev(nullptr), profiling(false), profileUsed(0) {
    launches = 0;
    pop[0] = pop[1] = nullptr;
    std::memset(&view, 0, sizeof(view));
    view.nx = l.nx;
    view.ny = l.ny;
    view.nz = l.nz;
    view.n = (long long) l.nx*l.ny*l.nz;
    // The dense kernel indexes nodes with 32-bit unsigned integers (4.29e9 nodes: 163 GB of FP16 populations).
    if (view.n >= (1LL << 32) || (long long) l.nx*l.ny >= (1LL << 31))
        throw Error(LBM_ERR_INVALID_ARGUMENT, "The lattice has too many nodes for one device (at most 2^32 nodes, "
                    "and nx*ny below 2^31)");
    view.wordsPerRow = (l.nx + 31)/32;
    view.tilesX = (l.nx + TX - 1)/TX;
    view.tilesY = (l.ny + TY - 1)/TY;
    view.numTiles = (long long) view.tilesX*view.tilesY*l.nz;
    view.numFluid = (double) (view.n - (long long) g.solidNodes.size());
    solidNodes = g.solidNodes;
    try {
        CUDA_CHECK(cudaMalloc(&faceDev, sizeof(double)*32));
        setParameters(l);
        size_t bytes = (size_t) 19*view.n*elementSize;
        CUDA_CHECK(cudaMalloc(&pop[0], bytes));
        CUDA_CHECK(cudaMalloc(&pop[1], bytes));
        int device = 0, sms = 0;
        CUDA_CHECK(cudaGetDevice(&device));
        CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        int occupancy = 1;
        dispatchStorage(storage, [&](auto L) { occupancy = decltype(L)::occupancy(); });
        long long wanted = (long long) sms*occupancy;
        gridBlocks = (int) std::max(1LL, std::min(wanted, view.numTiles));
        extraBlocks = kGridWall + kGridSparse;
        CUDA_CHECK(cudaMalloc(&partialsDev, sizeof(double)*NPART*(size_t) (gridBlocks + extraBlocks + 1)));
        CUDA_CHECK(cudaMalloc(&statsDev, sizeof(StepStats)));
        CUDA_CHECK(cudaMemsetAsync(statsDev, 0, sizeof(StepStats), stream));
        view.partials = partialsDev;
        view.stats = statsDev;

        // Solid mask, rows padded to 32-bit words.
        char* fluidDev = nullptr;
        if (!g.solidNodes.empty()) {
            size_t words = (size_t) view.wordsPerRow*l.ny*l.nz;
            std::vector<uint32_t> mask(words, 0u);
            for (int sn : g.solidNodes) {
                long long row = sn/l.nx;
                int x = (int) (sn%l.nx);
                mask[row*view.wordsPerRow + x/32] |= 1u << (x%32);
            }
            CUDA_CHECK(cudaMalloc(&solidMaskDev, sizeof(uint32_t)*words));
            CUDA_CHECK(cudaMemcpyAsync(solidMaskDev, mask.data(), sizeof(uint32_t)*words, cudaMemcpyHostToDevice, stream));
            CUDA_CHECK(cudaMalloc(&fluidDev, view.n));
            CUDA_CHECK(cudaMemcpyAsync(fluidDev, g.fluid.data(), view.n, cudaMemcpyHostToDevice, stream));
        }
        view.solidMask = solidMaskDev;
        numWall = (int) g.wallNodes.size();
        if (numWall > 0) {
            std::vector<int> w(2*numWall);
            for (int i = 0; i < numWall; i++) {
                w[2*i] = g.wallNodes[i];
                w[2*i+1] = g.wallLinks[i];
            }
            CUDA_CHECK(cudaMalloc(&wallDev, sizeof(int)*w.size()));
            CUDA_CHECK(cudaMemcpyAsync(wallDev, w.data(), sizeof(int)*w.size(), cudaMemcpyHostToDevice, stream));
        }
        numBoundary = (int) g.boundaryNodes.size();
        if (numBoundary > 0) {
            std::vector<int> b(4*numBoundary);
            for (int i = 0; i < numBoundary; i++) {
                b[4*i] = g.boundaryNodes[i];
                b[4*i+1] = g.unknown[i];
                b[4*i+2] = g.solidBits[i];
                b[4*i+3] = g.kind[i] | ((g.face[i] + 1) << 8);
                equilibriumNoise = equilibriumNoise || hasEquilibriumNoise(g.kind[i]);
            }
            CUDA_CHECK(cudaMalloc(&boundaryDev, sizeof(int)*b.size()));
            CUDA_CHECK(cudaMemcpyAsync(boundaryDev, b.data(), sizeof(int)*b.size(), cudaMemcpyHostToDevice, stream));
        }
        double u[3] = {l.initial_velocity[0], l.initial_velocity[1], l.initial_velocity[2]};
        dispatchStorage(storage, [&](auto L) { decltype(L)::init(pop[0], pop[1], view, fluidDev, u, stream); });
        CUDA_CHECK(cudaGetLastError());
        if (fluidDev) {
            CUDA_CHECK(cudaStreamSynchronize(stream));
            cudaFree(fluidDev);
        }
        momentsPass(true);
        CUDA_CHECK(cudaStreamSynchronize(stream));
    }
    catch (...) {
        this->~FluidEngine();
        throw;
    }
}

FluidEngine::~FluidEngine() {
    cudaFree(pop[0]);
    cudaFree(pop[1]);
    cudaFree(solidMaskDev);
    cudaFree(reactMaskDev);
    cudaFree(reactionDev);
    cudaFree(partialsDev);
    cudaFree(statsDev);
    cudaFree(wallDev);
    cudaFree(boundaryDev);
    cudaFree(stagingDev);
    cudaFree(faceDev);
    cudaFree(residualPrevDev);
    residualPrevDev = nullptr;
    faceDev = nullptr;
    for (cudaEvent_t e : profileEvents)
        cudaEventDestroy(e);
    profileEvents.clear();
    pop[0] = pop[1] = nullptr;
    solidMaskDev = reactMaskDev = nullptr;
    reactionDev = stagingDev = nullptr;
    partialsDev = nullptr;
    statsDev = nullptr;
    wallDev = boundaryDev = nullptr;
}

void FluidEngine::setParameters(const LbmLatticeParameters& l) {
    lattice = l;
    view.omega = l.omega;
    for (int a = 0; a < 3; a++)
        view.g[a] = l.body_acceleration[a];
    uint32_t seed = (uint32_t) l.random_number_seed;
    view.seed = seed;
    view.faceOpen = 0;
    for (int f = 0; f < 6; f++)
        if (l.face_boundary[f] != LBM_BOUNDARY_PERIODIC)
            view.faceOpen = 1;
    double cellMass = l.density*l.dx*l.dx*l.dx;
    bool fluctuate = l.fluid_fluctuations && l.fluid_kT > 0;
    view.mu = fluctuate ? 3.0*l.fluid_kT*l.dt*l.dt/(cellMass*l.dx*l.dx) : 0.0;
    // Face velocities and densities, and the boundary stress weight c = (1 - omega)^2/(omega (2 - omega))
    // (D3Q19.h:206-208), for the boundary kernel.
    for (int f = 0; f < 6; f++) {
        for (int a = 0; a < 3; a++)
            faceHost[4*f + a] = l.face_velocity[f][a];
        faceHost[4*f + 3] = l.face_density[f];
    }
    faceHost[24] = (1.0-l.omega)*(1.0-l.omega)/(l.omega*(2.0-l.omega));
    CUDA_CHECK(cudaMemcpyAsync(faceDev, faceHost, sizeof(double)*25, cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

void FluidEngine::enableReaction() {
    if (reactionDev != nullptr)
        return;
    size_t words = (size_t) view.wordsPerRow*lattice.ny*lattice.nz;
    size_t r = (storageType == LBM_STORAGE_F64 ? 8 : 4);
    CUDA_CHECK(cudaMalloc(&reactMaskDev, sizeof(uint32_t)*words));
    CUDA_CHECK(cudaMemsetAsync(reactMaskDev, 0, sizeof(uint32_t)*words, stream));
    CUDA_CHECK(cudaMalloc(&reactionDev, 4*r*(size_t) view.n));
    CUDA_CHECK(cudaMemsetAsync(reactionDev, 0, 4*r*(size_t) view.n, stream));
    view.reactMask = reactMaskDev;
    view.reaction = reactionDev;
}

void FluidEngine::clearReactMask(cudaStream_t s) {
    if (reactMaskDev != nullptr)
        CUDA_CHECK(cudaMemsetAsync(reactMaskDev, 0, sizeof(uint32_t)*(size_t) view.wordsPerRow*lattice.ny*lattice.nz, s));
}

void FluidEngine::step(long long stepIndex, bool remove, bool react) {
    const void* A = pop[cur];
    void* B = pop[1-cur];
    bool fluct = view.mu > 0;
    bool solids = solidMaskDev != nullptr;
    if (profiling) {
        if (profileUsed + 2 > profileEvents.size())
            for (int i = 0; i < 2; i++) {
                cudaEvent_t e;
                CUDA_CHECK(cudaEventCreate(&e));
                profileEvents.push_back(e);
            }
        CUDA_CHECK(cudaEventRecord(profileEvents[profileUsed], stream));
    }
    int denseGrid = gridBlocks;
    dispatchStorage(storageType, [&](auto L) {
        denseGrid = decltype(L)::denseAny(solids, react && reactionDev != nullptr, fluct, A, B, view, remove ? 1 : 0,
                                          stepIndex, gridBlocks, stream);
    });
    CUDA_CHECK(cudaGetLastError());
    launches++;
    if (profiling) {
        CUDA_CHECK(cudaEventRecord(profileEvents[profileUsed + 1], stream));
        profileUsed += 2;
    }
    int count = denseGrid;
    if (numWall > 0) {
        int grid = std::min(kGridWall, (numWall + THREADS - 1)/THREADS);
        double* part = partialsDev + NPART*(size_t) count;
        dispatchStorage(storageType, [&](auto L) { decltype(L)::bounceBack(B, wallDev, numWall, view, part, grid, stream); });
        CUDA_CHECK(cudaGetLastError());
        launches++;
        count += grid;
    }
    if (numBoundary > 0) {
        int grid = std::min(kGridSparse, (numBoundary + 127)/128);
        double* part = partialsDev + NPART*(size_t) count;
        // Face velocities and densities, and the boundary stress weight c (D3Q19.h:206-208), in a small table
        // that lives in the partials buffer tail (read-only for the kernel).
        dispatchStorage(storageType, [&](auto L) {
            decltype(L)::boundary(fluct, A, B, boundaryDev, numBoundary, view, remove ? 1 : 0, stepIndex, part,
                                  faceDev, grid, stream);
        });
        CUDA_CHECK(cudaGetLastError());
        launches++;
        count += grid;
    }
    finishKernel<<<1, THREADS, 0, stream>>>(partialsDev, count, view, 0);
    CUDA_CHECK(cudaGetLastError());
    launches++;
    cur = 1-cur;
}

void FluidEngine::profileDense(bool enable) {
    profiling = enable;
    if (enable)
        profileUsed = 0;
}

void FluidEngine::denseTime(long long* launches, double* totalMs) {
    CUDA_CHECK(cudaStreamSynchronize(stream));
    double total = 0;
    for (size_t i = 0; i + 1 < profileUsed; i += 2) {
        float ms = 0;
        CUDA_CHECK(cudaEventElapsedTime(&ms, profileEvents[i], profileEvents[i+1]));
        total += ms;
    }
    *launches = (long long) (profileUsed/2);
    *totalMs = total;
}

void FluidEngine::momentsPass(bool setSums) {
    dispatchStorage(storageType, [&](auto L) { decltype(L)::moments(pop[cur], view, gridBlocks, stream); });
    CUDA_CHECK(cudaGetLastError());
    finishKernel<<<1, THREADS, 0, stream>>>(partialsDev, gridBlocks, view, setSums ? 1 : 2);
    CUDA_CHECK(cudaGetLastError());
    launches += 2;
}

double FluidEngine::steadyResidual(int interval) {
    bool first = residualPrevDev == nullptr;
    if (first)
        CUDA_CHECK(cudaMalloc(&residualPrevDev, sizeof(double)*3*(size_t) view.n));
    dispatchStorage(storageType, [&](auto L) {
        decltype(L)::residual(pop[cur], view, residualPrevDev, first ? 1 : 0, gridBlocks, stream);
    });
    CUDA_CHECK(cudaGetLastError());
    launches++;
    std::vector<double> partials((size_t) NPART*gridBlocks);
    CUDA_CHECK(cudaMemcpyAsync(partials.data(), partialsDev, sizeof(double)*partials.size(), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    double maxDiff2 = 0, maxU2 = 0;
    for (int b = 0; b < gridBlocks; b++) {
        maxDiff2 = std::max(maxDiff2, partials[(size_t) NPART*b]);
        maxU2 = std::max(maxU2, partials[(size_t) NPART*b + 7]);
    }
    if (first || maxU2 == 0)
        return HUGE_VAL;
    return std::sqrt(maxDiff2)/(interval*std::sqrt(maxU2));
}

void FluidEngine::restoreStats(const StepStats& stats) {
    statsHost = stats;
    CUDA_CHECK(cudaMemcpyAsync(statsDev, &statsHost, sizeof(StepStats), cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

StepStats FluidEngine::readStats() {
    StepStats s;
    CUDA_CHECK(cudaMemcpyAsync(&s, statsDev, sizeof(StepStats), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    return s;
}

void FluidEngine::getState(double* host) {
    getStateByDirection([&](int q, const double* values) {
        std::memcpy(host + (size_t) q*view.n, values, sizeof(double)*view.n);
    });
}

void FluidEngine::getStateByDirection(const std::function<void(int, const double*)>& sink) {
    if (stagingDev == nullptr)
        CUDA_CHECK(cudaMalloc(&stagingDev, sizeof(double)*4*(size_t) view.n));
    std::vector<double> plane((size_t) view.n);
    for (int q = 0; q < 19; q++) {
        dispatchStorage(storageType, [&](auto L) { decltype(L)::gather(pop[cur], q, view, (double*) stagingDev, stream); });
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaMemcpyAsync(plane.data(), stagingDev, sizeof(double)*view.n, cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
        sink(q, plane.data());
    }
}

void FluidEngine::setState(const double* host) {
    setStateByDirection([&](int q, double* values) {
        std::memcpy(values, host + (size_t) q*view.n, sizeof(double)*view.n);
    });
}

void FluidEngine::setStateByDirection(const std::function<void(int, double*)>& source) {
    if (stagingDev == nullptr)
        CUDA_CHECK(cudaMalloc(&stagingDev, sizeof(double)*4*(size_t) view.n));
    int* changedDev = reinterpret_cast<int*>(partialsDev);
    CUDA_CHECK(cudaMemsetAsync(changedDev, 0, sizeof(int), stream));
    std::vector<double> plane((size_t) view.n);
    for (int q = 0; q < 19; q++) {
        source(q, plane.data());
        CUDA_CHECK(cudaMemcpyAsync(stagingDev, plane.data(), sizeof(double)*view.n, cudaMemcpyHostToDevice, stream));
        dispatchStorage(storageType, [&](auto L) {
            decltype(L)::scatter(pop[cur], pop[1-cur], q, view, (const double*) stagingDev, changedDev, stream);
        });
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaStreamSynchronize(stream));
    }
    int changed = 0;
    CUDA_CHECK(cudaMemcpy(&changed, changedDev, sizeof(int), cudaMemcpyDeviceToHost));
    if (changed)
        momentsPass(true);
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

void FluidEngine::setEquilibrium(const double* density, const double* velocity, bool onDevice, double densityScale,
                                 double velocityScale, bool strain) {
    const double* rho = density;
    const double* u = velocity;
    if (!onDevice) {
        if (stagingDev == nullptr)
            CUDA_CHECK(cudaMalloc(&stagingDev, sizeof(double)*4*(size_t) view.n));
        double* staging = (double*) stagingDev;
        CUDA_CHECK(cudaMemcpyAsync(staging, density, sizeof(double)*view.n, cudaMemcpyHostToDevice, stream));
        CUDA_CHECK(cudaMemcpyAsync(staging + view.n, velocity, sizeof(double)*3*view.n, cudaMemcpyHostToDevice, stream));
        rho = staging;
        u = staging + view.n;
    }
    dispatchStorage(storageType, [&](auto L) {
        decltype(L)::equilibrium(pop[cur], pop[1-cur], view, rho, u, densityScale, velocityScale, strain ? 1 : 0, stream);
    });
    CUDA_CHECK(cudaGetLastError());
    launches++;
    momentsPass(true);
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

void FluidEngine::fields(double* density, double* velocity, double densityScale, double velocityScale) {
    if (stagingDev == nullptr)
        CUDA_CHECK(cudaMalloc(&stagingDev, sizeof(double)*4*(size_t) view.n));
    dispatchStorage(storageType, [&](auto L) {
        decltype(L)::fields(pop[cur], view, (double*) stagingDev, densityScale, velocityScale, stream);
    });
    CUDA_CHECK(cudaGetLastError());
    std::vector<double> all(4*(size_t) view.n);
    CUDA_CHECK(cudaMemcpyAsync(all.data(), stagingDev, sizeof(double)*all.size(), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    for (long long x = 0; x < view.n; x++) {
        density[x] = all[4*x];
        for (int a = 0; a < 3; a++)
            velocity[3*x+a] = all[4*x+1+a];
    }
}

void FluidEngine::copyStateOut(void* host) {
    CUDA_CHECK(cudaMemcpyAsync(host, pop[cur], stateBytes(), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

void FluidEngine::copyStateIn(const void* host) {
    CUDA_CHECK(cudaMemcpyAsync(pop[cur], host, stateBytes(), cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaMemcpyAsync(pop[1-cur], pop[cur], stateBytes(), cudaMemcpyDeviceToDevice, stream));
    momentsPass(true);
    CUDA_CHECK(cudaStreamSynchronize(stream));
}

} // namespace lbm
