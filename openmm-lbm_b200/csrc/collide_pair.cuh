// The paired collision of two x-adjacent nodes in packed FP32 arithmetic (FFMA2 / FADD2 / FMUL2 of sm_100), shared by
// the single-lattice dense kernel (fluid.cu) and the replica batch (batch.cu).
#pragma once

#include "collide.cuh"
#include "fluid.cuh"
#include "lbm_device.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace lbm {
namespace {

// A float from global memory: through L2 when COHERENT (data written by other blocks of the same launch).
template <bool COHERENT>
__device__ __forceinline__ float loadValue(const float* p) {
    if constexpr (COHERENT)
        return __ldcg(p);
    else
        return *p;
}

// ---------------------------------------------------------------------------------------------------
// The dense step for 16-bit storage without fluctuations: two x-adjacent nodes per thread, their arithmetic in
// packed FP32 pairs (FFMA2 / FADD2 / FMUL2 of sm_100), their populations loaded and stored as 32-bit pairs.  For a
// direction with c_x = 0 the pair of sources is one aligned word of the source row; with c_x = +1 it is the high half
// of the word to the left and the low half of this word, with c_x = -1 the high half of this word and the low half
// of the word to the right (the lattice has an even nx, so the periodic wrap keeps the pairs aligned).  The
// algebra is that of collideNode (collide.cuh), written for the pairs.
// ---------------------------------------------------------------------------------------------------

struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 f2(float a) { return F2{make_float2(a, a)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2{__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)}; }

// Words of two x-adjacent nodes of one direction: a 32-bit word for 16-bit storage (stochastic rounding on store),
// a float2 for FP32 storage.  left(l, c) is the pair (x0 - 1, x0) from the word to the left and this one, right(c, r)
// the pair (x0 + 1, x0 + 2).
template <typename T> struct PairIO;
template <> struct PairIO<__half> {
    typedef uint32_t Word;
    static constexpr float scale = kHalfScale;
    static __device__ __forceinline__ Word left(Word l, Word c) { return __byte_perm(l, c, 0x5432); }
    static __device__ __forceinline__ Word right(Word c, Word r) { return __byte_perm(c, r, 0x5432); }
    static __device__ __forceinline__ F2 decode(Word w) {
        __half2 h = *reinterpret_cast<__half2*>(&w);
        return F2{__half22float2(h)};
    }
    static __device__ __forceinline__ uint32_t pack(float lo, float hi, uint32_t rbits) {
        return stochasticHalf2(lo, hi, rbits);
    }
};
template <> struct PairIO<__nv_bfloat16> {
    typedef uint32_t Word;
    static constexpr float scale = 1.0f;
    static __device__ __forceinline__ Word left(Word l, Word c) { return __byte_perm(l, c, 0x5432); }
    static __device__ __forceinline__ Word right(Word c, Word r) { return __byte_perm(c, r, 0x5432); }
    static __device__ __forceinline__ F2 decode(Word w) {
        return F2{make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xFFFF0000u))};
    }
    static __device__ __forceinline__ uint32_t pack(float lo, float hi, uint32_t rbits) {
        return stochasticBf162(lo, hi, rbits);
    }
};
template <> struct PairIO<float> {
    typedef float2 Word;
    static __device__ __forceinline__ Word left(Word l, Word c) { return make_float2(l.y, c.x); }
    static __device__ __forceinline__ Word right(Word c, Word r) { return make_float2(c.y, r.x); }
    static __device__ __forceinline__ F2 decode(Word w) { return F2{w}; }
};

// Factor from a deviation to the stored value of direction q.
template <typename T, int q> __device__ __forceinline__ constexpr float storeScale() {
    if constexpr (sizeof(T) == 2)
        return PairIO<T>::scale*storeFactorOf(q);
    else
        return 1.0f;
}

constexpr int PAIR_TX = 64;         // nodes per tile row: 2 per lane

// Stores the pair `value` (stored units) of one direction; the half of a solid node stays untouched (as in the
// one-node kernel).  16-bit storage rounds stochastically with the dither bits of the two nodes, node A's in the low
// half of `dither` and node B's in the high half.
// The packed 16-bit word w of two nodes; the half of a solid node stays untouched.
template <bool SOLID>
__device__ __forceinline__ void storeWord16(uint32_t* p, uint32_t w, bool solidA, bool solidB) {
    if (SOLID && (solidA || solidB)) {
        unsigned short* h = reinterpret_cast<unsigned short*>(p);
        if (!solidA)
            h[0] = (unsigned short) (w & 0xFFFFu);
        if (!solidB)
            h[1] = (unsigned short) (w >> 16);
        return;
    }
    *p = w;
}

template <typename T, bool SOLID>
__device__ __forceinline__ void storePair(typename PairIO<T>::Word* p, F2 value, uint32_t dither, bool solidA,
                                          bool solidB) {
    if constexpr (sizeof(T) == 2)
        storeWord16<SOLID>(p, PairIO<T>::pack(value.v.x, value.v.y, dither), solidA, solidB);
    else {
        if (SOLID && (solidA || solidB)) {
            float* h = reinterpret_cast<float*>(p);
            if (!solidA)
                h[0] = value.v.x;
            if (!solidB)
                h[1] = value.v.y;
            return;
        }
        *p = value.v;
    }
}

// Where collidePair puts the post-collision values of direction q (stored units, with their dither bits): the pair's
// word in each direction plane (`out` is its word in plane 0, planes `halfN` words apart).
template <typename T, bool SOLID>
struct PairStore {
    typename PairIO<T>::Word* out;
    unsigned halfN;
    bool solidA, solidB;
    template <int q> __device__ __forceinline__ void put(F2 value, uint32_t dither) {
        storePair<T, SOLID>(out + (size_t) q*halfN, value, dither, solidA, solidB);
    }
};

// Ghost-mode parts of direction q for a pair of nodes, without the weight: sums over the odd and the even modes
// k = 10..18 of e_k(c_q) a_k.
template <int q>
__device__ __forceinline__ void ghostSums2(const F2 a[15], F2& even, F2& odd) {
    even = f2(0.0f);
    odd = f2(0.0f);
    staticFor<9>([&](auto kc) {
        constexpr int k = decltype(kc)::value + 10;
        constexpr float m = (float) modeValue(k, q);
        if (m != 0.0f) {
            if (k <= 15)
                odd = fma2(f2(m), a[k-4], odd);
            else
                even = fma2(f2(m), a[k-4], even);
        }
    });
}

// Resident blocks of 256 threads per SM the paired kernel is compiled for: 3 for 16-bit storage without
// fluctuations (it fits in 80 registers without spilling and waits on its loads, so more warps help: FP16 channel
// step 0.584 -> 0.569 ms, BF16 0.581 -> 0.561 ms), 2 otherwise (FP32 storage at 3 blocks: channel step 0.722 ->
// 0.852 ms, 256^3 0.473 -> 0.483 ms; the noise needs more registers).
#ifndef LBM_PAIR_MIN_BLOCKS
#define LBM_PAIR_MIN_BLOCKS 2
#endif
#ifndef LBM_PAIR_MIN_BLOCKS_16BIT
#define LBM_PAIR_MIN_BLOCKS_16BIT 3
#endif

// Per-launch constants of the paired kernels.
struct PairConstants {
    float om1, mu, stressFactor;
    F2 gx, gy, gz, nux0, nuy0, nuz0;
    uint32_t stepHash;
};

// The removal velocity ucm is that of the fluid's step statistics (a launch of a persistent kernel passes the value
// that it read through L2).
__device__ __forceinline__ PairConstants pairConstants(const FluidView& v, int remove, long long step,
                                                       const double* ucm = nullptr) {
    if (ucm == nullptr)
        ucm = v.stats->ucm;
    PairConstants c;
    const float om = (float) v.omega;
    c.om1 = 1.0f - om;
    c.mu = (float) v.mu;
    c.stressFactor = om*(2.0f - om);
    c.gx = f2((float) v.g[0]);
    c.gy = f2((float) v.g[1]);
    c.gz = f2((float) v.g[2]);
    c.nux0 = c.nuy0 = c.nuz0 = f2(0.0f);
    if (remove) {
        c.nux0 = f2(-(float) ucm[0]);
        c.nuy0 = f2(-(float) ucm[1]);
        c.nuz0 = f2(-(float) ucm[2]);
    }
    c.stepHash = Dither::fmix32((uint32_t) step + 0x9E3779B9u*(uint32_t) ((unsigned long long) step >> 32));
    return c;
}

// The collision of the x-adjacent nodes `node` and `node + 1` from their pulled words r (stored units): hands the 19
// post-collision pairs to out.put<q>() and adds the pair's mass and momentum to sums.
// reactA, reactB flag nodes whose reaction force the coupling left in v.reaction.
// hi + t as the rounded sum hi and its exact rounding error, added to lo (Knuth's TwoSum: six rounded operations, valid
// whatever the magnitudes; the packed intrinsics are never re-associated by the compiler).
__device__ __forceinline__ void twoSumInto(F2& hi, F2& lo, F2 t) {
    const F2 s = hi + t;
    const F2 bb = s - hi;
    lo = lo + ((hi - (s - bb)) + (t - bb));
    hi = s;
}

// How the paired kernel carries the momentum in two floats (hi + lo).  In FP32 arithmetic the momentum sums and
// j + F are rounded every step, and a flow accelerated by a small force drifts by the accumulated rounding (2.5e-4 of
// u after 20,000 steps of the precision channel, against FP64, in the column emulation tests/channel_column.py and on
// the GPU): with level 2 the momentum sums and j + F are formed with their rounding errors, and the odd part of every
// direction adds the errors' share before the rounded momentum (1.6e-5 in the emulation, 2.6e-5 on the GPU).  Level 1
// compensates j + F only: the decoded values of 16-bit storage are multiples of a coarse quantum, so their momentum
// sums are exact or nearly so in FP32.  A fluctuating fluid takes level 0: its thermal noise dwarfs the drift, and the
// extra arithmetic would slow its instruction-bound kernel by 18%.
#ifndef LBM_COMPENSATED_16BIT
#define LBM_COMPENSATED_16BIT 1
#endif
template <typename T, bool FLUCT> LBM_HD constexpr int compensationLevel() {
    return FLUCT ? 0 : (sizeof(T) == 4 ? 2 : LBM_COMPENSATED_16BIT);
}

// The pulled values of a pair as collidePair reads them (stored units): from decoded pairs, or from packed 16-bit words
// decoded where the moment sums use them (so that the 19 decoded pairs need not be live at once).
struct PulledPairs {
    const F2 (&r)[19];
    template <int q> __device__ __forceinline__ F2 get() const { return r[q]; }
};
template <typename T>
struct PulledWords {
    const uint32_t (&w)[19];
    template <int q> __device__ __forceinline__ F2 get() const { return PairIO<T>::decode(w[q]); }
};

template <typename T, bool SOLID, bool REACT, bool FLUCT, bool COHERENT = false, typename Out>
__device__ __forceinline__ void collidePair(const F2 (&r)[19], const FluidView& v, const PairConstants& c, int remove,
                                            long long step, unsigned node, bool solidA, bool solidB, bool reactA,
                                            bool reactB, Out& out, float (&sums)[4]);
template <typename T, bool SOLID, bool REACT, bool FLUCT, bool COHERENT = false, typename In, typename Out>
__device__ __forceinline__ void collidePulled(const In& in, const FluidView& v, const PairConstants& c, int remove,
                                            long long step, unsigned node, bool solidA, bool solidB, bool reactA,
                                            bool reactB, Out& out, float (&sums)[4]) {
    constexpr bool dithered = sizeof(T) == 2;
    constexpr int level = compensationLevel<T, FLUCT>();
    constexpr bool comp = level >= 1, compSums = level >= 2;
    // Moments (deviations), the storage factors folded into the FMAs.  With comp the momentum is summed with its
    // rounding errors in jxl, jyl, jzl (the terms cx s D are exact: s is a power of two).
    F2 dr = f2(Storage<T>::template scale<0>())*in.template get<0>();
    F2 jx = f2(0), jy = f2(0), jz = f2(0), sxx = f2(0), syy = f2(0), szz = f2(0), sxy = f2(0), sxz = f2(0), syz = f2(0);
    F2 jxl = f2(0), jyl = f2(0), jzl = f2(0);
    staticFor<9>([&](auto pc) {
        constexpr int q = 2*decltype(pc)::value + 1;
        constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
        constexpr float s = Storage<T>::template scale<q>();
        const F2 rq = in.template get<q>(), rq1 = in.template get<q + 1>();
        const F2 S = rq + rq1, D = rq - rq1;
        dr = fma2(f2(s), S, dr);
        if constexpr (compSums) {
            // The first term of each component (q = 1, 3, 5) starts the sum exactly.
            if (cx != 0) { if (q == 1) jx = D*f2(cx*s); else twoSumInto(jx, jxl, D*f2(cx*s)); sxx = fma2(f2(s), S, sxx); }
            if (cy != 0) { if (q == 3) jy = D*f2(cy*s); else twoSumInto(jy, jyl, D*f2(cy*s)); syy = fma2(f2(s), S, syy); }
            if (cz != 0) { if (q == 5) jz = D*f2(cz*s); else twoSumInto(jz, jzl, D*f2(cz*s)); szz = fma2(f2(s), S, szz); }
        }
        else {
            if (cx != 0) { jx = fma2(f2(cx*s), D, jx); sxx = fma2(f2(s), S, sxx); }
            if (cy != 0) { jy = fma2(f2(cy*s), D, jy); syy = fma2(f2(s), S, syy); }
            if (cz != 0) { jz = fma2(f2(cz*s), D, jz); szz = fma2(f2(s), S, szz); }
        }
        if (cx*cy != 0) sxy = fma2(f2(cx*cy*s), S, sxy);
        if (cx*cz != 0) sxz = fma2(f2(cx*cz*s), S, sxz);
        if (cy*cz != 0) syz = fma2(f2(cy*cz*s), S, syz);
    });
    const F2 rho = dr + f2(1.0f);
    const F2 inv = F2{make_float2(__fdividef(1.0f, rho.v.x), __fdividef(1.0f, rho.v.y))};
    const F2 ninv = F2{make_float2(-inv.v.x, -inv.v.y)};
    const F2 dr3 = dr*f2(-1.0f/3.0f);
    // Pi_neq = S2 - dr/3 - j j/rho.
    const F2 jxi = jx*ninv, jyi = jy*ninv;
    const F2 pxx = fma2(jx, jxi, sxx + dr3), pyy = fma2(jy, jyi, syy + dr3), pzz = fma2(jz, jz*ninv, szz + dr3);
    const F2 pxy = fma2(jy, jxi, sxy), pxz = fma2(jz, jxi, sxz), pyz = fma2(jz, jyi, syz);
    if (remove) {
        if constexpr (compSums) {
            twoSumInto(jx, jxl, rho*c.nux0);
            twoSumInto(jy, jyl, rho*c.nuy0);
            twoSumInto(jz, jzl, rho*c.nuz0);
        }
        else {
            jx = fma2(rho, c.nux0, jx);
            jy = fma2(rho, c.nuy0, jy);
            jz = fma2(rho, c.nuz0, jz);
        }
    }
    F2 Fx = rho*c.gx, Fy = rho*c.gy, Fz = rho*c.gz;
    if (REACT) {
        const float* rp = reinterpret_cast<const float*>(v.reaction) + 4*(size_t) node;
        if (reactA) {
            Fx.v.x += loadValue<COHERENT>(rp); Fy.v.x += loadValue<COHERENT>(rp + 1); Fz.v.x += loadValue<COHERENT>(rp + 2);
        }
        if (reactB) {
            Fx.v.y += loadValue<COHERENT>(rp + 4); Fy.v.y += loadValue<COHERENT>(rp + 5); Fz.v.y += loadValue<COHERENT>(rp + 6);
        }
    }
    const F2 ux = fma2(Fx, f2(0.5f), jx)*inv, uy = fma2(Fy, f2(0.5f), jy)*inv, uz = fma2(Fz, f2(0.5f), jz)*inv;
    const F2 uu = fma2(uz, uz, fma2(uy, uy, ux*ux)), uf = fma2(uz, Fz, fma2(uy, Fy, ux*Fx));
    // The momentum after the force, p = j + F, and with comp its low part (the rounding error of the sum and that of
    // the momentum sums).
    F2 px = jx, py = jy, pz = jz, pxl = jxl, pyl = jyl, pzl = jzl;
    if constexpr (comp) {
        twoSumInto(px, pxl, Fx);
        twoSumInto(py, pyl, Fy);
        twoSumInto(pz, pzl, Fz);
    }
    else {
        px = jx + Fx;
        py = jy + Fy;
        pz = jz + Fz;
    }
    const F2 s45 = f2(c.om1*4.5f), s9 = f2(c.om1*9.0f);
    F2 qxx = s45*pxx, qyy = s45*pyy, qzz = s45*pzz, qxy = s9*pxy, qxz = s9*pxz, qyz = s9*pyz;
    // Fluctuations: the amplitudes a_k = phi_k r_k/sqrt(b_k) of the 15 non-conserved modes of each node (Philox
    // normals of the node and step), the stress modes merged into Q, the ghost modes added per direction.
    F2 a[15];
    if (FLUCT) {
        float rnA[15], rnB[15];
        philoxNormals<float, 15>(v.seed, PurposeFluid, node, step, rnA);
        philoxNormals<float, 15>(v.seed, PurposeFluid, node + 1, step, rnB);
        const float stressA = approxSqrt(c.mu*rho.v.x*c.stressFactor), stressB = approxSqrt(c.mu*rho.v.y*c.stressFactor);
        const float ghostA = approxSqrt(c.mu*rho.v.x), ghostB = approxSqrt(c.mu*rho.v.y);
#pragma unroll
        for (int k = 4; k < 19; k++) {
            const float norm = (float) invSqrtModeNorm(k);
            a[k-4] = F2{make_float2(rnA[k-4]*(k < 10 ? stressA : ghostA)*norm, rnB[k-4]*(k < 10 ? stressB : ghostB)*norm)};
        }
        qxx = qxx + a[0]; qyy = qyy + a[1]; qzz = qzz + a[2];
        qxy = qxy + a[3]; qxz = qxz + a[4]; qyz = qyz + a[5];
    }
    const F2 qtr = (qxx + qyy + qzz)*f2(1.0f/3.0f);
    const F2 base = fma2(fma2(rho, uu, uf), f2(-1.5f), dr);
    // The even part of direction q (before the weight), base - qtr + 4.5 (c.u)(rho c.u + c.F) + c.Q.c, as
    // base - qtr + sum_{c_a != 0} P_aa + sum_{a < b} c_a c_b P_ab with the symmetric tensor
    // P_aa = 4.5 u_a (rho u_a + F_a) + q_aa and P_ab = 4.5 (u_a (2 rho u_b + F_b) + u_b F_a) + q_ab: the axis
    // directions take E_a = base - qtr + P_aa, the diagonal ones S_ab +- P_ab with S_ab = E_a + P_bb.
    const F2 rho2 = rho + rho, base1 = base - qtr;
    const F2 Ex = base1 + fma2(ux*fma2(rho, ux, Fx), f2(4.5f), qxx);
    const F2 Pyy = fma2(uy*fma2(rho, uy, Fy), f2(4.5f), qyy), Pzz = fma2(uz*fma2(rho, uz, Fz), f2(4.5f), qzz);
    const F2 Ey = base1 + Pyy, Ez = base1 + Pzz;
    const F2 Pxy = fma2(fma2(ux, fma2(rho2, uy, Fy), uy*Fx), f2(4.5f), qxy);
    const F2 Pxz = fma2(fma2(ux, fma2(rho2, uz, Fz), uz*Fx), f2(4.5f), qxz);
    const F2 Pyz = fma2(fma2(uy, fma2(rho2, uz, Fz), uz*Fy), f2(4.5f), qyz);
    const F2 Sxy = Ex + Pyy, Sxz = Ex + Pzz, Syz = Ey + Pzz;
    // Dither words of the two nodes (the hash of collideNode's Dither, per node).
    uint32_t hashA = 0, hashB = 0;
    if (dithered) {
        hashA = Dither::fmix32(node ^ c.stepHash);
        hashB = Dither::fmix32((node + 1) ^ c.stepHash);
    }
    {
        F2 value = (base - qtr)*f2(1.0f/3.0f);
        if (FLUCT) {
            F2 e, o;
            ghostSums2<0>(a, e, o);
            value = fma2(e, f2(wOf<float>(0)), value);
        }
        out.template put<0>(value*f2(storeScale<T, 0>()), __byte_perm(hashA*0x9E3779B1u, hashB*0x9E3779B1u, 0x5410));
    }
    staticFor<9>([&](auto pc) {
        constexpr int p = decltype(pc)::value;
        constexpr int q = 2*p + 1;
        constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
        constexpr float k = storeScale<T, q>();
        constexpr float w = wOf<float>(q);
        F2 evenRaw;
        if constexpr (cy == 0 && cz == 0)
            evenRaw = Ex;
        else if constexpr (cx == 0 && cz == 0)
            evenRaw = Ey;
        else if constexpr (cx == 0 && cy == 0)
            evenRaw = Ez;
        else if constexpr (cz == 0)
            evenRaw = cx*cy > 0 ? Sxy + Pxy : Sxy - Pxy;
        else if constexpr (cy == 0)
            evenRaw = cx*cz > 0 ? Sxz + Pxz : Sxz - Pxz;
        else
            evenRaw = cy*cz > 0 ? Syz + Pyz : Syz - Pyz;
        // The odd part in stored units, k 3 w c.(j + F) (3 w rounded as oddOf); with comp the low parts of j + F come
        // first in the FMA chain, so that the high parts are added to their contribution and rounded once.
        constexpr float ko = k*oddOf<float>(q);
        F2 odd = f2(0.0f);
        if constexpr (comp) {
            if constexpr (cx != 0) odd = fma2(pxl, f2(cx*ko), odd);
            if constexpr (cy != 0) odd = fma2(pyl, f2(cy*ko), odd);
            if constexpr (cz != 0) odd = fma2(pzl, f2(cz*ko), odd);
            if constexpr (cx != 0) odd = fma2(px, f2(cx*ko), odd);
            if constexpr (cy != 0) odd = fma2(py, f2(cy*ko), odd);
            if constexpr (cz != 0) odd = fma2(pz, f2(cz*ko), odd);
        }
        else if constexpr (cx != 0) {
            odd = px*f2(cx*ko);
            if constexpr (cy != 0) odd = fma2(py, f2(cy*ko), odd);
            if constexpr (cz != 0) odd = fma2(pz, f2(cz*ko), odd);
        }
        else if constexpr (cy != 0) {
            odd = py*f2(cy*ko);
            if constexpr (cz != 0) odd = fma2(pz, f2(cz*ko), odd);
        }
        else
            odd = pz*f2(cz*ko);
        // Plus k w times the ghost sums with fluctuations; even in stored units is k w evenRaw.
        if (FLUCT) {
            F2 e, o;
            ghostSums2<q>(a, e, o);
            evenRaw = evenRaw + e;
            odd = fma2(o, f2(k*w), odd);
        }
        const F2 even = evenRaw*f2(k*w);
        uint32_t wa = 0, wb = 0;
        if (dithered) {
            wa = hashA*(0x9E3779B1u + 0x3C6EF372u*(uint32_t) (p + 1));
            wb = hashB*(0x9E3779B1u + 0x3C6EF372u*(uint32_t) (p + 1));
        }
        // Direction q takes the low halves of the nodes' words, q + 1 the high halves.
        out.template put<q>(even + odd, __byte_perm(wa, wb, 0x5410));
        out.template put<q + 1>(even - odd, __byte_perm(wa, wb, 0x7632));
    });
    if (!solidA) {
        sums[0] += dr.v.x; sums[1] += px.v.x; sums[2] += py.v.x; sums[3] += pz.v.x;
    }
    if (!solidB) {
        sums[0] += dr.v.y; sums[1] += px.v.y; sums[2] += py.v.y; sums[3] += pz.v.y;
    }
}

template <typename T, bool SOLID, bool REACT, bool FLUCT, bool COHERENT, typename Out>
__device__ __forceinline__ void collidePair(const F2 (&r)[19], const FluidView& v, const PairConstants& c, int remove,
                                            long long step, unsigned node, bool solidA, bool solidB, bool reactA,
                                            bool reactB, Out& out, float (&sums)[4]) {
    collidePulled<T, SOLID, REACT, FLUCT, COHERENT>(PulledPairs{r}, v, c, remove, step, node, solidA, solidB, reactA,
                                                    reactB, out, sums);
}

} // namespace
} // namespace lbm
