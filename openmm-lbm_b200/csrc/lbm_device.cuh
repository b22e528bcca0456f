// Device helpers of the B200 LBM kernels: the D3Q19 velocity set, storage conversion of the population
// deviations, the Philox4x32 counter-based generator and the collision algebra.
//
// The algebra is that of the reference's D3Q19 class (openmmapi/include/internal/D3Q19.h): equilibrium
// deviation (:55), regularized non-equilibrium part (:116), Guo forcing (:127) and the Lulli et al.
// orthogonal basis of the fluctuations (:136-190).  Loops over the 19 velocities are unrolled, so the
// velocity components and weights are compile-time constants.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>

namespace lbm {

#define LBM_HD __host__ __device__ __forceinline__

LBM_HD constexpr int cxOf(int q) { return (q == 1 || q == 7 || q == 9 || q == 15 || q == 18) ? 1 : (q == 2 || q == 8 || q == 10 || q == 16 || q == 17) ? -1 : 0; }
LBM_HD constexpr int cyOf(int q) { return (q == 3 || q == 7 || q == 10 || q == 11 || q == 13) ? 1 : (q == 4 || q == 8 || q == 9 || q == 12 || q == 14) ? -1 : 0; }
LBM_HD constexpr int czOf(int q) { return (q == 5 || q == 11 || q == 14 || q == 15 || q == 17) ? 1 : (q == 6 || q == 12 || q == 13 || q == 16 || q == 18) ? -1 : 0; }
LBM_HD constexpr int oppOf(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
template <typename R> LBM_HD constexpr R wOf(int q) { return q == 0 ? R(1.0/3.0) : (q <= 6 ? R(1.0/18.0) : R(1.0/36.0)); }
// Power-of-two stand-ins for 1/w_q (4, 16, 32): the 16-bit formats store the deviation times this factor, so
// that decoding is the exact inverse of encoding.
LBM_HD constexpr float storeFactorOf(int q) { return q == 0 ? 4.0f : (q <= 6 ? 16.0f : 32.0f); }
LBM_HD constexpr float loadFactorOf(int q) { return q == 0 ? 0.25f : (q <= 6 ? 0.0625f : 0.03125f); }
// Coefficients 3 w_q of the odd (momentum) part of the equilibrium, rounded so that the momentum they
// rebuild is exact: sum_q c_qx c_qx 3 w_q = 2 (axis + 4 diagonal) = 1 holds in floating point, with the
// diagonal value the nearest to 1/12 and the axis value 1/2 - 4 diag (exact).  With the rounded 3 w_q of
// float, each step would scale the momentum by 1 + 3e-8, which a flow accelerated from rest accumulates.
template <typename R> LBM_HD constexpr R oddDiagonal() { return R(1.0/12.0); }
template <typename R> LBM_HD constexpr R oddAxis() { return R(0.5) - R(4)*oddDiagonal<R>(); }
template <typename R> LBM_HD constexpr R oddOf(int q) { return q <= 6 ? oddAxis<R>() : oddDiagonal<R>(); }

// ------------------------------------------------------------------------------------------------------
// Storage of the deviations f_q - w_q.  FP64 and FP32 store the deviation itself, rounded to nearest.
// The 16-bit formats store v = (f_q - w_q) k_q with k_q = 4, 16, 32 (rest, axis, diagonal), powers of two
// near 1/w_q, which give all 19 directions values of one magnitude and make decoding exact.  FP16 stores
// v * 2^10, so that the binary16 normal range starts at |v| = 2^-24 and ends at |v| = 64, and BF16 (the
// exponent range of FP32) stores v itself.
//
// The dense kernel rounds its 16-bit stores stochastically: 13 (FP16) or 16 (BF16) dither bits are added to
// the magnitude of the FP32 value below the 16-bit mantissa, which is then truncated (one `cvt.rs` conversion
// per pair of values).  The stored value is the upper or the lower neighbour of v with probabilities
// proportional to the distances, so the expected rounding error is zero.
// Round-to-nearest would lose every change of a population smaller than half an ulp (1/2048 of the value in
// FP16, 1/256 in BF16): a flow accelerated from rest by a small body force stalls once the per-step change
// of its populations falls below that.  The dither bits of a store are a hash of (node, step), so runs are
// reproducible and restarts from a checkpoint are bitwise.  The sparse kernels (boundaries, state transfer)
// round to nearest.
// ------------------------------------------------------------------------------------------------------

constexpr float kHalfScale = 1024.0f;

// Stochastic rounding of two FP32 values to a packed 16-bit pair by the conversion of sm_100a (`cvt.rs`): the low
// half of the result is `lo` rounded with the low 16 bits of `rbits`, the high half `hi` with the high 16 bits.  The
// conversion adds those bits to the part of the FP32 magnitude below the 16-bit mantissa (FP16: their low 13 bits,
// BF16: all 16) and truncates, which for normal results is the same as adding them to the FP32 bit pattern and
// rounding toward zero (checked on B200 over 10^6 random operands).  Unlike that integer form it also rounds
// stochastically into the FP16 subnormal range, where the integer form truncates to zero.  `.satfinite` keeps the
// saturation of round-toward-zero at the largest finite value.
__device__ __forceinline__ uint32_t stochasticHalf2(float lo, float hi, uint32_t rbits) {
    uint32_t r;
    asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
    return r;
}
__device__ __forceinline__ uint32_t stochasticBf162(float lo, float hi, uint32_t rbits) {
    uint32_t r;
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
    return r;
}

// Storage<T>: raw<q>(p) loads the stored value in storage units, scale<q>() converts storage units to a
// deviation (a compile-time constant that the moment sums fold into their FMAs), storePair<q> stores the
// deviations of directions q and q+1 (equal weights) and returns what was stored, in storage units.
template <typename T> struct Storage;
template <> struct Storage<double> {
    template <int q> static LBM_HD constexpr double scale() { return 1.0; }
    template <int q> static __device__ __forceinline__ double raw(const double* p) { return __ldg(p); }
    // The load of data that the same launch writes (persistent kernels): through L2, never the read-only path.
    template <int q> static __device__ __forceinline__ double rawCoherent(const double* p) { return __ldcg(p); }
    template <int q> static __device__ __forceinline__ double storeOne(double* p, double v, uint32_t) { *p = v; return v; }
    template <int q> static __device__ __forceinline__ void storePair(double* pa, double* pb, double a, double b, uint32_t,
                                                                      double& ra, double& rb) {
        *pa = a; *pb = b; ra = a; rb = b;
    }
};
template <> struct Storage<float> {
    template <int q> static LBM_HD constexpr float scale() { return 1.0f; }
    template <int q> static __device__ __forceinline__ float raw(const float* p) { return __ldg(p); }
    template <int q> static __device__ __forceinline__ float rawCoherent(const float* p) { return __ldcg(p); }
    template <int q> static __device__ __forceinline__ float storeOne(float* p, float v, uint32_t) { *p = v; return v; }
    template <int q> static __device__ __forceinline__ void storePair(float* pa, float* pb, float a, float b, uint32_t,
                                                                      float& ra, float& rb) {
        *pa = a; *pb = b; ra = a; rb = b;
    }
};
template <> struct Storage<__half> {
    template <int q> static LBM_HD constexpr float scale() { return loadFactorOf(q)*(1.0f/kHalfScale); }
    template <int q> static __device__ __forceinline__ float raw(const __half* p) { return __half2float(__ldg(p)); }
    template <int q> static __device__ __forceinline__ float storeOne(__half* p, float v, uint32_t dither) {
        uint32_t packed = stochasticHalf2(v*(kHalfScale*storeFactorOf(q)), 0.0f, dither);
        *reinterpret_cast<unsigned short*>(p) = (unsigned short) (packed & 0xFFFFu);
        return __half2float(__ushort_as_half((unsigned short) (packed & 0xFFFFu)));
    }
    template <int q> static __device__ __forceinline__ void storePair(__half* pa, __half* pb, float a, float b,
                                                                      uint32_t dither, float& ra, float& rb) {
        uint32_t packed = stochasticHalf2(a*(kHalfScale*storeFactorOf(q)), b*(kHalfScale*storeFactorOf(q)), dither);
        *reinterpret_cast<unsigned short*>(pa) = (unsigned short) (packed & 0xFFFFu);
        *reinterpret_cast<unsigned short*>(pb) = (unsigned short) (packed >> 16);
        __half2 h2 = *reinterpret_cast<__half2*>(&packed);
        float2 back = __half22float2(h2);
        ra = back.x;
        rb = back.y;
    }
};
template <> struct Storage<__nv_bfloat16> {
    template <int q> static LBM_HD constexpr float scale() { return loadFactorOf(q); }
    template <int q> static __device__ __forceinline__ float raw(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
    template <int q> static __device__ __forceinline__ float storeOne(__nv_bfloat16* p, float v, uint32_t dither) {
        uint32_t packed = stochasticBf162(v*storeFactorOf(q), 0.0f, dither);
        *reinterpret_cast<unsigned short*>(p) = (unsigned short) (packed & 0xFFFFu);
        return __uint_as_float(packed << 16);
    }
    template <int q> static __device__ __forceinline__ void storePair(__nv_bfloat16* pa, __nv_bfloat16* pb, float a, float b,
                                                                      uint32_t dither, float& ra, float& rb) {
        uint32_t packed = stochasticBf162(a*storeFactorOf(q), b*storeFactorOf(q), dither);
        *reinterpret_cast<unsigned short*>(pa) = (unsigned short) (packed & 0xFFFFu);
        *reinterpret_cast<unsigned short*>(pb) = (unsigned short) (packed >> 16);
        ra = __uint_as_float(packed << 16);
        rb = __uint_as_float(packed & 0xFFFF0000u);
    }
};

// Dither words of the stores of one node and step: the MurmurHash3 32-bit finaliser (Appleby) of the node and
// step mixed together; word k is that hash times an odd constant, a bijection of the hash, so each word is uniform
// when the hash is (one multiply per word).  Each word serves two stores (low and high halves).
struct Dither {
    uint32_t hash;
    static __device__ __forceinline__ uint32_t fmix32(uint32_t h) {
        h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
        return h;
    }
    __device__ __forceinline__ Dither(long long node, long long step) {
        hash = fmix32((uint32_t) node ^ fmix32((uint32_t) step + 0x9E3779B9u*(uint32_t) ((unsigned long long) node >> 32)));
    }
    template <int k> __device__ __forceinline__ uint32_t word() const {
        return hash*(0x9E3779B1u + 0x3C6EF372u*(uint32_t) k);
    }
};

// Runtime-q versions (slow paths: boundaries, state transfer), rounded to nearest.
template <typename T, typename R> __device__ __forceinline__ R loadq(const T* p, int q);
template <typename T, typename R> __device__ __forceinline__ void storeq(T* p, int q, R v);

template <> __device__ __forceinline__ double loadq<double, double>(const double* p, int) { return *p; }
template <> __device__ __forceinline__ float loadq<float, float>(const float* p, int) { return *p; }
template <> __device__ __forceinline__ float loadq<__half, float>(const __half* p, int q) {
    return __half2float(*p)*(loadFactorOf(q)*(1.0f/kHalfScale));
}
template <> __device__ __forceinline__ float loadq<__nv_bfloat16, float>(const __nv_bfloat16* p, int q) {
    return __bfloat162float(*p)*loadFactorOf(q);
}
template <> __device__ __forceinline__ void storeq<double, double>(double* p, int, double v) { *p = v; }
template <> __device__ __forceinline__ void storeq<float, float>(float* p, int, float v) { *p = v; }
template <> __device__ __forceinline__ void storeq<__half, float>(__half* p, int q, float v) {
    *p = __float2half_rn(v*(kHalfScale*storeFactorOf(q)));
}
template <> __device__ __forceinline__ void storeq<__nv_bfloat16, float>(__nv_bfloat16* p, int q, float v) {
    *p = __float2bfloat16_rn(v*storeFactorOf(q));
}

// ------------------------------------------------------------------------------------------------------
// Philox4x32 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11) with the
// published multipliers 0xD2511F53, 0xCD9E8D57 and Weyl increments 0x9E3779B9, 0xBB67AE85, and kPhiloxRounds = 7
// rounds: the smallest round count that the paper reports to pass the BigCrush battery (10 is its default, with a
// safety margin); the thermal noise of the fluid takes about half the instructions of the fluctuating dense step.
//
// Normal number m of (purpose, index, step): block b is Philox of the counter (index, step low, step high,
// purpose*256 + b) under the key (seed, 0x4C424D32); word k of the draw is lane k%4 of block k/4.  The normals come in
// Box-Muller pairs i = m/2, two pairs per three words: pair i takes the radius word w_a, a = 3(m/4) + i%2, with
// u = (w_a + 1/2) 2^-32 and r = sqrt(-2 ln u), and the 16-bit half h of word 3(m/4) + 2 (the low half for even i,
// the high half for odd i), with the angle t = 2 pi ((h + 1/2) 2^-16 - 1/2); normal m is r cos t (m even) or r sin t
// (m odd).  15 normals take 3 blocks, 19 take 4, 3 take 1.
// ------------------------------------------------------------------------------------------------------

enum { PurposeFluid = 0, PurposeBoundary = 1, PurposeParticle = 2 };

constexpr int kPhiloxRounds = 7;

template <int ROUNDS>
__device__ __forceinline__ uint4 philox4x32(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < ROUNDS; round++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u*c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u*c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint4 philoxBlock(uint32_t seed, int purpose, long long index, long long step, int block) {
    uint4 c = make_uint4((uint32_t) index, (uint32_t) step, (uint32_t) ((unsigned long long) step >> 32),
                         (uint32_t) (purpose*256 + block));
    return philox4x32<kPhiloxRounds>(c, seed, 0x4C424D32u);
}

// Square root by the hardware approximation (sqrt.approx.f32: one special-function instruction, relative error of
// order 2^-23) for the amplitudes of the thermal noise, where the IEEE-rounded sqrtf would take a multi-instruction
// sequence; x >= 0.
__device__ __forceinline__ float approxSqrt(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// The square root of a noise amplitude in the compute precision: the approximation in float, IEEE in double.
__device__ __forceinline__ float noiseSqrt(float x) { return approxSqrt(x); }
__device__ __forceinline__ double noiseSqrt(double x) { return sqrt(x); }

// One Box-Muller pair from a 32-bit radius word and a 16-bit angle half-word, in the compute precision.
__device__ __forceinline__ void boxMullerPair(uint32_t a, uint32_t h, float& n0, float& n1) {
    const float below1 = 0.99999994f;                   // 1 - 2^-24: keeps log(u) < 0 after rounding to float
    const float u = fminf(fmaf((float) a, 2.3283064365386963e-10f, 1.1641532182693481e-10f), below1);
    const float t = fmaf((float) h, 9.587379924285257e-05f, -3.1415447166901718f);   // 2 pi ((h + 1/2)/2^16 - 1/2)
#ifdef LBM_ACCURATE_FLOAT_NORMALS
    const float r = sqrtf(-2.0f*logf(u));
    float s, c;
    sincosf(t, &s, &c);
#else
    // Hardware approximations (MUFU): -2 ln u = -2 ln2 log2(u), and sin/cos of an angle in (-pi, pi), where their
    // absolute error is about 2^-21.
    const float r = approxSqrt(fmaxf(-1.3862943611198906f*__log2f(u), 0.0f));
    float s, c;
    __sincosf(t, &s, &c);
#endif
    n0 = r*c;
    n1 = r*s;
}
__device__ __forceinline__ void boxMullerPair(uint32_t a, uint32_t h, double& n0, double& n1) {
    const double u = ((double) a + 0.5)*2.3283064365386963e-10;
    const double v = ((double) h + 0.5)*1.52587890625e-05;
    const double r = sqrt(-2.0*log(u));
    double s, c;
    sincospi(2.0*v - 1.0, &s, &c);
    n0 = r*c;
    n1 = r*s;
}

// The first COUNT normals (COUNT <= 20) of (purpose, index, step).
template <typename R, int COUNT>
__device__ __forceinline__ void philoxNormals(uint32_t seed, int purpose, long long index, long long step, R* out) {
    constexpr int PAIRS = (COUNT + 1)/2, GROUPS = (PAIRS + 1)/2, BLOCKS = (3*GROUPS + 3)/4;
    uint32_t w[4*BLOCKS];
#pragma unroll
    for (int b = 0; b < BLOCKS; b++) {
        const uint4 x = philoxBlock(seed, purpose, index, step, b);
        w[4*b] = x.x; w[4*b+1] = x.y; w[4*b+2] = x.z; w[4*b+3] = x.w;
    }
#pragma unroll
    for (int i = 0; i < PAIRS; i++) {
        const uint32_t angles = w[3*(i/2) + 2];
        R n0, n1;
        boxMullerPair(w[3*(i/2) + i%2], (i%2) ? (angles >> 16) : (angles & 0xFFFFu), n0, n1);
        out[2*i] = n0;
        if (2*i + 1 < COUNT)
            out[2*i + 1] = n1;
    }
}

// ------------------------------------------------------------------------------------------------------
// Collision algebra.
// ------------------------------------------------------------------------------------------------------

// Value of the basis polynomial e_k at c_q (D3Q19.h:145-169), k = 4..18, as a compile-time constant.
LBM_HD constexpr double modeValue(int k, int q) {
    double x = cxOf(q), y = cyOf(q), z = czOf(q);
    double x2 = x*x, y2 = y*y, z2 = z*z;
    return k == 4 ? x2 - 1.0/3.0 : k == 5 ? y2 - 1.0/3.0 : k == 6 ? z2 - 1.0/3.0 : k == 7 ? x*y : k == 8 ? x*z :
           k == 9 ? y*z : k == 10 ? y*(x2 - 1.0/3.0) : k == 11 ? z*(x2 - 1.0/3.0) : k == 12 ? x*(y2 - 1.0/3.0) :
           k == 13 ? 0.5*x*(y2 + 2.0*z2 - 1.0) : k == 14 ? 0.5*y*(x2 + 2.0*z2 - 1.0) :
           k == 15 ? 0.5*z*(x2 + 2.0*y2 - 1.0) : k == 16 ? x2*y2 - x2/3.0 - y2/3.0 + z2/6.0 + 1.0/18.0 :
           k == 17 ? (2.0/7.0)*x2*y2 + x2*z2 - (3.0/7.0)*x2 + y2/14.0 - (2.0/7.0)*z2 + 1.0/14.0 :
           0.4*x2*y2 + 0.4*x2*z2 + y2*z2 - 0.1*x2 - 0.4*y2 - 0.4*z2 + 0.1;
}

// 1/sqrt(b_k) of the mode norms b_k (D3Q19.h:136-137), k = 4..18.
LBM_HD constexpr double invSqrtModeNorm(int k) {
    return k <= 6 ? 2.1213203435596424 : k <= 9 ? 3.0 : k <= 12 ? 3.6742346141747673 : k <= 15 ? 4.242640687119285 :
           k == 16 ? 4.810702354423639 : k == 17 ? 5.019960159204453 : 5.477225575051661;
}

// Random part xi_q of a collision (D3Q19::fluctuation, D3Q19.h:179-190) for the 15 normals r[0..14]:
// xi_q = w_q sum_k e_k(c_q) a_k with a_k = phi_k r_{k-4}/sqrt(b_k).
template <typename R, int q>
__device__ __forceinline__ R fluctuationTerm(const R a[15]) {
    R sum = 0;
#pragma unroll
    for (int k = 4; k < 19; k++) {
        const R e = R(modeValue(k, q));
        if (modeValue(k, q) != 0.0)
            sum += e*a[k-4];
    }
    return wOf<R>(q)*sum;
}

} // namespace lbm
