// Device helpers of the B200 LBM kernels: the D3Q19 velocity set, storage conversion of the population
// deviations, the Philox4x32-10 counter-based generator and the collision algebra.
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

// ------------------------------------------------------------------------------------------------------
// Storage of the deviations f_q - w_q.  FP64 and FP32 store the deviation itself.  FP16 stores the
// deviation divided by w_q, which lifts the small deviations of the diagonal directions away from the
// subnormal range of binary16; BF16 stores the same scaled value.
// ------------------------------------------------------------------------------------------------------

template <typename T> struct Storage;
template <> struct Storage<double> {
    template <int q> static __device__ __forceinline__ double load(const double* p) { return __ldg(p); }
    template <int q> static __device__ __forceinline__ double store(double* p, double v) { *p = v; return v; }
    template <int q> static __device__ __forceinline__ double decode(double v) { return v; }
    template <int q> static __device__ __forceinline__ double encode(double v) { return v; }
};
template <> struct Storage<float> {
    template <int q> static __device__ __forceinline__ float load(const float* p) { return __ldg(p); }
    template <int q> static __device__ __forceinline__ float store(float* p, float v) { *p = v; return v; }
    template <int q> static __device__ __forceinline__ float decode(float v) { return v; }
    template <int q> static __device__ __forceinline__ float encode(float v) { return v; }
};
template <> struct Storage<__half> {
    template <int q> static __device__ __forceinline__ float decode(__half h) { return __half2float(h)*wOf<float>(q); }
    template <int q> static __device__ __forceinline__ __half encode(float v) { return __float2half_rn(v*(1.0f/wOf<float>(q))); }
    template <int q> static __device__ __forceinline__ float load(const __half* p) { return decode<q>(__ldg(p)); }
    // Returns the value actually stored, so that sums see what the next step reads.
    template <int q> static __device__ __forceinline__ float store(__half* p, float v) { __half h = encode<q>(v); *p = h; return decode<q>(h); }
};
template <> struct Storage<__nv_bfloat16> {
    template <int q> static __device__ __forceinline__ float decode(__nv_bfloat16 h) { return __bfloat162float(h)*wOf<float>(q); }
    template <int q> static __device__ __forceinline__ __nv_bfloat16 encode(float v) { return __float2bfloat16_rn(v*(1.0f/wOf<float>(q))); }
    template <int q> static __device__ __forceinline__ float load(const __nv_bfloat16* p) { return decode<q>(__ldg(p)); }
    template <int q> static __device__ __forceinline__ float store(__nv_bfloat16* p, float v) { __nv_bfloat16 h = encode<q>(v); *p = h; return decode<q>(h); }
};

// Runtime-q versions (slow paths: boundaries, state transfer).
template <typename T, typename R> __device__ __forceinline__ R loadq(const T* p, int q);
template <typename T, typename R> __device__ __forceinline__ void storeq(T* p, int q, R v);

template <> __device__ __forceinline__ double loadq<double, double>(const double* p, int) { return *p; }
template <> __device__ __forceinline__ float loadq<float, float>(const float* p, int) { return *p; }
template <> __device__ __forceinline__ float loadq<__half, float>(const __half* p, int q) {
    return __half2float(*p)*(q == 0 ? 1.0f/3.0f : (q <= 6 ? 1.0f/18.0f : 1.0f/36.0f));
}
template <> __device__ __forceinline__ float loadq<__nv_bfloat16, float>(const __nv_bfloat16* p, int q) {
    return __bfloat162float(*p)*(q == 0 ? 1.0f/3.0f : (q <= 6 ? 1.0f/18.0f : 1.0f/36.0f));
}
template <> __device__ __forceinline__ void storeq<double, double>(double* p, int, double v) { *p = v; }
template <> __device__ __forceinline__ void storeq<float, float>(float* p, int, float v) { *p = v; }
template <> __device__ __forceinline__ void storeq<__half, float>(__half* p, int q, float v) {
    *p = __float2half_rn(v*(q == 0 ? 3.0f : (q <= 6 ? 18.0f : 36.0f)));
}
template <> __device__ __forceinline__ void storeq<__nv_bfloat16, float>(__nv_bfloat16* p, int q, float v) {
    *p = __float2bfloat16_rn(v*(q == 0 ? 3.0f : (q <= 6 ? 18.0f : 36.0f)));
}

// ------------------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11),
// with the published multipliers 0xD2511F53, 0xCD9E8D57 and Weyl increments 0x9E3779B9, 0xBB67AE85.
// The normal number m of (purpose, index, step) comes from the counter (index, step low, step high,
// purpose*256 + m/4) and the key (seed, 0x4C424D32): lanes (0,1) and (2,3) of the output are Box-Muller
// pairs, u = (x + 1/2) 2^-32, r = sqrt(-2 ln u_a), normals r cos(2 pi (u_b - 1/2)) and r sin(2 pi (u_b - 1/2)).
// ------------------------------------------------------------------------------------------------------

enum { PurposeFluid = 0, PurposeBoundary = 1, PurposeParticle = 2 };

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; round++) {
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
    return philox4x32_10(c, seed, 0x4C424D32u);
}

// Four normals from one Philox block, in the compute precision R.  Angles are taken in (-pi, pi):
// normals r cos(2 pi (u_b - 1/2)) and r sin(2 pi (u_b - 1/2)).
__device__ __forceinline__ void boxMuller(uint4 x, float out[4]) {
    const float scale = 2.3283064365386963e-10f;        // 2^-32
    const float below1 = 0.99999994f;                   // 1 - 2^-24: keeps log(u) < 0 after rounding to float
    float ua = fminf(fmaf((float) x.x, scale, 0.5f*scale), below1), ub = fmaf((float) x.y, scale, 0.5f*scale);
    float uc = fminf(fmaf((float) x.z, scale, 0.5f*scale), below1), ud = fmaf((float) x.w, scale, 0.5f*scale);
#ifdef LBM_ACCURATE_FLOAT_NORMALS
    float r0 = sqrtf(-2.0f*logf(ua)), r1 = sqrtf(-2.0f*logf(uc));
    float s0, c0, s1, c1;
    sincospif(2.0f*ub - 1.0f, &s0, &c0);
    sincospif(2.0f*ud - 1.0f, &s1, &c1);
#else
    // Hardware approximations (MUFU): -2 ln u = -2 ln2 log2(u), and sin/cos of an angle in (-pi, pi), where their
    // absolute error is about 2^-21.
    float r0 = sqrtf(fmaxf(-1.3862943611198906f*__log2f(ua), 0.0f));
    float r1 = sqrtf(fmaxf(-1.3862943611198906f*__log2f(uc), 0.0f));
    float s0, c0, s1, c1;
    __sincosf(6.283185307179586f*(ub - 0.5f), &s0, &c0);
    __sincosf(6.283185307179586f*(ud - 0.5f), &s1, &c1);
#endif
    out[0] = r0*c0; out[1] = r0*s0; out[2] = r1*c1; out[3] = r1*s1;
}
__device__ __forceinline__ void boxMuller(uint4 x, double out[4]) {
    const double scale = 2.3283064365386963e-10;
    double ua = ((double) x.x + 0.5)*scale, ub = ((double) x.y + 0.5)*scale;
    double uc = ((double) x.z + 0.5)*scale, ud = ((double) x.w + 0.5)*scale;
    double r0 = sqrt(-2.0*log(ua)), r1 = sqrt(-2.0*log(uc));
    double s0, c0, s1, c1;
    sincospi(2.0*ub - 1.0, &s0, &c0);
    sincospi(2.0*ud - 1.0, &s1, &c1);
    out[0] = r0*c0; out[1] = r0*s0; out[2] = r1*c1; out[3] = r1*s1;
}

// The first `count` normals (count <= 20) of (purpose, index, step).
template <typename R, int COUNT>
__device__ __forceinline__ void philoxNormals(uint32_t seed, int purpose, long long index, long long step, R* out) {
#pragma unroll
    for (int b = 0; b < (COUNT + 3)/4; b++) {
        R v[4];
        boxMuller(philoxBlock(seed, purpose, index, step, b), v);
#pragma unroll
        for (int l = 0; l < 4; l++)
            if (4*b + l < COUNT)
                out[4*b + l] = v[l];
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
