// Collision algebra of the dense step, shared by the kernel of one lattice (fluid.cu) and the replica batch
// (batch.cu): the moments of the pulled populations, the regularized collision with Guo forcing and the Philox
// fluctuations of the non-conserved modes, after the reference's D3Q19 class (openmmapi/include/internal/D3Q19.h:
// equilibrium :55, regularized part :116, Guo forcing :127, fluctuation basis :136-190) and collideNode
// (platforms/reference/src/ReferenceLBMKernels.cpp:1066-1120).
#pragma once

#include "lbm_device.cuh"
#include <utility>

namespace lbm {
namespace {

template <typename F, int... I>
__device__ __forceinline__ void staticForImpl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void staticFor(F&& f) {
    staticForImpl(f, std::make_integer_sequence<int, N>{});
}

__device__ __forceinline__ double reciprocal(double x) { return 1.0/x; }
__device__ __forceinline__ float reciprocal(float x) { return __fdividef(1.0f, x); }

// Moments of 19 post-stream deviations: density deviation, momentum and non-equilibrium second moment
// Pi_neq = sum_q H2(c_q) df_q - j j/rho (xx, yy, zz, xy, xz, yz).  For the D3Q19 second-order
// equilibrium, sum_q H2(c_q) (feq_q - w_q) = j j/rho exactly, so this equals the reference's
// sum_q H2(c_q) (df_q - dfeq_q) (D3Q19.h:98-110).
template <typename R>
struct Moments {
    R dr, jx, jy, jz, pxx, pyy, pzz, pxy, pxz, pyz;
};

template <typename R>
__device__ __forceinline__ Moments<R> momentsOf(const R f[19]) {
    Moments<R> m;
    R dr = 0, jx = 0, jy = 0, jz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    staticFor<19>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
        R fq = f[q];
        dr += fq;
        if (cx == 1) jx += fq; else if (cx == -1) jx -= fq;
        if (cy == 1) jy += fq; else if (cy == -1) jy -= fq;
        if (cz == 1) jz += fq; else if (cz == -1) jz -= fq;
        if (cx != 0) sxx += fq;
        if (cy != 0) syy += fq;
        if (cz != 0) szz += fq;
        if (cx*cy == 1) sxy += fq; else if (cx*cy == -1) sxy -= fq;
        if (cx*cz == 1) sxz += fq; else if (cx*cz == -1) sxz -= fq;
        if (cy*cz == 1) syz += fq; else if (cy*cz == -1) syz -= fq;
    });
    R inv = R(1)/(R(1) + dr);
    R third = dr*R(1.0/3.0);
    m.dr = dr; m.jx = jx; m.jy = jy; m.jz = jz;
    m.pxx = sxx - third - jx*jx*inv;
    m.pyy = syy - third - jy*jy*inv;
    m.pzz = szz - third - jz*jz*inv;
    m.pxy = sxy - jx*jy*inv;
    m.pxz = sxz - jx*jz*inv;
    m.pyz = syz - jy*jz*inv;
    return m;
}

// Amplitudes a_k = phi_k r_k/sqrt(b_k) of the 15 non-conserved modes (D3Q19::fluctuation).
template <typename R>
__device__ __forceinline__ void modeAmplitudes(const R r[15], R stress, R ghost, R a[15]) {
#pragma unroll
    for (int k = 4; k < 19; k++)
        a[k-4] = r[k-4]*(k < 10 ? stress : ghost)*R(invSqrtModeNorm(k));
}

// Even and odd parts (in c_q) of xi_q = w_q sum_k e_k(c_q) a_k for one direction q.
template <typename R, int q>
__device__ __forceinline__ void fluctuationParts(const R a[15], R& even, R& odd) {
    R e = 0, o = 0;
    staticFor<15>([&](auto kc) {
        constexpr int k = decltype(kc)::value + 4;
        constexpr double m = modeValue(k, q);
        if (m != 0.0) {
            if (k >= 10 && k <= 15)
                o += R(m)*a[k-4];
            else
                e += R(m)*a[k-4];
        }
    });
    even = wOf<R>(q)*e;
    odd = wOf<R>(q)*o;
}

// Even and odd parts of the ghost-mode part (k = 10..18) of xi_q; the stress modes are merged into the
// non-equilibrium tensor of the dense kernel.
template <typename R, int q>
__device__ __forceinline__ void ghostParts(const R a[15], R& even, R& odd) {
    R e = 0, o = 0;
    staticFor<9>([&](auto kc) {
        constexpr int k = decltype(kc)::value + 10;
        constexpr double m = modeValue(k, q);
        if (m != 0.0) {
            if (k <= 15)
                o += R(m)*a[k-4];
            else
                e += R(m)*a[k-4];
        }
    });
    even = wOf<R>(q)*e;
    odd = wOf<R>(q)*o;
}

// Moments of the 19 pulled values r_q in storage units (deviation = scale_q r_q), summed over the opposite
// pairs (q, q+1): S = r_q + r_{q+1} feeds the even moments and D = r_q - r_{q+1} the momentum, with the
// scales folded into the FMAs.
template <typename T, typename R>
__device__ __forceinline__ Moments<R> momentsOfRaw(const R r[19]) {
    R dr = R(Storage<T>::template scale<0>())*r[0];
    R jx = 0, jy = 0, jz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    staticFor<9>([&](auto pc) {
        constexpr int q = 2*decltype(pc)::value + 1;
        constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
        constexpr R s = R(Storage<T>::template scale<q>());
        R S = r[q] + r[q+1], D = r[q] - r[q+1];
        dr += s*S;
        if (cx != 0) { jx += R(cx)*s*D; sxx += s*S; }
        if (cy != 0) { jy += R(cy)*s*D; syy += s*S; }
        if (cz != 0) { jz += R(cz)*s*D; szz += s*S; }
        if (cx*cy != 0) sxy += R(cx*cy)*s*S;
        if (cx*cz != 0) sxz += R(cx*cz)*s*S;
        if (cy*cz != 0) syz += R(cy*cz)*s*S;
    });
    Moments<R> m;
    R inv = reciprocal(R(1) + dr);
    R third = dr*R(1.0/3.0);
    m.dr = dr; m.jx = jx; m.jy = jy; m.jz = jz;
    m.pxx = sxx - third - jx*jx*inv;
    m.pyy = syy - third - jy*jy*inv;
    m.pzz = szz - third - jz*jz*inv;
    m.pxy = sxy - jx*jy*inv;
    m.pxz = sxz - jx*jz*inv;
    m.pyz = syz - jy*jz*inv;
    return m;
}


// Constants of the collision for one lattice, in the arithmetic type.
template <typename R>
struct CollideConstants {
    R om1, gx, gy, gz, ux0, uy0, uz0, mu, stressFactor;
    int remove;
    uint32_t seed;
};

template <typename R>
__device__ __forceinline__ CollideConstants<R> collideConstants(double omega, const double g[3], const double ucm[3],
                                                                int remove, double mu, uint32_t seed) {
    CollideConstants<R> k;
    R om = R(omega);
    k.om1 = R(1) - om;
    k.gx = R(g[0]); k.gy = R(g[1]); k.gz = R(g[2]);
    k.remove = remove;
    k.ux0 = remove ? R(ucm[0]) : R(0);
    k.uy0 = remove ? R(ucm[1]) : R(0);
    k.uz0 = remove ? R(ucm[2]) : R(0);
    k.mu = R(mu);
    k.stressFactor = om*(R(2) - om);
    k.seed = seed;
    return k;
}

// One fluid node of the dense step: pull streaming from the periodic neighbours in A, moments, momentum removal,
// regularized collision with Guo forcing (body force plus the extra force e, the particle reaction), Philox
// fluctuations when FLUCT, and the store into B.  Node indices are 32-bit; (x, y, z) are the node's coordinates in
// an nx x ny x nz lattice of N nodes.  The node's mass and momentum deviations after the collision are added to the
// sums: the collision conserves mass and gives the momentum j + F (the fluctuation modes carry neither), so they are
// dr and j + F, equal to the sums of the stored values up to the rounding of the stores.
// COHERENT: A was written by the same launch (a persistent kernel), so it is read through L2, not the read-only path.
template <typename T, typename R, bool FLUCT, bool COHERENT = false>
__device__ __forceinline__ void collideNode(const T* __restrict__ A, T* __restrict__ B, unsigned N, unsigned node,
                                            int x, int y, int z, int nx, int ny, int nz, const CollideConstants<R>& k,
                                            R ex, R ey, R ez, long long step, R& sumMass, R& sumX, R& sumY, R& sumZ) {
    constexpr bool dithered = sizeof(T) == 2;
    const unsigned sxy = (unsigned) nx*(unsigned) ny;
    // Offsets (mod 2^32) from the node to the pull sources x - c: index 0 for c = +1, 2 for c = -1.
    const unsigned ox[3] = {x == 0 ? (unsigned) (nx - 1) : ~0u, 0u, x == nx - 1 ? (unsigned) (1 - nx) : 1u};
    const unsigned oy[3] = {y == 0 ? (unsigned) (ny - 1)*nx : (unsigned) -nx, 0u,
                            y == ny - 1 ? (unsigned) (1 - ny)*nx : (unsigned) nx};
    const unsigned oz[3] = {z == 0 ? (unsigned) (nz - 1)*sxy : 0u - sxy, 0u, z == nz - 1 ? 0u - (unsigned) (nz - 1)*sxy : sxy};
    R r[19];
    staticFor<19>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
        const unsigned src = node + ox[1-cx] + oy[1-cy] + oz[1-cz];
        if constexpr (COHERENT)
            r[q] = Storage<T>::template rawCoherent<q>(A + ((size_t) q*N + src));
        else
            r[q] = Storage<T>::template raw<q>(A + ((size_t) q*N + src));
    });
    Moments<R> m = momentsOfRaw<T, R>(r);
    R rho = R(1) + m.dr, inv = reciprocal(rho);
    R jx = m.jx, jy = m.jy, jz = m.jz;
    if (k.remove) {
        jx -= rho*k.ux0;
        jy -= rho*k.uy0;
        jz -= rho*k.uz0;
    }
    R Fx = rho*k.gx + ex, Fy = rho*k.gy + ey, Fz = rho*k.gz + ez;
    R ux = (jx + R(0.5)*Fx)*inv, uy = (jy + R(0.5)*Fy)*inv, uz = (jz + R(0.5)*Fz)*inv;
    R uu = ux*ux + uy*uy + uz*uz, uf = ux*Fx + uy*Fy + uz*Fz;
    // The odd part 3 w_q (rho c.u + c.F/2) = 3 w_q c.(j + F) is built from the momentum after the force, not
    // through u = (j + F/2)/rho: a rounded rho*(1/rho) would scale the momentum by a fixed factor every step.
    const R px = jx + Fx, py = jy + Fy, pz = jz + Fz;
    // The regularized non-equilibrium part (1 - omega) 4.5 w_q H2(c_q):Pi_neq and the random stress modes
    // w_q sum_{k=4..9} e_k(c_q) a_k are both quadratic forms in c_q: they are merged into one tensor Q, so that
    // each direction evaluates w_q (c Q c - tr Q/3) once.  The ghost modes (k = 10..18) are added per direction.
    const R s45 = k.om1*R(4.5), s9 = k.om1*R(9);
    R qxx = s45*m.pxx, qyy = s45*m.pyy, qzz = s45*m.pzz;
    R qxy = s9*m.pxy, qxz = s9*m.pxz, qyz = s9*m.pyz;
    R a[15];
    if (FLUCT) {
        R rn[15];
        philoxNormals<R, 15>(k.seed, PurposeFluid, node, step, rn);
        R ghost = noiseSqrt(k.mu*rho);
        modeAmplitudes<R>(rn, noiseSqrt(k.mu*rho*k.stressFactor), ghost, a);
        qxx += a[0]; qyy += a[1]; qzz += a[2];
        qxy += a[3]; qxz += a[4]; qyz += a[5];
    }
    R qtr = (qxx + qyy + qzz)*R(1.0/3.0);
    // Terms common to all directions: dr - 1.5 rho u.u - 1.5 u.F.
    const R base = m.dr - R(1.5)*(rho*uu + uf);
    // Stochastic rounding of the 16-bit stores: one dither word per pair of directions.
    Dither dither(dithered ? node : 0, dithered ? step : 0);
    // q = 0
    {
        R value = R(1.0/3.0)*(base - qtr);
        if (FLUCT) {
            R e, o;
            ghostParts<R, 0>(a, e, o);
            value += e;
        }
        Storage<T>::template storeOne<0>(B + node, value, dithered ? dither.template word<0>() : 0u);
    }
    // Pairs (q, q+1) with c_{q+1} = -c_q.
    staticFor<9>([&](auto pc) {
        constexpr int q = 2*decltype(pc)::value + 1;
        constexpr int cx = cxOf(q), cy = cyOf(q), cz = czOf(q);
        constexpr R w = wOf<R>(q);
        R cu = R(cx)*ux + R(cy)*uy + R(cz)*uz;
        R cf = R(cx)*Fx + R(cy)*Fy + R(cz)*Fz;
        R cqc = R(cx*cx)*qxx + R(cy*cy)*qyy + R(cz*cz)*qzz - qtr
              + R(cx*cy)*qxy + R(cx*cz)*qxz + R(cy*cz)*qyz;
        R even = w*(base + cqc + R(4.5)*cu*(rho*cu + cf));
        R odd = oddOf<R>(q)*(R(cx)*px + R(cy)*py + R(cz)*pz);
        if (FLUCT) {
            R e, o;
            ghostParts<R, q>(a, e, o);
            even += e;
            odd += o;
        }
        R s1, s2;
        Storage<T>::template storePair<q>(B + ((size_t) q*N + node), B + ((size_t) (q+1)*N + node), even + odd,
                                          even - odd, dithered ? dither.template word<(q + 1)/2>() : 0u, s1, s2);
    });
    sumMass += m.dr;
    sumX += px;
    sumY += py;
    sumZ += pz;
}

} // namespace
} // namespace lbm
