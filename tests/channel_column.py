"""TEST INFRASTRUCTURE: the precision channel (a Poiseuille channel between bounce-back planes z = 0 and z = nz - 1,
driven by the Guo body force g_x, started from rest) reduced to its column of nz nodes, with the arithmetic of the
paired FP32 dense kernel (streamCollidePairKernel, openmm-lbm_b200/csrc/fluid.cu) emulated operation by operation in
numpy, for any floating-point type.

The channel is homogeneous in x and y, so the populations of a plane z are the same at every (x, y) and the pull
streaming of the lattice moves them only along z: the column is the exact reduced system.  Every operation of the
kernel is rounded to the type: a fused multiply-add fma(a, b, c) is computed in float64 (a float32 product is exact
there) and rounded once.  The walls are the halfway bounce-back of the kernel's bounceBackKernel: the value a fluid
node pulls from a solid node is its own post-collision value of the opposite direction.  Storage types narrower than
the arithmetic are emulated with round-to-nearest (FP32) or with the kernel's unbiased stochastic rounding (FP16,
BF16: the upper or lower neighbour with probabilities proportional to the distances).

This shows what FP32 collide arithmetic alone gives on the 20,000 steps of the precision configuration, without the
GPU: the floor under every storage format whose collision computes in FP32."""
import numpy as np

# D3Q19 velocities in the kernel's order (openmm-lbm_b200/csrc/lbm_device.cuh cxOf/cyOf/czOf).
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1])
W = np.array([1/3] + [1/18]*6 + [1/36]*12)


def _fma(a, b, c, t):
    return (np.float64(a)*np.float64(b) + np.float64(c)).astype(t)


def _store16(v, fmt, rng):
    """Unbiased stochastic rounding of float32 values v to FP16 or BF16 (stored back as float32)."""
    v = np.asarray(v, dtype=np.float32)
    if fmt == 'bfloat16':
        bits = v.view(np.uint32).astype(np.uint64)
        lo = (bits & ~np.uint64(0xFFFF)).astype(np.uint32).view(np.float32)
        hi = ((bits & ~np.uint64(0xFFFF)) + np.uint64(0x10000)).astype(np.uint32).view(np.float32)
    else:
        lo = v.astype(np.float16)
        lo = np.where(lo.astype(np.float32) > v, np.nextafter(lo, np.float16(-np.inf)), lo)
        hi = np.nextafter(lo, np.float16(np.inf))
        lo, hi = lo.astype(np.float32), hi.astype(np.float32)
    # The two neighbours bracket v (for BF16 in the order of the magnitudes, so the span may be negative).
    span = hi.astype(np.float64) - lo.astype(np.float64)
    p = np.where(span != 0, (v.astype(np.float64) - lo)/np.where(span != 0, span, 1.0), 0.0)
    return np.where(rng.random(v.shape) < p, hi, lo).astype(np.float32)


def _two_sum(hi, lo, b, t):
    """hi + b rounded, and its exact rounding error added to lo (TwoSum, each operation rounded to t)."""
    s = (hi + b).astype(t)
    bb = (s - hi).astype(t)
    e = ((hi - (s - bb).astype(t)).astype(t) + (b - bb).astype(t)).astype(t)
    return s, (lo + e).astype(t)


def collide(r, t, gx, omega, compensated=True):
    """Post-collision populations (deviations, [19, nodes]) of the pulled populations r, the paired kernel's order;
    compensated: the momentum carried in two numbers (hi + lo) as the kernel does for FP32 storage (True: the momentum
    sums and j + F), or only j + F (the kernel's choice for 16-bit storage, 'p'), or neither (False)."""
    sums_compensated = compensated is True
    compensated = bool(compensated)
    one = t(1)
    dr = r[0].copy()
    jx = np.zeros_like(dr); jy = np.zeros_like(dr); jz = np.zeros_like(dr)
    jxl = np.zeros_like(dr); jyl = np.zeros_like(dr); jzl = np.zeros_like(dr)
    sxx = np.zeros_like(dr); syy = np.zeros_like(dr); szz = np.zeros_like(dr)
    sxy = np.zeros_like(dr); sxz = np.zeros_like(dr); syz = np.zeros_like(dr)
    for q in range(1, 19, 2):
        S = (r[q] + r[q+1]).astype(t)
        D = (r[q] - r[q+1]).astype(t)
        dr = _fma(one, S, dr, t)
        if CX[q]:
            if sums_compensated:
                jx, jxl = _two_sum(jx, jxl, (t(CX[q])*D).astype(t), t)
            else:
                jx = _fma(t(CX[q]), D, jx, t)
            sxx = _fma(one, S, sxx, t)
        if CY[q]:
            if sums_compensated:
                jy, jyl = _two_sum(jy, jyl, (t(CY[q])*D).astype(t), t)
            else:
                jy = _fma(t(CY[q]), D, jy, t)
            syy = _fma(one, S, syy, t)
        if CZ[q]:
            if sums_compensated:
                jz, jzl = _two_sum(jz, jzl, (t(CZ[q])*D).astype(t), t)
            else:
                jz = _fma(t(CZ[q]), D, jz, t)
            szz = _fma(one, S, szz, t)
        if CX[q]*CY[q]:
            sxy = _fma(t(CX[q]*CY[q]), S, sxy, t)
        if CX[q]*CZ[q]:
            sxz = _fma(t(CX[q]*CZ[q]), S, sxz, t)
        if CY[q]*CZ[q]:
            syz = _fma(t(CY[q]*CZ[q]), S, syz, t)
    rho = (dr + one).astype(t)
    inv = (one/rho).astype(t)
    ninv = -inv
    dr3 = (dr*t(-1.0/3.0)).astype(t)
    jxi, jyi = (jx*ninv).astype(t), (jy*ninv).astype(t)
    pxx = _fma(jx, jxi, (sxx + dr3).astype(t), t)
    pyy = _fma(jy, jyi, (syy + dr3).astype(t), t)
    pzz = _fma(jz, (jz*ninv).astype(t), (szz + dr3).astype(t), t)
    pxy, pxz, pyz = _fma(jy, jxi, sxy, t), _fma(jz, jxi, sxz, t), _fma(jz, jyi, syz, t)
    Fx = (rho*t(gx)).astype(t)
    Fy = np.zeros_like(Fx)
    Fz = np.zeros_like(Fx)
    ux = (_fma(Fx, t(0.5), jx, t)*inv).astype(t)
    uy = (_fma(Fy, t(0.5), jy, t)*inv).astype(t)
    uz = (_fma(Fz, t(0.5), jz, t)*inv).astype(t)
    uu = _fma(uz, uz, _fma(uy, uy, (ux*ux).astype(t), t), t)
    uf = _fma(uz, Fz, _fma(uy, Fy, (ux*Fx).astype(t), t), t)
    if compensated:
        (px, pxl), (py, pyl), (pz, pzl) = _two_sum(jx, jxl, Fx, t), _two_sum(jy, jyl, Fy, t), _two_sum(jz, jzl, Fz, t)
    else:
        px, py, pz = (jx + Fx).astype(t), (jy + Fy).astype(t), (jz + Fz).astype(t)
        pxl = pyl = pzl = None
    om1 = t(1) - t(omega)
    s45, s9 = t(om1*t(4.5)), t(om1*t(9))
    qxx, qyy, qzz = (s45*pxx).astype(t), (s45*pyy).astype(t), (s45*pzz).astype(t)
    qxy, qxz, qyz = (s9*pxy).astype(t), (s9*pxz).astype(t), (s9*pyz).astype(t)
    qtr = (((qxx + qyy).astype(t) + qzz).astype(t)*t(1.0/3.0)).astype(t)
    base = _fma(_fma(rho, uu, uf, t), t(-1.5), dr, t)
    rho2 = (rho + rho).astype(t)
    base1 = (base - qtr).astype(t)
    Ex = (base1 + _fma((ux*_fma(rho, ux, Fx, t)).astype(t), t(4.5), qxx, t)).astype(t)
    Pyy = _fma((uy*_fma(rho, uy, Fy, t)).astype(t), t(4.5), qyy, t)
    Pzz = _fma((uz*_fma(rho, uz, Fz, t)).astype(t), t(4.5), qzz, t)
    Ey, Ez = (base1 + Pyy).astype(t), (base1 + Pzz).astype(t)
    Pxy = _fma(_fma(ux, _fma(rho2, uy, Fy, t), (uy*Fx).astype(t), t), t(4.5), qxy, t)
    Pxz = _fma(_fma(ux, _fma(rho2, uz, Fz, t), (uz*Fx).astype(t), t), t(4.5), qxz, t)
    Pyz = _fma(_fma(uy, _fma(rho2, uz, Fz, t), (uz*Fy).astype(t), t), t(4.5), qyz, t)
    Sxy, Sxz, Syz = (Ex + Pyy).astype(t), (Ex + Pzz).astype(t), (Ey + Pzz).astype(t)
    out = np.empty_like(r)
    out[0] = ((base - qtr).astype(t)*t(1.0/3.0)).astype(t)
    odd_diag = t(1.0/12.0)
    odd_axis = t(t(0.5) - t(4)*odd_diag)
    for q in range(1, 19, 2):
        cx, cy, cz = CX[q], CY[q], CZ[q]
        if cy == 0 and cz == 0:
            even_raw = Ex
        elif cx == 0 and cz == 0:
            even_raw = Ey
        elif cx == 0 and cy == 0:
            even_raw = Ez
        elif cz == 0:
            even_raw = (Sxy + Pxy if cx*cy > 0 else Sxy - Pxy).astype(t)
        elif cy == 0:
            even_raw = (Sxz + Pxz if cx*cz > 0 else Sxz - Pxz).astype(t)
        else:
            even_raw = (Syz + Pyz if cy*cz > 0 else Syz - Pyz).astype(t)
        ko = odd_axis if q <= 6 else odd_diag
        terms = [(p, c) for p, c in ((px, cx), (py, cy), (pz, cz)) if c != 0]
        if compensated:
            terms = [(p, c) for p, c in ((pxl, cx), (pyl, cy), (pzl, cz)) if c != 0] + terms
        odd = (terms[0][0]*t(terms[0][1]*ko)).astype(t)
        for p, c in terms[1:]:
            odd = _fma(p, t(c*ko), odd, t)
        even = (even_raw*t(W[q])).astype(t)
        out[q] = (even + odd).astype(t)
        out[q+1] = (even - odd).astype(t)
    return out


def run(nz=192, steps=20000, arithmetic=np.float32, storage=None, tau=0.55, gx=5e-7, seed=1, compensated=None):
    """The column after `steps` steps from rest; returns u_x(z) = (j_x + F_x/2)/rho in float64 at every node (0 at the
    solid planes).  storage: None (the arithmetic type) or 'half' / 'bfloat16' (stochastic rounding of the stores);
    compensated: the kernel's two-number momentum (see collide); None: the kernel's choice for the storage (True for
    FP32, 'p' for 16-bit storage)."""
    if compensated is None:
        compensated = True if storage is None else 'p'
    t = arithmetic
    rng = np.random.default_rng(seed)
    f = np.zeros((19, nz), dtype=t)          # post-collision deviations, pull layout: f[q][z] produced at z
    fluid = slice(1, nz - 1)
    opp = np.array([0] + [q + 1 if q % 2 else q - 1 for q in range(1, 19)])
    omega = 1.0/tau
    for _ in range(steps):
        r = np.empty((19, nz - 2), dtype=t)
        z = np.arange(1, nz - 1)
        for q in range(19):
            src = z - CZ[q]
            pulled = f[q, src]
            solid = (src == 0) | (src == nz - 1)
            # halfway bounce-back: from a solid node the node gets back its own value of the opposite direction
            r[q] = np.where(solid, f[opp[q], z], pulled)
        out = collide(r, t, gx, omega, compensated)
        if storage is not None:
            out = _store16(out, storage, rng)
        f[:, fluid] = out
    rho = 1.0 + f[:, fluid].astype(np.float64).sum(axis=0)
    jx = (CX[:, None]*f[:, fluid].astype(np.float64)).sum(axis=0)
    u = np.zeros(nz)
    u[fluid] = (jx + 0.5*gx*rho)/rho
    return u
