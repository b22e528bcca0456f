"""Bead dynamics on the device (include/lbm_b200_md.h) for torch CUDA tensors: the bond and pair forces and the
leapfrog integrator that OpenMM would provide around the LBM force kernel in the benchmark configurations."""
import ctypes

import numpy as np

from .abi import check, load_library

PAIR = {'none': 0, 'wca': 1, 'lj': 2}

_SIGNATURES = {
    'lbm_md_create': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                     ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]),
    'lbm_md_destroy': (None, [ctypes.c_void_p]),
    'lbm_md_compute_forces': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    'lbm_md_integrate': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    'lbm_md_kinetic': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                      ctypes.c_void_p]),
    'lbm_md_kernel_launches': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
}


def _lib():
    lib = load_library()
    if not getattr(lib, '_md_bound', False):
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        lib._md_bound = True
    return lib


class BeadDynamics:
    """Bonds (pairs of indices) with constant k and length r0, a pair force ('wca', 'lj' or 'none') with sigma,
    epsilon and cutoff, in a periodic box; positions, velocities and forces are (n, 3) float64 CUDA tensors."""

    def __init__(self, masses, box, bonds, k, r0, pair='wca', sigma=1.0, epsilon=1.0, cutoff=2.5, device=0):
        self.lib = _lib()
        masses = np.ascontiguousarray(masses, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64)
        bonds = np.ascontiguousarray(np.asarray(bonds, dtype=np.int32).reshape(-1))
        self.n = len(masses)
        handle = ctypes.c_void_p()
        dp = ctypes.POINTER(ctypes.c_double)
        check(self.lib.lbm_md_create(self.n, masses.ctypes.data_as(dp), box.ctypes.data_as(dp), len(bonds)//2,
                                     bonds.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), k, r0, PAIR[pair], sigma,
                                     epsilon, cutoff, device, ctypes.byref(handle)), self.lib)
        self.handle = handle

    def close(self):
        if getattr(self, 'handle', None):
            self.lib.lbm_md_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def compute_forces(self, positions, forces, stream=None):
        check(self.lib.lbm_md_compute_forces(self.handle, positions.data_ptr(), forces.data_ptr(), stream), self.lib)

    def integrate(self, dt, positions, velocities, forces, stream=None):
        check(self.lib.lbm_md_integrate(self.handle, dt, positions.data_ptr(), velocities.data_ptr(),
                                        forces.data_ptr(), stream), self.lib)

    def launches(self):
        out = ctypes.c_longlong()
        check(self.lib.lbm_md_kernel_launches(self.handle, ctypes.byref(out)), self.lib)
        return out.value

    def twice_kinetic(self, velocities, stream=None):
        out = ctypes.c_double()
        check(self.lib.lbm_md_kinetic(self.handle, velocities.data_ptr(), ctypes.byref(out), stream), self.lib)
        return out.value


def random_walk_chains(num_chains, length, box, seed, min_distance=0.8, step=1.0):
    """Seeded random-walk chains: unit steps in uniform directions, a step rejected (and drawn again) when it comes
    within min_distance of any earlier bead; chain starts uniform in the box.  Returns (positions (n,3), bonds)."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=float)
    ncell = np.maximum((box//max(min_distance, 1e-9)).astype(int), 1)
    cell = box/ncell                     # cells no smaller than min_distance, an integer number per axis
    grid = {}
    positions = []

    def key(p):
        w = np.mod(p, box)
        return tuple(np.minimum((w//cell).astype(int), ncell - 1))

    def clear(p):
        k = key(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    kk = ((k[0] + dx) % ncell[0], (k[1] + dy) % ncell[1], (k[2] + dz) % ncell[2])
                    for q in grid.get(kk, ()):
                        d = p - q
                        d -= box*np.round(d/box)
                        if d.dot(d) < min_distance*min_distance:
                            return False
        return True

    def add(p):
        positions.append(p)
        grid.setdefault(key(p), []).append(p)

    bonds = []
    for c in range(num_chains):
        # A bounded number of attempts: in a box too dense for the exclusion the last candidate is kept.
        for _ in range(1000):
            p = rng.uniform(0, 1, 3)*box
            if clear(p):
                break
        add(p)
        for b in range(1, length):
            for _ in range(1000):
                v = rng.normal(size=3)
                q = positions[-1] + step*v/np.linalg.norm(v)
                if clear(q):
                    break
            add(q)
            bonds.append((len(positions) - 2, len(positions) - 1))
    return np.array(positions), np.array(bonds, dtype=np.int32)
