"""TEST INFRASTRUCTURE: Python access to the two CPU oracles, with the kernel protocol of lbm_b200.B200Kernel.

    ReferenceKernel  the reference's own Reference-platform kernel (ReferenceCalcLBMForceKernel) compiled
                     unmodified from the reference sources against the OpenMM shim (oracle/_ref/libref_lbm.so,
                     `make -C oracle ref`, only where the reference sources are present).
    OracleKernel     the C restatement oracle/lbm_oracle.c (oracle/liblbm_oracle.so, `make -C oracle oracle`).

Only tests/, the smoke check and the CPU-baseline leg of bench.py use this module; the product never does.
The package lbm_b200 (openmm-lbm_b200/) must be imported first (for the ABI structures).
"""
import ctypes
import os

import numpy as np

from lbm_b200.abi import LbmLatticeParameters, LbmParticleArrays, MEMORY_HOST, check, dptr  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
REF_PATH = os.path.join(HERE, '_ref', 'libref_lbm.so')
ADAPTER_PATH = os.path.join(HERE, '_ref', 'libadapter_lbm.so')
ORACLE_PATH = os.path.join(HERE, 'liblbm_oracle.so')

RANDOM_SEQUENTIAL, RANDOM_PHILOX = 0, 1

_libs = {}


class _Lib:
    def __init__(self, path, prefix):
        self.cdll = ctypes.CDLL(path)
        self.prefix = prefix
        P, D, I = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        LP = ctypes.POINTER(LbmLatticeParameters)
        PA = ctypes.POINTER(LbmParticleArrays)
        sig = {
            'last_error': (ctypes.c_char_p, []),
            'destroy': (None, [P]),
            'begin_step': (ctypes.c_int, [P, ctypes.c_longlong, PA]),
            'execute': (ctypes.c_int, [P, ctypes.c_longlong, PA, ctypes.c_int, ctypes.c_int, D]),
            'get_fluid_fields': (ctypes.c_int, [P, D, D]),
            'get_fluid_mach_number': (ctypes.c_int, [P, D]),
            'get_wall_force': (ctypes.c_int, [P, D]),
            'get_fluid_state': (ctypes.c_int, [P, D]),
            'set_fluid_state': (ctypes.c_int, [P, D]),
        }
        if prefix in ('refdrv_', 'adapterdrv_'):
            sig['create'] = (ctypes.c_int, [LP, ctypes.c_int, D, ctypes.c_int, I, ctypes.POINTER(P)])
            sig['create_with_storage'] = (ctypes.c_int, [LP, ctypes.c_int, D, ctypes.c_int, I, ctypes.c_int,
                                                         ctypes.POINTER(P)])
            sig['get_fluid_fields_halo'] = (ctypes.c_int, [P, D, D])
            sig['copy_parameters'] = (ctypes.c_int, [P, LP, ctypes.c_int, I])
            sig['create_checkpoint'] = (ctypes.c_int, [P, P, ctypes.POINTER(ctypes.c_size_t)])
            sig['load_checkpoint'] = (ctypes.c_int, [P, P, ctypes.c_size_t])
        else:
            sig['create'] = (ctypes.c_int, [LP, ctypes.c_int, ctypes.c_int, D, ctypes.c_int, I, ctypes.POINTER(P)])
            sig['copy_parameters'] = (ctypes.c_int, [P, LP])
            sig['philox4x32_10'] = (None, [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                           ctypes.POINTER(ctypes.c_uint32)])
            sig['philox_normal'] = (ctypes.c_double, [ctypes.c_uint32, ctypes.c_int, ctypes.c_longlong,
                                                      ctypes.c_longlong, ctypes.c_int])
            sig['axis_weights'] = (None, [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, I, D])
            sig['stencil_kernel'] = (ctypes.c_double, [ctypes.c_int, ctypes.c_double])
            sig['fluctuation'] = (None, [D, ctypes.c_double, ctypes.c_double, D])
            sig['find_boundaries'] = (ctypes.c_int, [LP, ctypes.c_int, I, I, I, I, I, I])
        for name, (restype, argtypes) in sig.items():
            fn = getattr(self.cdll, prefix + name)
            fn.restype = restype
            fn.argtypes = argtypes
            setattr(self, name, fn)

    def check(self, status):
        if status != 0:
            from lbm_b200.abi import LbmError
            raise LbmError(status, self.last_error().decode())


def library(kind):
    """'reference' (oracle/_ref), 'adapter' (the B200 platform kernel through the same driver) or 'oracle' (the C
    restatement)."""
    if kind not in _libs:
        path, prefix = {'reference': (REF_PATH, 'refdrv_'), 'adapter': (ADAPTER_PATH, 'adapterdrv_'),
                        'oracle': (ORACLE_PATH, 'oracle_')}[kind]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        _libs[kind] = _Lib(path, prefix)
    return _libs[kind]


def reference_available():
    return os.path.exists(REF_PATH)


def adapter_available():
    return os.path.exists(ADAPTER_PATH)


class _CpuKernel:
    """Common part of the two CPU kernels: host particle arrays, the kernel protocol of B200Kernel."""

    def __init__(self, lib, handle, lattice, num_particles):
        self.lib = lib
        self.handle = handle
        self.lattice = lattice.copy()
        self.num_particles = num_particles
        self.num_nodes = lattice.nx*lattice.ny*lattice.nz

    def close(self):
        if getattr(self, 'handle', None):
            self.lib.destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    @staticmethod
    def _arrays(p, v, f):
        if p is None:
            return None
        arrays = LbmParticleArrays()
        arrays.positions, arrays.velocities, arrays.forces = p.ctypes.data, v.ctypes.data, f.ctypes.data
        arrays.memory = MEMORY_HOST
        return arrays

    def begin_step(self, step, positions=None, velocities=None, forces=None):
        a = self._arrays(positions, velocities, forces)
        self.lib.check(self.lib.begin_step(self.handle, step, ctypes.byref(a) if a else None))

    def execute(self, step, positions=None, velocities=None, forces=None, include_forces=True, include_energy=False):
        a = self._arrays(positions, velocities, forces)
        e = ctypes.c_double()
        self.lib.check(self.lib.execute(self.handle, step, ctypes.byref(a) if a else None, int(include_forces),
                                        int(include_energy), ctypes.byref(e)))
        return e.value

    def get_fluid_fields(self):
        d = np.zeros(self.num_nodes)
        v = np.zeros((self.num_nodes, 3))
        self.lib.check(self.lib.get_fluid_fields(self.handle, dptr(d), dptr(v)))
        return d, v

    def get_fluid_mach_number(self):
        m = ctypes.c_double()
        self.lib.check(self.lib.get_fluid_mach_number(self.handle, ctypes.byref(m)))
        return m.value

    def get_wall_force(self):
        f = np.zeros(3)
        self.lib.check(self.lib.get_wall_force(self.handle, dptr(f)))
        return f

    def get_fluid_state(self):
        s = np.zeros(19*self.num_nodes)
        self.lib.check(self.lib.get_fluid_state(self.handle, dptr(s)))
        return s

    def set_fluid_state(self, state):
        s = np.ascontiguousarray(state, dtype=np.float64)
        if s.size != 19*self.num_nodes:
            raise ValueError('LBMForce: setFluidState() was called with a state of the wrong size')
        self.lib.check(self.lib.set_fluid_state(self.handle, dptr(s)))


class ReferenceKernel(_CpuKernel):
    """The reference's ReferenceCalcLBMForceKernel, compiled unmodified (oracle/_ref)."""

    name = 'Reference'

    def __init__(self, lattice, masses, solid_nodes):
        lib = library('reference')
        masses = np.ascontiguousarray(masses, dtype=np.float64)
        self.solid = np.ascontiguousarray(solid_nodes, dtype=np.int32)
        h = ctypes.c_void_p()
        lat = lattice.copy()
        lib.check(lib.create(ctypes.byref(lat), len(masses), dptr(masses), len(self.solid),
                             self.solid.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(h)))
        super().__init__(lib, h, lattice, len(masses))

    def copy_parameters(self, lattice):
        self.lattice = lattice.copy()
        self.lib.check(self.lib.copy_parameters(self.handle, ctypes.byref(self.lattice), len(self.solid),
                                                self.solid.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    def create_checkpoint(self):
        size = ctypes.c_size_t(0)
        self.lib.check(self.lib.create_checkpoint(self.handle, None, ctypes.byref(size)))
        buf = ctypes.create_string_buffer(size.value)
        self.lib.check(self.lib.create_checkpoint(self.handle, buf, ctypes.byref(size)))
        return buf.raw

    def load_checkpoint(self, data):
        buf = ctypes.create_string_buffer(data, len(data))
        self.lib.check(self.lib.load_checkpoint(self.handle, buf, len(data)))


class AdapterKernel(ReferenceKernel):
    """The project's B200 platform kernel (openmm-lbm_b200/openmm/B200LBMKernels.cpp, CalcLBMForceKernel over
    liblbm_b200.so), created by its kernel factory and driven through OpenMM's kernel interface by the same driver as
    the reference's kernel (oracle/_ref/libadapter_lbm.so; a GPU is needed).  storage: 'double', 'single', 'half' or
    'bfloat16'."""

    name = 'B200 adapter'

    def __init__(self, lattice, masses, solid_nodes, storage='double'):
        from lbm_b200.abi import STORAGE
        lib = library('adapter')
        masses = np.ascontiguousarray(masses, dtype=np.float64)
        self.solid = np.ascontiguousarray(solid_nodes, dtype=np.int32)
        h = ctypes.c_void_p()
        lat = lattice.copy()
        lib.check(lib.create_with_storage(ctypes.byref(lat), len(masses), dptr(masses), len(self.solid),
                                          self.solid.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), STORAGE[storage],
                                          ctypes.byref(h)))
        _CpuKernel.__init__(self, lib, h, lattice, len(masses))


def fields_with_halo(kernel):
    """getFluidFields() with the halo of a ReferenceKernel or AdapterKernel: density and velocity on the lattice
    extended by one node on every side, (nz + 2, ny + 2, nx + 2) and (nz + 2, ny + 2, nx + 2, 3)."""
    l = kernel.lattice
    shape = (l.nz + 2, l.ny + 2, l.nx + 2)
    d = np.zeros(shape)
    v = np.zeros(shape + (3,))
    kernel.lib.check(kernel.lib.get_fluid_fields_halo(kernel.handle, dptr(d), dptr(v)))
    return d, v


class OracleKernel(_CpuKernel):
    """The C restatement of the reference kernel (oracle/lbm_oracle.c); random='philox' uses the counter-based
    normals of the CUDA kernels, random='sequential' the stream of the shimmed reference."""

    name = 'Oracle'

    def __init__(self, lattice, masses, solid_nodes, random='philox'):
        lib = library('oracle')
        masses = np.ascontiguousarray(masses, dtype=np.float64)
        solid = np.ascontiguousarray(solid_nodes, dtype=np.int32)
        h = ctypes.c_void_p()
        lat = lattice.copy()
        mode = RANDOM_PHILOX if random == 'philox' else RANDOM_SEQUENTIAL
        lib.check(lib.create(ctypes.byref(lat), mode, len(masses), dptr(masses), len(solid),
                             solid.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(h)))
        super().__init__(lib, h, lattice, len(masses))

    def copy_parameters(self, lattice):
        self.lattice = lattice.copy()
        self.lib.check(self.lib.copy_parameters(self.handle, ctypes.byref(self.lattice)))


def philox4x32_10(counter, key):
    lib = library('oracle')
    c = (ctypes.c_uint32*4)(*counter)
    k = (ctypes.c_uint32*2)(*key)
    out = (ctypes.c_uint32*4)()
    lib.philox4x32_10(c, k, out)
    return list(out)


def philox_normal(seed, purpose, index, step, m):
    return library('oracle').philox_normal(seed, purpose, index, step, m)


def axis_weights(stencil, s, n, is_open):
    index = (ctypes.c_int*4)()
    weight = (ctypes.c_double*4)()
    library('oracle').axis_weights(stencil, s, n, int(is_open), index, weight)
    width = {0: 1, 1: 2, 2: 3, 3: 4}[stencil]
    return list(index)[:width], list(weight)[:width]


def stencil_kernel(stencil, r):
    return library('oracle').stencil_kernel(stencil, r)


def fluctuation(normals, stress, ghost):
    r = np.ascontiguousarray(normals, dtype=np.float64)
    xi = np.zeros(19)
    library('oracle').fluctuation(dptr(r), stress, ghost, dptr(xi))
    return xi


def md_forces(positions, box, bonds, k, r0, pair, sigma, eps, cutoff):
    """Bead forces on the CPU (oracle_md_forces): bonds and WCA ('wca') or Lennard-Jones ('lj') pairs."""
    lib = library('oracle')
    fn = lib.cdll.oracle_md_forces
    D = ctypes.POINTER(ctypes.c_double)
    fn.restype = None
    fn.argtypes = [ctypes.c_int, D, D, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_double, ctypes.c_double,
                   ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, D]
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    box = np.ascontiguousarray(box, dtype=np.float64)
    bonds = np.ascontiguousarray(np.asarray(bonds, dtype=np.int32).reshape(-1))
    forces = np.zeros_like(pos)
    fn(len(pos), dptr(pos), dptr(box), len(bonds)//2, bonds.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), k, r0,
       {'none': 0, 'wca': 1, 'lj': 2}[pair], sigma, eps, cutoff, dptr(forces))
    return forces


def find_boundaries(lattice, solid_nodes):
    lib = library('oracle')
    solid = np.ascontiguousarray(solid_nodes, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    lat = lattice.copy()
    count = lib.find_boundaries(ctypes.byref(lat), len(solid), solid.ctypes.data_as(ip), None, None, None, None, None)
    arrays = [np.zeros(max(count, 1), dtype=np.int32) for _ in range(5)]
    lib.find_boundaries(ctypes.byref(lat), len(solid), solid.ctypes.data_as(ip), *[a.ctypes.data_as(ip) for a in arrays])
    return [a[:count] for a in arrays]
