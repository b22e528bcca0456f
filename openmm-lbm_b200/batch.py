"""Replica batches (include/lbm_b200_batch.h): many independent periodic lattices of uneven sizes, each with its own
coupled beads, advanced together on one device, every phase of a step one launch over all replicas and runs of steps
replayed from a CUDA graph.  Each replica follows the step of a B200Kernel with the same lattice parameters, driven
by the bead forces and a leapfrog with the lattice time step."""
import ctypes

import numpy as np

from .abi import LbmLatticeParameters, LbmOptions, STORAGE, check, load_library
from .md import PAIR


class LbmBatchPairForce(ctypes.Structure):
    _fields_ = [('pair_type', ctypes.c_int), ('sigma', ctypes.c_double), ('epsilon', ctypes.c_double),
                ('cutoff', ctypes.c_double)]


_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_SIGNATURES = {
    'lbm_batch_create': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(LbmLatticeParameters), ctypes.POINTER(ctypes.c_int),
                                        _D, _D, ctypes.POINTER(LbmBatchPairForce), ctypes.POINTER(LbmOptions),
                                        ctypes.POINTER(_P)]),
    'lbm_batch_destroy': (None, [_P]),
    'lbm_batch_step': (ctypes.c_int, [_P, ctypes.c_int]),
    'lbm_batch_autotune': (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _D]),
    'lbm_batch_get_particles': (ctypes.c_int, [_P, _D, _D]),
    'lbm_batch_set_velocities': (ctypes.c_int, [_P, _D]),
    'lbm_batch_get_fluid_state': (ctypes.c_int, [_P, ctypes.c_int, _D]),
    'lbm_batch_temperatures': (ctypes.c_int, [_P, _D, _D]),
    'lbm_batch_set_persistent': (ctypes.c_int, [_P, ctypes.c_int]),
    'lbm_batch_set_barrier_polls': (ctypes.c_int, [_P, ctypes.c_longlong]),
    'lbm_batch_info': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)]),
}


def _lib():
    lib = load_library()
    if not getattr(lib, '_batch_bound', False):
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        lib._batch_bound = True
    return lib


def _dp(a):
    return a.ctypes.data_as(_D)


class ReplicaBatch:
    """lattices: one LbmLatticeParameters per replica (LBMForce.latticeParameters); particles: the number of beads of
    each replica; masses (Da) and positions (nm, (n, 3)) of all beads, replica by replica; pair: ('lj' | 'wca' |
    'none', sigma, epsilon, cutoff); precision 'double' or 'single'."""

    def __init__(self, lattices, particles, masses, positions, pair=('none', 1.0, 1.0, 2.5), precision='single',
                 device=0, stream=None):
        self.lib = _lib()
        self.num_replicas = len(lattices)
        array = (LbmLatticeParameters*self.num_replicas)(*[l.copy() for l in lattices])
        self.particles = np.ascontiguousarray(particles, dtype=np.int32)
        self.offsets = np.concatenate([[0], np.cumsum(self.particles)])
        self.nodes = np.array([l.nx*l.ny*l.nz for l in lattices])
        masses = np.ascontiguousarray(masses, dtype=np.float64)
        positions = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        if len(masses) != self.offsets[-1] or len(positions) != self.offsets[-1]:
            raise ValueError('masses and positions must hold every bead of every replica')
        self.num_beads = int(self.offsets[-1])
        kind, sigma, epsilon, cutoff = pair
        force = LbmBatchPairForce(PAIR[kind], sigma, epsilon, cutoff)
        options = LbmOptions(STORAGE[precision], device, stream)
        handle = ctypes.c_void_p()
        check(self.lib.lbm_batch_create(self.num_replicas, array, self.particles.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                        _dp(masses), _dp(positions), ctypes.byref(force), ctypes.byref(options),
                                        ctypes.byref(handle)), self.lib)
        self.handle = handle

    def close(self):
        if getattr(self, 'handle', None):
            self.lib.lbm_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def step(self, steps):
        check(self.lib.lbm_batch_step(self.handle, int(steps)), self.lib)

    def autotune(self, graph_steps=0):
        """Returns (threads per block of the dense kernel, its time per launch in ms)."""
        threads, ms = ctypes.c_int(), ctypes.c_double()
        check(self.lib.lbm_batch_autotune(self.handle, int(graph_steps), ctypes.byref(threads), ctypes.byref(ms)),
              self.lib)
        return threads.value, ms.value

    def particles_state(self):
        pos = np.zeros((max(1, self.num_beads), 3))
        vel = np.zeros((max(1, self.num_beads), 3))
        check(self.lib.lbm_batch_get_particles(self.handle, _dp(pos), _dp(vel)), self.lib)
        return pos[:self.num_beads], vel[:self.num_beads]

    def set_velocities(self, velocities):
        v = np.ascontiguousarray(np.asarray(velocities, dtype=np.float64).reshape(-1, 3))
        check(self.lib.lbm_batch_set_velocities(self.handle, _dp(v)), self.lib)

    def fluid_state(self, replica):
        state = np.zeros(19*int(self.nodes[replica]))
        check(self.lib.lbm_batch_get_fluid_state(self.handle, int(replica), _dp(state)), self.lib)
        return state

    def temperatures(self):
        fluid = np.zeros(self.num_replicas)
        beads = np.zeros(self.num_replicas)
        check(self.lib.lbm_batch_temperatures(self.handle, _dp(fluid), _dp(beads)), self.lib)
        return fluid, beads

    def set_persistent(self, enable=True):
        """One persistent launch per graph_steps steps (True, the default) or the seven phase kernels of a step."""
        check(self.lib.lbm_batch_set_persistent(self.handle, int(enable)), self.lib)

    def set_barrier_polls(self, polls=0):
        """Poll limit of the persistent step's grid barriers (0: the default)."""
        check(self.lib.lbm_batch_set_barrier_polls(self.handle, int(polls)), self.lib)

    def info(self):
        nodes, steps, launches = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        threads, graph = ctypes.c_int(), ctypes.c_int()
        check(self.lib.lbm_batch_info(self.handle, ctypes.byref(nodes), ctypes.byref(steps), ctypes.byref(launches),
                                      ctypes.byref(threads), ctypes.byref(graph)), self.lib)
        return {'nodes': nodes.value, 'steps': steps.value, 'launches': launches.value, 'threads': threads.value,
                'graph_steps': graph.value}
