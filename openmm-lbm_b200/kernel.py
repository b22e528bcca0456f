"""The B200 kernel behind the C ABI, as a Python object with the methods of the reference's platform kernel
interface CalcLBMForceKernel (openmmapi/include/LBMKernels.h:97-189).

Particle arrays are (n, 3) float64 numpy arrays in host memory (positions nm, velocities nm/ps, forces
kJ/mol/nm, coupled particles in coupling order), or, for device-resident runs, torch CUDA tensors of the
same shape, which are passed to the library as device pointers.
"""
import ctypes

import numpy as np

from .abi import (LbmOptions, LbmParticleArrays, MEMORY_DEVICE, MEMORY_HOST, STORAGE, check, dptr, load_library)


def _arrays(positions, velocities, forces):
    """LbmParticleArrays for numpy (host) or torch CUDA (device) arrays."""
    arrays = LbmParticleArrays()
    if positions is None:
        return None
    if isinstance(positions, np.ndarray):
        for a in (positions, velocities, forces):
            assert a.dtype == np.float64 and a.flags['C_CONTIGUOUS']
        arrays.positions = positions.ctypes.data
        arrays.velocities = velocities.ctypes.data
        arrays.forces = forces.ctypes.data
        arrays.memory = MEMORY_HOST
    else:
        for a in (positions, velocities, forces):
            assert a.is_cuda and a.is_contiguous() and str(a.dtype) == 'torch.float64'
        arrays.positions = positions.data_ptr()
        arrays.velocities = velocities.data_ptr()
        arrays.forces = forces.data_ptr()
        arrays.memory = MEMORY_DEVICE
    return arrays


class B200Kernel:
    """CalcLBMForceKernel on one B200 (the product path).

    lattice: LbmLatticeParameters; masses: masses (Da) of the coupled particles in coupling order;
    solid_nodes: indices of the solid nodes; precision: 'double', 'single', 'half' or 'bfloat16' storage of the
    populations; stream: an optional cudaStream_t (int) to launch on.
    """

    name = 'B200'
    # The platform whose CalcLBMForceKernel this kernel replaces, as checkpoints record it.
    platform_name = 'CUDA'

    def __init__(self, lattice, masses, solid_nodes, precision='single', device=0, stream=None):
        self.lib = load_library()
        self.lattice = lattice.copy()
        self.num_particles = len(masses)
        self.num_nodes = lattice.nx*lattice.ny*lattice.nz
        options = LbmOptions(STORAGE[precision], device, stream)
        masses = np.ascontiguousarray(masses, dtype=np.float64)
        solid = np.ascontiguousarray(solid_nodes, dtype=np.int32)
        handle = ctypes.c_void_p()
        check(self.lib.lbm_create(ctypes.byref(self.lattice), ctypes.byref(options), self.num_particles, dptr(masses),
                                  len(solid), solid.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  ctypes.byref(handle)), self.lib)
        self.handle = handle

    def close(self):
        if getattr(self, 'handle', None):
            self.lib.lbm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def stream(self):
        return self.lib.lbm_get_stream(self.handle)

    def begin_step(self, step, positions=None, velocities=None, forces=None):
        arrays = _arrays(positions, velocities, forces)
        check(self.lib.lbm_begin_step(self.handle, step, ctypes.byref(arrays) if arrays else None), self.lib)

    def execute(self, step, positions=None, velocities=None, forces=None, include_forces=True, include_energy=False):
        arrays = _arrays(positions, velocities, forces)
        energy = ctypes.c_double()
        check(self.lib.lbm_execute(self.handle, step, ctypes.byref(arrays) if arrays else None, int(include_forces),
                                   int(include_energy), ctypes.byref(energy)), self.lib)
        return energy.value

    def copy_parameters(self, lattice):
        self.lattice = lattice.copy()
        check(self.lib.lbm_copy_parameters(self.handle, ctypes.byref(self.lattice)), self.lib)

    def get_fluid_fields(self):
        density = np.zeros(self.num_nodes)
        velocity = np.zeros((self.num_nodes, 3))
        check(self.lib.lbm_get_fluid_fields(self.handle, dptr(density), dptr(velocity)), self.lib)
        return density, velocity

    def steady_residual(self, interval=100):
        """max|u - u_prev|/(interval max|u|) against the previous call (infinity on the first), FP64 on the device."""
        r = ctypes.c_double()
        check(self.lib.lbm_steady_residual(self.handle, int(interval), ctypes.byref(r)), self.lib)
        return r.value

    def solve_steady(self, first_step=0, interval=100, tolerance=1e-6, max_steps=10**6):
        """Steps until the steady residual is at most `tolerance`; returns (steps taken, last residual)."""
        steps, r = ctypes.c_longlong(), ctypes.c_double()
        check(self.lib.lbm_steady_solve(self.handle, int(first_step), int(interval), float(tolerance), int(max_steps),
                                        ctypes.byref(steps), ctypes.byref(r)), self.lib)
        return steps.value, r.value

    def set_fluid_equilibrium(self, density, velocity, strain=True):
        """The populations of the fields (units of get_fluid_fields): numpy arrays, or float64 torch CUDA tensors;
        the equilibrium plus, with strain, the non-equilibrium part of the velocity's strain rate."""
        if hasattr(density, 'data_ptr'):
            assert density.is_cuda and density.dtype.itemsize == 8 and density.is_contiguous()
            assert velocity.is_cuda and velocity.dtype.itemsize == 8 and velocity.is_contiguous()
            check(self.lib.lbm_set_fluid_equilibrium(self.handle, density.data_ptr(), velocity.data_ptr(), MEMORY_DEVICE,
                                                     int(strain)), self.lib)
            return
        density = np.ascontiguousarray(density, dtype=np.float64)
        velocity = np.ascontiguousarray(velocity, dtype=np.float64)
        if density.size != self.num_nodes or velocity.size != 3*self.num_nodes:
            raise ValueError('set_fluid_equilibrium: one density and three velocity components per node')
        check(self.lib.lbm_set_fluid_equilibrium(self.handle, density.ctypes.data, velocity.ctypes.data, MEMORY_HOST,
                                                 int(strain)), self.lib)

    def solver_iterations(self):
        """Conjugate-gradient iterations of the last centred stencil drag solve."""
        n = ctypes.c_int()
        check(self.lib.lbm_solver_iterations(self.handle, ctypes.byref(n)), self.lib)
        return n.value

    def set_solver_limits(self, max_iterations=0, barrier_polls=0):
        """Iteration cap and barrier poll limit of the centred stencil drag's solve (0 restores the default)."""
        check(self.lib.lbm_set_solver_limits(self.handle, int(max_iterations), int(barrier_polls)), self.lib)

    def solver_fallback_steps(self):
        """Steps whose centred stencil drag was solved by spread and gather on the nodes (capacity overflow)."""
        n = ctypes.c_longlong()
        check(self.lib.lbm_solver_fallback_steps(self.handle, ctypes.byref(n)), self.lib)
        return n.value

    def get_fluid_mach_number(self):
        mach = ctypes.c_double()
        check(self.lib.lbm_get_fluid_mach_number(self.handle, ctypes.byref(mach)), self.lib)
        return mach.value

    def get_wall_force(self):
        force = np.zeros(3)
        check(self.lib.lbm_get_wall_force(self.handle, dptr(force)), self.lib)
        return force

    def get_fluid_state(self):
        state = np.zeros(19*self.num_nodes)
        check(self.lib.lbm_get_fluid_state(self.handle, dptr(state)), self.lib)
        return state

    def set_fluid_state(self, state):
        state = np.ascontiguousarray(state, dtype=np.float64)
        if state.size != 19*self.num_nodes:
            raise ValueError('LBMForce: setFluidState() was called with a state of the wrong size')
        check(self.lib.lbm_set_fluid_state(self.handle, dptr(state)), self.lib)

    def create_checkpoint(self):
        size = ctypes.c_size_t()
        check(self.lib.lbm_checkpoint_size(self.handle, ctypes.byref(size)), self.lib)
        buffer = ctypes.create_string_buffer(size.value)
        check(self.lib.lbm_create_checkpoint(self.handle, buffer, size.value), self.lib)
        return buffer.raw

    def load_checkpoint(self, data):
        buffer = ctypes.create_string_buffer(data, len(data))
        check(self.lib.lbm_load_checkpoint(self.handle, buffer, len(data)), self.lib)

    def set_checkpoint_element_size(self, element_size):
        """The element size of the checkpoint stream: 8 as the reference's GPU platforms write it in double and mixed
        precision, 4 in single precision."""
        check(self.lib.lbm_set_checkpoint_element_size(self.handle, int(element_size)), self.lib)

    def checkpoint_layout(self):
        """(bytes of the reference's kernel stream, bytes of this kernel's trailer) of a checkpoint."""
        stream, trailer = ctypes.c_size_t(), ctypes.c_size_t()
        check(self.lib.lbm_checkpoint_layout(self.handle, ctypes.byref(stream), ctypes.byref(trailer)), self.lib)
        return stream.value, trailer.value
