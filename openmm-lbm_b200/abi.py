"""ctypes mirror of the C ABI in include/lbm_b200.h, and the loader of liblbm_b200.so.

The structures have the field order of the header; the library is the product's CUDA build in this
folder.  Loading it needs no GPU: the entry points that need one fail with LBM_ERR_CUDA on a machine
without a device, and lbm_compute_lattice_parameters (host logic) works everywhere.
"""
import ctypes
import os

import numpy as np

LBM_OK = 0
LBM_ERR_INVALID_ARGUMENT = 1
LBM_ERR_MACH_LIMIT = 2
LBM_ERR_CG_NOT_CONVERGED = 3
LBM_ERR_DEVICE_TIMEOUT = 4
LBM_ERR_CUDA = 5
LBM_ERR_OUT_OF_MEMORY = 6
LBM_ERR_NOT_SUPPORTED = 7
LBM_ERR_CHECKPOINT = 8

STORAGE = {'double': 0, 'single': 1, 'half': 2, 'bfloat16': 3}
MEMORY_HOST, MEMORY_DEVICE = 0, 1


class LbmError(RuntimeError):
    """A failed call of the C ABI: `status` is the LbmStatus code and the message that of lbm_last_error()."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class LbmOpenMMBuffers(ctypes.Structure):
    """The particle buffers of an OpenMM CUDA-platform Context (device pointers)."""
    _fields_ = [('posq', ctypes.c_void_p), ('posq_correction', ctypes.c_void_p), ('velm', ctypes.c_void_p),
                ('force', ctypes.c_void_p), ('atom_index', ctypes.c_void_p), ('num_atoms', ctypes.c_int),
                ('padded_num_atoms', ctypes.c_int), ('precision', ctypes.c_int)]


OPENMM_PRECISION = {'single': 0, 'mixed': 1, 'double': 2}


class LbmLatticeParameters(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int), ('ny', ctypes.c_int), ('nz', ctypes.c_int),
                ('dx', ctypes.c_double), ('dt', ctypes.c_double), ('density', ctypes.c_double),
                ('tau', ctypes.c_double), ('omega', ctypes.c_double),
                ('initial_velocity', ctypes.c_double*3), ('body_acceleration', ctypes.c_double*3),
                ('friction', ctypes.c_double), ('kT', ctypes.c_double),
                ('drag_scheme', ctypes.c_int), ('interpolation_stencil', ctypes.c_int),
                ('fluid_fluctuations', ctypes.c_int), ('fluid_kT', ctypes.c_double),
                ('random_number_seed', ctypes.c_int), ('momentum_removal_frequency', ctypes.c_int),
                ('mach_check_frequency', ctypes.c_int), ('mach_number_limit', ctypes.c_double),
                ('wall_scheme', ctypes.c_int), ('face_boundary', ctypes.c_int*6),
                ('face_velocity', (ctypes.c_double*3)*6), ('face_density', ctypes.c_double*6)]

    def copy(self):
        other = LbmLatticeParameters()
        ctypes.memmove(ctypes.byref(other), ctypes.byref(self), ctypes.sizeof(self))
        return other


class LbmOptions(ctypes.Structure):
    _fields_ = [('storage', ctypes.c_int), ('device', ctypes.c_int), ('stream', ctypes.c_void_p)]


class LbmParticleArrays(ctypes.Structure):
    _fields_ = [('positions', ctypes.c_void_p), ('velocities', ctypes.c_void_p), ('forces', ctypes.c_void_p),
                ('memory', ctypes.c_int)]


class LbmForceDescription(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int), ('ny', ctypes.c_int), ('nz', ctypes.c_int),
                ('fluid_density', ctypes.c_double), ('kinematic_viscosity', ctypes.c_double),
                ('friction', ctypes.c_double), ('temperature', ctypes.c_double),
                ('coupling_scheme', ctypes.c_int), ('drag_scheme', ctypes.c_int),
                ('interpolation_stencil', ctypes.c_int), ('fluid_fluctuations', ctypes.c_int),
                ('wall_scheme', ctypes.c_int), ('face_boundary', ctypes.c_int*6),
                ('face_velocity', (ctypes.c_double*3)*6), ('face_density', ctypes.c_double*6),
                ('random_number_seed', ctypes.c_int), ('body_acceleration', ctypes.c_double*3),
                ('initial_velocity', ctypes.c_double*3), ('momentum_removal_frequency', ctypes.c_int),
                ('mach_check_frequency', ctypes.c_int), ('mach_number_limit', ctypes.c_double)]


# Every entry point that include/lbm_b200.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    'lbm_last_error': (ctypes.c_char_p, []),
    'lbm_default_force_description': (None, [ctypes.POINTER(LbmForceDescription)]),
    'lbm_compute_lattice_parameters': (ctypes.c_int, [ctypes.POINTER(LbmForceDescription), _D, ctypes.c_double,
                                                      ctypes.c_int, _D, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                      ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                      ctypes.POINTER(LbmLatticeParameters)]),
    'lbm_create': (ctypes.c_int, [ctypes.POINTER(LbmLatticeParameters), ctypes.POINTER(LbmOptions), ctypes.c_int, _D,
                                  ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_P)]),
    'lbm_destroy': (None, [_P]),
    'lbm_begin_step': (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(LbmParticleArrays)]),
    'lbm_execute': (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(LbmParticleArrays), ctypes.c_int,
                                   ctypes.c_int, _D]),
    'lbm_copy_parameters': (ctypes.c_int, [_P, ctypes.POINTER(LbmLatticeParameters)]),
    'lbm_get_fluid_fields': (ctypes.c_int, [_P, _D, _D]),
    'lbm_get_fluid_mach_number': (ctypes.c_int, [_P, _D]),
    'lbm_get_wall_force': (ctypes.c_int, [_P, _D]),
    'lbm_get_fluid_state': (ctypes.c_int, [_P, _D]),
    'lbm_set_fluid_state': (ctypes.c_int, [_P, _D]),
    'lbm_checkpoint_size': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_size_t)]),
    'lbm_create_checkpoint': (ctypes.c_int, [_P, _P, ctypes.c_size_t]),
    'lbm_load_checkpoint': (ctypes.c_int, [_P, _P, ctypes.c_size_t]),
    'lbm_set_checkpoint_element_size': (ctypes.c_int, [_P, ctypes.c_int]),
    'lbm_checkpoint_layout': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    'lbm_get_info': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]),
    'lbm_get_stream': (_P, [_P]),
    'lbm_profile_dense_kernel': (ctypes.c_int, [_P, ctypes.c_int]),
    'lbm_dense_kernel_time': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_longlong), _D]),
    'lbm_kernel_launches': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    'lbm_solver_iterations': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    'lbm_set_coupled_atoms': (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    'lbm_begin_step_openmm': (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(LbmOpenMMBuffers)]),
    'lbm_execute_openmm': (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(LbmOpenMMBuffers), ctypes.c_int,
                                          ctypes.c_int, _D]),
    'lbm_set_solver_limits': (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_longlong]),
    'lbm_solver_fallback_steps': (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    'lbm_steady_residual': (ctypes.c_int, [_P, ctypes.c_int, _D]),
    'lbm_steady_solve': (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.c_int, ctypes.c_double, ctypes.c_longlong,
                                        ctypes.POINTER(ctypes.c_longlong), _D]),
    'lbm_set_fluid_equilibrium': (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_int]),
    'lbm_fluid_moments_noalloc': (ctypes.c_int, [_P, ctypes.c_longlong, _P, _P, _P]),
}

# LBM_B200_LIBRARY selects another build of the library (for example one compiled with other kernel options).
LIBRARY_PATH = os.environ.get('LBM_B200_LIBRARY',
                              os.path.join(os.path.dirname(os.path.abspath(__file__)), 'liblbm_b200.so'))
_library = None


def load_library():
    """Load liblbm_b200.so (built by `make` in this folder, or by __graft_entry__.build()).

    Raises if the library is missing: there is no fallback implementation.
    """
    global _library
    if _library is None:
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError('liblbm_b200.so is not built: run make in %s' % os.path.dirname(LIBRARY_PATH))
        lib = ctypes.CDLL(LIBRARY_PATH)
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _library = lib
    return _library


def check(status, lib=None):
    if status != LBM_OK:
        lib = lib or load_library()
        raise LbmError(status, lib.lbm_last_error().decode())


def dptr(array):
    """Pointer to the data of a C-contiguous float64 numpy array."""
    assert array.dtype == np.float64 and array.flags['C_CONTIGUOUS']
    return array.ctypes.data_as(_D)
