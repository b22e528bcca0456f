"""CPU tests of the host logic of the C ABI and of the library itself: the conversion into lattice units and its
checks (the reference's LBMForceImpl::computeLatticeParameters, openmmapi/src/LBMForceImpl.cpp:44-214), and the
exports of liblbm_b200.so against include/lbm_b200.h."""
import os
import re

import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from lbm_b200.abi import SIGNATURES, load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for header in sorted(os.listdir(os.path.join(ROOT, 'include'))):
        if header.endswith('.h'):
            text = open(os.path.join(ROOT, 'include', header)).read()
            names.update(re.findall(r'^\w[\w\s\*]*?\b(lbm_\w+)\s*\(', text, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from lbm_b200.md import _SIGNATURES as MD_SIGNATURES
    from lbm_b200.batch import _SIGNATURES as BATCH_SIGNATURES
    from lbm_b200.warmstart import _SIGNATURES as WARMSTART_SIGNATURES
    lib = load_library()
    names = declared_functions()
    assert len(names) >= 40
    for name in names:
        assert hasattr(lib, name), name
        assert (name in SIGNATURES or name in MD_SIGNATURES or name in BATCH_SIGNATURES
                or name in WARMSTART_SIGNATURES), name


def lattice_of(force, box=(3.0, 3.0, 3.0), dt=0.01, masses=(1.0,)):
    return force.latticeParameters(np.array(box), dt, np.array(masses))


def test_lattice_units():
    force = LBMForce()
    force.setGridSize(6, 6, 6)
    force.setKinematicViscosity(0.3/3*0.25/0.01)
    force.setBodyAcceleration((0.5, -0.2, 0.1))
    force.setInitialFluidVelocity((0.5, 0.2, -0.3))
    force.setFaceDensity(LBMForce.XMin, 0.0)
    lattice = lattice_of(force)
    assert lattice.dx == 0.5 and lattice.dt == 0.01
    assert abs(lattice.tau - 0.8) < 1e-14 and abs(lattice.omega - 1/0.8) < 1e-14
    assert abs(lattice.body_acceleration[0] - 0.5*0.01**2/0.5) < 1e-18
    assert abs(lattice.initial_velocity[2] + 0.3*0.01/0.5) < 1e-18
    assert abs(lattice.kT - 0.0083144626181532*300) < 1e-9
    assert lattice.fluid_kT == 0.0 and lattice.face_density[0] == 1.0
    assert lattice.momentum_removal_frequency == 1 and lattice.mach_check_frequency == 100


@pytest.mark.parametrize('setup,message', [
    (lambda f: f.setGridSize(0, 4, 4), 'grid size'),
    (lambda f: f.setKinematicViscosity(-1), 'viscosity'),
    (lambda f: f.setFriction(-1), 'friction'),
    (lambda f: f.setFaceBoundary(LBMForce.XMin, LBMForce.Velocity), 'both periodic or both open'),
    (lambda f: (f.setFaceBoundary(LBMForce.XMin, LBMForce.Velocity),
                f.setFaceBoundary(LBMForce.XMax, LBMForce.Velocity)), 'momentum cannot be removed'),
    (lambda f: (f.setFluidFluctuations(True), f.setFaceBoundary(LBMForce.ZMin, LBMForce.Density),
                f.setFaceBoundary(LBMForce.ZMax, LBMForce.Density), f.setFluidMomentumRemovalFrequency(0)),
     'Density faces cannot be used with fluid fluctuations'),
    (lambda f: f.setSolidNodes([1, 1]), 'more than once'),
    (lambda f: f.setSolidNodes([64]), 'out of range'),
    (lambda f: f.setSolidNodes(list(range(64))), 'all lattice nodes are solid'),
    (lambda f: f.setMachNumberLimit(0), 'Mach number limit'),
    (lambda f: f.addParticle(5), 'out of range'),
])
def test_lattice_checks(setup, message):
    force = LBMForce()
    force.setGridSize(4, 4, 4)
    setup(force)
    with pytest.raises(lbm_b200.LbmError) as error:
        lattice_of(force, box=(2.0, 2.0, 2.0))
    assert message in str(error.value)
    assert error.value.status == 1


def test_cells_must_be_cubic():
    force = LBMForce()
    force.setGridSize(4, 4, 4)
    with pytest.raises(lbm_b200.LbmError, match='cubic'):
        lattice_of(force, box=(2.0, 2.0, 2.5))


def test_kernel_calls_fail_cleanly_without_a_device():
    """Without a CUDA device the product path reports LBM_ERR_CUDA: there is no CPU fallback."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a device is present')
    force = LBMForce()
    force.setGridSize(4, 4, 4)
    with pytest.raises(lbm_b200.LbmError) as error:
        lbm_b200.B200Kernel(lattice_of(force, box=(2.0, 2.0, 2.0)), [], [])
    assert error.value.status == 5


def test_coupled_lattice_above_2_31_nodes_is_rejected():
    """The coupling keeps 32-bit signed node indices: lbm_create refuses a lattice of 2^31 nodes or more with coupled
    particles (before it touches a device), while the same lattice without particles passes that check."""
    import ctypes
    from lbm_b200.abi import LBM_ERR_INVALID_ARGUMENT, LbmOptions, STORAGE, dptr
    lib = load_library()
    force = LBMForce()
    force.setGridSize(8, 8, 8)
    lattice = lattice_of(force)
    lattice.nx, lattice.ny, lattice.nz = 1291, 1291, 1291          # 2.15e9 nodes
    options = LbmOptions(STORAGE['half'], 0, None)
    masses = np.ones(1)
    handle = ctypes.c_void_p()
    status = lib.lbm_create(ctypes.byref(lattice), ctypes.byref(options), 1, dptr(masses), 0, None,
                            ctypes.byref(handle))
    assert status == LBM_ERR_INVALID_ARGUMENT
    assert '2^31 - 1 nodes' in lib.lbm_last_error().decode()
    assert not handle.value
