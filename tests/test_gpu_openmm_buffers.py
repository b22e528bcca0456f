"""GPU tests of the OpenMM Context interface of the C ABI (lbm_set_coupled_atoms, lbm_begin_step_openmm,
lbm_execute_openmm): the kernel reads the coupled atoms from OpenMM CUDA-platform buffers -- posq (+ posqCorrection in
mixed precision) and velm in the platform's storage order, which is shuffled again before every call as OpenMM's atom
reordering would -- writes the reflected velocities back into velm and adds the coupling forces to the fixed-point
force buffer as (long long) (F 2^32), as the reference's CUDA kernels do (platforms/common/src/kernels/
lbmCoupling.cc:47-54, 148-171, 2043-2053).  The same run through the host-array entry points (lbm_begin_step,
lbm_execute) is the expectation: the same fluid (FP64 storage: bit for bit), the same velocities, and forces within the
fixed-point resolution."""
import ctypes

import numpy as np
import pytest
import torch

import lbm_b200
from lbm_b200 import LBMForce
from lbm_b200.abi import OPENMM_PRECISION, LbmOpenMMBuffers, check

pytestmark = pytest.mark.gpu

NUM_ATOMS, COUPLED = 7, [5, 1, 3, 6]
FIELD = np.array([3.0, -2.0, 1.0])


def lattice_case(drag, stencil):
    """4 coupled atoms of a System of 7 (mass 100) on an 8^3 lattice with the wall plane j = 0, friction 10/ps: the
    reference's coupling test case (TestLBMForce.py:573-635) with atoms that are not coupled around the coupled ones."""
    force = LBMForce()
    force.setGridSize(8, 8, 8)
    for atom in COUPLED:
        force.addParticle(atom)
    force.setDragScheme(getattr(LBMForce, drag))
    force.setInterpolationStencil(getattr(LBMForce, stencil))
    force.setFriction(10.0)
    force.setTemperature(0.0)
    force.setFluidMomentumRemovalFrequency(0)
    force.setSolidNodes([i + 64*k for k in range(8) for i in range(8)])
    masses = np.full(NUM_ATOMS, 100.0)
    lattice = force.latticeParameters(np.array([4.0, 4.0, 4.0]), 0.01, masses)
    return lattice, force.solid_nodes


def rounded(a, precision):
    return a.astype(np.float32).astype(np.float64) if precision == 'single' else a


@pytest.mark.parametrize('precision', ['double', 'mixed', 'single'])
@pytest.mark.parametrize('drag,stencil', [('Explicit', 'NearestNode'), ('Centered', 'Keys'),
                                          ('Centered', 'NearestNode'), ('Explicit', 'ThreePoint')])
def test_openmm_buffers_follow_host_arrays(drag, stencil, precision):
    lattice, solid = lattice_case(drag, stencil)
    masses = np.full(len(COUPLED), 100.0)
    host = lbm_b200.B200Kernel(lattice, masses, solid, 'double')
    dev = lbm_b200.B200Kernel(lattice, masses, solid, 'double')
    lib = dev.lib
    coupled = np.array(COUPLED, dtype=np.int32)
    check(lib.lbm_set_coupled_atoms(dev.handle, NUM_ATOMS, len(COUPLED),
                                    coupled.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), lib)
    rng = np.random.default_rng(5)
    pos = rng.uniform(0.2, 3.8, (NUM_ATOMS, 3))
    pos[COUPLED[2]] = (3.98, 0.52, 3.96)          # next to the wall plane: reflected
    vel = rng.normal(0.0, 1.0, (NUM_ATOMS, 3))
    vel[COUPLED[2]] = (2.0, -1.5, 1.0)
    padded = 32
    real = torch.float64 if precision == 'double' else torch.float32
    vreal = torch.float32 if precision == 'single' else torch.float64
    dt = 0.01
    for step in range(12):
        order = rng.permutation(NUM_ATOMS).astype(np.int32)          # atom stored at slot j
        pos, vel = rounded(pos, precision), rounded(vel, precision)
        posq = torch.zeros((NUM_ATOMS, 4), dtype=real)
        posq[:, :3] = torch.as_tensor(pos[order], dtype=real)
        correction = None
        if precision == 'mixed':
            correction = torch.zeros((NUM_ATOMS, 4), dtype=torch.float32)
            correction[:, :3] = torch.as_tensor(pos[order] - posq[:, :3].double().numpy(), dtype=torch.float32)
        velm = torch.zeros((NUM_ATOMS, 4), dtype=vreal)
        velm[:, :3] = torch.as_tensor(vel[order], dtype=vreal)
        velm[:, 3] = 1.0/100.0
        fixed = torch.zeros((3, padded), dtype=torch.int64)
        fixed[:, :NUM_ATOMS] = torch.as_tensor((np.tile(FIELD, (NUM_ATOMS, 1))[order]*2.0**32).T, dtype=torch.int64)
        # The positions the kernel reads: posq, plus posqCorrection (summed in double) in mixed precision.
        seen = posq[:, :3].double().numpy() + (correction[:, :3].double().numpy() if correction is not None else 0.0)
        pos[order] = seen
        w_in = velm[:, 3].double().numpy().copy()
        gpu = [t.cuda() if t is not None else None for t in (posq, correction, velm, fixed, torch.as_tensor(order))]
        buffers = LbmOpenMMBuffers(gpu[0].data_ptr(), gpu[1].data_ptr() if gpu[1] is not None else None,
                                   gpu[2].data_ptr(), gpu[3].data_ptr(), gpu[4].data_ptr(), NUM_ATOMS, padded,
                                   OPENMM_PRECISION[precision])
        # The host-array run on the same (already rounded) particles, in coupling order.
        p = np.ascontiguousarray(pos[COUPLED])
        v = np.ascontiguousarray(vel[COUPLED])
        f = np.ascontiguousarray(np.tile(FIELD, (len(COUPLED), 1)))
        host.begin_step(step, p, v, f)
        host.execute(step, p, v, f)
        check(lib.lbm_begin_step_openmm(dev.handle, step, ctypes.byref(buffers)), lib)
        check(lib.lbm_execute_openmm(dev.handle, step, ctypes.byref(buffers), 1, 0, None), lib)
        torch.cuda.synchronize()
        velm_out = gpu[2].cpu().double().numpy()
        force_out = gpu[3].cpu().numpy()[:, :NUM_ATOMS].T.astype(np.float64)/2.0**32
        slot = {int(a): j for j, a in enumerate(order)}
        for i, atom in enumerate(COUPLED):
            j = slot[atom]
            assert abs(velm_out[j, :3] - v[i]).max() <= 1e-6*max(1.0, abs(v[i]).max()), (step, atom)
            assert velm_out[j, 3] == w_in[j]
            # (long long) (F 2^32) truncates: the sum of the field and the coupling force within 2 units of 2^-32.
            assert abs(force_out[j] - f[i]).max() <= 2.0**-31 + 1e-12*abs(f[i]).max(), (step, atom)
        for atom in set(range(NUM_ATOMS)) - set(COUPLED):
            assert (force_out[slot[atom]] == FIELD).all()
        # Both runs integrate the same forces (the host run's), so that they stay on one trajectory.
        vel[COUPLED] = v
        acc = np.tile(FIELD, (NUM_ATOMS, 1))
        acc[COUPLED] = f
        vel = vel + dt*acc/100.0
        pos = pos + dt*vel
    state_host, state_dev = host.get_fluid_state(), dev.get_fluid_state()
    host.close()
    dev.close()
    scale = abs(state_host).max()
    tol = 0.0 if precision == 'double' else 1e-12
    assert abs(state_dev - state_host).max() <= tol*scale
