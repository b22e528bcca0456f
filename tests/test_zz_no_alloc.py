"""GPU test of lbm_fluid_moments_noalloc, the entry point for callers that cannot allocate device memory (a plugin
whose host program owns the device memory through its own allocator, or a time-critical loop that cannot take the
synchronization of cudaMalloc/cudaFree).  It keeps its partial sums in a fixed device array of the library instead
of allocated scratch.

Its results are checked, through the C ABI, against those of the existing entry points on the same fluid: the Mach
number of lbm_get_fluid_mach_number and the mass and momentum of the state of lbm_get_fluid_state, on two calls in a
row (two lattices of different size, so the second call cannot pass on what the first left in the shared array).
The file is named to be collected last; it passes alone in a fresh process as well."""
import ctypes

import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from lbm_b200.abi import LBM_ERR_INVALID_ARGUMENT, load_library
from cases import FLUID_DX, FLUID_DT, fluid_system, make_context, total_moments, wall_plane

pytestmark = pytest.mark.gpu


def fluid(nx, ny, nz, steps):
    system, force = fluid_system(nx, ny, nz, 0.7)
    force.setSolidNodes(wall_plane(nx, ny, nz))
    force.setInitialFluidVelocity(np.array([0.03, -0.01, 0.02])*(FLUID_DX/FLUID_DT))
    force.setBodyAcceleration(np.array([2e-4, 1e-4, 0.0])*(FLUID_DX/FLUID_DT**2))
    context = make_context(system, properties={'Precision': 'double'})
    context.integrator.step(steps)
    return context, force


def noalloc_moments(state, is_fluid):
    import torch
    lib = load_library()
    s = torch.tensor(state, device='cuda', dtype=torch.float64)
    m = torch.tensor(is_fluid.astype(np.uint8), device='cuda')
    out = torch.full((5,), float('nan'), device='cuda', dtype=torch.float64)
    torch.cuda.synchronize()
    status = lib.lbm_fluid_moments_noalloc(s.data_ptr(), len(is_fluid), m.data_ptr(), out.data_ptr(), None)
    assert status == 0, lib.lbm_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_moments_match_existing_entry_points():
    # Two lattices of different size, in a row: 70,000 nodes (3 chunks), then 6x5x4.
    for nx, ny, nz, steps in ((50, 40, 35, 12), (6, 5, 4, 7)):
        context, force = fluid(nx, ny, nz, steps)
        state = force.getFluidState(context)
        mach = force.getFluidMachNumber(context)
        n = nx*ny*nz
        is_fluid = np.ones(n, dtype=bool)
        is_fluid[wall_plane(nx, ny, nz)] = False
        f = state.reshape(19, n)[:, is_fluid]
        mass, momentum = total_moments(f.reshape(-1))
        got = noalloc_moments(state, is_fluid)
        context.close()
        # FP64 state: the tolerance of the other double-precision parity tests.
        assert abs(got[4] - mach) <= 1e-12*mach
        assert abs(got[0] - (mass - is_fluid.sum())) <= 1e-12*n
        assert abs(got[1:4] - momentum).max() <= 1e-12*max(1.0, abs(momentum).max())


def test_noalloc_rejects_lattices_beyond_its_scratch():
    lib = load_library()
    status = lib.lbm_fluid_moments_noalloc(ctypes.c_void_p(16), 67108864 + 1, None, ctypes.c_void_p(16), None)
    assert status == LBM_ERR_INVALID_ARGUMENT
    assert 'fixed scratch array' in lib.lbm_last_error().decode()
