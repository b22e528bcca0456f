"""CPU tests of the reference's Python helpers (python/openmmlbm.i:513-800) as lbm_b200.reporters restates them,
driven by the CPU oracle's kernel: the temperature reporter (the full-step velocity with the explicit drag, the State's
velocity with the centred one), and the VTK reporter's files, read back against getFluidFields() and the State."""
import io
import os

import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce
from lbm_b200.reporters import KB, read_vtk_arrays
from cases import coupling_case
from oracle import OracleKernel


@pytest.mark.parametrize('drag', ['Explicit', 'Centered'])
def test_temperature_reporter(drag):
    context, force = coupling_case(True, drag, 'Trilinear', OracleKernel, temperature=300.0)
    simulation = lbm_b200.Simulation(context)
    out = io.StringIO()
    simulation.reporters.append(lbm_b200.LBMTemperatureReporter(out, 5, force))
    simulation.step(10)
    lines = out.getvalue().splitlines()
    assert lines[0].startswith('#"Step"') and len(lines) == 3
    step, time, temperature = lines[-1].split()
    assert int(step) == 10 and abs(float(time) - 0.1) < 1e-12
    v = context.velocities.copy()
    if drag == 'Explicit':
        v = v + context.getForces()*(0.5*0.01/100.0)
    expected = 0.5*100.0*(v**2).sum()*2/(3*4*KB)
    assert abs(float(temperature) - expected) <= 1e-3*max(1.0, expected)


def test_vtk_reporter_files_hold_the_fields(tmp_path):
    context, force = coupling_case(True, 'Explicit', 'Keys', OracleKernel, temperature=300.0)
    simulation = lbm_b200.Simulation(context)
    prefix = os.path.join(str(tmp_path), 'run')
    simulation.reporters.append(lbm_b200.LBMVTKReporter(prefix, 4, force, double=True))
    simulation.step(8)
    density, velocity = force.getFluidFields(context)
    blocks = read_vtk_arrays(prefix + '_density_8.vti')
    assert np.array_equal(np.frombuffer(blocks[0], '<f8'), density)
    solid = np.frombuffer(blocks[1], np.uint8)
    assert solid.sum() == len(force.getSolidNodes()) and solid[force.getSolidNodes()].all()
    blocks = read_vtk_arrays(prefix + '_velocity_8.vti')
    assert np.array_equal(np.frombuffer(blocks[0], '<f8').reshape(-1, 3), velocity)
    blocks = read_vtk_arrays(prefix + '_particles_8.vtp')
    positions = np.frombuffer(blocks[0], '<f8').reshape(-1, 3)
    box = context.system.box
    assert np.allclose(positions, context.positions - box*np.floor(context.positions/box), rtol=0, atol=1e-12)
    assert np.array_equal(np.frombuffer(blocks[1], '<f8').reshape(-1, 3), context.velocities)
    assert list(np.frombuffer(blocks[4], np.uint8)) == [1, 1, 1, 1]
    pvd = open(prefix + '.pvd').read()
    for step in (4, 8):
        for name in ('density', 'velocity'):
            assert 'file="run_%s_%d.vti"' % (name, step) in pvd
        assert 'file="run_particles_%d.vtp"' % step in pvd
    header = open(prefix + '_density_8.vti', 'rb').read(400).decode('ascii', 'replace')
    assert 'WholeExtent="0 7 0 7 0 7"' in header and 'Spacing="0.5 0.5 0.5"' in header
