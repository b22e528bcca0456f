"""The reference's Python helpers around LBMForce (python/openmmlbm.i:513-800), over the Context of lbm_b200.harness:
saveCheckpoint / loadCheckpoint, and the reporters LBMCheckpointReporter, LBMTemperatureReporter and LBMVTKReporter,
with OpenMM's reporter protocol (describeNextReport(simulation) -> {'steps', ...}; report(simulation, state)).

OpenMM is not part of this build, so Simulation (below) is the minimal driver that calls reporters as
openmm.app.Simulation does: after the steps that a reporter asked for, with a State of the Context.  Quantities are
plain floats in OpenMM's units (nm, ps, Da, kJ/mol, K).
"""
import os
import struct

import numpy as np

from . import checkpoint
from .force import LBMForce

# Boltzmann's constant in kJ/mol/K (OpenMM's MOLAR_GAS_CONSTANT_R).
KB = 6.02214076e23*1.380649e-23/1000.0

class State:
    """The State of a Context: step count, time (ps), positions (nm), velocities (nm/ps) and forces (kJ/mol/nm),
    (n, 3) arrays of all particles."""

    def __init__(self, context, forces=False):
        self.step = context.getStepCount()
        self.time = self.step*context.integrator.getStepSize()
        self.positions = context.positions.copy()
        self.velocities = context.velocities.copy()
        self.forces = context.getForces() if forces else None

    def getTime(self):
        return self.time

    def getPositions(self):
        return self.positions

    def getVelocities(self):
        return self.velocities

    def getForces(self):
        return self.forces


class Simulation:
    """A Context advanced by its integrator, with reporters called as openmm.app.Simulation calls them."""

    def __init__(self, context):
        self.context = context
        self.system = context.system
        self.integrator = context.integrator
        self.reporters = []

    @property
    def currentStep(self):
        return self.context.getStepCount()

    def step(self, steps):
        end = self.currentStep + steps
        while self.currentStep < end:
            nexts = [(r.describeNextReport(self), r) for r in self.reporters]
            advance = min([d['steps'] for d, _ in nexts] + [end - self.currentStep])
            self.integrator.step(advance)
            due = [(d, r) for d, r in nexts if d['steps'] == advance]
            if due:
                forces = any('forces' in d.get('include', []) for d, _ in due)
                state = State(self.context, forces=forces)
                for _, reporter in due:
                    reporter.report(self, state)


def saveCheckpoint(file, context, force):
    """Save the state of a Context with an LBMForce in the reference's file format for one domain
    (python/openmmlbm.i:513-550): the tag, the lengths, the Context's checkpoint (here the particles: step count,
    positions, velocities) and LBMForce.createCheckpoint() (the header and the kernel's stream), written to file +
    '.tmp' and then renamed, so that an interrupted write never replaces a valid checkpoint.  Like the reference's,
    the file is specific to the platform, the precision and the System."""
    data = checkpoint.pack_file(context.createCheckpoint(), force.createCheckpoint(context))
    temporary = file + '.tmp'
    with open(temporary, 'wb') as out:
        out.write(data)
    os.replace(temporary, file)


def loadCheckpoint(file, context, force):
    """Load a file written by saveCheckpoint() into a Context built from the same System (python/openmmlbm.i:553-586):
    the run continues exactly, bit for bit."""
    with open(file, 'rb') as stream:
        data = stream.read()
    openmm_data, force_data = checkpoint.unpack_file(data, file)
    context.loadCheckpoint(openmm_data)
    force.loadCheckpoint(context, force_data)


class LBMCheckpointReporter:
    """Saves a checkpoint of the run, fluid included, every reportInterval steps (python/openmmlbm.i:589-618)."""

    def __init__(self, file, reportInterval, force):
        self._file = file
        self._reportInterval = reportInterval
        self._force = force

    def describeNextReport(self, simulation):
        steps = self._reportInterval - simulation.currentStep%self._reportInterval
        return {'steps': steps, 'periodic': None, 'include': []}

    def report(self, simulation, state):
        saveCheckpoint(self._file, simulation.context, self._force)


class LBMTemperatureReporter:
    """Writes the temperature of the particles coupled to an LBMForce (python/openmmlbm.i:621-680), from the velocity
    that has the right temperature for the drag scheme: with the Explicit drag the full-step velocity v + dt F/(2m),
    with the Centered drag the velocity of the State.  Three degrees of freedom per coupled particle.  Each line: the
    step, the time (ps) and the temperature (K); the header only at the start of a file (a file opened for appending
    continues)."""

    def __init__(self, file, reportInterval, force):
        self._reportInterval = reportInterval
        self._force = force
        self._openedFile = isinstance(file, str)
        self._out = open(file, 'w') if self._openedFile else file
        self._particles = None

    def __del__(self):
        if getattr(self, '_openedFile', False):
            self._out.close()

    def describeNextReport(self, simulation):
        steps = self._reportInterval - simulation.currentStep%self._reportInterval
        include = ['velocities'] if self._force.getDragScheme() == LBMForce.Centered else ['velocities', 'forces']
        return {'steps': steps, 'periodic': None, 'include': include}

    def report(self, simulation, state):
        if self._particles is None:
            self._particles = np.array(self._force.particles, dtype=np.int64)
            self._masses = np.array([simulation.system.getParticleMass(int(i)) for i in self._particles])
            try:
                new = self._out.tell() == 0
            except (AttributeError, OSError, ValueError):
                new = True
            if new:
                print('#"Step","Time (ps)","Temperature (K)"', file=self._out)
        velocities = state.getVelocities()[self._particles]
        if self._force.getDragScheme() != LBMForce.Centered:
            forces = state.getForces()[self._particles]
            dt = simulation.integrator.getStepSize()
            velocities = velocities + forces*(0.5*dt/self._masses[:, None])
        energy = 0.5*np.sum(self._masses[:, None]*velocities**2)
        temperature = 2*energy/(3*len(self._particles)*KB)
        print('%d %.4f %.3f' % (simulation.currentStep, state.getTime(), temperature), file=self._out)
        self._out.flush()


def _vtk_units_field(lines):
    """VTK field data: the string array "units", one line per array (VTK writes ASCII strings as character codes,
    each string ended by 0)."""
    codes = ' '.join(' '.join(str(ord(c)) for c in line) + ' 0' for line in lines)
    return ('    <FieldData>\n      <DataArray type="String" Name="units" NumberOfTuples="%d" format="ascii">\n'
            '        %s\n      </DataArray>\n    </FieldData>\n' % (len(lines), codes))


def _write_vtk(path, kind, body, arrays):
    """A VTK XML file whose data arrays (numpy arrays, in the order of the {offsetN} fields of body) are appended
    raw, little endian, each after its UInt64 byte count."""
    blocks = [np.ascontiguousarray(a).astype(a.dtype.newbyteorder('<'), copy=False).tobytes() for a in arrays]
    offsets, offset = {}, 0
    for i, block in enumerate(blocks):
        offsets['offset%d' % i] = offset
        offset += 8 + len(block)
    head = ('<?xml version="1.0"?>\n<!-- lbm_b200.LBMVTKReporter, in OpenMM units: see the field data array "units" -->\n'
            '<VTKFile type="%s" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n' % kind +
            body.format(**offsets) + '  <AppendedData encoding="raw">\n_')
    with open(path, 'wb') as out:
        out.write(head.encode('ascii'))
        for block in blocks:
            out.write(struct.pack('<Q', len(block)))
            out.write(block)
        out.write(b'\n  </AppendedData>\n</VTKFile>\n')


class LBMVTKReporter:
    """Writes the fluid of an LBMForce and the particles in VTK XML files (python/openmmlbm.i:713-800), in OpenMM units,
    every reportInterval steps: <prefix>_density_<step>.vti and <prefix>_velocity_<step>.vti (ImageData, point
    (i, j, k) the node at (i dx, j dx, k dx); with solid nodes also "solid", 1 for a solid node), <prefix>_particles_
    <step>.vtp (PolyData: positions in nm, wrapped into the box unless wrap=False, "velocity", "mass", "index" and
    "coupled") and <prefix>.pvd, the list of the files with their times.  Single precision unless double=True.  The
    reporter does not change the run (getFluidFields neither advances the fluid nor draws random numbers)."""

    def __init__(self, prefix, reportInterval, force, fluid=True, particles=True, double=False, wrap=True,
                 append=False, density=True, velocity=True):
        self._prefix = prefix
        self._reportInterval = reportInterval
        self._force = force
        self._density = fluid and density
        self._velocity = fluid and velocity
        self._particles = particles
        self._double = double
        self._wrap = wrap
        self._datasets = []
        if append and os.path.exists(prefix + '.pvd'):
            with open(prefix + '.pvd') as pvd:
                self._datasets = [line for line in pvd if '<DataSet ' in line]

    def describeNextReport(self, simulation):
        steps = self._reportInterval - simulation.currentStep%self._reportInterval
        include = ['positions', 'velocities'] if self._particles else []
        return {'steps': steps, 'periodic': (self._wrap if self._particles else None), 'include': include}

    def report(self, simulation, state):
        real = np.float64 if self._double else np.float32
        name = 'Float64' if self._double else 'Float32'
        step, time = simulation.currentStep, state.getTime()
        nx, ny, nz = self._force.getGridSize()
        files = []
        solid = None
        if self._force.solid_nodes:
            solid = np.zeros(nx*ny*nz, dtype=np.uint8)
            solid[np.asarray(self._force.solid_nodes, dtype=np.int64)] = 1
        if self._density or self._velocity:
            density, velocity = self._force.getFluidFields(simulation.context)
            dx = simulation.context.lattice.dx
            extent = '0 %d 0 %d 0 %d' % (nx - 1, ny - 1, nz - 1)
            for field, data, components, unit in (('density', density, 1, 'Da/nm^3'),
                                                  ('velocity', velocity, 3, 'nm/ps')):
                if not (self._density if field == 'density' else self._velocity):
                    continue
                units = ['Origin, Spacing: nm', '%s: %s' % (field, unit)]
                arrays = [np.asarray(data, dtype=real).reshape(-1)]
                points = ('        <DataArray type="%s" Name="%s" NumberOfComponents="%d" format="appended" '
                          'offset="{offset0}"/>\n' % (name, field, components))
                if solid is not None:
                    units.append('solid: 1 for a solid node, 0 for a fluid node')
                    arrays.append(solid)
                    points += ('        <DataArray type="UInt8" Name="solid" format="appended" '
                               'offset="{offset1}"/>\n')
                body = ('  <ImageData WholeExtent="%s" Origin="0 0 0" Spacing="%.17g %.17g %.17g">\n' %
                        (extent, dx, dx, dx) + _vtk_units_field(units) +
                        '    <Piece Extent="%s">\n      <PointData Scalars="%s">\n' % (extent, field) + points +
                        '      </PointData>\n    </Piece>\n  </ImageData>\n')
                path = '%s_%s_%d.vti' % (self._prefix, field, step)
                _write_vtk(path, 'ImageData', body, arrays)
                files.append(path)
        if self._particles:
            positions = state.getPositions().copy()
            if self._wrap:
                box = simulation.system.box
                positions -= box*np.floor(positions/box)
            n = len(positions)
            coupled = np.zeros(n, dtype=np.uint8)
            coupled[np.asarray(self._force.particles, dtype=np.int64)] = 1
            masses = np.array(simulation.system.masses)
            arrays = [positions.astype(real).reshape(-1), state.getVelocities().astype(real).reshape(-1),
                      masses.astype(real), np.arange(n, dtype=np.int64), coupled,
                      np.arange(n, dtype=np.int64), np.arange(1, n + 1, dtype=np.int64)]
            units = ['Points: nm', 'velocity: nm/ps', 'mass: Da']
            body = ('  <PolyData>\n' + _vtk_units_field(units) +
                    '    <Piece NumberOfPoints="%d" NumberOfVerts="%d">\n' % (n, n) +
                    '      <Points>\n        <DataArray type="%s" NumberOfComponents="3" format="appended" '
                    'offset="{offset0}"/>\n      </Points>\n' % name +
                    '      <PointData>\n'
                    '        <DataArray type="%s" Name="velocity" NumberOfComponents="3" format="appended" '
                    'offset="{offset1}"/>\n' % name +
                    '        <DataArray type="%s" Name="mass" format="appended" offset="{offset2}"/>\n' % name +
                    '        <DataArray type="Int64" Name="index" format="appended" offset="{offset3}"/>\n'
                    '        <DataArray type="UInt8" Name="coupled" format="appended" offset="{offset4}"/>\n'
                    '      </PointData>\n      <Verts>\n'
                    '        <DataArray type="Int64" Name="connectivity" format="appended" offset="{offset5}"/>\n'
                    '        <DataArray type="Int64" Name="offsets" format="appended" offset="{offset6}"/>\n'
                    '      </Verts>\n    </Piece>\n  </PolyData>\n')
            path = '%s_particles_%d.vtp' % (self._prefix, step)
            _write_vtk(path, 'PolyData', body, arrays)
            files.append(path)
        for path in files:
            self._datasets.append('    <DataSet timestep="%.17g" part="0" file="%s"/>\n' % (time, os.path.basename(path)))
        with open(self._prefix + '.pvd', 'w') as pvd:
            pvd.write('<?xml version="1.0"?>\n<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">\n'
                      '  <Collection>\n' + ''.join(self._datasets) + '  </Collection>\n</VTKFile>\n')


def read_vtk_arrays(path):
    """The appended arrays of a file written by LBMVTKReporter, as raw bytes in order (for tests and tools)."""
    with open(path, 'rb') as stream:
        data = stream.read()
    start = data.index(b'<AppendedData encoding="raw">\n_') + len(b'<AppendedData encoding="raw">\n_')
    blocks = []
    while True:
        if data[start:start + 2] == b'\n ' or start >= len(data) - 8:
            break
        size, = struct.unpack_from('<Q', data, start)
        blocks.append(data[start + 8:start + 8 + size])
        start += 8 + size
    return blocks
