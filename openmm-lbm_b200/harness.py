"""A minimal stand-in for the parts of OpenMM that drive the LBM force kernel: a System of particles with masses
and a rectangular periodic box, extra forces, and a Context advanced by OpenMM's leapfrog VerletIntegrator.

OpenMM is not part of this build.  The step follows OpenMM's order for a VerletIntegrator: the force's
updateContextState (the kernel's beginStep), then the force evaluation (every other force, then the LBM
kernel's execute, since LBMForce must come last), then v(t + dt/2) = v(t - dt/2) + dt F(t)/m and
x(t + dt) = x(t) + dt v(t + dt/2), then the step count is incremented.  A kernel factory selects the
implementation (the B200 kernel by default); the parity tests pass the oracle's.
"""
import struct

import numpy as np

from .force import LBMForce
from .kernel import B200Kernel


class System:
    """Particles (masses in Da) in a rectangular periodic box (nm) with a list of forces."""

    def __init__(self):
        self.masses = []
        self.box = np.zeros(3)
        self.forces = []

    def addParticle(self, mass):
        self.masses.append(float(mass))
        return len(self.masses) - 1

    def getNumParticles(self):
        return len(self.masses)

    def getParticleMass(self, index):
        return self.masses[index]

    def setDefaultPeriodicBoxVectors(self, a, b, c):
        if a[1] != 0 or a[2] != 0 or b[0] != 0 or b[2] != 0 or c[0] != 0 or c[1] != 0:
            raise ValueError('LBMForce: the periodic box must be rectangular')
        self.box = np.array([a[0], b[1], c[2]], dtype=np.float64)

    def addForce(self, force):
        self.forces.append(force)
        return len(self.forces) - 1


class ExternalForce:
    """A force on particles from a callable f(positions (n,3) nm) -> forces (n,3) kJ/mol/nm."""

    def __init__(self, function, particles=None):
        self.function = function
        self.particles = particles

    def compute(self, positions, box):
        forces = np.zeros_like(positions)
        idx = self.particles if self.particles is not None else np.arange(len(positions))
        forces[idx] = self.function(positions[idx])
        return forces


class PairForce:
    """A central pair force between all particles with minimum-image periodic distances: the force along r of
    magnitude -dU/dr for U(r) given by dudr(r), within a cutoff."""

    def __init__(self, dudr, cutoff):
        self.dudr = dudr
        self.cutoff = cutoff

    def compute(self, positions, box):
        n = len(positions)
        forces = np.zeros_like(positions)
        for i in range(n):
            d = positions[i] - positions[i+1:]
            d -= box*np.round(d/box)
            r = np.sqrt((d*d).sum(axis=1))
            mask = (r < self.cutoff) & (r > 0)
            if not mask.any():
                continue
            f = (-self.dudr(r[mask])/r[mask])[:, None]*d[mask]
            forces[i] += f.sum(axis=0)
            forces[i+1:][mask] -= f
        return forces


class VerletIntegrator:
    def __init__(self, step_size):
        self.step_size = float(step_size)
        self.context = None

    def getStepSize(self):
        return self.step_size

    def step(self, steps):
        for _ in range(steps):
            self.context._step()


class _Platform:
    def __init__(self, name):
        self.name = name

    def getName(self):
        return self.name


class Context:
    """A System integrated with a VerletIntegrator, whose LBMForce runs on a kernel from kernel_factory
    (lattice, coupled masses, solid nodes) -> kernel; the default is the B200 kernel with
    properties['Precision'] ('single', 'double', 'half', 'bfloat16')."""

    def __init__(self, system, integrator, kernel_factory=None, properties=None):
        self.system = system
        self.integrator = integrator
        integrator.context = self
        lbm = [f for f in system.forces if isinstance(f, LBMForce)]
        if len(lbm) != 1:
            raise ValueError('the System must contain one LBMForce')
        self.force = lbm[0]
        self.others = [f for f in system.forces if not isinstance(f, LBMForce)]
        if self.force.getDragScheme() == LBMForce.Centered and system.forces[-1] is not self.force:
            raise ValueError('LBMForce: with the Centered drag scheme LBMForce must be the last force of the System; '
                             'add it after all the other forces')
        n = system.getNumParticles()
        self.positions = np.zeros((n, 3))
        self.velocities = np.zeros((n, 3))
        self.masses = np.array(system.masses)
        self.step_count = 0
        self.coupled = np.array(self.force.particles, dtype=np.int64)
        self.lattice = self.force.latticeParameters(system.box, integrator.getStepSize(), self.masses)
        coupled_masses = self.masses[self.coupled] if len(self.coupled) else np.zeros(0)
        properties = properties or {}
        if kernel_factory is None:
            precision = properties.get('Precision', 'single')
            self.kernel = B200Kernel(self.lattice, coupled_masses, self.force.solid_nodes, precision)
        else:
            self.kernel = kernel_factory(self.lattice, coupled_masses, self.force.solid_nodes)

    def getPlatform(self):
        """The platform of the Context: the one whose CalcLBMForceKernel the kernel stands for (the B200 kernel replaces
        the CUDA platform's), by name, as checkpoints record it."""
        return _Platform(getattr(self.kernel, 'platform_name', self.kernel.name))

    def createCheckpoint(self):
        """The particle part of a checkpoint, in place of OpenMM's Context.createCheckpoint(): the step count, then the
        positions and velocities (float64, little-endian)."""
        return (struct.pack('<qq', self.step_count, len(self.positions)) +
                np.concatenate([self.positions.ravel(), self.velocities.ravel()]).astype('<f8').tobytes())

    def loadCheckpoint(self, data):
        step, n = struct.unpack_from('<qq', data, 0)
        if n != len(self.positions) or len(data) != 16 + 48*n:
            raise ValueError('the checkpoint was written for another System')
        values = np.frombuffer(data, dtype='<f8', count=6*n, offset=16).reshape(2, n, 3)
        self.setPositions(values[0])
        self.setVelocities(values[1])
        self.step_count = step

    def setPositions(self, positions):
        self.positions = np.array(positions, dtype=np.float64).reshape(-1, 3)

    def setVelocities(self, velocities):
        self.velocities = np.array(velocities, dtype=np.float64).reshape(-1, 3)

    def getStepCount(self):
        return self.step_count

    def setStepCount(self, count):
        self.step_count = count

    def updateLatticeParameters(self):
        self.lattice = self.force.latticeParameters(self.system.box, self.integrator.getStepSize(), self.masses)
        self.kernel.copy_parameters(self.lattice)

    def _coupled_arrays(self, forces):
        if len(self.coupled) == 0:
            return None, None, None
        return (np.ascontiguousarray(self.positions[self.coupled]), np.ascontiguousarray(self.velocities[self.coupled]),
                np.ascontiguousarray(forces[self.coupled]))

    def _forces(self, include_lbm=True):
        forces = np.zeros_like(self.positions)
        for f in self.others:
            forces += f.compute(self.positions, self.system.box)
        if include_lbm:
            p, v, f = self._coupled_arrays(forces)
            self.kernel.execute(self.step_count, p, v, f, True, False)
            if f is not None:
                forces[self.coupled] = f
        return forces

    def _step(self):
        p, v, f = self._coupled_arrays(np.zeros_like(self.positions))
        self.kernel.begin_step(self.step_count, p, v, f)
        if v is not None:
            self.velocities[self.coupled] = v
        forces = self._forces()
        dt = self.integrator.step_size
        self.velocities += dt*forces/self.masses[:, None]
        self.positions += dt*self.velocities
        self.step_count += 1

    def getForces(self):
        """The forces of the current state (an evaluation between steps)."""
        return self._forces()

    def close(self):
        self.kernel.close()
