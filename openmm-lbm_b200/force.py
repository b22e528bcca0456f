"""LBMForce: the parameter store of the reference's public API (openmmapi/include/LBMForce.h:41-691), with the
same enumerations, setters, getters and defaults (openmmapi/src/LBMForce.cpp:19-29), and the conversion into
lattice units through the C ABI (lbm_compute_lattice_parameters, the reference's
LBMForceImpl::computeLatticeParameters, openmmapi/src/LBMForceImpl.cpp:44-214).

The methods that act on a Context (getFluidState, setFluidState, getFluidFields, getFluidMachNumber,
getWallForce, createCheckpoint, loadCheckpoint, updateParametersInContext) call the kernel of the Context.
"""
import ctypes

import numpy as np

from . import checkpoint
from .abi import LbmForceDescription, LbmLatticeParameters, check, dptr, load_library


class LBMForce:
    # CouplingScheme (LBMForce.h:46)
    EulerMaruyama, NVE = 0, 1
    # DragScheme (LBMForce.h:61)
    Explicit, Centered = 0, 1
    # InterpolationStencil (LBMForce.h:83)
    NearestNode, Trilinear, ThreePoint, Keys = 0, 1, 2, 3
    # WallScheme (LBMForce.h:106)
    BounceBack, Regularized = 0, 1
    # Face (LBMForce.h:127)
    XMin, XMax, YMin, YMax, ZMin, ZMax = 0, 1, 2, 3, 4, 5
    # BoundaryType (LBMForce.h:138)
    Periodic, Velocity, Density, DensityVelocity = 0, 1, 2, 3

    def __init__(self):
        self.description = LbmForceDescription()
        load_library().lbm_default_force_description(ctypes.byref(self.description))
        self.particles = []
        self.solid_nodes = []
        self.force_group = 0
        self.name = 'LBMForce'
        self.decomposition = (1, 1, 1)
        self.particle_copies_check = True
        self.density_halo_exchange = False
        self.velocity_halo_exchange = False

    # Name (OpenMM's Force::getName / setName: the class name by default)
    def getName(self):
        return self.name

    def setName(self, name):
        self.name = str(name)

    # Grid and fluid
    def getGridSize(self):
        d = self.description
        return d.nx, d.ny, d.nz

    def setGridSize(self, nx, ny, nz):
        d = self.description
        d.nx, d.ny, d.nz = nx, ny, nz

    # Domain decomposition (LBMForce.h:180-263).  This library runs the whole lattice on one GPU: the settings are kept
    # (and serialized), and a Context rejects more than one domain as the reference does without MPI.
    def getDomainDecomposition(self):
        return tuple(self.decomposition)

    def setDomainDecomposition(self, px, py, pz):
        if px < 0 or py < 0 or pz < 0:
            raise ValueError('LBMForce: the domain decomposition (setDomainDecomposition()) cannot be negative')
        self.decomposition = (int(px), int(py), int(pz))

    @staticmethod
    def isMPIAvailable():
        return False

    def getParticleCopiesCheck(self):
        return self.particle_copies_check

    def setParticleCopiesCheck(self, check):
        self.particle_copies_check = bool(check)

    def getDensityHaloExchange(self):
        return self.density_halo_exchange

    def setDensityHaloExchange(self, exchange):
        self.density_halo_exchange = bool(exchange)

    def getVelocityHaloExchange(self):
        return self.velocity_halo_exchange

    def setVelocityHaloExchange(self, exchange):
        self.velocity_halo_exchange = bool(exchange)

    def getFluidDensity(self):
        return self.description.fluid_density

    def setFluidDensity(self, density):
        self.description.fluid_density = density

    def getKinematicViscosity(self):
        return self.description.kinematic_viscosity

    def setKinematicViscosity(self, viscosity):
        self.description.kinematic_viscosity = viscosity

    # Coupling
    def getFriction(self):
        return self.description.friction

    def setFriction(self, friction):
        self.description.friction = friction

    def getTemperature(self):
        return self.description.temperature

    def setTemperature(self, temperature):
        self.description.temperature = temperature

    def getCouplingScheme(self):
        return self.description.coupling_scheme

    def setCouplingScheme(self, scheme):
        self.description.coupling_scheme = scheme

    def getDragScheme(self):
        return self.description.drag_scheme

    def setDragScheme(self, scheme):
        self.description.drag_scheme = scheme

    def getInterpolationStencil(self):
        return self.description.interpolation_stencil

    def setInterpolationStencil(self, stencil):
        self.description.interpolation_stencil = stencil

    def getFluidFluctuations(self):
        return bool(self.description.fluid_fluctuations)

    def setFluidFluctuations(self, fluctuations):
        self.description.fluid_fluctuations = int(bool(fluctuations))

    # Walls and faces
    def getWallScheme(self):
        return self.description.wall_scheme

    def setWallScheme(self, scheme):
        self.description.wall_scheme = scheme

    @staticmethod
    def _check_face(face):
        if face < LBMForce.XMin or face > LBMForce.ZMax:
            raise ValueError('LBMForce: unknown face of the box')

    def getFaceBoundary(self, face):
        self._check_face(face)
        return self.description.face_boundary[face]

    def setFaceBoundary(self, face, boundary):
        self._check_face(face)
        self.description.face_boundary[face] = boundary

    def getFaceVelocity(self, face):
        self._check_face(face)
        return tuple(self.description.face_velocity[face])

    def setFaceVelocity(self, face, velocity):
        self._check_face(face)
        for a in range(3):
            self.description.face_velocity[face][a] = velocity[a]

    def getFaceDensity(self, face):
        self._check_face(face)
        return self.description.face_density[face]

    def setFaceDensity(self, face, density):
        self._check_face(face)
        self.description.face_density[face] = density

    def getSolidNodes(self):
        return list(self.solid_nodes)

    def setSolidNodes(self, nodes):
        self.solid_nodes = [int(n) for n in nodes]

    # Fluid state and options
    def getRandomNumberSeed(self):
        return self.description.random_number_seed

    def setRandomNumberSeed(self, seed):
        self.description.random_number_seed = seed

    def getBodyAcceleration(self):
        return tuple(self.description.body_acceleration)

    def setBodyAcceleration(self, acceleration):
        for a in range(3):
            self.description.body_acceleration[a] = acceleration[a]

    def getInitialFluidVelocity(self):
        return tuple(self.description.initial_velocity)

    def setInitialFluidVelocity(self, velocity):
        for a in range(3):
            self.description.initial_velocity[a] = velocity[a]

    def getFluidMomentumRemovalFrequency(self):
        return self.description.momentum_removal_frequency

    def setFluidMomentumRemovalFrequency(self, frequency):
        self.description.momentum_removal_frequency = frequency

    def getMachCheckFrequency(self):
        return self.description.mach_check_frequency

    def setMachCheckFrequency(self, frequency):
        self.description.mach_check_frequency = frequency

    def getMachNumberLimit(self):
        return self.description.mach_number_limit

    def setMachNumberLimit(self, limit):
        self.description.mach_number_limit = limit

    # Particles
    def getNumParticles(self):
        return len(self.particles)

    def addParticle(self, particle):
        self.particles.append(int(particle))
        return len(self.particles) - 1

    def getParticle(self, index):
        return self.particles[index]

    def setParticle(self, index, particle):
        self.particles[index] = int(particle)

    def getForceGroup(self):
        return self.force_group

    def setForceGroup(self, group):
        self.force_group = group

    # Lattice units
    def latticeParameters(self, box, step_size, system_masses):
        """LBMForceImpl::computeLatticeParameters for a rectangular box (nm) and a step size (ps).  More than one
        domain is rejected as by the reference built without MPI (LBMDecomposition.cpp:113-124)."""
        if any(p < 0 for p in self.decomposition):
            raise ValueError('LBMForce: the domain decomposition (setDomainDecomposition()) cannot be negative')
        if tuple(self.decomposition) != (1, 1, 1):
            raise ValueError('LBMForce: setDomainDecomposition() asks for more than one domain, but this library runs '
                             'the whole lattice on one GPU (no MPI decomposition)')
        lib = load_library()
        lattice = LbmLatticeParameters()
        masses = np.ascontiguousarray(system_masses, dtype=np.float64)
        coupled = np.ascontiguousarray(self.particles, dtype=np.int32)
        solid = np.ascontiguousarray(self.solid_nodes, dtype=np.int32)
        box = np.ascontiguousarray(box, dtype=np.float64)
        ip = ctypes.POINTER(ctypes.c_int)
        check(lib.lbm_compute_lattice_parameters(ctypes.byref(self.description), dptr(box), step_size, len(masses),
                                                 dptr(masses), len(coupled), coupled.ctypes.data_as(ip), len(solid),
                                                 solid.ctypes.data_as(ip), ctypes.byref(lattice)), lib)
        return lattice

    # Context access (LBMForce.h:516-666)
    def getFluidState(self, context):
        return context.kernel.get_fluid_state()

    def setFluidState(self, context, state):
        context.kernel.set_fluid_state(state)

    def getFluidFields(self, context):
        return context.kernel.get_fluid_fields()

    def getFluidMachNumber(self, context):
        return context.kernel.get_fluid_mach_number()

    def getWallForce(self, context):
        return context.kernel.get_wall_force()

    def createCheckpoint(self, context):
        """LBMForceImpl::createCheckpoint (LBMForceImpl.cpp:568-573): the header, then the kernel's stream."""
        header = checkpoint.write_header(context.getPlatform().getName(), context.lattice, len(self.particles))
        return header + context.kernel.create_checkpoint()

    def loadCheckpoint(self, context, data):
        """LBMForceImpl::loadCheckpoint (LBMForceImpl.cpp:575-580): the header is checked against the Context."""
        start = checkpoint.read_header(data, context.getPlatform().getName(), context.lattice, len(self.particles))
        context.kernel.load_checkpoint(bytes(data[start:]))

    def getLatticeParametersInContext(self, context):
        lattice = context.lattice
        return lattice.dx, lattice.dt, lattice.tau

    def updateParametersInContext(self, context):
        context.updateLatticeParameters()
