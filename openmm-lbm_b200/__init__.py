"""B200-native LBM force kernel: the per-step fluid and particle-coupling path of openmm-lbm on one B200.

    abi      ctypes mirror of include/lbm_b200.h and the loader of liblbm_b200.so (the CUDA build)
    force    LBMForce, the reference's parameter API, and its conversion into lattice units
    kernel   B200Kernel, the platform kernel (CalcLBMForceKernel) behind the C ABI
    harness  System / Context / VerletIntegrator: the OpenMM call order that drives the kernel
    md       BeadDynamics: bead forces and the leapfrog on the device (the benchmark's stand-in for OpenMM)
    batch    ReplicaBatch: many independent periodic replicas with their beads, advanced together
    reporters  saveCheckpoint / loadCheckpoint and the reference's reporters (checkpoints, temperature, VTK files),
             with a Simulation driver that calls them as OpenMM's does
    checkpoint the reference's checkpoint header and checkpoint file around the kernel's stream
    serialization  XmlSerializer: the reference's XML form of LBMForce (LBMForceProxy, version 9; reads 1 to 9)
"""
from .batch import ReplicaBatch  # noqa: F401
from .abi import LbmError, LbmLatticeParameters, load_library  # noqa: F401
from .force import LBMForce  # noqa: F401
from .harness import Context, ExternalForce, PairForce, System, VerletIntegrator  # noqa: F401
from .kernel import B200Kernel  # noqa: F401
from .md import BeadDynamics, random_walk_chains  # noqa: F401
from .reporters import (LBMCheckpointReporter, LBMTemperatureReporter, LBMVTKReporter, Simulation,  # noqa: F401
                        loadCheckpoint, saveCheckpoint)
from .serialization import XmlSerializer  # noqa: F401
