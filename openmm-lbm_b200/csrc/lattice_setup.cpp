// Host-side setup of the B200 LBM force kernel: conversion of an LBMForce description in OpenMM units
// into lattice units, with the checks of the reference (LBMForceImpl::computeLatticeParameters,
// openmmapi/src/LBMForceImpl.cpp:44-214), and the defaults of the LBMForce constructor
// (openmmapi/src/LBMForce.cpp:19-29).  No GPU is needed.
#include "lbm_internal.h"
#include <algorithm>
#include <cmath>
#include <limits>
#include <set>
#include <sstream>
#include <vector>

namespace lbm {

// Boltzmann's constant in kJ/(mol K): the molar gas constant R = N_A k_B (exact SI values) / 1000.
static const double kBoltz = 6.02214076e23*1.380649e-23/1000.0;

void defaultForceDescription(LbmForceDescription* f) {
    *f = LbmForceDescription();
    f->nx = f->ny = f->nz = 0;
    f->fluid_density = 602.214;
    f->kinematic_viscosity = 1.0035;
    f->friction = 1.0;
    f->temperature = 300.0;
    f->coupling_scheme = 0;
    f->drag_scheme = LBM_DRAG_EXPLICIT;
    f->interpolation_stencil = LBM_STENCIL_NEAREST;
    f->fluid_fluctuations = 0;
    f->wall_scheme = LBM_WALL_BOUNCEBACK;
    for (int face = 0; face < 6; face++) {
        f->face_boundary[face] = LBM_BOUNDARY_PERIODIC;
        f->face_velocity[face][0] = f->face_velocity[face][1] = f->face_velocity[face][2] = 0.0;
        f->face_density[face] = 0.0;
    }
    f->random_number_seed = 0;
    f->momentum_removal_frequency = 1;
    f->mach_check_frequency = 100;
    f->mach_number_limit = 0.3;
}

static bool isOpenAxis(const LbmLatticeParameters& l, int axis) {
    return l.face_boundary[2*axis] != LBM_BOUNDARY_PERIODIC;
}

void computeLatticeParameters(const LbmForceDescription& force, const double box[3], double stepSize,
                              int numSystemParticles, const double* systemMasses, int numCoupled,
                              const int* coupled, int numSolid, const int* solid, LbmLatticeParameters& l) {
    l = LbmLatticeParameters();
    l.nx = force.nx;
    l.ny = force.ny;
    l.nz = force.nz;
    if (l.nx <= 0 || l.ny <= 0 || l.nz <= 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the grid size must be set to positive values with setGridSize()");

    // The reference's 2^31 node limit (LBMForceImpl.cpp:56-78) comes from its 32-bit indexing.  The dense kernels
    // here index nodes with 32-bit unsigned integers, so the fluid may have up to 2^32 nodes (lbm_create checks it);
    // a lattice with coupled particles stays below 2^31 nodes, because the coupling keeps signed 32-bit node indices.

    // The lattice spans the periodic box with cubic cells (:80-92).
    l.dx = box[0]/l.nx;
    double dy = box[1]/l.ny, dz = box[2]/l.nz;
    if (std::fabs(dy-l.dx) > 1e-6*l.dx || std::fabs(dz-l.dx) > 1e-6*l.dx) {
        std::stringstream msg;
        msg << "LBMForce: the lattice cells must be cubic, but the box and grid sizes give spacings " << l.dx << ", "
            << dy << ", " << dz << " nm";
        throw Error(LBM_ERR_INVALID_ARGUMENT, msg.str());
    }

    // Time step and relaxation time (:94-105).
    if (stepSize <= 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the integrator step size must be positive");
    l.dt = stepSize;
    if (force.fluid_density <= 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the fluid density must be positive");
    if (force.kinematic_viscosity <= 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the kinematic viscosity must be positive");
    l.density = force.fluid_density;
    l.tau = 3.0*force.kinematic_viscosity*l.dt/(l.dx*l.dx) + 0.5;
    l.omega = 1.0/l.tau;

    // Velocities and accelerations in lattice units (:107-110).
    for (int a = 0; a < 3; a++) {
        l.initial_velocity[a] = force.initial_velocity[a]*(l.dt/l.dx);
        l.body_acceleration[a] = force.body_acceleration[a]*(l.dt*l.dt/l.dx);
    }

    // Coupling and checks (:112-128).
    if (force.friction < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the friction must not be negative");
    if (force.temperature < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the temperature must not be negative");
    if (force.momentum_removal_frequency < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the fluid momentum removal frequency must not be negative");
    if (force.mach_check_frequency < 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the Mach number check frequency must not be negative");
    if (force.mach_number_limit <= 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the Mach number limit must be positive");
    l.mach_check_frequency = force.mach_check_frequency;
    l.mach_number_limit = force.mach_number_limit;

    // Solid nodes (:130-144).
    long long numNodes = (long long) l.nx*l.ny*l.nz;
    std::vector<int> solidNodes(solid, solid + numSolid);
    std::sort(solidNodes.begin(), solidNodes.end());
    for (size_t i = 0; i < solidNodes.size(); i++) {
        if (solidNodes[i] < 0 || solidNodes[i] >= numNodes)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: a solid node index is out of range");
        if (i > 0 && solidNodes[i] == solidNodes[i-1])
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: a solid node is listed more than once");
    }
    if ((long long) solidNodes.size() == numNodes)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: all lattice nodes are solid");
    if (force.wall_scheme != LBM_WALL_BOUNCEBACK && force.wall_scheme != LBM_WALL_REGULARIZED)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: unknown wall scheme");
    l.wall_scheme = force.wall_scheme;

    // Faces of the box (:146-172).
    const char* axisName[3] = {"x", "y", "z"};
    int size[3] = {l.nx, l.ny, l.nz};
    for (int face = 0; face < 6; face++) {
        int type = force.face_boundary[face];
        if (type != LBM_BOUNDARY_PERIODIC && type != LBM_BOUNDARY_VELOCITY && type != LBM_BOUNDARY_DENSITY &&
                type != LBM_BOUNDARY_DENSITY_VELOCITY)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: unknown boundary type of a face");
        l.face_boundary[face] = type;
        for (int a = 0; a < 3; a++)
            l.face_velocity[face][a] = force.face_velocity[face][a]*(l.dt/l.dx);
        double density = force.face_density[face];
        if (density < 0)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: the density of a face must not be negative");
        l.face_density[face] = (density == 0 ? 1.0 : density/l.density);
    }
    for (int axis = 0; axis < 3; axis++) {
        if ((l.face_boundary[2*axis] == LBM_BOUNDARY_PERIODIC) != (l.face_boundary[2*axis+1] == LBM_BOUNDARY_PERIODIC))
            throw Error(LBM_ERR_INVALID_ARGUMENT, std::string("LBMForce: the two faces perpendicular to ") + axisName[axis] +
                        " must be both periodic or both open (Velocity, Density or DensityVelocity)");
        if (isOpenAxis(l, axis) && size[axis] < 3)
            throw Error(LBM_ERR_INVALID_ARGUMENT, std::string("LBMForce: with open faces perpendicular to ") +
                        axisName[axis] + " the grid needs at least 3 nodes along " + axisName[axis]);
    }
    bool openFaces = isOpenAxis(l, 0) || isOpenAxis(l, 1) || isOpenAxis(l, 2);
    if (openFaces && force.momentum_removal_frequency > 0)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: with open faces the fluid exchanges momentum with the outside, "
                    "and its momentum cannot be removed: call setFluidMomentumRemovalFrequency(0)");
    l.friction = force.friction;
    if (force.coupling_scheme != 0 && force.coupling_scheme != 1)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: unknown coupling scheme");
    l.kT = (force.coupling_scheme == 1 ? 0.0 : kBoltz*force.temperature);
    if (force.drag_scheme != LBM_DRAG_EXPLICIT && force.drag_scheme != LBM_DRAG_CENTERED)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: unknown drag scheme");
    l.drag_scheme = force.drag_scheme;
    if (force.interpolation_stencil < LBM_STENCIL_NEAREST || force.interpolation_stencil > LBM_STENCIL_KEYS)
        throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: unknown interpolation stencil");
    l.interpolation_stencil = force.interpolation_stencil;
    l.fluid_fluctuations = force.fluid_fluctuations ? 1 : 0;
    l.fluid_kT = (l.fluid_fluctuations ? kBoltz*force.temperature : 0.0);
    if (l.fluid_fluctuations)
        for (int face = 0; face < 6; face++)
            if (l.face_boundary[face] == LBM_BOUNDARY_DENSITY)
                throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: Density faces cannot be used with fluid fluctuations: they "
                            "do not keep the fluctuating fluid next to the face at equilibrium (its momentum fluctuates more "
                            "than at the temperature of the force, and coupled particles near the face are hotter). Use "
                            "DensityVelocity faces, which impose the density and the velocity, or Velocity faces");
    l.random_number_seed = force.random_number_seed;
    l.momentum_removal_frequency = force.momentum_removal_frequency;

    // Coupled particles (:200-211).
    std::set<int> seen;
    for (int i = 0; i < numCoupled; i++) {
        int particle = coupled[i];
        if (particle < 0 || particle >= numSystemParticles)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: a coupled particle index is out of range");
        if (seen.count(particle))
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: a particle is coupled more than once");
        if (systemMasses[particle] <= 0)
            throw Error(LBM_ERR_INVALID_ARGUMENT, "LBMForce: coupled particles must have a positive mass");
        seen.insert(particle);
    }
}

} // namespace lbm
