"""GPU tests of the replica batch (include/lbm_b200_batch.h).  Replicas of the batching configuration (periodic
fluctuating fluids, tau 0.7, kT = 1e-4, distinct Philox seeds; Lennard-Jones beads sigma 1, epsilon kT, cutoff 2.5,
mass 1; three-point stencil, explicit drag 0.8; lattice units dx = 1 nm, dt = 1 ps, rho0 = 1 Da/nm^3) on small lattices
of uneven sizes:

- pathwise against the CPU oracle (its Philox mode and its bead forces), FP64 and FP32;
- pathwise: each replica of a batch follows a B200Kernel with the same lattice parameters and the bead dynamics of
  the benchmark (BeadDynamics), step for step, within 1e-9 relative in FP64 over 30 steps (the bead pair forces are
  summed in another order, and the chaotic bead dynamics amplify the last bits);
- a run replayed from the CUDA graph equals the same run launched step by step;
- the fluid temperature of every replica is kT (equipartition of the fluctuating fluid)."""
import numpy as np
import pytest

import lbm_b200
from lbm_b200 import LBMForce, ReplicaBatch

pytestmark = pytest.mark.gpu

BOLTZ = 6.02214076e23*1.380649e-23/1000.0
KT, TAU, FRICTION, SIGMA, CUTOFF = 1e-4, 0.7, 0.8, 1.0, 2.5


def replica_lattice(n, num_beads, seed, kT=KT):
    force = LBMForce()
    force.setGridSize(n, n, n)
    force.setFluidDensity(1.0)
    force.setKinematicViscosity((TAU - 0.5)/3.0)
    force.setFluidFluctuations(kT > 0)
    force.setTemperature(kT/BOLTZ)
    force.setRandomNumberSeed(seed)
    force.setInterpolationStencil(LBMForce.ThreePoint)
    force.setDragScheme(LBMForce.Explicit)
    force.setFriction(FRICTION)
    for i in range(num_beads):
        force.addParticle(i)
    return force.latticeParameters(np.array([n, n, n], dtype=float), 1.0, np.ones(max(1, num_beads)))


def bead_positions(n, count, rng, min_distance=1.1):
    """Uniform positions in an n^3 periodic box at least min_distance apart (minimum image)."""
    out = []
    while len(out) < count:
        x = rng.uniform(0, n, 3)
        if all(np.linalg.norm((x - y) - n*np.round((x - y)/n)) >= min_distance for y in out):
            out.append(x)
    return np.array(out)


def make_replicas(sizes, beads, seed=2026):
    rng = np.random.Generator(np.random.PCG64(seed))
    lattices = [replica_lattice(n, b, 1000 + r) for r, (n, b) in enumerate(zip(sizes, beads))]
    positions = [bead_positions(n, b, rng) for n, b in zip(sizes, beads)]
    return lattices, positions


def run_separately(lattice, positions, steps):
    import torch
    n = lattice.nx
    count = len(positions)
    masses = np.ones(count)
    kernel = lbm_b200.B200Kernel(lattice, masses, [], 'double')
    md = lbm_b200.BeadDynamics(masses, (n, n, n), np.zeros((0, 2), dtype=np.int32), k=0.0, r0=1.0, pair='lj',
                               sigma=SIGMA, epsilon=KT, cutoff=CUTOFF)
    stream = kernel.stream()
    pos = torch.tensor(positions, device='cuda', dtype=torch.float64)
    vel = torch.zeros_like(pos)
    frc = torch.zeros_like(pos)
    for s in range(steps):
        kernel.begin_step(s, pos, vel, frc)
        md.compute_forces(pos, frc, stream)
        kernel.execute(s, pos, vel, frc)
        md.integrate(1.0, pos, vel, frc, stream)
    torch.cuda.synchronize()
    out = kernel.get_fluid_state(), pos.cpu().numpy(), vel.cpu().numpy()
    kernel.close()
    md.close()
    return out


def run_oracle(lattice, positions, steps):
    """One replica on the CPU oracle (Philox mode: the same random numbers as the device), its Lennard-Jones bead
    forces from the oracle's bead forces, and the leapfrog of a VerletIntegrator with the lattice time step."""
    from oracle import OracleKernel, md_forces
    n = lattice.nx
    count = len(positions)
    masses = np.ones(count)
    kernel = OracleKernel(lattice, masses, [])
    pos = np.array(positions, dtype=np.float64)
    vel = np.zeros_like(pos)
    box = np.array([n, n, n], dtype=np.float64)
    for s in range(steps):
        kernel.begin_step(s, pos, vel, np.zeros_like(pos))
        frc = md_forces(pos, box, np.zeros((0, 2), dtype=np.int32), 0.0, 1.0, 'lj', SIGMA, KT, CUTOFF)
        kernel.execute(s, pos, vel, frc)
        vel += frc/masses[:, None]
        pos += vel
    out = kernel.get_fluid_state(), pos, vel
    kernel.close()
    return out


@pytest.mark.parametrize('precision,steps,tolerance,sizes', [('double', 30, 1e-9, (12, 16, 10, 14)),
                                                               ('single', 10, 1e-5, (12, 16, 10, 14)),
                                                               ('single', 10, 1e-5, (13, 16, 9, 15))])
def test_batch_follows_oracle(precision, steps, tolerance, sizes):
    """Each replica of a batch of the batching configuration (fluctuating fluid, three-point stencil, explicit drag,
    Lennard-Jones beads) follows the CPU oracle path by path: FP64 within 1e-9 over 30 steps (the bead pair forces
    are summed in another order and the bead dynamics amplify the last bits), FP32 storage within 1e-5 over 10.  FP32
    replicas of an odd edge pair the nodes within each row, the row's last node alone."""
    beads = [20, 35, 8, 26]
    lattices, positions = make_replicas(sizes, beads, seed=99)
    batch = ReplicaBatch(lattices, beads, np.ones(sum(beads)), np.concatenate(positions), pair=('lj', SIGMA, KT, CUTOFF),
                         precision=precision)
    batch.step(steps)
    pos, vel = batch.particles_state()
    offsets = np.concatenate([[0], np.cumsum(beads)])
    for r, n in enumerate(sizes):
        state, ref_pos, ref_vel = run_oracle(lattices[r], positions[r], steps)
        got = batch.fluid_state(r)
        assert abs(got - state).max() <= tolerance*abs(state).max(), r
        b = slice(offsets[r], offsets[r+1])
        d = pos[b] - ref_pos
        d -= n*np.round(d/n)
        assert abs(d).max() <= tolerance*abs(ref_pos).max(), r
        assert abs(vel[b] - ref_vel).max() <= tolerance*abs(ref_vel).max(), r
    batch.close()


def test_batch_follows_separate_kernels():
    sizes, beads, steps = [12, 16, 10, 14], [20, 35, 8, 26], 30
    lattices, positions = make_replicas(sizes, beads)
    batch = ReplicaBatch(lattices, beads, np.ones(sum(beads)), np.concatenate(positions), pair=('lj', SIGMA, KT, CUTOFF),
                         precision='double')
    batch.step(steps)
    pos, vel = batch.particles_state()
    offsets = np.concatenate([[0], np.cumsum(beads)])
    for r in range(len(sizes)):
        state, ref_pos, ref_vel = run_separately(lattices[r], positions[r], steps)
        got = batch.fluid_state(r)
        assert abs(got - state).max() <= 1e-9*abs(state).max(), r
        b = slice(offsets[r], offsets[r+1])
        assert abs(pos[b] - ref_pos).max() <= 1e-9*abs(ref_pos).max(), r
        assert abs(vel[b] - ref_vel).max() <= 1e-9*abs(ref_vel).max(), r
    batch.close()


@pytest.mark.parametrize('persistent', [True, False])
def test_graph_replay_equals_direct_launches(persistent):
    """The persistent step runs graph_steps steps per launch: 25 + 15 steps with graphs of 10 steps are two graph
    replays and two direct launches (the 15 start at an odd step, off the graph's buffer parity), with graphs of 1000
    steps two direct launches; the seven-kernel form launches 7 kernels per step.  Every way gives the same run."""
    sizes, beads = [16, 20, 12], [30, 50, 10]
    lattices, positions = make_replicas(sizes, beads, seed=7)
    runs = []
    for graph_steps in (10, 1000):
        batch = ReplicaBatch(lattices, beads, np.ones(sum(beads)), np.concatenate(positions),
                             pair=('lj', SIGMA, KT, CUTOFF), precision='double')
        batch.set_persistent(persistent)
        batch.autotune(graph_steps)
        launches = batch.info()['launches']
        batch.step(25)
        batch.step(15)
        info = batch.info()
        expected = ({10: 4, 1000: 2}[graph_steps] if persistent else 7*40)
        assert info['steps'] == 40 and info['launches'] - launches == expected
        runs.append((batch.fluid_state(1), batch.particles_state()[1]))
        batch.close()
    (state_a, vel_a), (state_b, vel_b) = runs
    # The reactions of beads that share a node are added with atomics, in any order.
    assert abs(state_a - state_b).max() <= 1e-12*abs(state_a).max()
    assert abs(vel_a - vel_b).max() <= 1e-12*abs(vel_a).max()


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_persistent_step_equals_phase_kernels(precision):
    """The persistent step (phases separated by grid barriers, per-replica sums by the last block of each replica,
    double-buffered reactions) computes what the seven phase kernels compute (reactions summed with atomics in any
    order: 1e-12 in FP64, 1e-6 in FP32, over 30 steps of the chaotic bead dynamics)."""
    sizes, beads = [12, 17, 14, 9], [25, 40, 30, 6]
    lattices, positions = make_replicas(sizes, beads, seed=13)
    runs = []
    for persistent in (True, False):
        batch = ReplicaBatch(lattices, beads, np.ones(sum(beads)), np.concatenate(positions),
                             pair=('lj', SIGMA, KT, CUTOFF), precision=precision)
        batch.set_persistent(persistent)
        batch.autotune(10)
        batch.step(30)
        runs.append([batch.fluid_state(r) for r in range(len(sizes))] + list(batch.particles_state()))
        batch.close()
    tol = 1e-12 if precision == 'double' else 1e-6
    for a, b in zip(*runs):
        assert abs(a - b).max() <= tol*abs(a).max()


def test_persistent_barrier_timeout_is_reported():
    """A poll limit of one makes the blocks that wait at a grid barrier of the persistent step give up: the launch
    stops, the next synchronizing call reports LBM_ERR_DEVICE_TIMEOUT, and with the default limit the batch steps
    again (the fluid temperature of every replica stays finite)."""
    from lbm_b200.abi import LBM_ERR_DEVICE_TIMEOUT, LbmError
    sizes, beads = [16, 20, 12], [30, 50, 10]
    lattices, positions = make_replicas(sizes, beads, seed=5)
    batch = ReplicaBatch(lattices, beads, np.ones(sum(beads)), np.concatenate(positions),
                         pair=('lj', SIGMA, KT, CUTOFF), precision='single')
    batch.set_barrier_polls(1)
    batch.step(4)
    with pytest.raises(LbmError) as failure:
        batch.particles_state()
    assert failure.value.status == LBM_ERR_DEVICE_TIMEOUT
    batch.set_barrier_polls(0)
    batch.step(6)
    fluid, _ = batch.temperatures()
    batch.close()
    assert np.isfinite(fluid).all()


@pytest.mark.parametrize('precision', ['single', 'double'])
def test_fluid_temperature_of_every_replica(precision):
    sizes = [16, 20, 24, 18, 22, 16]
    beads = [20, 40, 60, 30, 50, 25]
    lattices, positions = make_replicas(sizes, beads, seed=11)
    batch = ReplicaBatch(lattices, beads, np.ones(sum(beads)), np.concatenate(positions), pair=('lj', SIGMA, KT, CUTOFF),
                         precision=precision)
    batch.autotune(20)
    batch.step(300)
    samples = []
    for _ in range(10):
        batch.step(20)
        samples.append(batch.temperatures()[0])
    batch.close()
    fluid = np.mean(samples, axis=0)
    # One snapshot of N nodes has a relative spread sqrt(2/(3N)) (1.3 % at 16^3); ten snapshots 20 steps apart.
    assert np.all(abs(fluid/KT - 1) < 0.05), fluid/KT
