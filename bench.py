"""Benchmark of the per-step fluid and particle-coupling path on B200: MLUPS, and the HBM roofline of the dense
stream-collide kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload coupled|fluid|channel|batch|warmstart] [--precision double|single|half|bfloat16]
                    [--size EDGE]
                    [--graph-steps G] [--replicas R] [--separate]

Workload "coupled" (default, the scale configuration): a 256^3 periodic fluctuating D3Q19 fluid (tau 0.6, kT 1e-4 in
lattice units, Philox seed), FP32 storage, momentum removal every step, Mach check every 100 steps; 512 bead-spring
chains of 100 beads (51,200 beads, mass 1) placed as seeded random walks, harmonic bonds (k = 100 kT/sigma^2, r0 = 1)
and WCA repulsion (sigma 1, epsilon = kT), coupled through the Keys stencil with the centred drag (friction 1 per
lattice step, solved by conjugate gradients on the device).  One step: beginStep, bead forces, execute (coupling +
fluid) and the leapfrog of the beads, all on the device.  "fluid": the fluid alone (kernel profiling).  "channel": the
precision configuration, a 384x384x192 Poiseuille channel between bounce-back planes (g_x 5e-7, tau 0.55), for the
MLUPS of each storage format.  "batch": the batching configuration, 256 periodic fluctuating replicas of uneven sizes
with Lennard-Jones beads, every phase one launch over all replicas, G steps per CUDA graph (--separate also times the
replicas as separate kernels).  The default run also reports the plain fluid of the same lattice ("plain_fluid") and,
when openmm-lbm_b200/warmstart_net/weights.pt exists, the metric's time-to-steady part ("warm_start": held-out obstacle
channels solved to the residual 1e-6 from rest and from the learned warm start); "warmstart" runs that alone, on
--steps channels.

value = fluid nodes x steps / device time (MLUPS).  e2e = the same metric through the C ABI with the beads' positions
and velocities in pinned host memory: copied to the device before and back after every step.  With N > 1 (torchrun,
one rank per GPU) every rank advances its own replica; value = all ranks' node updates / the slowest rank's time.
--impl reference times the reference's own Reference-platform kernel (oracle/_ref, compiled unmodified from the
reference sources) on the host, with the beads integrated by the CPU bead forces of the oracle, on a bounded sample.
"""
import argparse
import ctypes
import importlib.util
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PACKAGE = os.path.join(ROOT, 'openmm-lbm_b200')
BOLTZ = 6.02214076e23*1.380649e-23/1000.0
STORAGE_BYTES = {'double': 8, 'single': 4, 'half': 2, 'bfloat16': 2}
DTYPE = {'double': 'f64', 'single': 'f32', 'half': 'f16 storage, f32 compute', 'bfloat16': 'bf16 storage, f32 compute'}


def load_package():
    if 'lbm_b200' in sys.modules:
        return sys.modules['lbm_b200']
    spec = importlib.util.spec_from_file_location('lbm_b200', os.path.join(PACKAGE, '__init__.py'),
                                                  submodule_search_locations=[PACKAGE])
    module = importlib.util.module_from_spec(spec)
    sys.modules['lbm_b200'] = module
    spec.loader.exec_module(module)
    return module


class Workload:
    """The scale configuration, or a sample of it with the same densities (n^3 nodes, chains scaled with volume)."""

    def __init__(self, n=256, chains=512, length=100, coupled=True, fluctuations=True, seed=2026):
        self.n, self.chains, self.length = n, chains if coupled else 0, length
        self.tau, self.kT, self.seed = 0.6, (1e-4 if fluctuations else 0.0), seed
        self.friction = 1.0
        self.coupled = coupled

    def name(self):
        fluid = '%d^3 periodic %sD3Q19 fluid, tau 0.6%s' % (self.n, 'fluctuating ' if self.kT > 0 else '',
                                                          ', kT 1e-4' if self.kT > 0 else '')
        if not self.coupled:
            return fluid + ' (lattice units)'
        return (fluid + ' + %d chains x %d beads (harmonic k = 100 kT, WCA), Keys stencil, centred drag 1.0 '
                '(lattice units)' % (self.chains, self.length))

    def lattice(self, lbm):
        n = self.n
        force = lbm.LBMForce()
        force.setGridSize(n, n, n)
        force.setFluidDensity(1.0)
        force.setKinematicViscosity((self.tau - 0.5)/3.0)
        force.setFluidFluctuations(self.kT > 0)
        force.setTemperature(self.kT/BOLTZ if self.kT > 0 else 0.0)
        force.setRandomNumberSeed(self.seed)
        force.setInterpolationStencil(force.Keys)
        force.setDragScheme(force.Centered)
        force.setFriction(self.friction)
        for i in range(self.chains*self.length):
            force.addParticle(i)
        masses = np.ones(max(1, self.chains*self.length))
        return force.latticeParameters(np.array([n, n, n], dtype=float), 1.0, masses)

    def beads(self, lbm):
        return lbm.random_walk_chains(self.chains, self.length, (self.n,)*3, self.seed)

    def md_parameters(self):
        kT = self.kT if self.kT > 0 else 1e-4
        return dict(k=100.0*kT, r0=1.0, pair='wca', sigma=1.0, epsilon=kT, cutoff=2.0**(1/6))

    @property
    def shape(self):
        return (self.n,)*3

    def solids(self):
        return []

    def fluid_nodes(self):
        return self.n**3

    def profile_tag(self):
        return '%s_%d' % ('fluct' if self.kT > 0 else 'plain', self.n)

    def sample(self, n):
        """A sample on an n^3 lattice with the same bead density."""
        chains = int(round(self.chains*(n/self.n)**3)) if self.coupled else 0
        return Workload(n=n, chains=chains, length=self.length, coupled=self.coupled, fluctuations=self.kT > 0,
                        seed=self.seed)


class ChannelWorkload:
    """The precision configuration: a Poiseuille channel between bounce-back planes z = 0 and z = nz - 1, Guo body
    force g_x = 5e-7, tau 0.55, no fluctuations, no momentum removal, started from rest (lattice units)."""

    def __init__(self, shape=(384, 384, 192)):
        self.shape = tuple(shape)
        self.n = max(shape)
        self.chains, self.length, self.coupled = 0, 0, False
        self.tau, self.kT, self.g, self.seed = 0.55, 0.0, 5e-7, 2026

    def name(self):
        return ('%dx%dx%d Poiseuille channel, bounce-back planes z = 0 and z = %d, g_x 5e-7, tau 0.55, no fluctuations '
                '(lattice units)' % (self.shape + (self.shape[2] - 1,)))

    def lattice(self, lbm):
        nx, ny, nz = self.shape
        force = lbm.LBMForce()
        force.setGridSize(nx, ny, nz)
        force.setFluidDensity(1.0)
        force.setKinematicViscosity((self.tau - 0.5)/3.0)
        force.setBodyAcceleration((self.g, 0.0, 0.0))
        force.setFluidMomentumRemovalFrequency(0)
        return force.latticeParameters(np.array(self.shape, dtype=float), 1.0, np.ones(1))

    def solids(self):
        nx, ny, nz = self.shape
        plane = np.arange(nx*ny, dtype=np.int64)
        return np.concatenate([plane, plane + nx*ny*(nz - 1)])

    def fluid_nodes(self):
        nx, ny, nz = self.shape
        return nx*ny*(nz - 2)

    def profile_tag(self):
        return 'channel_%dx%dx%d' % self.shape

    def sample(self, n):
        """A sample with the same aspect ratio and edge n in x."""
        return ChannelWorkload((n, n, max(4, n//2)))


class BatchWorkload:
    """The batching configuration: replicas with seeded-uniform cubic edges 16..64 and bead counts 20..200 (numpy PCG64,
    seed 2026), each a periodic fluctuating fluid (tau 0.7, kT 1e-4, its own Philox seed) with Lennard-Jones beads
    (sigma 1, epsilon kT, cutoff 2.5, mass 1) at random non-overlapping positions, three-point stencil, explicit drag
    0.8 (lattice units)."""

    def __init__(self, replicas=256, seed=2026):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.replicas, self.seed = replicas, seed
        self.sizes = rng.integers(16, 65, replicas)
        self.beads = rng.integers(20, 201, replicas)
        self.tau, self.kT, self.friction = 0.7, 1e-4, 0.8
        self.coupled, self.chains, self.length = True, 0, 0
        self.n = int(self.sizes.max())

    def name(self):
        return ('%d replicas, cubic edges U{16..64} and U{20..200} Lennard-Jones beads (seed %d): periodic fluctuating '
                'D3Q19, tau 0.7, kT 1e-4, three-point stencil, explicit drag 0.8 (lattice units)' % (self.replicas, self.seed))

    def fluid_nodes(self):
        return int((self.sizes.astype(np.int64)**3).sum())

    def lattices(self, lbm):
        out = []
        for r, (n, b) in enumerate(zip(self.sizes, self.beads)):
            force = lbm.LBMForce()
            force.setGridSize(int(n), int(n), int(n))
            force.setFluidDensity(1.0)
            force.setKinematicViscosity((self.tau - 0.5)/3.0)
            force.setFluidFluctuations(True)
            force.setTemperature(self.kT/BOLTZ)
            force.setRandomNumberSeed(self.seed + 1 + r)
            force.setInterpolationStencil(force.ThreePoint)
            force.setDragScheme(force.Explicit)
            force.setFriction(self.friction)
            for i in range(int(b)):
                force.addParticle(i)
            out.append(force.latticeParameters(np.array([n, n, n], dtype=float), 1.0, np.ones(int(b))))
        return out

    def positions(self, min_distance=1.0):
        rng = np.random.Generator(np.random.PCG64(self.seed + 1))
        out = []
        for n, b in zip(self.sizes, self.beads):
            pts = np.zeros((0, 3))
            while len(pts) < b:
                x = rng.uniform(0, n, 3)
                d = pts - x
                d -= n*np.round(d/n)
                if len(pts) == 0 or (d*d).sum(axis=1).min() >= min_distance**2:
                    pts = np.vstack([pts, x])
            out.append(pts)
        return out

    def sample(self, n):
        return BatchWorkload(replicas=n, seed=self.seed)


def run_batch(args, w, rank, world, device):
    """The replica batch: every phase one launch over all replicas, runs of graph_steps steps replayed from a CUDA
    graph; the dense kernel's block size chosen by the autotuner."""
    import torch
    lbm = load_package()
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream()
    lattices = w.lattices(lbm)
    positions = w.positions()
    beads = int(w.beads.sum())
    batch = lbm.ReplicaBatch(lattices, w.beads, np.ones(beads), np.concatenate(positions),
                             pair=('lj', 1.0, w.kT, 2.5), precision=args.precision, device=device,
                             stream=stream.cuda_stream)
    graph_steps = args.graph_steps
    threads, dense_ms = batch.autotune(graph_steps)
    batch.step(max(args.warmup, 3)*graph_steps)
    torch.cuda.synchronize()
    launches0 = batch.info()['launches']
    clock_path = os.path.join(tempfile.gettempdir(), 'lbm_clocks_%d.csv' % rank)
    sampler = start_clock_sampler(clock_path) if rank == 0 else None
    time.sleep(0.5 if sampler else 0.0)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    batch.step(args.steps)
    stop.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = stop_clock_sampler(sampler, clock_path, device) if sampler else None
    ms = start.elapsed_time(stop)
    launches = batch.info()['launches'] - launches0
    if world > 1:
        ms = max_over_ranks(ms)
    # End to end through the C ABI: every run of graph_steps steps takes the beads' velocities from host memory and
    # returns their positions and velocities to host memory.
    pos_h, vel_h = batch.particles_state()
    chunks = max(1, args.steps//graph_steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(chunks):
        batch.set_velocities(vel_h)
        batch.step(graph_steps)
        pos_h, vel_h = batch.particles_state()
    e2e_s = time.perf_counter() - t0
    fluid_kT, bead_kT = batch.temperatures()
    nodes = w.fluid_nodes()
    observables = {'fluid_kT_over_kT_mean': float(np.mean(fluid_kT)/w.kT),
                   'fluid_kT_over_kT_range': [float(fluid_kT.min()/w.kT), float(fluid_kT.max()/w.kT)],
                   'bead_kT_over_kT_mean': float(np.mean(bead_kT)/w.kT),
                   'steps_run': int(batch.info()['steps'])}
    batch.close()
    if args.separate:
        observables['separate_launches_mlups'] = separate_launch_mlups(lbm, w, lattices, positions, args.precision, 3)
    bytes_per_node = 2*19*STORAGE_BYTES[args.precision]
    achieved = bytes_per_node*nodes/(dense_ms*1e-3)/1e9
    peak, peak_kind = peaks()
    v3 = 3*8*beads
    return {
        'metric': 'MLUPS (fluid nodes x lattice steps / s) of the batched replica step',
        'value': world*nodes*args.steps/(ms*1e-3)/1e6, 'unit': 'MLUPS', 'n_gpus': world, 'steps': args.steps,
        'warmup': max(args.warmup, 3)*graph_steps, 'ms_per_step': ms/args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': DTYPE[args.precision],
        'data': 'synthetic: seeded replica sizes, bead counts and positions, thermal noise from Philox',
        'config': {'workload': w.name(), 'replicas': w.replicas, 'nodes_per_gpu': nodes, 'beads_per_gpu': beads,
                   'storage': args.precision, 'graph_steps': graph_steps, 'dense_threads_per_block': threads,
                   'l2': 'inputs larger than L2 (2 x %.2f GB of populations)' % (19*nodes*STORAGE_BYTES[args.precision]/1e9),
                   'parallelism': 'independent replica batches, one per GPU' if world > 1 else 'single GPU'},
        'roofline': {'bound': 'hbm', 'kernel': 'batchStreamCollideKernel', 'achieved': achieved, 'peak': peak,
                     'unit': 'GB/s', 'frac': achieved/peak, 'peak_kind': peak_kind,
                     'algorithmic_bytes_per_launch': bytes_per_node*nodes, 'algorithmic_bytes_per_node': bytes_per_node,
                     'avg_launch_ms': dense_ms, 'launches': 5, 'traffic': None},
        'e2e': {'value': world*nodes*chunks*graph_steps/e2e_s/1e6, 'unit': 'MLUPS',
                'h2d_bytes_per_step': v3/graph_steps, 'd2h_bytes_per_step': 2*v3/graph_steps,
                'steps': chunks*graph_steps},
        'gpu_launches': launches,
        'clocks': clocks,
        'observables': observables,
    }


def separate_launch_mlups(lbm, w, lattices, positions, precision, steps):
    """The same replicas as separate kernels (one B200Kernel and one BeadDynamics each, launched replica after
    replica on one stream): MLUPS over `steps` steps after one warm-up step."""
    import torch
    stream = torch.cuda.Stream()
    runs = []
    for lattice, pos, n in zip(lattices, positions, w.sizes):
        m = np.ones(len(pos))
        kernel = lbm.B200Kernel(lattice, m, [], precision, stream=stream.cuda_stream)
        md = lbm.BeadDynamics(m, (n, n, n), np.zeros((0, 2), dtype=np.int32), k=0.0, r0=1.0, pair='lj', sigma=1.0,
                              epsilon=w.kT, cutoff=2.5)
        p = torch.tensor(pos, device='cuda', dtype=torch.float64)
        runs.append((kernel, md, p, torch.zeros_like(p), torch.zeros_like(p)))

    def advance(s):
        for kernel, md, p, v, f in runs:
            kernel.begin_step(s, p, v, f)
            md.compute_forces(p, f, stream.cuda_stream)
            kernel.execute(s, p, v, f)
            md.integrate(1.0, p, v, f, stream.cuda_stream)

    advance(0)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for s in range(1, steps + 1):
        advance(s)
    stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    for kernel, md, *_ in runs:
        kernel.close()
        md.close()
    return w.fluid_nodes()*steps/(ms*1e-3)/1e6


def max_over_ranks(value):
    """The largest of a value over the ranks of the job (a time: the slowest rank sets the job's time).  Every rank
    takes this collective at the same point; with the NCCL backend the value goes through the rank's GPU."""
    import torch
    device = 'cuda' if torch.distributed.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_mlups(world, nodes, steps, ms):
    """Node updates per second of the whole job: every rank advances its own replica of `nodes` nodes (replicas only,
    no exchange), so the job updates world x nodes x steps nodes in the slowest rank's time."""
    return world*nodes*steps/(ms*1e-3)/1e6


def peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return float(data['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


def start_clock_sampler(path):
    try:
        return subprocess.Popen(
            ['nvidia-smi', '--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap',
             '--format=csv,noheader,nounits', '-lms', '200'], stdout=open(path, 'w'), stderr=subprocess.DEVNULL)
    except (FileNotFoundError, OSError):
        return None


def stop_clock_sampler(proc, path, device):
    if proc is None:
        return None
    proc.terminate()
    proc.wait()
    sm, smax, reasons = [], 0.0, set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
    for line in open(path):
        parts = [p.strip() for p in line.split(',')]
        if len(parts) < 9 or parts[0] != str(device):
            continue
        try:
            sm.append(float(parts[1]))
            smax = max(smax, float(parts[2]))
        except ValueError:
            continue
        for name, flag in zip(names, parts[5:9]):
            if flag.lower() == 'active':
                reasons.add(name)
    if not sm:
        return None
    return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': smax, 'reasons': sorted(reasons), 'samples': len(sm)}


def run_b200(args, w, rank, world, device):
    import torch
    lbm = load_package()
    torch.cuda.set_device(device)
    lattice = w.lattice(lbm)
    np_ = w.chains*w.length
    masses = np.ones(np_)
    # The kernel launches on a stream that torch owns, so that the pinned copies of the e2e loop (which torch
    # orders with events on that stream) outlive nothing they depend on.
    stream = torch.cuda.Stream()
    stream_ptr = stream.cuda_stream
    kernel = lbm.B200Kernel(lattice, masses, w.solids(), args.precision, device=device, stream=stream_ptr)
    lib = kernel.lib
    nodes = w.fluid_nodes()
    md = None
    if np_ > 0:
        pos0, bonds = w.beads(lbm)
        md = lbm.BeadDynamics(masses, w.shape, bonds, device=device, **w.md_parameters())
        pos = torch.tensor(pos0, device='cuda', dtype=torch.float64)
        vel = torch.zeros_like(pos)
        frc = torch.zeros_like(pos)
    dist = world > 1

    def barrier():
        if dist:
            torch.distributed.barrier()

    def step(s, after_begin=None):
        if md is None:
            kernel.begin_step(s)
            kernel.execute(s)
            return
        kernel.begin_step(s, pos, vel, frc)
        if after_begin is not None:
            after_begin()
        md.compute_forces(pos, frc, stream_ptr)
        kernel.execute(s, pos, vel, frc)
        md.integrate(1.0, pos, vel, frc, stream_ptr)

    s = 0
    for _ in range(args.warmup):
        step(s)
        s += 1
    torch.cuda.synchronize()
    launches0 = ctypes.c_longlong()
    lib.lbm_kernel_launches(kernel.handle, ctypes.byref(launches0))
    md0 = md.launches() if md else 0
    lib.lbm_profile_dense_kernel(kernel.handle, 1)
    clock_path = os.path.join(tempfile.gettempdir(), 'lbm_clocks_%d.csv' % rank)
    sampler = start_clock_sampler(clock_path) if rank == 0 else None
    time.sleep(0.5 if sampler else 0.0)
    barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step(s)
        s += 1
    stop.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = stop_clock_sampler(sampler, clock_path, device) if sampler else None
    ms = start.elapsed_time(stop)
    dense_launches, dense_ms = ctypes.c_longlong(), ctypes.c_double()
    lib.lbm_dense_kernel_time(kernel.handle, ctypes.byref(dense_launches), ctypes.byref(dense_ms))
    lib.lbm_profile_dense_kernel(kernel.handle, 0)
    launches1 = ctypes.c_longlong()
    lib.lbm_kernel_launches(kernel.handle, ctypes.byref(launches1))
    gpu_launches = int(launches1.value - launches0.value) + ((md.launches() - md0) if md else 0)
    if dist:
        ms = max_over_ranks(ms)

    # End to end through the C ABI with the particles in pinned host memory: every step copies the beads'
    # positions and velocities to the device, runs the step, and reads them back.  Without solid nodes begin_step
    # reads the positions only (the reflection at walls also changes velocities), so the velocities' copy is issued
    # after it and overlaps the stencil pass that begin_step starts on the kernel's second stream.
    e2e_steps = max(3, args.steps//2)
    late_velocities = md is not None and len(w.solids()) == 0

    def copy_velocities():
        with torch.cuda.stream(stream):
            vel.copy_(vel_h, non_blocking=True)

    h2d = d2h = 0
    if md is not None:
        pos_h = pos.cpu().pin_memory()
        vel_h = vel.cpu().pin_memory()
        h2d = d2h = 2*pos.numel()*8
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        if md is not None:
            with torch.cuda.stream(stream):
                pos.copy_(pos_h, non_blocking=True)
                if not late_velocities:
                    vel.copy_(vel_h, non_blocking=True)
        step(s, copy_velocities if late_velocities else None)
        if md is not None:
            with torch.cuda.stream(stream):
                pos_h.copy_(pos, non_blocking=True)
                vel_h.copy_(vel, non_blocking=True)
        stream.synchronize()
        s += 1
    e2e_s = time.perf_counter() - t0
    if dist:
        e2e_s = max_over_ranks(e2e_s)

    observables = {}
    if rank == 0 and args.observables:
        density, velocity = kernel.get_fluid_fields()
        rho = density/1.0
        u = velocity - (velocity*rho[:, None]).sum(axis=0)/rho.sum()
        observables['fluid_kT'] = float((rho[:, None]*u*u).mean())
        if md is not None:
            observables['bead_kT'] = md.twice_kinetic(vel, stream_ptr)/(3*np_)
            observables['steps_run'] = s
            iterations = ctypes.c_int()
            lib.lbm_solver_iterations(kernel.handle, ctypes.byref(iterations))
            observables['cg_iterations_last_step'] = iterations.value
    kernel.close()

    value = job_mlups(world, nodes, args.steps, ms)
    e2e_value = job_mlups(world, nodes, e2e_steps, e2e_s*1e3)
    bytes_per_node = 2*19*STORAGE_BYTES[args.precision]
    avg_dense_s = dense_ms.value*1e-3/max(1, dense_launches.value)
    achieved = bytes_per_node*nodes/avg_dense_s/1e9
    peak, peak_kind = peaks()
    config = {'workload': w.name(), 'nodes_per_gpu': nodes, 'beads_per_gpu': np_, 'storage': args.precision,
              'momentum_removal_frequency': 0 if isinstance(w, ChannelWorkload) else 1, 'mach_check_frequency': 100,
              'l2': 'inputs larger than L2 (2 x %.2f GB of populations)' % (19*nodes*STORAGE_BYTES[args.precision]/1e9),
              'parallelism': 'independent replicas, one per GPU' if world > 1 else 'single GPU'}
    return {
        'metric': metric_name(w),
        'value': value, 'unit': 'MLUPS', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms/args.steps, 'coupled_steps_per_s': 1e3*args.steps/ms, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': DTYPE[args.precision],
        'data': data_name(w), 'config': config,
        'roofline': {'bound': 'hbm', 'kernel': dense_kernel_name(args, w), 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved/peak, 'peak_kind': peak_kind, 'algorithmic_bytes_per_launch': bytes_per_node*nodes,
                     'algorithmic_bytes_per_node': bytes_per_node, 'avg_launch_ms': avg_dense_s*1e3,
                     'launches': dense_launches.value, 'traffic': traffic_per_launch(args, w)},
        'e2e': {'value': e2e_value, 'unit': 'MLUPS', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                'steps': e2e_steps},
        'gpu_launches': gpu_launches,
        'clocks': clocks,
        'observables': observables,
    }


def plain_fluid_record(args, w, rank, world, device):
    """The dense step of the plain fluid of the same lattice (no particles, no fluctuations, the same storage), timed
    like the main record: its MLUPS and the roofline fraction of its dense kernel."""
    import copy
    plain = Workload(n=w.n, coupled=False, fluctuations=False, seed=w.seed)
    sub = copy.copy(args)
    sub.observables = False
    r = run_b200(sub, plain, rank, world, device)
    return {'workload': plain.name(), 'value': r['value'], 'unit': 'MLUPS', 'ms_per_step': r['ms_per_step'],
            'dense_kernel_ms': r['roofline']['avg_launch_ms'], 'roofline_frac': r['roofline']['frac'],
            'achieved_gbs': r['roofline']['achieved'], 'peak_gbs': r['roofline']['peak'],
            'gpu_launches': r['gpu_launches'], 'clocks': r['clocks']}


WARMSTART_WEIGHTS = os.path.join(PACKAGE, 'warmstart_net', 'weights.pt')


def warm_start_record(cases, first_seed=300001):
    """The metric's time-to-steady part: `cases` obstacle channels (128x64x64, seeds the network never saw) solved to
    the steady residual 1e-6 from rest and from the learned warm start (openmm-lbm_b200/warmstart_net/weights.pt), one
    solve at a time; value = total cold wall time / total warm wall time (the prediction included)."""
    load_package()
    from lbm_b200 import warmstart
    net = warmstart.load_network(WARMSTART_WEIGHTS)
    rows = warmstart.time_to_steady(net, list(range(first_seed, first_seed + cases)))
    cold = sum(r['cold_seconds'] for r in rows)
    warm = sum(r['warm_seconds'] for r in rows)
    return {'metric': 'time to steady state (residual 1e-6) from rest / from the learned warm start',
            'value': cold/warm, 'unit': 'x', 'cases': len(rows),
            'workload': '128x64x64 obstacle channel, 5-20 spheres of radius 4-10, Velocity inlet 0.02, Density outlet, '
                        'tau 0.6, FP32 (held-out seeds %d..%d)' % (first_seed, first_seed + cases - 1),
            'cold_seconds_mean': cold/len(rows), 'warm_seconds_mean': warm/len(rows),
            'cold_steps_mean': float(np.mean([r['cold_steps'] for r in rows])),
            'warm_steps_mean': float(np.mean([r['warm_steps'] for r in rows])),
            'speedup_per_case': [round(r['speedup'], 3) for r in rows],
            'final_velocity_error_max': float(max(r['final_velocity_error'] for r in rows))}


def host_description():
    """The host's logical core count and CPU model (the CPU baseline runs on one of these cores)."""
    model = 'unknown'
    try:
        for line in open('/proc/cpuinfo'):
            if line.startswith('model name'):
                model = line.split(':', 1)[1].strip()
                break
    except OSError:
        pass
    return {'nproc': os.cpu_count(), 'cpu_model': model, 'threads_used': 1}


def metric_name(w):
    return 'MLUPS (fluid nodes x lattice steps / s) of the %s lattice step' % ('coupled' if w.coupled else 'fluid')


def data_name(w):
    if w.coupled:
        return 'synthetic: seeded random-walk chains in a fluid at rest, thermal noise from Philox'
    if w.kT > 0:
        return 'synthetic: a fluid at rest, thermal noise from Philox'
    return 'synthetic: a fluid started from rest'


def dense_kernel_name(args, w):
    """The dense kernel that the library launches for this workload: four nodes per thread for 16-bit storage without
    fluctuations (nx a multiple of 4), two for FP32 and 16-bit storage (nx even), else one."""
    nx = w.shape[0]
    fluct = getattr(w, 'kT', 0) > 0
    if args.precision in ('half', 'bfloat16') and not fluct and nx % 4 == 0 and os.environ.get('LBM_B200_QUAD16') != '0':
        return 'streamCollideQuadKernel'
    if args.precision != 'double' and nx % 2 == 0:
        return 'streamCollidePairKernel'
    return 'streamCollideKernel'


def traffic_per_launch(args, w):
    """DRAM bytes per launch of the dense kernel from the committed ncu summary of this variant, if there is one."""
    name = 'stream_collide_%s_%s.md' % ({'double': 'f64', 'single': 'f32', 'half': 'f16', 'bfloat16': 'bf16'}[args.precision],
                                       w.profile_tag())
    path = os.path.join(ROOT, 'profiles', name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith('traffic_bytes_per_launch:'):
            return float(line.split(':')[1])
    return None


def cpu_step_fn(lbm, oracle, w, kernel, pos, vel, bonds, masses):
    params = w.md_parameters() if len(pos) else None
    box = np.array(w.shape, dtype=float)
    frc = np.zeros_like(pos)

    def step(s):
        kernel.begin_step(s, pos, vel, frc)
        if len(pos):
            frc[:] = oracle.md_forces(pos, box, bonds, params['k'], params['r0'], params['pair'], params['sigma'],
                                      params['epsilon'], params['cutoff'])
        kernel.execute(s, pos, vel, frc)
        if len(pos):
            vel[:] += frc/masses[:, None]
            pos[:] += vel
    return step


def run_cpu(args, w, steps, warmup):
    """The reference's kernel (oracle/_ref; the C restatement where the reference was not built) on the host cores,
    on the sample w of the workload; single-threaded, as the reference.  Returns (MLUPS, kind, seconds per step)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    lbm = load_package()
    import oracle
    kind = 'reference' if oracle.reference_available() else 'port'
    factory = oracle.ReferenceKernel if kind == 'reference' else oracle.OracleKernel
    lattice = w.lattice(lbm)
    np_ = w.chains*w.length
    masses = np.ones(np_)
    kernel = factory(lattice, masses, w.solids())
    if np_:
        pos, bonds = w.beads(lbm)
    else:
        pos, bonds = np.zeros((0, 3)), np.zeros((0, 2), dtype=np.int32)
    pos = np.ascontiguousarray(pos)
    vel = np.zeros_like(pos)
    step = cpu_step_fn(lbm, oracle, w, kernel, pos, vel, bonds, masses)
    s = 0
    for _ in range(warmup):
        step(s)
        s += 1
    t0 = time.perf_counter()
    for _ in range(steps):
        step(s)
        s += 1
    dt = (time.perf_counter() - t0)/steps
    kernel.close()
    return w.fluid_nodes()/dt/1e6, kind, dt


def run_cpu_batch(w, steps, warmup, count=4):
    """The reference's kernel (oracle/_ref; else the C restatement) on the first `count` replicas of the batch, one
    after another on one core, with the oracle's CPU bead forces and leapfrog.  Returns (MLUPS, kind, seconds per
    step of the sample, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    lbm = load_package()
    import oracle
    kind = 'reference' if oracle.reference_available() else 'port'
    factory = oracle.ReferenceKernel if kind == 'reference' else oracle.OracleKernel
    lattices = w.lattices(lbm)[:count]
    positions = w.positions()[:count]
    runs = []
    for lattice, pos, n in zip(lattices, positions, w.sizes[:count]):
        m = np.ones(len(pos))
        runs.append((factory(lattice, m, []), np.ascontiguousarray(pos), np.zeros_like(pos), m, float(n)))
    no_bonds = np.zeros((0, 2), dtype=np.int32)

    def advance(s):
        for kernel, pos, vel, m, n in runs:
            frc = np.zeros_like(pos)
            kernel.begin_step(s, pos, vel, frc)
            frc[:] = oracle.md_forces(pos, np.array([n, n, n]), no_bonds, 0.0, 1.0, 'lj', 1.0, w.kT, 2.5)
            kernel.execute(s, pos, vel, frc)
            vel[:] += frc/m[:, None]
            pos[:] += vel

    for s in range(warmup):
        advance(s)
    t0 = time.perf_counter()
    for s in range(warmup, warmup + steps):
        advance(s)
    dt = (time.perf_counter() - t0)/steps
    for kernel, *_ in runs:
        kernel.close()
    nodes = int((w.sizes[:count].astype(np.int64)**3).sum())
    sample = ('per step, the first %d replicas (%d nodes, %d beads) one after another' %
              (count, nodes, int(w.beads[:count].sum())))
    return nodes/dt/1e6, kind, dt, sample


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument('--gpus', type=int, default=1)
    parser.add_argument('--steps', type=int, default=30)
    parser.add_argument('--warmup', type=int, default=5)
    parser.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    parser.add_argument('--workload', default='coupled', choices=['coupled', 'fluid', 'channel', 'batch', 'warmstart'])
    parser.add_argument('--precision', default='single', choices=list(STORAGE_BYTES))
    parser.add_argument('--size', type=int, default=0, help='lattice edge in x (smaller cases for profiling)')
    parser.add_argument('--no-fluctuations', action='store_true')
    parser.add_argument('--no-cpu-baseline', action='store_true')
    parser.add_argument('--no-observables', dest='observables', action='store_false',
                        help='skip the fluid and bead temperatures after the run')
    parser.add_argument('--no-plain-fluid', action='store_true',
                        help='skip the record of the plain fluid (no particles, no fluctuations) of the same size')
    parser.add_argument('--warm-start-cases', type=int, default=4,
                        help='held-out channels of the time-to-steady record (0: none)')
    parser.add_argument('--graph-steps', type=int, default=10, help='batch: lattice steps per CUDA graph')
    parser.add_argument('--replicas', type=int, default=256, help='batch: number of replicas')
    parser.add_argument('--separate', action='store_true', help='batch: also time the replicas as separate kernels')
    args = parser.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.workload == 'warmstart':
        # The learned warm start alone: time to the steady residual from rest and from the network's prediction.
        if rank == 0:
            record = warm_start_record(max(1, args.steps))
            record.update({'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True,
                           'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic obstacle channels'})
            print(json.dumps(record))
        return
    if args.workload == 'channel':
        base = ChannelWorkload()
    elif args.workload == 'batch':
        base = BatchWorkload(replicas=args.replicas)
    else:
        base = Workload(coupled=args.workload == 'coupled', fluctuations=not args.no_fluctuations)
    if args.workload == 'batch':
        w = base
    else:
        w = base.sample(args.size) if args.size and args.size != base.shape[0] else base
    if args.impl == 'reference' and args.workload == 'batch':
        if rank != 0:
            return
        value, kind, dt, sample = run_cpu_batch(w, args.steps, args.warmup)
        print(json.dumps({
            'metric': 'MLUPS (fluid nodes x lattice steps / s) of the batched replica step', 'impl': 'reference',
            'value': value, 'unit': 'MLUPS', 'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': dt*1e3, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic', 'config': {'workload': w.name(), 'sample': sample},
            'cpu_baseline': {'value': value, 'unit': 'MLUPS', 'cores': 1, 'kind': kind, 'sample': sample,
                             'host': host_description()},
            'e2e': {'value': value, 'unit': 'MLUPS', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}))
        return
    if args.impl == 'reference':
        if rank != 0:
            return
        # Each step is a bounded sample: a 128^3 lattice with 1/8 of the beads (the same densities and per-node
        # work); the reference takes ~30 s per step of the full 256^3 fluid on one core.
        sample = w.sample(min(w.shape[0], 128))
        value, kind, dt = run_cpu(args, sample, args.steps, args.warmup)
        print(json.dumps({
            'metric': metric_name(w), 'impl': 'reference',
            'value': value, 'unit': 'MLUPS', 'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': dt*1e3, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic', 'config': {'workload': w.name(), 'sample': sample.name()},
            'cpu_baseline': {'value': value, 'unit': 'MLUPS', 'cores': 1, 'kind': kind,
                             'sample': 'per step, %s (the same per-node and per-bead work)' % sample.name(),
                             'host': host_description()},
            'e2e': {'value': value, 'unit': 'MLUPS', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}))
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local)
        torch.distributed.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    if args.workload == 'batch':
        result = run_batch(args, w, rank, world, local)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            value, kind, dt, sample = run_cpu_batch(w, 1, 1)
            result['cpu_baseline'] = {'value': value, 'unit': 'MLUPS', 'cores': 1, 'kind': kind, 'sample': sample}
    else:
        result = run_b200(args, w, rank, world, local)
        if args.workload == 'coupled' and not args.no_plain_fluid:
            result['plain_fluid'] = plain_fluid_record(args, w, rank, world, local)
        if args.workload == 'coupled' and rank == 0 and args.warm_start_cases > 0 and os.path.exists(WARMSTART_WEIGHTS):
            result['warm_start'] = warm_start_record(args.warm_start_cases)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload != 'batch':
        sample = w.sample(min(w.shape[0], 128))
        value, kind, dt = run_cpu(args, sample, 2, 1)
        result['cpu_baseline'] = {'value': value, 'unit': 'MLUPS', 'cores': 1, 'kind': kind,
                                  'sample': 'two timed steps after one warm-up of %s' % sample.name(),
                                  'host': host_description()}
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == '__main__':
    main()
