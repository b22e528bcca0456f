"""Benchmark of the per-step fluid and particle-coupling path on B200: MLUPS, and the HBM roofline of the dense
stream-collide kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload coupled|fluid|channel]
                    [--precision double|single|half|bfloat16] [--size EDGE]

Workload "coupled" (default, the scale configuration): a 256^3 periodic fluctuating D3Q19 fluid (tau 0.6, kT 1e-4 in
lattice units, Philox seed), FP32 storage, momentum removal every step, Mach check every 100 steps; 512 bead-spring
chains of 100 beads (51,200 beads, mass 1) placed as seeded random walks, harmonic bonds (k = 100 kT/sigma^2, r0 = 1)
and WCA repulsion (sigma 1, epsilon = kT), coupled through the Keys stencil with the centred drag (friction 1 per
lattice step, solved by conjugate gradients on the device).  One step: beginStep, bead forces, execute (coupling +
fluid) and the leapfrog of the beads, all on the device.  "fluid": the fluid alone (kernel profiling).  "channel": the
precision configuration, a 384x384x192 Poiseuille channel between bounce-back planes (g_x 5e-7, tau 0.55), for the
MLUPS of each storage format.

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

    def step(s):
        if md is None:
            kernel.begin_step(s)
            kernel.execute(s)
            return
        kernel.begin_step(s, pos, vel, frc)
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
        t = torch.tensor([ms], device='cuda')
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())

    # End to end through the C ABI with the particles in pinned host memory: every step copies the beads'
    # positions and velocities to the device, runs the step, and reads them back.
    e2e_steps = max(3, args.steps//2)
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
                vel.copy_(vel_h, non_blocking=True)
        step(s)
        if md is not None:
            with torch.cuda.stream(stream):
                pos_h.copy_(pos, non_blocking=True)
                vel_h.copy_(vel, non_blocking=True)
        stream.synchronize()
        s += 1
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device='cuda')
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())

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

    value = world*nodes*args.steps/(ms*1e-3)/1e6
    e2e_value = world*nodes*e2e_steps/e2e_s/1e6
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
        'roofline': {'bound': 'hbm', 'kernel': 'streamCollideKernel', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved/peak, 'peak_kind': peak_kind, 'algorithmic_bytes_per_launch': bytes_per_node*nodes,
                     'algorithmic_bytes_per_node': bytes_per_node, 'avg_launch_ms': avg_dense_s*1e3,
                     'launches': dense_launches.value, 'traffic': traffic_per_launch(args, w)},
        'e2e': {'value': e2e_value, 'unit': 'MLUPS', 'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
                'steps': e2e_steps},
        'gpu_launches': gpu_launches,
        'clocks': clocks,
        'observables': observables,
    }


def metric_name(w):
    return 'MLUPS (fluid nodes x lattice steps / s) of the %s lattice step' % ('coupled' if w.coupled else 'fluid')


def data_name(w):
    if w.coupled:
        return 'synthetic: seeded random-walk chains in a fluid at rest, thermal noise from Philox'
    if w.kT > 0:
        return 'synthetic: a fluid at rest, thermal noise from Philox'
    return 'synthetic: a fluid started from rest'


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


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument('--gpus', type=int, default=1)
    parser.add_argument('--steps', type=int, default=30)
    parser.add_argument('--warmup', type=int, default=5)
    parser.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    parser.add_argument('--workload', default='coupled', choices=['coupled', 'fluid', 'channel'])
    parser.add_argument('--precision', default='single', choices=list(STORAGE_BYTES))
    parser.add_argument('--size', type=int, default=0, help='lattice edge in x (smaller cases for profiling)')
    parser.add_argument('--no-fluctuations', action='store_true')
    parser.add_argument('--no-cpu-baseline', action='store_true')
    parser.add_argument('--observables', action='store_true', help='fluid and bead temperatures after the run')
    args = parser.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.workload == 'channel':
        base = ChannelWorkload()
    else:
        base = Workload(coupled=args.workload == 'coupled', fluctuations=not args.no_fluctuations)
    w = base.sample(args.size) if args.size and args.size != base.shape[0] else base
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
                             'sample': 'per step, %s (the same per-node and per-bead work)' % sample.name()},
            'e2e': {'value': value, 'unit': 'MLUPS', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}))
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local)
        torch.distributed.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    result = run_b200(args, w, rank, world, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = w.sample(min(w.shape[0], 128))
        value, kind, dt = run_cpu(args, sample, 2, 1)
        result['cpu_baseline'] = {'value': value, 'unit': 'MLUPS', 'cores': 1, 'kind': kind,
                                  'sample': 'two timed steps after one warm-up of %s' % sample.name()}
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == '__main__':
    main()
