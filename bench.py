"""Benchmark of the per-step fluid and coupling path on B200: MLUPS and the HBM roofline of the dense kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--precision single]

Workload: the 256^3 periodic fluctuating fluid of the scale configuration (tau = 0.6, kT = 1e-4 in lattice
units, Philox seed), FP32 storage, momentum removal every step, Mach check every 100 steps.  One step is
one lattice step (beginStep + execute through the C ABI).  With N > 1 (torchrun, one rank per GPU) every rank
advances its own lattice (replicas, no collective on the data path); value = all ranks' node updates / the
slowest rank's time.  --impl reference times the reference's own Reference-platform kernel (oracle/_ref,
compiled unmodified from the reference sources) on the host cores, on a bounded sample of the same workload.
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


def load_package():
    if 'lbm_b200' in sys.modules:
        return sys.modules['lbm_b200']
    spec = importlib.util.spec_from_file_location('lbm_b200', os.path.join(PACKAGE, '__init__.py'),
                                                  submodule_search_locations=[PACKAGE])
    module = importlib.util.module_from_spec(spec)
    sys.modules['lbm_b200'] = module
    spec.loader.exec_module(module)
    return module


WORKLOAD = {'name': '256^3 periodic fluctuating D3Q19 fluid, tau 0.6, kT 1e-4 (lattice units)',
            'n': 256, 'tau': 0.6, 'kT': 1e-4, 'seed': 2026}
STORAGE_BYTES = {'double': 8, 'single': 4, 'half': 2, 'bfloat16': 2}


def lattice_parameters(lbm, n, tau, kT, seed):
    """The workload in lattice units: dx = dt = 1, rho0 = 1, temperature with BOLTZ T = kT."""
    force = lbm.LBMForce()
    force.setGridSize(n, n, n)
    force.setFluidDensity(1.0)
    force.setKinematicViscosity((tau - 0.5)/3.0)
    force.setFluidFluctuations(kT > 0)
    force.setTemperature(kT/BOLTZ)
    force.setRandomNumberSeed(seed)
    return force.latticeParameters(np.array([n, n, n], dtype=float), 1.0, np.array([1.0]))


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


def workload(args):
    w = dict(WORKLOAD)
    if args.size != w['n'] or args.no_fluctuations:
        w['n'] = args.size
        w['kT'] = 0.0 if args.no_fluctuations else w['kT']
        w['name'] = '%d^3 periodic D3Q19 fluid, tau 0.6%s (lattice units)' % (
            args.size, '' if args.no_fluctuations else ', kT 1e-4, fluctuating')
    return w


def run_b200(args, rank, world, device):
    import torch
    lbm = load_package()
    torch.cuda.set_device(device)
    w = workload(args)
    lattice = lattice_parameters(lbm, w['n'], w['tau'], w['kT'], w['seed'] + rank)
    kernel = lbm.B200Kernel(lattice, [], [], args.precision, device=device)
    lib = kernel.lib
    nodes = w['n']**3
    stream = torch.cuda.ExternalStream(kernel.stream())
    dist = world > 1

    def barrier():
        if dist:
            torch.distributed.barrier()

    step = 0
    for _ in range(args.warmup):
        kernel.begin_step(step)
        kernel.execute(step)
        step += 1
    torch.cuda.synchronize()
    launches0 = ctypes.c_longlong()
    lib.lbm_kernel_launches(kernel.handle, ctypes.byref(launches0))
    lib.lbm_profile_dense_kernel(kernel.handle, 1)
    clock_path = os.path.join(tempfile.gettempdir(), 'lbm_clocks_%d.csv' % rank)
    sampler = start_clock_sampler(clock_path) if rank == 0 else None
    time.sleep(0.5 if sampler else 0.0)
    barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        kernel.begin_step(step)
        kernel.execute(step)
        step += 1
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
    if dist:
        t = torch.tensor([ms], device='cuda')
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())

    # End to end through the C ABI with host buffers: each step is driven from the host, and a device-to-host
    # read of the step's wall-force statistics (24 bytes) closes it.
    e2e_steps = max(3, args.steps//2)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        kernel.begin_step(step)
        kernel.execute(step)
        kernel.get_wall_force()
        step += 1
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device='cuda')
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    kernel.close()

    value = world*nodes*args.steps/(ms*1e-3)/1e6
    e2e_value = world*nodes*e2e_steps/e2e_s/1e6
    bytes_per_node = 2*19*STORAGE_BYTES[args.precision]
    avg_dense_s = dense_ms.value*1e-3/max(1, dense_launches.value)
    achieved = bytes_per_node*nodes/avg_dense_s/1e9
    peak, peak_kind = peaks()
    result = {
        'metric': 'MLUPS (lattice node updates per second, fluid nodes x steps / time)',
        'value': value, 'unit': 'MLUPS', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms/args.steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': {'double': 'f64', 'single': 'f32', 'half': 'f16 storage, f32 compute',
                  'bfloat16': 'bf16 storage, f32 compute'}[args.precision],
        'data': 'synthetic: fluid at rest with thermal fluctuations from Philox (seeded)',
        'config': {'workload': w['name'], 'nodes_per_gpu': nodes, 'storage': args.precision,
                   'momentum_removal_frequency': 1, 'mach_check_frequency': 100,
                   'l2': 'inputs larger than L2 (2 x %.2f GB of populations)' % (19*nodes*STORAGE_BYTES[args.precision]/1e9),
                   'parallelism': 'replicas' if world > 1 else 'single GPU'},
        'roofline': {'bound': 'hbm', 'kernel': 'streamCollideKernel', 'achieved': achieved, 'peak': peak,
                     'unit': 'GB/s', 'frac': achieved/peak, 'peak_kind': peak_kind,
                     'algorithmic_bytes_per_launch': bytes_per_node*nodes,
                     'avg_launch_ms': avg_dense_s*1e3, 'launches': dense_launches.value, 'traffic': None},
        'e2e': {'value': e2e_value, 'unit': 'MLUPS', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 24,
                'steps': e2e_steps},
        'gpu_launches': int(launches1.value - launches0.value),
        'clocks': clocks,
    }
    return result


def run_cpu_baseline(precision_unused=None):
    """The reference's Reference-platform kernel (oracle/_ref) on the host: one warm-up and one timed step of the
    full 256^3 workload (FP64, single-threaded: the reference has no threads)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    lbm = load_package()
    import oracle
    kind = 'reference' if oracle.reference_available() else 'port'
    factory = oracle.ReferenceKernel if kind == 'reference' else oracle.OracleKernel
    w = WORKLOAD
    n = w['n']
    lattice = lattice_parameters(lbm, n, w['tau'], w['kT'], w['seed'])
    kernel = factory(lattice, [], [])
    kernel.begin_step(0)
    kernel.execute(0)
    t0 = time.perf_counter()
    kernel.begin_step(1)
    kernel.execute(1)
    dt = time.perf_counter() - t0
    kernel.close()
    return {'value': n**3/dt/1e6, 'unit': 'MLUPS', 'cores': 1, 'kind': kind,
            'sample': 'one timed lattice step of the full %d^3 workload after one warm-up step (FP64)' % n}


def run_reference_arm(args, rank):
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    lbm = load_package()
    import oracle
    kind = 'reference' if oracle.reference_available() else 'port'
    factory = oracle.ReferenceKernel if kind == 'reference' else oracle.OracleKernel
    # Each step is a bounded sample of the workload: a 128^3 lattice with the same per-node work (the reference is
    # single-threaded and takes ~28 s per 256^3 step), so that K + W steps end within a few minutes.
    w = WORKLOAD
    n = 128
    lattice = lattice_parameters(lbm, n, w['tau'], w['kT'], w['seed'])
    kernel = factory(lattice, [], [])
    step = 0
    for _ in range(args.warmup):
        kernel.begin_step(step)
        kernel.execute(step)
        step += 1
    t0 = time.perf_counter()
    for _ in range(args.steps):
        kernel.begin_step(step)
        kernel.execute(step)
        step += 1
    dt = time.perf_counter() - t0
    kernel.close()
    value = n**3*args.steps/dt/1e6
    return {'metric': 'MLUPS (lattice node updates per second, fluid nodes x steps / time)', 'impl': 'reference',
            'value': value, 'unit': 'MLUPS', 'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': dt*1e3/args.steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f64', 'data': 'synthetic', 'config': {'workload': w['name'], 'sample_nodes': n**3},
            'cpu_baseline': {'value': value, 'unit': 'MLUPS', 'cores': 1, 'kind': kind,
                             'sample': '%d^3 sub-lattice of the workload per step (same per-node work)' % n},
            'e2e': {'value': value, 'unit': 'MLUPS', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument('--gpus', type=int, default=1)
    parser.add_argument('--steps', type=int, default=50)
    parser.add_argument('--warmup', type=int, default=5)
    parser.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    parser.add_argument('--precision', default='single', choices=list(STORAGE_BYTES))
    parser.add_argument('--no-cpu-baseline', action='store_true')
    parser.add_argument('--size', type=int, default=WORKLOAD['n'], help='lattice edge (profiling of smaller cases)')
    parser.add_argument('--no-fluctuations', action='store_true', help='plain fluid (profiling of the kernel variant)')
    args = parser.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        result = run_reference_arm(args, rank)
        if result is not None:
            print(json.dumps(result))
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local)
        torch.distributed.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    result = run_b200(args, rank, world, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result['cpu_baseline'] = run_cpu_baseline()
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == '__main__':
    main()
