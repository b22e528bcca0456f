"""CPU test of the multi-rank plumbing of bench.py, with two gloo ranks: the time every rank reports is the slowest
rank's (the MAX all-reduce that `bench.py --gpus N` takes under torchrun with NCCL), and the job's throughput counts
the replicas of every rank (replicas only: no exchange between ranks)."""
import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location('bench_under_test', os.path.join(ROOT, 'bench.py'))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, results):
    import datetime
    import torch.distributed as dist
    os.environ.update({'MASTER_ADDR': '127.0.0.1', 'MASTER_PORT': str(port)})
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = load_bench()
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + 5.0*rank)
        results[rank] = (ms, bench.job_mlups(world, 1000000, 20, ms))
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest_time_and_the_job_throughput():
    world = 2
    with mp.get_context('spawn').Manager() as manager:
        results = manager.dict()
        mp.start_processes(rank_main, args=(world, free_port(), results), nprocs=world, join=True,
                           start_method='spawn')
        got = dict(results)
    assert set(got) == {0, 1}
    for ms, mlups in got.values():
        assert ms == 15.0
        # 2 ranks x 1e6 nodes x 20 steps in 15 ms.
        assert mlups == pytest.approx(2*1e6*20/15e-3/1e6)
