"""Multi-rank bench logic on CPU: world size 2 over gloo.

bench.py --gpus N runs one replica of the event per rank (the path has no
exchange step); the ranks meet only to take the slowest rank's time. These
tests cover that reduction and the reference arm's rank handling without a
GPU.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 10 + 5 r ms; every rank must see the slowest
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
        value = bench.aggregate_rate(1000, 4, ms, world)
        dist.barrier()
        with open(os.path.join(out_dir, 'rank%d.json' % rank), 'w') as f:
            json.dump({'ms': ms, 'value': value}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method='spawn')
    got = [json.load(open(os.path.join(str(tmp_path), 'rank%d.json' % r))) for r in range(world)]
    for g in got:
        assert g['ms'] == 15.0
        # 2 replicas x 1000 cells x 4 steps in 15 ms
        assert g['value'] == pytest.approx(2 * 1000 * 4 / 15e-3)


def test_single_rank_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.aggregate_rate(10, 2, 4.0, 1) == pytest.approx(10 * 2 / 4e-3)


def test_reference_arm_two_ranks(tmp_path):
    """Under torchrun with two ranks, rank 0 alone times the CPU path and
    prints one JSON line; rank 1 exits 0 without work."""
    env = dict(os.environ, OMP_NUM_THREADS='4')
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1', '--nproc-per-node', '2',
           '--master-addr', '127.0.0.1', '--master-port', str(_free_port()),
           os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--gpus', '2', '--steps', '1',
           '--warmup', '0', '--grid', '41,41,8']
    r = subprocess.run(cmd, cwd=str(tmp_path), env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith('{')]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d['impl'] == 'reference'
    assert d['n_gpus'] == 2
    assert d['value'] > 0 and d['e2e']['value'] == d['value']
    assert d['e2e']['h2d_bytes_per_step'] == 0 and d['e2e']['d2h_bytes_per_step'] == 0
    assert d['cpu_baseline']['kind'] == 'port' and d['cpu_baseline']['cores'] == 4
    assert '41x41x8' in d['cpu_baseline']['sample']
