"""Multi-rank host logic on CPU (gloo, world_size 2): replica seeding, the
max-over-ranks timing reduction, the whole-job rate, and the reference arm's
rank-0-only output under torchrun."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from shock_turbulence_b200.replicas import aggregate_rate, max_over_ranks, replica_seed
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = max_over_ranks(100.0 + 25.0 * rank, dist, "cpu")
        rate = aggregate_rate(1000, 4, ms, world)
        out.put((rank, replica_seed(1, rank), ms, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [1, 2]               # independent replicas
    assert all(r[2] == 125.0 for r in res)             # the slowest rank's time on every rank
    assert all(abs(r[3] - 2 * 1000 * 4 / 0.125 / 1e6) < 1e-12 for r in res)


def test_single_process_needs_no_group():
    from shock_turbulence_b200.replicas import aggregate_rate, max_over_ranks
    assert max_over_ranks(3.5) == 3.5
    assert aggregate_rate(10 ** 6, 2, 1000.0, 1) == 2.0
    with pytest.raises(ValueError):
        aggregate_rate(1, 1, 0.0, 1)


def test_reference_arm_prints_once_under_torchrun(oracle_mod):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0", "--cpu-n", "16"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
