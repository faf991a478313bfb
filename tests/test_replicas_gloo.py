"""The N > 1 path on CPU: two gloo ranks through the replica bookkeeping of bench.py.

bench.py --gpus N runs one independent replica per rank; the ranks share
only their timing (the job's time is the maximum over ranks) and the
whole-job throughput counts every replica's simulated time.  Two processes
rendezvous over 127.0.0.1 with the gloo backend and run exactly those
helpers; the reference arm's rule that only rank 0 runs and prints is
checked by launching it as rank 1 of 2.
"""
import os
import socket
import subprocess
import sys

import pytest

from td1c_b200 import replicas

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local = 0.25 + 0.5 * rank  # rank 1 is the slower replica
        sec = replicas.max_over_ranks(local, dist, None)
        dist.barrier()
        out.put((rank, sec, replicas.replica_seed(7, rank), replicas.job_throughput(world, 10, 0.004, sec)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_only_the_timing():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks see the slower rank's time; distinct seeds; throughput of both replicas
    assert [r[1] for r in res] == [0.75, 0.75]
    assert [r[2] for r in res] == [7, 8]
    expect = 2 * 10 * 0.004 * replicas.AU2FS / 0.75
    assert all(abs(r[3] - expect) < 1e-15 * expect for r in res)


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(1.5) == 1.5
    assert replicas.job_throughput(1, 100, 0.004, 2.0) == pytest.approx(100 * 0.004 * replicas.AU2FS / 2.0, rel=1e-15)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
