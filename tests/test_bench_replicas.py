"""The multi-GPU form of the bench on CPU: world_size-2 gloo ranks.

The path does not shard: under torchrun every rank advances its own channel
(a different seed, no data-path collective), and the job's time is the
maximum over ranks.  Here each rank advances its replica on the CPU oracle,
times it, and takes the bench's own reduction helpers over gloo; the test
checks that both ranks agree on the max-over-ranks time and on the whole-job
rate, and that the replicas differ.  The reference arm under torchrun runs on
rank 0 only; other ranks exit 0 without output.
"""
import math
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import time
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import bench
    from oracle import Oracle
    from chapsim.mesh import channel_setup
    from chapsim.fields import initial_field
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    L = M = N = 32
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, bench.replica_seed(rank), 0.1)
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, DT0=0.02, threads=1)
    o.set_fields(Q, PR)
    o.substep(0)
    dist.barrier()
    t0 = time.perf_counter()
    o.run_steps(2 + 2 * rank)  # uneven work: rank 1 is the slow one
    ms_local = 1000.0 * (time.perf_counter() - t0)
    ms = bench.max_over_ranks(ms_local, dist, "cpu")
    value = bench.aggregate_rate(L * M * N, 2, ws, ms)
    Qs, _, _ = o.get_fields()
    q.put((rank, ms_local, ms, value, float(np.abs(Qs).sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_reduce_max_time_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, l0, m0, v0, c0), (r1, l1, m1, v1, c1) = out
    assert m0 == m1 == max(l0, l1)
    assert v0 == v1 == 32 ** 3 * 2 * 2 / (m0 / 1000.0)
    assert c0 != c1  # independent replicas (different seeds)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
