"""The multi-GPU arm of bench.py runs independent replicas, one per rank
(no collective in the data path): the job time is the slowest rank's, the
job value counts every replica's points, and the reference arm works on
rank 0 only.  Exercised here with two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 10.0 + 5.0 * rank   # the second replica is slower
        ms = bench.max_over_ranks(local_ms, dist, device="cpu")
        out.put((rank, ms, bench.job_value(1000, 30, world, ms * 1e-3)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [15.0, 15.0]                 # both ranks see the slowest
    assert got[0][2] == got[1][2] == 1000 * 30 * 2 / 0.015 / 1e6   # both replicas' points count


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
