"""Host side of the N-GPU bench path on the CPU: two ranks over the gloo
backend.  Each rank owns a disjoint block of noise seeds (trajectories are
independent: replicas, no data-path collective), the timed region is the max
over ranks, and the reference arm runs on rank 0 only while the other ranks
exit without work."""
import multiprocessing as mp
import os
import socket
import subprocess
import sys
from datetime import timedelta

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        import bench
        m = bench.max_over_ranks(10.0 + 3.0 * rank, "cpu")
        seeds = bench.rank_seeds(rank, 4)
        rec = bench.e2e_record(4, world, m, 2, 2 * 640, 2 * 320)
        q.put((rank, m, seeds, rec["value"], rec["h2d_bytes_per_step"]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_timing_and_disjoint_seeds():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, s0, v0, b0), (r1, m1, s1, v1, b1) = out
    assert (r0, r1) == (0, 1)
    assert m0 == m1 == 13.0                       # both ranks see the slowest rank
    assert not set(s0) & set(s1) and len(s0) == len(s1) == 4
    assert v0 == v1 == round(4 * 2 * 2 / 13.0, 2)  # whole-job throughput
    assert b0 == b1 == 640


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
