"""Multi-process plumbing of the replica form (one process per GPU), on the
CPU with the gloo backend and two ranks: rank layout from the launcher's
environment, distinct captures per rank, the max-over-ranks elapsed time
every rank agrees on, and the reference arm's non-zero ranks exiting
without work."""

import os
import socket
import subprocess
import sys
from datetime import timedelta

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "ld-decode_b200"))
    import torch.distributed as dist
    from ldgpu.replicas import barrier, capture_seed, dist_env, max_over_ranks
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    r, w, local = dist_env()
    elapsed = 10.0 + 5.0 * r          # rank 1 is the slower one
    agreed = max_over_ranks(elapsed, w)
    barrier(w)
    q.put((r, w, local, agreed, capture_seed(7, r)))
    dist.destroy_process_group()


def test_two_rank_max_and_seeds():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[3] == 15.0 for o in out)          # both ranks report the slowest rank's time
    assert out[0][4] != out[1][4]                  # each replica decodes its own capture


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
