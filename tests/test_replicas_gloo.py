"""The replica (N > 1) bookkeeping of bench.py on CPU with the gloo backend, world size 2:
every rank times its own solve, the job time is the maximum over ranks, value is that
time over the number of replicas, and the reference arm prints from rank 0 only."""
import importlib.util
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b = _bench()
    local = [120.0, 175.5][rank]
    m = b.max_over_ranks(local)
    # the ensemble partition: every rank's members, gathered on every rank
    mine = b.members_of_rank(rank, world, 3)
    got = [None] * world
    dist.all_gather_object(got, mine)
    q.put((rank, m, b.job_time_per_solve(m, world), got))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[:3] for g in got] == [(0, 175.5, 87.75), (1, 175.5, 87.75)]
    # members sharded with no overlap, the job covering 0 .. world * per_gpu - 1
    for g in got:
        parts = g[3]
        assert parts == [[0, 1, 2], [3, 4, 5]]
        flat = [m for p in parts for m in p]
        assert sorted(flat) == list(range(6)) and len(set(flat)) == len(flat)


def test_single_process_needs_no_group():
    b = _bench()
    assert b.max_over_ranks(3.5) == 3.5
    assert b.job_time_per_solve(10.0, 1) == 10.0
    assert b.members_of_rank(0, 1, 64) == list(range(64))
    with pytest.raises(ValueError):
        b.members_of_rank(2, 2, 4)


def test_reference_arm_prints_from_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
