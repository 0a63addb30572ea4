"""The multi-rank path of bench.py on the CPU (gloo, two ranks): `bench.py --gpus N` runs N
independent replicas with no collective in the data path, only a barrier and the MAX over ranks
of the step time; under torchrun the reference arm runs on rank 0 alone."""
import contextlib
import io
import multiprocessing as mp
import os
import socket
import sys
from datetime import timedelta

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(1.5 + rank, 2, device="cpu")   # rank 1 is the slower one
        dist.barrier()
        q.put((rank, slowest))
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}


def test_one_rank_keeps_its_value():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(0.25, 1) == 0.25


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Ranks other than 0 leave the reference arm at once, printing nothing."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = bench.argparse.Namespace(workload="rand400", steps=1, warmup=0, gpus=2)
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.run_reference(args)
    assert out.getvalue() == ""
