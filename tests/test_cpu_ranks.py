"""bench.py's whole-job numbers under torchrun (one process per GPU, replicas only): every
rank takes part in the same barrier and max-reduction, so rank 0 reports the slowest
rank's time per tree and end-to-end wall time.  Two gloo ranks on CPU stand in for the
NCCL ranks of a multi-GPU run."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    from datetime import timedelta

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench

        # rank r: time per tree 1 + r ms, wall 10 - r s
        q.put((rank, bench.max_over_ranks([1.0 + rank, 10.0 - rank], "cpu")))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = dict(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert got[0] == got[1] == [2.0, 10.0]


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3.5, 1.0], "cpu") == [3.5, 1.0]
