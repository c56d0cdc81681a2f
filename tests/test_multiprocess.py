"""The multi-rank plumbing of bench.py on the host (gloo, world size 2): the
device time reported is the maximum over ranks, and the reference arm runs on
rank 0 only.  The hot path does not exchange data between GPUs ("replicas
only"), so the time reduction and rank gating are all there is to test."""

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    got = bench._max_over_ranks(10.0 + rank * 5.0)
    args = type("A", (), {"steps": 1, "warmup": 0, "dtype": "float64"})()
    ref = bench.run_reference(args) if rank == 1 else "skipped"
    q.put((rank, got, ref))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_and_rank0_only_reference_arm():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]
    assert out[1][2] is None          # rank 1 prints nothing and does no work
