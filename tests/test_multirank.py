"""The multi-GPU bench path on CPU: two gloo ranks run the bench's rank
logic (independent photon streams per rank, max-over-ranks timing, whole-job
throughput); on GPUs the same functions run over NCCL."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank's step times differ; the job is as slow as its slowest rank
        ms, e2e = bench.max_over_ranks([10.0 + rank, 20.0 - rank], world)
        seeds = [bench.step_seed(5, rank, i) for i in range(3)]
        all_seeds = [None] * world
        dist.all_gather_object(all_seeds, seeds)
        out[rank] = (ms, e2e, bench.job_mphotons(world, 10_000_000, ms), all_seeds)
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    for r in range(world):
        ms, e2e, v, all_seeds = out[r]
        assert ms == 11.0 and e2e == 20.0          # max over ranks, the same on every rank
        assert abs(v - 2 * 10_000_000 / 11e-3 / 1e6) < 1e-9
        flat = [s for rank_seeds in all_seeds for s in rank_seeds]
        assert len(set(flat)) == len(flat)       # no two ranks or steps share a photon stream


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.0], 1) == [3.0, 4.0]
    assert bench.job_mphotons(1, 10_000_000, 10.0) == pytest.approx(1000.0)
