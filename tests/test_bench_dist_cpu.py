"""The bench's multi-rank plumbing on the CPU: two gloo ranks run the same
setup, barrier and max-over-ranks helpers bench.py uses under torchrun (the
GPU arms use NCCL; the solve itself does not shard, so ranks are replicas)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "QCU_BENCH_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    # each rank's time differs; every rank must see the largest
    got = bench.max_over_ranks(1.0 + rank, w)
    bench.barrier(w)
    with open(f"{out_path}.{rank}", "w") as f:
        f.write(repr(got))
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_max_time(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    out = str(tmp_path / "res")
    mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    vals = [float(open(f"{out}.{r}").read()) for r in range(2)]
    assert vals == [2.0, 2.0]


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_setup() == (1, 0, 0)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    bench.barrier(1)  # no-op
