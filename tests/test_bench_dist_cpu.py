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


def test_gpus_flag_against_the_launcher():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.check_world(1, {}) == "run"
    assert bench.check_world(2, {}) == "relaunch"
    assert bench.check_world(2, {"WORLD_SIZE": "2"}) == "run"
    with pytest.raises(SystemExit):
        bench.check_world(2, {"WORLD_SIZE": "1"})
    with pytest.raises(SystemExit):
        bench.check_world(1, {"WORLD_SIZE": "4"})
    cmd = bench.relaunch_argv(2, ["--gpus", "2"])
    assert "--nproc-per-node=2" in cmd and "127.0.0.1" in cmd and cmd[-2:] == ["--gpus", "2"]


def test_gpus_two_outside_torchrun_starts_two_ranks():
    """`bench.py --gpus 2` without torchrun relaunches itself with two ranks
    (gloo here), so its line can never claim n_gpus 1."""
    import json
    import subprocess
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_PORT")}
    env["QCU_BENCH_BACKEND"] = "gloo"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--plan"], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(v) for v in r.stdout.splitlines() if v.startswith("{")]
    assert sorted(d["rank"] for d in lines) == [0, 1]
    assert all(d["world"] == 2 and d["n_gpus"] == 2 for d in lines)
