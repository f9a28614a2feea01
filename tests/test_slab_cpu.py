"""The t-slab decomposition's host logic without a GPU: the slab geometry
(qcuSlabGeometry, host arithmetic in the C library) and the host transport's
exchange and sum over a two-rank gloo process group, checked on marked
buffers: every rank's first slices must land in the ghost above rank - 1's
slab and its last slices in the ghost below rank + 1's."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_slab_geometry(qcu_lib):
    q = qcu_lib
    L = (8, 8, 8, 16)
    face = 4 * 8 * 8
    for n in (1, 2, 4):
        vh = 0
        for r in range(n):
            g = q.slab_geometry(L, n, r)
            assert g["t0"] == r * 16 // n and g["lt"] == 16 // n and g["face"] == face
            assert g["vh"] == face * g["lt"] and g["ghost_fwd"] == g["vh"] and g["ghost_bwd"] == g["vh"] + face
            vh += g["vh"]
        assert vh == 8 * 8 * 8 * 16 // 2
    for bad in (((8, 8, 8, 16), 16, 0),   # one slice per rank (odd)
                ((8, 8, 8, 6), 2, 0),     # three slices per rank
                ((6, 2, 2, 8), 2, 0),     # a slice of 12 sites: not whole 32-site blocks
                ((8, 8, 8, 16), 2, 2)):   # no such rank
        with pytest.raises(q.QcuError):
            q.slab_geometry(*bad)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import qcu_cg_inverter_b200 as q
    dist.init_process_group("gloo", rank=rank, world_size=world)
    exchange, allreduce = q.dist_transport()
    nb = 24
    send_lo = np.full(nb, 10 * rank + 1, np.uint8)  # my first slices
    send_hi = np.full(nb, 10 * rank + 2, np.uint8)  # my last slices
    recv_lo, recv_hi = np.zeros(nb, np.uint8), np.zeros(nb, np.uint8)
    exchange(send_lo, send_hi, recv_lo, recv_hi)
    v = np.array([1.0 + rank, 0.5], np.float64)
    allreduce(v)
    np.savez(f"{out_path}.{rank}.npz", lo=recv_lo, hi=recv_hi, v=v)
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_host_transport_moves_faces_to_the_neighbours(tmp_path, world):
    import torch.multiprocessing as mp
    out = str(tmp_path / "x")
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        d = np.load(f"{out}.{r}.npz")
        lo, hi = (r - 1) % world, (r + 1) % world
        assert np.all(d["hi"] == 10 * hi + 1)  # rank + 1's first slices above my slab
        assert np.all(d["lo"] == 10 * lo + 2)  # rank - 1's last slices below it
        assert np.allclose(d["v"], [sum(1.0 + k for k in range(world)), 0.5 * world])
