"""Domain decomposition along t on the GPU (SlabContext).

One GPU serves these tests, so the multi-rank cases run two or four
processes on it with the host transport (their kernels never wait on one another: the halo
exchange and the sums go through the host, over a gloo process group). The
NCCL transport runs with one rank, which sends its faces to itself.

Checked against the whole-lattice context on the same seeded fields (the
slab generators give the slab's part of the global field):
  * the hop with the antiperiodic time boundary and the operator M = A -
    kappa D, D and D^dag: bit-identical (the ghost slices hold the very values
    the periodic wrap reads);
  * solves (16-bit and FP64): every rank's part stitched together reaches
    true residual < 1e-10 by the oracle's FP64 operator on the global
    lattice, and agrees with the whole-lattice solution to 1e-8 relative.
"""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L = (8, 8, 8, 16)
GSEED, EPS, PSEED = 11, 0.4, 5
KAPPA, CSW, BC = 0.13, 1.0, -1.0
KAPPAS2 = (0.125, 0.1375)


def whole_lattice(q, torch):
    """Gauge field, source, hop, operator and solutions on one context."""
    V = L[0] * L[1] * L[2] * L[3]
    res = {}
    with q.Context(L) as c:
        c.generate_gauge(GSEED, EPS)
        U = np.zeros((4, 2, V // 2, 3, 3), complex)
        c.export_gauge(U)
        res["U"] = U
        psi = torch.empty(V * 12, dtype=torch.complex128, device="cuda")
        c.generate_spinor(psi, 1, PSEED)
        res["psi"] = psi.cpu().numpy().reshape(2, V // 2, 12)
        for dag in (0, 1):
            out = torch.zeros_like(psi)
            c.apply_operator(out, psi, KAPPA, CSW, BC, dag)
            res[f"op{dag}"] = out.cpu().numpy().reshape(2, V // 2, 12)
        half_out = torch.zeros(V * 6, dtype=torch.complex128, device="cuda")
        c.dslash(half_out, psi[V * 6:].clone(), 0, 0, BC)
        res["hop"] = half_out.cpu().numpy().reshape(V // 2, 12)
        for prec in ("half", "double"):
            x = torch.zeros_like(psi)
            rep = c.invert(x, psi, kappa=KAPPA, csw=CSW, bc_t=BC, tol=1e-10, precision=prec)[0]
            assert rep["converged"]
            res["x_" + prec] = x.cpu().numpy().reshape(2, V // 2, 12)
        # a batch of two sources with two kappas (the batched kernels and their faces)
        bb = torch.empty(2 * V * 12, dtype=torch.complex128, device="cuda")
        c.generate_spinor(bb, 2, PSEED + 10)
        xb = torch.zeros_like(bb)
        reps = c.invert(xb, bb, nrhs=2, kappas=KAPPAS2, csw=CSW, bc_t=BC, tol=1e-10, precision="half")
        assert all(r["converged"] for r in reps)
        res["bb"] = bb.cpu().numpy().reshape(2, 2, V // 2, 12)
        res["xb"] = xb.cpu().numpy().reshape(2, 2, V // 2, 12)
    return res


def slab_run(q, torch, comm):
    """The same computations on this rank's slab; local arrays."""
    out = {}
    with q.SlabContext(L, comm, 0) as s:
        s.generate_gauge(GSEED, EPS)
        vh = s.volume // 2
        psi = torch.empty(2 * vh * 12, dtype=torch.complex128, device="cuda")
        s.generate_spinor(psi, 1, PSEED)
        out["psi"] = psi.cpu().numpy().reshape(2, vh, 12)
        for dag in (0, 1):
            o = torch.zeros_like(psi)
            s.apply_operator(o, psi, KAPPA, CSW, BC, dag)
            out[f"op{dag}"] = o.cpu().numpy().reshape(2, vh, 12)
        h = torch.zeros(vh * 12, dtype=torch.complex128, device="cuda")
        s.dslash(h, psi[vh * 12:].clone(), 0, 0, BC)
        out["hop"] = h.cpu().numpy().reshape(vh, 12)
        for prec in ("half", "double"):
            x = torch.zeros_like(psi)
            rep = s.invert(x, psi, kappa=KAPPA, csw=CSW, bc_t=BC, tol=1e-10, precision=prec)[0]
            out["x_" + prec] = x.cpu().numpy().reshape(2, vh, 12)
            out["conv_" + prec] = rep["converged"]
        bb = torch.empty(2 * 2 * vh * 12, dtype=torch.complex128, device="cuda")
        s.generate_spinor(bb, 2, PSEED + 10)
        xb = torch.zeros_like(bb)
        reps = s.invert(xb, bb, nrhs=2, kappas=KAPPAS2, csw=CSW, bc_t=BC, tol=1e-10, precision="half")
        out["bb"] = bb.cpu().numpy().reshape(2, 2, vh, 12)
        out["xb"] = xb.cpu().numpy().reshape(2, 2, vh, 12)
        out["conv_b"] = all(r["converged"] for r in reps)
        out["t0"] = s.t0
        out["vh"] = vh
    return out


def stitch(parts, key):
    """Every rank's local [parity][sites] block at its slab's sites."""
    return np.concatenate([p[key] for p in parts], axis=-2)


def check_against_whole(oracle, whole, parts):
    for key in ("psi", "op0", "op1"):
        assert np.array_equal(stitch(parts, key), whole[key]), key
    assert np.array_equal(np.concatenate([p["hop"] for p in parts], axis=0), whole["hop"])
    C = oracle.clover_build(whole["U"], L, KAPPA * CSW)
    b = whole["psi"].reshape(2, -1, 4, 3)
    for prec in ("half", "double"):
        assert all(p["conv_" + prec] for p in parts)
        x = stitch(parts, "x_" + prec).reshape(b.shape)
        res = np.linalg.norm(b - oracle.apply_full(x, whole["U"], C, L, KAPPA, BC)) / np.linalg.norm(b)
        assert res < 1e-10, (prec, res)
        xw = whole["x_" + prec].reshape(b.shape)
        assert np.linalg.norm(x - xw) / np.linalg.norm(xw) < 1e-8, prec
    # the two-source, two-kappa batch
    assert all(p["conv_b"] for p in parts)
    assert np.array_equal(stitch(parts, "bb"), whole["bb"])
    xb = stitch(parts, "xb")
    for r, k in enumerate(KAPPAS2):
        Ck = oracle.clover_build(whole["U"], L, k * CSW)
        br = whole["bb"][r].reshape(2, -1, 4, 3)
        xr = xb[r].reshape(br.shape)
        res = np.linalg.norm(br - oracle.apply_full(xr, whole["U"], Ck, L, k, BC)) / np.linalg.norm(br)
        assert res < 1e-10, (r, res)
        xw = whole["xb"][r].reshape(br.shape)
        assert np.linalg.norm(xr - xw) / np.linalg.norm(xw) < 1e-8, r


@pytest.mark.parametrize("transport", ["host", "nccl"])
def test_one_rank_slab_equals_whole_lattice(cuda, qcu_lib, oracle, transport):
    import torch
    q = qcu_lib
    whole = whole_lattice(q, torch)
    comm = q.Comm.host(1, 0) if transport == "host" else q.Comm.nccl(q.Comm.nccl_unique_id(), 1, 0, 0)
    try:
        part = slab_run(q, torch, comm)
    finally:
        comm.close()
    check_against_whole(oracle, whole, [part])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import qcu_cg_inverter_b200 as q
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    comm = q.Comm.torch_distributed(0)  # gloo: the host transport
    try:
        part = slab_run(q, torch, comm)
    finally:
        comm.close()
    np.savez(f"{out_path}.{rank}.npz", **{k: np.asarray(v) for k, v in part.items()})
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_ranks_on_one_gpu_equal_whole_lattice(cuda, qcu_lib, oracle, tmp_path, world):
    """world processes on the one GPU over the host transport. With 2 ranks
    each rank's two neighbours are the same rank; with 4 (slabs of 4 time
    slices) every rank exchanges with two different ranks."""
    import torch
    import torch.multiprocessing as mp
    whole = whole_lattice(qcu_lib, torch)
    out = str(tmp_path / "slab")
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    parts = [dict(np.load(f"{out}.{r}.npz")) for r in range(world)]
    assert [int(p["t0"]) for p in parts] == [r * L[3] // world for r in range(world)]
    check_against_whole(oracle, whole, parts)
