"""Runs the unmodified reference library (oracle/_ref/libqcu_ref.so) on a GPU -
TEST INFRASTRUCTURE ONLY.

The reference keeps process-global state (its clover term is computed once per
process and never again, src/qcu_clover_dslash.cu:564-566, 794-825) and calls
exit(-1) on any CUDA error (include/qcu_macro.cuh:34-41), so every gauge field
is run in a fresh subprocess:

    python -m oracle.ref_runner --lattice 8 8 8 8 --gauge random:2024:0.3 \
        --ops dslash,full,invert,pre,newfull,round,mmv --out out.npz
    python -m oracle.ref_runner --lattice 8 8 8 8 --gauge pure:7 --ops cg --out cg.npz

Inputs come from the CPU oracle's seeded generators (identical on every
machine); outputs are written as complex128 arrays in the reference layouts.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402

MANGLED = {
    "invertCloverDslash": "_Z18invertCloverDslashPvS_S_P10QcuParam_si",
    "preCloverDslash": "_Z15preCloverDslashPvS_S_P10QcuParam_si",
    "cloverDslashOneRound": "_Z20cloverDslashOneRoundPvS_S_P10QcuParam_si",
    "fullCloverDslashOneRound": "_Z24fullCloverDslashOneRoundPvS_S_P10QcuParam_si",
    "newFullCloverDslashOneRound": "_Z27newFullCloverDslashOneRoundPvS_S_P10QcuParam_si",
    "MmV_one_round": "_Z13MmV_one_roundPvS_S_P10QcuParam_sS_",
}


class QcuParam(ctypes.Structure):
    _fields_ = [("lattice_size", ctypes.c_int * 4)]


class QcuGrid(ctypes.Structure):
    _fields_ = [("grid_size", ctypes.c_int * 4)]


def make_gauge(L, spec: str) -> np.ndarray:
    kind, *args = spec.split(":")
    if kind == "random":
        return O.gauge_random(L, int(args[0]), float(args[1]))
    if kind == "pure":
        return O.gauge_pure(L, int(args[0]))
    if kind == "unit":
        return O.gauge_unit(L)
    raise ValueError(spec)


def run_in_process(L, gauge_spec, ops, spinor_seed, out_path, timing_reps=0):
    import torch

    lib = ctypes.CDLL(O.REF_LIB_PATH)
    P = ctypes.c_void_p
    PP = ctypes.POINTER(QcuParam)
    lib.initGridSize.argtypes = [ctypes.POINTER(QcuGrid), PP, P, P, P]
    for n in ("dslashQcu", "fullDslashQcu"):
        getattr(lib, n).argtypes = [P, P, P, PP, ctypes.c_int]
    lib.cg_inverter.argtypes = [P, P, P, PP]
    lib.loadQcuGauge.argtypes = [P, PP]
    fns = {}
    for k, m in MANGLED.items():
        f = getattr(lib, m)
        f.argtypes = [P, P, P, PP, P] if k == "MmV_one_round" else [P, P, P, PP, ctypes.c_int]
        f.restype = None
        fns[k] = f

    V = L[0] * L[1] * L[2] * L[3]
    Vh = V // 2
    dev = torch.device("cuda:0")
    gauge_np = make_gauge(L, gauge_spec)
    gauge = torch.from_numpy(gauge_np.reshape(-1)).to(dev)
    psi_np = O.full_spinor_random(L, spinor_seed)
    psi = torch.from_numpy(psi_np.reshape(-1)).to(dev)
    p = QcuParam()
    for k in range(4):
        p.lattice_size[k] = L[k]
    g = QcuGrid()
    for k in range(4):
        g.grid_size[k] = 1
    fin = torch.zeros(V * 12, dtype=torch.complex128, device=dev)
    fout = torch.zeros(V * 12, dtype=torch.complex128, device=dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    lib.initGridSize(ctypes.byref(g), ctypes.byref(p), ptr(gauge), ptr(fin), ptr(fout))
    lib.loadQcuGauge(ptr(gauge), ctypes.byref(p))
    torch.cuda.synchronize()
    res = {"lattice": np.array(L), "spinor_seed": np.array(spinor_seed)}
    out = torch.zeros_like(psi)
    tmp = torch.zeros_like(psi)
    for op in ops:
        if op == "dslash":
            for par in (0, 1):
                half_in = psi[(1 - par) * Vh * 12:(2 - par) * Vh * 12].clone()
                half_out = torch.zeros_like(half_in)
                lib.dslashQcu(ptr(half_out), ptr(half_in), ptr(gauge), ctypes.byref(p), par)
                torch.cuda.synchronize()
                res[f"dslash_p{par}"] = half_out.cpu().numpy()
        elif op == "full":
            for dag in (0, 1):
                lib.fullDslashQcu(ptr(out), ptr(psi), ptr(gauge), ctypes.byref(p), dag)
                torch.cuda.synchronize()
                res[f"full_d{dag}"] = out.cpu().numpy()
        elif op in ("invert", "pre"):
            t = psi.clone()
            name = "invertCloverDslash" if op == "invert" else "preCloverDslash"
            fns[name](ptr(t), ptr(psi), ptr(gauge), ctypes.byref(p), 0)
            torch.cuda.synchronize()
            res[op] = t.cpu().numpy()
        elif op in ("newfull", "round"):
            name = "newFullCloverDslashOneRound" if op == "newfull" else "cloverDslashOneRound"
            for dag in (0, 1):
                fns[name](ptr(out), ptr(psi), ptr(gauge), ctypes.byref(p), dag)
                torch.cuda.synchronize()
                res[f"{op}_d{dag}"] = out.cpu().numpy()
        elif op == "mmv":
            fns["MmV_one_round"](ptr(out), ptr(psi), ptr(gauge), ctypes.byref(p), ptr(tmp))
            torch.cuda.synchronize()
            res["mmv"] = out.cpu().numpy()
        elif op == "cg":
            x = torch.zeros_like(psi)
            t0 = time.perf_counter()
            lib.cg_inverter(ptr(psi), ptr(x), ptr(gauge), ctypes.byref(p))
            torch.cuda.synchronize()
            res["cg_seconds"] = np.array(time.perf_counter() - t0)
            res["cg_x"] = x.cpu().numpy()
        elif op == "time_dslash":
            # API-level time of dslashQcu (its three kernels, transposes and syncs)
            half_in = psi[Vh * 12:].clone()
            half_out = torch.zeros_like(half_in)
            for _ in range(2):
                lib.dslashQcu(ptr(half_out), ptr(half_in), ptr(gauge), ctypes.byref(p), 0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(max(timing_reps, 1)):
                lib.dslashQcu(ptr(half_out), ptr(half_in), ptr(gauge), ctypes.byref(p), 0)
            torch.cuda.synchronize()
            res["dslash_api_seconds"] = np.array((time.perf_counter() - t0) / max(timing_reps, 1))
        elif op == "time_full":
            for _ in range(2):
                lib.fullDslashQcu(ptr(out), ptr(psi), ptr(gauge), ctypes.byref(p), 0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(max(timing_reps, 1)):
                lib.fullDslashQcu(ptr(out), ptr(psi), ptr(gauge), ctypes.byref(p), 0)
            torch.cuda.synchronize()
            res["full_api_seconds"] = np.array((time.perf_counter() - t0) / max(timing_reps, 1))
        else:
            raise ValueError(op)
    np.savez(out_path, **res)


def run(L, gauge_spec, ops, spinor_seed=11, timing_reps=0, timeout=1200):
    """Runs the reference in a subprocess; returns (dict of arrays, stdout)."""
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "out.npz")
        cmd = [sys.executable, "-m", "oracle.ref_runner", "--lattice", *map(str, L), "--gauge", gauge_spec,
               "--ops", ",".join(ops), "--seed", str(spinor_seed), "--reps", str(timing_reps), "--out", path]
        r = subprocess.run(cmd, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        d = dict(np.load(path))
    m = re.search(r"number of iteration (\d+)", r.stdout)
    d["cg_iterations"] = np.array(int(m.group(1)) if m else -1)
    d["cg_converged"] = np.array("cg success" in r.stdout)
    return d, r.stdout


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", type=int, nargs=4, required=True)
    ap.add_argument("--gauge", required=True)
    ap.add_argument("--ops", required=True)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--reps", type=int, default=0)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    run_in_process(tuple(a.lattice), a.gauge, a.ops.split(","), a.seed, a.out, a.reps)
