"""Benchmark: Wilson-clover CG to a true residual |r|/|b| < 1e-10 on B200.

Workload (one step = one complete solve): lattice 16^3x32, kappa = 0.1375,
c_sw = 1.0, seeded SU(3) links exp(0.4 i H), seeded Gaussian source,
antiperiodic in time; even-odd preconditioned CG with 16-bit inner storage,
FP32 arithmetic and FP64 reliable updates, stopping on the FP64 true residual
of the full system. Gauge field and source are resident in HBM when a step
starts (`value`); `e2e` repeats the solve through the public C API with the
source and solution in pinned HOST memory, so each step includes the
host->device copy of b and the device->host copy of x.

Printed JSON line (rank 0): metric/value (whole-job solves/s), the FP64
solver on the same system, the roofline of the dominant kernel (the fused
16-bit stencil, timed alone on the 32^3x64 lattice of the Dslash metric, whose
fields exceed L2), the CPU baseline (the oracle's FP64 Schur CG on all host
cores, stopping by the same true-residual rule, clover setup timed apart),
the error of each GPU solution against the oracle's, clocks sampled during
the timed region, and the number of kernels launched. At one GPU the line
also carries the other workloads of the metric: `large_solve` (32^3x64,
kappa 0.1370, eps 0.5, mixed vs FP64), `multi_rhs` (the 48-RHS 24^3x48 batch
against the FP64 single-RHS solve, every column's residual recomputed by the
oracle) and `serving` (the Poisson stream's p50/p99 and solves/s);
--no-extras leaves them out.

Other modes: --multi (the 48-RHS batch alone), --serve (the serving stream
alone, full record), --stencil (one stencil variant timed alone, for
rooflines and profiles).

`--impl reference` times the reference path on the host cores instead (the
reference library is GPU-only; its host-side restatement is the oracle's FP64
CG, run with every host thread) and adds the reference library's own Dslash
kernels (its printed kernel times) and entry points timed on the GPU.

Multi-GPU: by default N ranks run N independent replicas of the headline
solve (weak scaling); value = total solves / max-over-ranks time. --dd
instead splits one 32^3x64 lattice into N t-slabs (halo exchange and sums
over NCCL; strong scaling).
`--gpus N` outside torchrun relaunches this script under torchrun with N
local ranks; under torchrun it must equal WORLD_SIZE.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LATTICE = (16, 16, 16, 32)
KAPPA, CSW, EPS, BC_T, TOL = 0.1375, 1.0, 0.4, -1.0, 1e-10
GAUGE_SEED, SOURCE_SEED = 20241, 7
ROOF_LATTICE = (32, 32, 32, 64)
# DRAM bytes (read + write) per output site of the fused 16-bit stencil, per
# storage of links and clover, from ncu captures of one launch (the traffic
# grows with the number of sites): FP32 links and clover at 32^4 (592.9 MB for
# 524288 sites); 16-bit links and clover at 32^3x64 (561.1 MB for 1048576 sites)
ROOF_TRAFFIC_BYTES_PER_SITE = {"fast": 592.9e6 / 524288, "compact": 561.1e6 / 1048576}
# storage behind the 16-bit solves (qcuContextSetHalfOperator) and its description
STORAGE = {"auto": None, "fast": True, "compact": False}
DTYPE = {"fast": "f32 arithmetic; 16-bit spinors, FP32 links (18 reals) and FP32 clover; f64 reliable updates",
         "compact": "f32 arithmetic; 16-bit spinors, 16-bit 12-real links and 16-bit clover; f64 reliable updates"}
METRIC = "CG time to |r|/|b|<1e-10, mixed vs FP64 (16^3x32 Wilson-clover, kappa 0.1375, c_sw 1)"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons around the timed region.

    Started before the warm-up and given time to produce its first sample;
    samples every 20 ms with timestamps; mark() brackets the timed region and
    summary() keeps the samples inside it (or, if the region was shorter than
    one period, the nearest samples on either side)."""

    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            deadline = time.time() + 5
            while time.time() < deadline and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def start(self):
        self.t0 = time.time()

    def stop(self):
        self.t1 = time.time()
        time.sleep(0.05)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime
        rows = []
        try:
            for line in open(self.path):
                f = [v.strip() for v in line.split(",")]
                if len(f) < 8:
                    continue
                try:
                    ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    rows.append((ts, float(f[1]), float(f[2]), f[4:8]))
                except ValueError:
                    continue
            os.unlink(self.path)
        except Exception:
            pass
        inside = [r for r in rows if self.t0 is not None and self.t0 <= r[0] <= (self.t1 or r[0])]
        sel = inside
        if not sel and rows and self.t0 is not None:
            before = [r for r in rows if r[0] < self.t0]
            after = [r for r in rows if r[0] > (self.t1 or self.t0)]
            sel = before[-1:] + after[:1]
        reasons = sorted({n for r in sel for n, v in zip(self.REASONS, r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median([r[1] for r in sel]) if sel else None,
                "sm_max_mhz": max(r[2] for r in sel) if sel else None, "reasons": reasons,
                "samples_in_timed_region": len(inside), "samples_used": len(sel)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = os.environ.get("QCU_BENCH_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist
        if device is not None and dist.get_backend() == "nccl":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ---------------------------------------------------------------------------
def oracle_baseline(U, b, L, kappa, csw, threads=None, solves=3):
    """The CPU baseline: the oracle's FP64 Schur CG on the host cores, with the
    clover term built and factored once (timed apart, as `setup_s`) and then
    `solves` complete solves timed (median): the same work as a GPU step, which
    reuses the clover fields of the context. The solve stops by the GPU
    solver's rule (true residual checked where the iterated one predicts it).
    Returns the timings, iteration count and one solution."""
    from oracle import oracle as O
    if threads:
        O.set_threads(threads)
    t0 = time.perf_counter()
    C = O.clover_build(U, L, kappa * csw)
    Ci = O.clover_invert(C)
    setup_s = time.perf_counter() - t0
    times, x = [], None
    for _ in range(max(solves, 1)):
        t0 = time.perf_counter()
        x, iters, res, checks = O.solve_schur_cl(b, U, C, Ci, L, kappa, BC_T, TOL, 100000)
        times.append(time.perf_counter() - t0)
    return {"solve_s": statistics.median(times), "setup_s": setup_s, "iterations": iters, "true_residual": res,
            "checks": checks, "cores": O.num_threads(), "x": x, "solves": len(times)}


ORACLE_RULE = ("stops on the true residual |b-Mx|/|b| < 1e-10 of the full system, checked where the iterated "
               "residual predicts it (the GPU solver's rule); clover build and factorisation timed apart")


def time_drop_in(ctx, torch, device, reps=20):
    """The reference-signature entry points dslashQcu and fullDslashQcu on
    device AoS buffers at the headline lattice, wall time per call (each call
    is synchronous, as in the reference; the reference arm times the reference
    library's own calls the same way)."""
    import numpy as np

    import qcu_cg_inverter_b200 as q
    L, V = LATTICE, ctx.volume
    U = np.zeros((4, 2, V // 2, 3, 3), complex)
    ctx.export_gauge(U)
    gauge = torch.from_numpy(U.reshape(-1)).to(device)
    psi = torch.empty(V * 12, dtype=torch.complex128, device=device)
    ctx.generate_spinor(psi, 1, SOURCE_SEED)
    out = torch.zeros_like(psi)
    half_in, half_out = psi[V * 6:].clone(), torch.zeros(V * 6, dtype=torch.complex128, device=device)
    p = q.param(L)
    q.initGridSize((1, 1, 1, 1), p, gauge, psi, out)
    res = {"lattice": L}
    for name, call in (("dslashQcu_ms", lambda: q.dslashQcu(half_out, half_in, gauge, p, 0)),
                       ("fullDslashQcu_ms", lambda: q.fullDslashQcu(out, psi, gauge, p, 0))):
        for _ in range(3):
            call()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for _ in range(reps):
            call()
        torch.cuda.synchronize(device)
        res[name] = (time.perf_counter() - t0) / reps * 1e3
    return res


def timed_steps(torch, device, stream, flush, fn, steps):
    """steps x fn() with an L2 flush before each, CUDA events on the library
    stream; returns (total seconds, last result)."""
    total, rep = 0.0, None
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rep = fn()
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1) / 1e3
    return total, rep


LARGE_KAPPA, LARGE_EPS = 0.1370, 0.5


def run_large(roof, torch, device, flush, args):
    """The large single solve: 32^3x64 Wilson-clover (kappa 0.1370, c_sw 1,
    eps 0.5, antiperiodic t), seeded Gaussian source, mixed precision against
    the FP64 solver on the same GPU, each to true residual 1e-10."""
    V = roof.volume
    b = torch.empty(V * 12, dtype=torch.complex128, device=device)
    roof.generate_spinor(b, 1, SOURCE_SEED)
    x = torch.zeros_like(b)
    stream = torch.cuda.ExternalStream(roof.stream, device=device)
    kw = dict(kappa=LARGE_KAPPA, csw=CSW, bc_t=BC_T, tol=TOL, delta=args.delta)

    def solve(prec):  # --delta applies to the mixed-precision solve only
        rep = roof.invert(x, b, precision=prec, **(kw if prec != "double" else dict(kw, delta=0.0)))[0]
        assert rep["converged"], rep
        return rep

    out = {"workload": "32^3x64 Wilson-clover CG to true residual 1e-10", "lattice": ROOF_LATTICE,
           "kappa": LARGE_KAPPA, "csw": CSW, "eps": LARGE_EPS, "bc_t": "antiperiodic",
           "dtype": DTYPE[roof.half_storage(1)],
           "l2": "256 MB buffer written between timed steps (fields exceed L2)"}
    res = {}
    for prec, steps in ((args.precision, 3), ("double", 2)):
        solve(prec)  # warm-up: autotune, clover fields, graphs
        n0 = roof.launches
        t, rep = timed_steps(torch, device, stream, flush, lambda: solve(prec), steps)
        res[prec] = (t / steps, rep, (roof.launches - n0) // steps, x.clone())
    tm, rm, lm, xm = res[args.precision]
    td, rd, ld, xd = res["double"]
    out.update({"mixed_s": tm, "mixed_iterations": rm["iterations"], "mixed_reliable_updates": rm["reliable_updates"],
                "mixed_true_residual": rm["true_residual"], "mixed_gpu_launches": lm,
                "fp64_s": td, "fp64_iterations": rd["iterations"], "fp64_true_residual": rd["true_residual"],
                "speedup_vs_fp64": td / tm,
                "solution_rel_err_mixed_vs_fp64": float(torch.linalg.norm(xm - xd) / torch.linalg.norm(xd))})
    if not args.no_cpu_baseline:  # both solutions' true residuals by the oracle's FP64 operator
        import numpy as np

        from oracle import oracle as O
        U = np.zeros((4, 2, V // 2, 3, 3), complex)
        roof.export_gauge(U)
        C = O.clover_build(U, ROOF_LATTICE, LARGE_KAPPA * CSW)
        bh = b.cpu().numpy().reshape(2, V // 2, 4, 3)
        nb = np.linalg.norm(bh)
        for key, xx in (("mixed", xm), ("fp64", xd)):
            r = bh - O.apply_full(xx.cpu().numpy().reshape(bh.shape), U, C, ROOF_LATTICE, LARGE_KAPPA, BC_T)
            out[key + "_true_residual_by_oracle"] = float(np.linalg.norm(r) / nb)
    return out


def relaunch_argv(gpus, argv, port=29517):
    """The torchrun command that runs this script with `gpus` local ranks (one
    per GPU), used when --gpus N > 1 is given outside torchrun."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + list(argv)


def check_world(gpus, env):
    """--gpus N against the launcher: 'run' when they agree, 'relaunch' when
    N > 1 was asked for outside torchrun; raises when torchrun started a
    different number of ranks (the line would mislabel n_gpus)."""
    if "WORLD_SIZE" in env:
        world = int(env["WORLD_SIZE"])
        if world != gpus:
            raise SystemExit(f"bench.py: --gpus {gpus} but WORLD_SIZE={world}; pass the same number to both")
        return "run"
    return "relaunch" if gpus > 1 else "run"


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import qcu_cg_inverter_b200 as q
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ctx = q.Context(LATTICE, local)
    ctx.generate_gauge(GAUGE_SEED, EPS)
    ctx.set_half_operator(STORAGE[args.storage])
    V = ctx.volume
    b = torch.empty(V * 12, dtype=torch.complex128, device=device)
    ctx.generate_spinor(b, 1, SOURCE_SEED + rank)
    x = torch.zeros_like(b)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    kw = dict(kappa=KAPPA, csw=CSW, bc_t=BC_T, tol=TOL, delta=args.delta)

    def solve(xx, bb, prec):  # --delta applies to the mixed-precision solve only
        rep = ctx.invert(xx, bb, precision=prec, **(kw if prec != "double" else dict(kw, delta=0.0)))[0]
        assert rep["converged"], rep
        return rep

    def timed(fn, steps):
        return timed_steps(torch, device, stream, flush, fn, steps)

    with ClockSampler(local) as clk:
        # warm-up (also autotunes, builds the clover fields and captures the CUDA graphs)
        for _ in range(args.warmup):
            solve(x, b, args.precision)
        barrier(world, device)
        torch.cuda.synchronize(device)
        n0 = ctx.launches
        clk.start()
        t_mixed, rep = timed(lambda: solve(x, b, args.precision), args.steps)
        clk.stop()
    launches = (ctx.launches - n0) // max(args.steps, 1)
    t_mixed = max_over_ranks(t_mixed, world, device)
    barrier(world, device)
    # e2e through the public C API with host buffers
    bh = b.cpu().pin_memory()
    xh = torch.zeros_like(bh).pin_memory()
    solve(xh, bh, args.precision)
    t_e2e, _ = timed(lambda: solve(xh, bh, args.precision), args.steps)
    t_e2e = max_over_ranks(t_e2e, world, device)
    # FP64 solver on the same system
    solve(x, b, "double")
    fsteps = max(1, min(args.steps, 3))
    t_fp64, rep64 = timed(lambda: solve(x, b, "double"), fsteps)
    t_fp64 = max_over_ranks(t_fp64, world, device)
    x64 = x.clone()
    solve(x, b, args.precision)
    err_vs_fp64 = float(torch.linalg.norm(x - x64) / torch.linalg.norm(x64))

    out = None
    if rank == 0:
        # dominant kernel: the fused 16-bit stencil (hop + A^-1 + xpay + second output + norm)
        hbm, src = peaks()
        roof = q.Context(ROOF_LATTICE, local)
        V_roof = roof.volume
        roof.generate_gauge(GAUGE_SEED, LARGE_EPS)
        roof.set_half_operator(STORAGE[args.storage])
        for p in ("half", "double"):
            roof.autotune(p, 1)
        ms, nbytes = roof.bench_stencil("half", 2, 1, 50)
        ms_hop64, bytes_hop64 = roof.bench_stencil("double", 0, 1, 20)
        ms_hop16, bytes_hop16 = roof.bench_stencil("half", 0, 1, 50)
        achieved = nbytes / (ms / 1e3) / 1e9
        roof_storage = roof.half_storage(1)
        tps = ROOF_TRAFFIC_BYTES_PER_SITE[roof_storage]
        # in-solve kernels at the headline size (fields L2-resident)
        ms_small, nbytes_small = ctx.bench_stencil("half", 2, 1, 50)
        ms_hop64_small, _ = ctx.bench_stencil("double", 0, 1, 20)
        drop_in = time_drop_in(ctx, torch, device)
        steps = args.steps
        per = t_mixed / steps
        out = {
            "metric": METRIC, "value": world * steps / t_mixed, "unit": "solves/s", "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[ctx.half_storage(1)],
            "data": "synthetic (seeded SU(3) links exp(0.4iH), seeded Gaussian source)",
            "config": {"workload": "16^3x32 Wilson-clover even-odd CG to true residual 1e-10", "lattice": LATTICE,
                       "kappa": KAPPA, "csw": CSW, "bc_t": "antiperiodic", "precision": args.precision,
                       "l2": "256 MB buffer written between timed steps", "parallelism": f"replicas x{world}"},
            "time_to_solution_s": per, "iterations": rep["iterations"], "reliable_updates": rep["reliable_updates"],
            "true_residual": rep["true_residual"],
            "fp64": {"time_to_solution_s": t_fp64 / fsteps, "iterations": rep64["iterations"],
                     "true_residual": rep64["true_residual"]},
            "speedup_vs_fp64": (t_fp64 / fsteps) / per,
            "solution_rel_err_vs_fp64": err_vs_fp64,
            "e2e": {"value": world * steps / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": V * 12 * 16,
                    "d2h_bytes_per_step": V * 12 * 16},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": src, "frac_of_nominal_8000_GBps": achieved / 8000.0,
                         "traffic": tps * (V_roof // 2) if tps else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                           "per site, times the sites of this launch",
                         "kernel": "dslash half hop+A^-1+xpay+out2+norm, 32^3x64, 1 RHS", "storage": DTYPE[roof_storage],
                         "bytes_per_launch": nbytes, "ms_per_launch": ms},
            "dslash": {"lattice": ROOF_LATTICE,
                       "fp64_hop_GBps": bytes_hop64 / (ms_hop64 / 1e3) / 1e9, "fp64_hop_ms": ms_hop64,
                       "fp64_hop_16x32_ms": ms_hop64_small,
                       "half_hop_GBps": bytes_hop16 / (ms_hop16 / 1e3) / 1e9,
                       "half_fused_GBps": achieved,
                       "in_solve_16x32_half_fused_GBps": nbytes_small / (ms_small / 1e3) / 1e9},
            "drop_in": drop_in,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_extras:
            out["large_solve"] = run_large(roof, torch, device, flush, args)
        roof.close()
        if world == 1 and not args.no_cpu_baseline:
            U = np.zeros((4, 2, V // 2, 3, 3), complex)
            ctx.export_gauge(U)
            bnp = b.cpu().numpy().reshape(2, V // 2, 4, 3)
            cb = oracle_baseline(U, bnp, LATTICE, KAPPA, CSW, os.cpu_count(), 3)
            xo = cb["x"].reshape(-1)
            nrm = np.linalg.norm(xo)
            out["solution_rel_err_vs_oracle"] = float(np.linalg.norm(x.cpu().numpy() - xo) / nrm)
            out["fp64"]["solution_rel_err_vs_oracle"] = float(np.linalg.norm(x64.cpu().numpy() - xo) / nrm)
            out["cpu_baseline"] = {"value": 1.0 / cb["solve_s"], "unit": "solves/s", "cores": cb["cores"],
                                   "kind": "port", "solve_s": cb["solve_s"], "clover_setup_s": cb["setup_s"],
                                   "iterations": cb["iterations"],
                                   "sample": f"{cb['solves']} complete FP64 solves of the same 16^3x32 Schur system "
                                             f"by the oracle ({cb['iterations']} iterations, {cb['checks']} "
                                             f"true-residual checks, true residual {cb['true_residual']:.1e}), "
                                             f"median; {ORACLE_RULE}"}
    ctx.close()
    if rank == 0 and world == 1 and not args.no_extras:
        out["multi_rhs"] = run_multi(args, check_oracle=not args.no_cpu_baseline)
        out["serving"] = summarize_serve(run_serve(args))
    return out


def run_reference(args, world, rank, local):
    """The reference path on the host cores (the oracle port, all threads),
    plus the reference library's own Dslash kernels and entry points on the GPU."""
    if rank != 0:
        return None
    from oracle import oracle as O
    L = LATTICE
    U = O.gauge_random(L, GAUGE_SEED, EPS)
    b = O.full_spinor_random(L, SOURCE_SEED)
    ncores = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle_baseline(U, b, L, KAPPA, CSW, ncores, 1)
    cb = oracle_baseline(U, b, L, KAPPA, CSW, ncores, max(args.steps, 1))
    solve_s = cb["solve_s"]
    out = {
        "impl": "reference", "metric": METRIC, "value": 1.0 / solve_s, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": solve_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded SU(3) links exp(0.4iH), seeded Gaussian source)",
        "config": {"workload": "16^3x32 Wilson-clover even-odd CG to true residual 1e-10", "lattice": L,
                   "kappa": KAPPA, "csw": CSW, "bc_t": "antiperiodic", "precision": "double"},
        "cpu_baseline": {"value": 1.0 / solve_s, "unit": "solves/s", "cores": ncores, "kind": "port",
                         "clover_setup_s": cb["setup_s"],
                         "sample": f"{cb['solves']} complete FP64 solves of the 16^3x32 Schur system by the oracle "
                                   f"({cb['iterations']} iterations, true residual {cb['true_residual']:.1e}), "
                                   f"median; {ORACLE_RULE}"},
        "e2e": {"value": 1.0 / solve_s, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_note": "the reference library is GPU-only and its cg_inverter solves a different (kappa=1, "
                          "non-Hermitian) system; the timed reference path is the oracle's FP64 restatement",
    }
    if os.path.exists(O.REF_LIB_PATH) and not args.no_ref_gpu:
        out["reference_gpu"] = reference_gpu_kernels()
    return out


# FP64 hop: 8 neighbour spinors (192 B), 8 links (12 reals, 96 B), one output
# spinor per site; the reference's coalesced kernel reads exactly these
HOP64_BYTES_PER_SITE = 8 * 192 + 8 * 96 + 192


def reference_gpu_kernels():
    """The reference library (compiled unmodified for sm_100a) on the GPU:
    its own printed timing of its best Dslash kernel (mpiDslashCoalesce,
    src/qcu_wilson_dslash_neo.cu:649-661: a host clock around the launch and a
    device synchronisation) and of its naive kernel, per call of dslashQcu,
    at 16^3x32 and 32^3x64, in GB/s of the FP64 hop's algorithmic bytes; plus
    the API wall time of dslashQcu and fullDslashQcu (transposes, allocations
    and the extra kernels included)."""
    import re
    res = {"bytes_per_site": HOP64_BYTES_PER_SITE,
           "note": "kernel times are the reference's own printed host-clock times around launch + sync"}
    try:
        from oracle import ref_runner
        for L, eps in ((LATTICE, EPS), (ROOF_LATTICE, LARGE_EPS)):
            ops = ["time_dslash", "time_full"] if L == LATTICE else ["time_dslash"]
            d, stdout = ref_runner.run(L, f"random:{GAUGE_SEED}:{eps}", ops, SOURCE_SEED, timing_reps=20,
                                       timeout=900)
            vh = L[0] * L[1] * L[2] * L[3] // 2
            key = "x".join(map(str, L))
            r = {"dslashQcu_api_ms": float(d["dslash_api_seconds"]) * 1e3}
            if "full_api_seconds" in d:
                r["fullDslashQcu_api_ms"] = float(d["full_api_seconds"]) * 1e3
            for name, pat in (("mpiDslashCoalesce", r"coalescing total time: .*?: ([0-9.eE+-]+) sec"),
                              ("mpiDslashNaive", r"naive total time: .*?: ([0-9.eE+-]+) sec")):
                v = [float(m) for m in re.findall(pat, stdout)]
                if v:
                    ms = statistics.median(v[2:] if len(v) > 4 else v) * 1e3
                    r[name + "_ms"] = ms
                    r[name + "_GBps"] = HOP64_BYTES_PER_SITE * vh / (ms / 1e3) / 1e9
            res[key] = r
    except Exception as e:  # the CPU leg stands on its own
        res["error"] = str(e)[-300:]
    return res


MULTI_LATTICE = (24, 24, 24, 48)
MULTI_KAPPAS = (0.1360, 0.1365, 0.1370, 0.1375)
MULTI_EPS = 0.4  # not fixed by the workload description; recorded in the output


def point_sources(torch, V, site, device):
    """12 spin-colour point sources at checkerboard site `site` of parity 0,
    as full spinors [rhs][parity][Vh][4][3] (complex128)."""
    Vh = V // 2
    b = torch.zeros(12, 2, Vh, 12, dtype=torch.complex128, device=device)
    for k in range(12):
        b[k, 0, site, k] = 1.0
    return b.reshape(12, -1)


def run_multi(args, check_oracle=False):
    """The multi-RHS batch: 24^3x48 Wilson-clover (c_sw 1), 12 point sources at
    a seeded site x 4 kappas = 48 RHS, one mixed-precision batched solve (each
    RHS stops on its own at true residual 1e-10; mean of two timed solves after
    one warm-up) against the plain FP64 single-RHS CG on the same GPU (one RHS
    per kappa solved alone, the faster of two timings, scaled to 48). With
    check_oracle, every column's true residual is recomputed by the CPU
    oracle's FP64 operator."""
    import random

    import numpy as np
    import torch

    import qcu_cg_inverter_b200 as q
    device = torch.device("cuda", 0)
    ctx = q.Context(MULTI_LATTICE, 0)
    ctx.generate_gauge(GAUGE_SEED, MULTI_EPS)
    V = ctx.volume
    site = random.Random(SOURCE_SEED).randrange(V // 2)
    src12 = point_sources(torch, V, site, device)
    nr = 12 * len(MULTI_KAPPAS)
    b = src12.repeat(len(MULTI_KAPPAS), 1).contiguous()
    kap = [k for k in MULTI_KAPPAS for _ in range(12)]
    x = torch.zeros_like(b)
    kw = dict(csw=CSW, bc_t=BC_T, tol=TOL, delta=args.delta)
    kw64 = dict(kw, delta=0.0)  # --delta applies to the mixed-precision batch only
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)

    def timed(fn):
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, r

    # warm-up: autotune and clover for every kappa, graphs
    ctx.invert(x, b, nrhs=nr, kappas=kap, precision=args.precision, **kw)
    n0 = ctx.launches
    t_runs = []
    for _ in range(2):
        t, reps = timed(lambda: ctx.invert(x, b, nrhs=nr, kappas=kap, precision=args.precision, **kw))
        t_runs.append(t)
    t_multi = sum(t_runs) / len(t_runs)
    launches = (ctx.launches - n0) // len(t_runs)
    assert all(r["converged"] for r in reps), reps
    oracle_res = None
    if check_oracle:
        from oracle import oracle as O
        U = np.zeros((4, 2, V // 2, 3, 3), complex)
        ctx.export_gauge(U)
        oracle_res = []
        for j, k in enumerate(MULTI_KAPPAS):
            C = O.clover_build(U, MULTI_LATTICE, k * CSW)
            for c in range(12):
                r = 12 * j + c
                xr = x[r].cpu().numpy().reshape(2, V // 2, 4, 3)
                br = b[r].cpu().numpy().reshape(2, V // 2, 4, 3)
                res = br - O.apply_full(xr, U, C, MULTI_LATTICE, k, BC_T)
                oracle_res.append(float(np.linalg.norm(res) / np.linalg.norm(br)))
    # FP64 single-RHS sample: spin-colour 0 for each kappa
    x1 = torch.zeros_like(b[0])
    ctx.invert(x1, b[0].contiguous(), kappa=MULTI_KAPPAS[0], precision="double", **kw64)
    t64, it64 = [], []
    for j, k in enumerate(MULTI_KAPPAS):
        bb = b[12 * j].contiguous()
        ts = []
        for _ in range(2):  # two timings per kappa, the faster one kept
            t, r = timed(lambda: ctx.invert(x1, bb, kappa=k, precision="double", **kw64)[0])
            assert r["converged"], r
            ts.append(t)
        t64.append(min(ts))
        it64.append(r["iterations"])
    per64 = sum(t64) / len(t64)
    ctx.close()
    out = {
        "workload": "24^3x48 Wilson-clover multi-RHS: 12 point sources x 4 kappas = 48 RHS, true residual 1e-10",
        "lattice": MULTI_LATTICE, "kappas": MULTI_KAPPAS, "csw": CSW, "eps": MULTI_EPS, "source_site": site,
        "precision": args.precision, "nrhs": nr,
        "multi_s": t_multi, "multi_runs_s": t_runs, "multi_per_rhs_s": t_multi / nr,
        "iterations": [r["iterations"] for r in reps], "max_true_residual": max(r["true_residual"] for r in reps),
        "fp64_single_rhs_s": per64, "fp64_single_iterations": it64,
        "fp64_single_total_48_s": per64 * nr,
        "speedup_vs_fp64_single": per64 * nr / t_multi,
        "gpu_launches": launches,
    }
    if oracle_res is not None:
        out["max_true_residual_by_oracle"] = max(oracle_res)
        out["columns_checked_by_oracle"] = len(oracle_res)
    return out


SERVE_LATTICES = ((8, 8, 8, 8), (16, 16, 16, 32), (24, 24, 24, 48))
SERVE_WEIGHTS = (0.5, 0.3, 0.2)
SERVE_RATE = 50.0  # mean arrivals per second (Poisson)
SERVE_EPS = 0.4  # not fixed by the workload description; recorded in the output
SERVE_SEED = 2025


def serve_trace(n, seed):
    """n requests: Poisson arrivals (mean 50/s), lattice 8^4 / 16^3x32 / 24^3x48
    with weights .5/.3/.2, one of 3 gauge configurations per lattice, kappa
    uniform in [0.120, 0.1375], c_sw in {0, 1}, 1-12 RHS."""
    import numpy as np
    rng = np.random.default_rng(seed)
    arr = np.cumsum(rng.exponential(1.0 / SERVE_RATE, n))
    arr -= arr[0]
    lat = rng.choice(len(SERVE_LATTICES), n, p=SERVE_WEIGHTS)
    cfg = rng.integers(0, 3, n)
    kap = rng.uniform(0.120, 0.1375, n)
    csw = rng.choice([0.0, 1.0], n)
    nrhs = rng.integers(1, 13, n)
    return [dict(t=float(arr[i]), lat=int(lat[i]), cfg=int(cfg[i]), kappa=float(kap[i]), csw=float(csw[i]),
                 nrhs=int(nrhs[i])) for i in range(n)]


def run_serve(args):
    """The serving stream: a seeded Poisson trace run through the request
    server (continuous batching, one resident batch per gauge configuration).
    Sources are seeded Gaussian spinors in pinned host memory; solutions are
    copied back to pinned host memory; latency runs from each request's
    scheduled arrival to its solution being in host memory. The trace's
    offered load bounds the throughput of that run, so the same requests are
    then run all queued at once: their RHS solves per second are the server's
    capacity."""
    import numpy as np
    import torch

    import qcu_cg_inverter_b200 as q
    device = torch.device("cuda", 0)
    srv = q.Server(0, columns=args.columns, clover_slots=args.clover_slots, tol=TOL, bc_t=BC_T,
                   precision=q._PREC[args.precision], max_chunk=args.max_chunk, delta=args.delta)
    cids = {}
    for li, L in enumerate(SERVE_LATTICES):
        for c in range(3):
            cids[(li, c)] = srv.add_config(L, GAUGE_SEED + 1000 * li + c, SERVE_EPS)
    t_prep = time.time()
    for cid in cids.values():
        srv.prepare(cid)
    t_prep = time.time() - t_prep
    # pinned pools: 12 Gaussian sources per lattice, and output rings
    full = [2 * (L[0] * L[1] * L[2] * L[3] // 2) * 12 for L in SERVE_LATTICES]  # complex per full spinor
    src, out = [], []
    for li, L in enumerate(SERVE_LATTICES):
        pb = q.PinnedBuffer(12 * full[li] * 16)
        with q.Context(L, 0) as c:
            t = torch.empty(12 * full[li], dtype=torch.complex128, device=device)
            c.generate_spinor(t, 12, SOURCE_SEED + li)
            pb.array[:] = t.cpu().numpy()
            del t
        src.append(pb)
        out.append([q.PinnedBuffer(12 * full[li] * 16) for _ in range(args.out_ring)])

    def trace_args(tr):
        b = [src[r["lat"]].addr for r in tr]
        x = [out[r["lat"]][i % args.out_ring].addr for i, r in enumerate(tr)]
        return ([r["t"] for r in tr], [cids[(r["lat"], r["cfg"])] for r in tr], [r["kappa"] for r in tr],
                [r["csw"] for r in tr], [r["nrhs"] for r in tr], b, x)

    # warm-up trace (other seed): graphs and clover slots of every batch
    warm = serve_trace(max(args.warmup, 0) * 9, SERVE_SEED + 1)
    if warm:
        for r in warm:
            r["t"] = 0.0
        srv.run_trace(*trace_args(warm))
    tr = serve_trace(args.requests, SERVE_SEED)
    with ClockSampler(0) as clk:
        clk.start()
        t0 = time.time()
        lat, reps, code = srv.run_trace(*trace_args(tr), raise_on_fail=False)
        wall = time.time() - t0
        clk.stop()
    conv = all(r["converged"] for rr in reps for r in rr)
    nsol = sum(r["nrhs"] for r in tr)
    # capacity: the same requests all queued at once (the offered load of the
    # trace bounds the throughput of the timed run above)
    burst = [dict(r, t=0.0) for r in tr]
    t0 = time.time()
    _, breps, _ = srv.run_trace(*trace_args(burst), raise_on_fail=False)
    burst_wall = time.time() - t0
    conv = conv and all(r["converged"] for rr in breps for r in rr)
    lat_ms = sorted(v * 1e3 for v in lat)

    def pct(p):
        k = min(len(lat_ms) - 1, max(0, int(round(p / 100.0 * (len(lat_ms) - 1)))))
        return lat_ms[k]

    per_lat = {}
    for li, L in enumerate(SERVE_LATTICES):
        v = sorted(lat[i] * 1e3 for i, r in enumerate(tr) if r["lat"] == li)
        if v:
            per_lat["x".join(map(str, L))] = {"requests": len(v), "p50_ms": v[len(v) // 2],
                                              "p99_ms": v[min(len(v) - 1, int(round(0.99 * (len(v) - 1))))]}
    h2d = sum(r["nrhs"] * full[r["lat"]] * 16 for r in tr)
    res = {
        "metric": "serving p50/p99 latency and solves/s (Poisson 50 req/s; 8^4/16^3x32/24^3x48 mix)",
        "value": nsol / wall, "unit": "RHS solves/s", "requests_per_s": len(tr) / wall,
        "p50_ms": pct(50), "p99_ms": pct(99), "max_ms": lat_ms[-1], "per_lattice": per_lat,
        "requests": len(tr), "rhs_solves": nsol, "makespan_s": wall, "arrival_window_s": tr[-1]["t"],
        "capacity_rhs_per_s": nsol / burst_wall, "burst_makespan_s": burst_wall,
        "all_converged": conv, "status": code,
        "max_true_residual": max(r["true_residual"] for rr in reps for r in rr),
        "iterations_mean": float(np.mean([r["iterations"] for rr in reps for r in rr])),
        "config": {"workload": "serving stream", "lattices": SERVE_LATTICES, "weights": SERVE_WEIGHTS,
                   "rate_per_s": SERVE_RATE, "kappa": [0.120, 0.1375], "csw": [0.0, 1.0], "nrhs": [1, 12],
                   "configs_per_lattice": 3, "eps": SERVE_EPS, "tol": TOL, "precision": args.precision,
                   "columns_per_config": args.columns, "clover_slots_per_config": args.clover_slots,
                   "trace_seed": SERVE_SEED, "output_ring_per_lattice": args.out_ring,
                   "max_chunk": args.max_chunk},
        "e2e": {"h2d_bytes": h2d, "d2h_bytes": h2d},
        "device_bytes_resident": srv.device_bytes, "prepare_s": t_prep,
        "clocks": clk.summary(),
    }
    srv.close()
    return res


def summarize_serve(res):
    """The serving figures carried in the default bench line."""
    keep = ("value", "unit", "requests_per_s", "p50_ms", "p99_ms", "max_ms", "per_lattice", "requests",
            "rhs_solves", "makespan_s", "arrival_window_s", "capacity_rhs_per_s", "burst_makespan_s",
            "all_converged", "max_true_residual", "iterations_mean")
    out = {k: res[k] for k in keep if k in res}
    out["metric"] = res["metric"]
    out["offered_rhs_per_s"] = res["rhs_solves"] / max(res["arrival_window_s"], 1e-9)
    return out


def run_stencil(args):
    """Times one fused stencil variant alone (Dslash GB/s of the metric), e.g.
    for profiling: --stencil 24 24 24 48 --precision half --variant 2."""
    import qcu_cg_inverter_b200 as q
    hbm, src = peaks()
    with q.Context(tuple(args.stencil), 0) as c:
        c.generate_gauge(GAUGE_SEED, 0.5)
        c.set_half_operator(STORAGE[args.storage])
        if args.sb:
            c.set_shape(1, args.sb)
        elif not args.no_autotune:  # else: the shape from QCU_TUNE_CACHE or the default
            c.autotune(args.precision, args.nrhs)
        ms, nbytes = c.bench_stencil(args.precision, args.variant, args.nrhs, args.iters)
        storage = c.half_storage(args.nrhs)
    gbs = nbytes / (ms / 1e3) / 1e9
    print(json.dumps({"stencil": args.stencil, "precision": args.precision, "variant": args.variant,
                      "storage": storage,
                      "nrhs": args.nrhs, "ms_per_launch": ms, "bytes_per_launch": nbytes, "GBps": gbs,
                      "frac": gbs / hbm, "peak_source": src}), flush=True)


def run_dd(args, world, rank, local):
    """One lattice decomposed along t over the N ranks (strong scaling): the
    32^3x64 Wilson-clover solve of the large workload (kappa 0.1370, eps 0.5)
    on SlabContexts, halo exchange and sums over NCCL (one rank: NCCL to
    itself). Time per solve is the max over ranks of the CUDA-event time."""
    import torch
    import torch.distributed as dist

    import qcu_cg_inverter_b200 as q
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        comm = q.Comm.torch_distributed(local)
    else:
        comm = q.Comm.nccl(q.Comm.nccl_unique_id(), 1, 0, local)
    s = q.SlabContext(ROOF_LATTICE, comm, local)
    s.generate_gauge(GAUGE_SEED, LARGE_EPS)
    s.set_half_operator(STORAGE[args.storage])
    vh = s.volume // 2
    b = torch.empty(2 * vh * 12, dtype=torch.complex128, device=device)
    s.generate_spinor(b, 1, SOURCE_SEED)
    x = torch.zeros_like(b)
    stream = torch.cuda.ExternalStream(s.stream, device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    kw = dict(kappa=LARGE_KAPPA, csw=CSW, bc_t=BC_T, tol=TOL, delta=args.delta, precision=args.precision)
    for _ in range(max(args.warmup, 1)):
        rep = s.invert(x, b, **kw)[0]
    barrier(world, device)
    steps = max(1, min(args.steps, 5))
    t, rep = timed_steps(torch, device, stream, flush, lambda: s.invert(x, b, **kw)[0], steps)
    t = max_over_ranks(t, world, device)
    storage = s.half_storage(1)
    s.close()  # its CUDA graphs hold NCCL calls: released before the communicator
    comm.close()
    if rank != 0:
        return None
    return {"metric": "CG time to |r|/|b|<1e-10, one 32^3x64 lattice decomposed along t", "value": steps / t,
            "unit": "solves/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": t / steps * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": DTYPE[storage], "data": "synthetic",
            "config": {"workload": "32^3x64 Wilson-clover, t-slabs", "lattice": ROOF_LATTICE, "kappa": LARGE_KAPPA,
                       "csw": CSW, "eps": LARGE_EPS, "parallelism": f"t-slabs x{world}",
                       "transport": "nccl" if world == 1 or dist.get_backend() == "nccl" else "host"},
            "iterations": rep["iterations"], "reliable_updates": rep["reliable_updates"],
            "true_residual": rep["true_residual"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--stencil", type=int, nargs=4, default=None, help="time one stencil variant on this lattice")
    ap.add_argument("--variant", type=int, default=2, help="0 hop, 1 hop+A^-1, 2 hop+A^-1+xpay+out2+norm, 3 the CG update stencil (D^dag, xpay, x and r update, norm), 4 variant 2 without the norm")
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--sb", type=int, default=0, help="site lanes per block for --stencil (0 = library default)")
    ap.add_argument("--no-autotune", action="store_true", help="--stencil: keep the cached or default shape")
    ap.add_argument("--storage", default="auto", choices=sorted(STORAGE),
                    help="links and clover behind --precision half: 16-bit (compact), FP32 (fast), or the "
                         "library's choice by lattice size and RHS count (auto)")
    ap.add_argument("--multi", action="store_true", help="the 48-RHS 24^3x48 batch against FP64 single-RHS")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="half", choices=["half", "single", "double"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the large solve, the 48-RHS batch and the serving stream in the default line")
    ap.add_argument("--dd", action="store_true",
                    help="one 32^3x64 lattice decomposed along t over the --gpus ranks (strong scaling)")
    ap.add_argument("--plan", action="store_true",
                    help="print the rank layout each process sees (after any --gpus relaunch) and exit")
    ap.add_argument("--oracle-check", action="store_true", help="--multi: recompute each residual with the oracle")
    ap.add_argument("--delta", type=float, default=0.0, help="reliable-update factor (0 = library default)")
    ap.add_argument("--serve", action="store_true", help="the serving stream through the request server")
    ap.add_argument("--requests", type=int, default=300, help="--serve: requests in the timed trace")
    ap.add_argument("--columns", type=int, default=16, help="--serve: RHS columns per resident configuration")
    ap.add_argument("--clover-slots", type=int, default=8, help="--serve: clover fields per configuration")
    ap.add_argument("--out-ring", type=int, default=4, help="--serve: pinned output buffers per lattice")
    ap.add_argument("--max-chunk", type=int, default=8, help="--serve: most CG iterations between admissions")
    args = ap.parse_args()
    if args.serve:
        print(json.dumps(run_serve(args)), flush=True)
        return
    if args.stencil:
        run_stencil(args)
        return
    if args.multi:
        print(json.dumps(run_multi(args, check_oracle=args.oracle_check)), flush=True)
        return
    if check_world(args.gpus, os.environ) == "relaunch":
        cmd = relaunch_argv(args.gpus, sys.argv[1:])
        os.execv(cmd[0], cmd)
    world, rank, local = dist_setup()
    if args.plan:
        # launcher self-check: what each rank sees, no GPU work
        print(json.dumps({"rank": rank, "world": world, "local_rank": local, "n_gpus": world}), flush=True)
        barrier(world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.dd:
        out = run_dd(args, world, rank, local)
    elif args.impl == "reference":
        out = run_reference(args, world, rank, local)
    else:
        out = run_ours(args, world, rank, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
