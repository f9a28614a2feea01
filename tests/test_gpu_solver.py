"""The even-odd mixed-precision CG (qcuInvert) on the GPU.

Every solve is checked independently: the returned x is fed to the CPU
oracle's full operator M = A - kappa D and |b - M x| / |b| must be below the
requested tolerance (1e-10). Solutions are compared with the oracle's own FP64
Schur solve at 1e-8 relative (both are solutions to 1e-10 of a system with a
modest condition number).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda")


def host(t, shape):
    return t.cpu().numpy().reshape(shape)


def true_residual(oracle, x, b, U, L, kappa, csw, bc=-1.0):
    C = oracle.clover_build(U, L, kappa * csw)
    r = b - oracle.apply_full(x, U, C, L, kappa, bc)
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["double", "single", "half"])
def test_config1_wilson_even_source(cuda, qcu_lib, oracle, prec):
    """8^3x8 Wilson, kappa 0.12, no clover, antiperiodic t, eps 0.3, source on
    the even sites only, stop at true residual 1e-10."""
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 1, 0.3)
    b = oracle.full_spinor_random(L, 2)
    b[1] = 0
    with qcu_lib.Context(L) as c:
        c.load_gauge(dev(U))
        x = dev(np.zeros_like(b))
        rep = c.invert(x, dev(b), kappa=0.12, csw=0.0, bc_t=-1.0, tol=1e-10, precision=prec)[0]
    xh = host(x, b.shape)
    assert rep["converged"] and rep["true_residual"] < 1e-10
    assert true_residual(oracle, xh, b, U, L, 0.12, 0.0) < 1e-10
    xo, it, res = oracle.solve_schur(b, U, L, 0.12, 0.0, -1.0, 1e-11)
    assert np.linalg.norm(xh - xo) / np.linalg.norm(xo) < 1e-8


@pytest.mark.parametrize("prec", ["double", "single", "half", "half-compact"])
def test_clover_solve(cuda, qcu_lib, oracle, prec):
    """half = 16-bit spinors with FP32 links/clover; half-compact = all 16-bit."""
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 3, 0.4)
    b = oracle.full_spinor_random(L, 4)
    with qcu_lib.Context(L) as c:
        c.load_gauge(dev(U))
        if prec == "half-compact":
            c.set_half_operator(False)
            prec = "half"
        x = dev(np.zeros_like(b))
        rep = c.invert(x, dev(b), kappa=0.1375, csw=1.0, bc_t=-1.0, tol=1e-10, precision=prec)[0]
    xh = host(x, b.shape)
    assert rep["converged"], rep
    assert true_residual(oracle, xh, b, U, L, 0.1375, 1.0) < 1e-10
    if prec == "half":
        assert rep["reliable_updates"] >= 2


def test_multi_rhs_multi_kappa_equals_single(cuda, qcu_lib, oracle):
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 5, 0.4)
    kappas = [0.1360, 0.1365, 0.1370, 0.1375]
    bs = np.stack([oracle.full_spinor_random(L, 10 + r) for r in range(4)])
    with qcu_lib.Context(L) as c:
        c.load_gauge(dev(U))
        xb = dev(np.zeros_like(bs))
        reps = c.invert(xb, dev(bs), nrhs=4, kappas=kappas, csw=1.0, tol=1e-10, precision="half")
        xs = host(xb, bs.shape)
        for r in range(4):
            assert reps[r]["converged"]
            assert true_residual(oracle, xs[r], bs[r], U, L, kappas[r], 1.0) < 1e-10
            x1 = dev(np.zeros_like(bs[r]))
            c.invert(x1, dev(bs[r]), kappa=kappas[r], csw=1.0, tol=1e-10, precision="half")
            x1 = host(x1, bs[r].shape)
            assert np.linalg.norm(xs[r] - x1) / np.linalg.norm(x1) < 1e-8


@pytest.mark.parametrize("stage", [1, 2])
def test_batched_solve_with_staged_neighbours_is_bit_identical(cuda, qcu_lib, oracle, stage):
    """The RHS-paired stencils that stage far neighbours in shared memory
    store the same bits, so a whole batched solve (fresh context: its graphs
    are captured with the staged kernels) gives the same solution bits and
    iteration counts as with the unstaged kernels (both on the default launch
    shape: the sums of the solver's reductions depend on the shape)."""
    L = (8, 8, 8, 16)
    U = oracle.gauge_random(L, 6, 0.4)
    kappas = [0.1360, 0.1360, 0.1375, 0.1375, 0.1375]
    bs = np.stack([oracle.full_spinor_random(L, 40 + r) for r in range(len(kappas))])
    out = {}
    for st in (0, stage):
        qcu_lib.lib().qcuDebugSetPairStage(st)
        try:
            with qcu_lib.Context(L) as c:
                c.load_gauge(dev(U))
                xb = dev(np.zeros_like(bs))
                reps = c.invert(xb, dev(bs), nrhs=len(kappas), kappas=kappas, csw=1.0, tol=1e-10, precision="half",
                                autotune=0)
                out[st] = (host(xb, bs.shape), [r["iterations"] for r in reps])
        finally:
            qcu_lib.lib().qcuDebugSetPairStage(-1)
    assert np.array_equal(out[0][0], out[stage][0])
    assert out[0][1] == out[stage][1]
    for r, k in enumerate(kappas):
        assert true_residual(oracle, out[stage][0][r], bs[r], U, L, k, 1.0) < 1e-10


def test_successive_solves_with_different_parameters(cuda, qcu_lib, oracle):
    """One context, one batch size, solves that differ only in parameters the
    captured CUDA graphs would bake in (boundary, clover on/off, tolerance):
    each must solve its own system."""
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 8, 0.4)
    b = oracle.full_spinor_random(L, 9)
    cases = [dict(csw=1.0, bc_t=-1.0, tol=1e-10), dict(csw=0.0, bc_t=-1.0, tol=1e-10),
             dict(csw=1.0, bc_t=1.0, tol=1e-10), dict(csw=1.0, bc_t=-1.0, tol=1e-6)]
    with qcu_lib.Context(L) as c:
        c.load_gauge(dev(U))
        for kw in cases:
            x = dev(np.zeros_like(b))
            rep = c.invert(x, dev(b), kappa=0.13, precision="half", **kw)[0]
            xh = host(x, b.shape)
            C = oracle.clover_build(U, L, 0.13 * kw["csw"])
            res = np.linalg.norm(b - oracle.apply_full(xh, U, C, L, 0.13, kw["bc_t"])) / np.linalg.norm(b)
            assert rep["converged"] and res < kw["tol"], (kw, rep, res)


def test_bad_solve_arguments_are_rejected(cuda, qcu_lib, oracle):
    """Empty batches, non-positive or non-finite kappa, a zero tolerance, and a
    batch whose fields would pass 2^32 chunks: each returns INVALID_ARG and
    leaves the context usable."""
    import ctypes
    q = qcu_lib
    L = (8, 8, 8, 8)
    b = oracle.full_spinor_random(L, 4)
    with q.Context(L) as c:
        c.generate_gauge(1, 0.3)
        x, bd = dev(np.zeros_like(b)), dev(b)
        sp = q.solve_params(kappa=0.12)
        reps = (q.SolveReport * 1)()
        assert q.lib().qcuInvert(c._h, q._ptr(x), q._ptr(bd), 0, None, ctypes.byref(sp), reps) == q.QCU_ERR_INVALID_ARG
        for kw in (dict(kappa=0.0), dict(kappa=-0.1), dict(kappa=float("nan")), dict(kappa=0.12, tol=0.0)):
            with pytest.raises(q.QcuError) as e:
                c.invert(x, bd, **kw)
            assert e.value.code == q.QCU_ERR_INVALID_ARG, kw
        rep = c.invert(x, bd, kappa=0.12, csw=1.0)[0]
        assert rep["converged"]
    big = (32, 32, 32, 64)  # 1048576 sites per parity x 12 chunks x 400 RHS > 2^32
    with q.Context(big) as c:
        c.generate_gauge(1, 0.3)
        one = dev(np.zeros(1, complex))
        sp = q.solve_params(kappa=0.12)
        reps = (q.SolveReport * 400)()
        code = q.lib().qcuInvert(c._h, q._ptr(one), q._ptr(one), 400, None, ctypes.byref(sp), reps)
        assert code == q.QCU_ERR_INVALID_ARG


def test_nan_source_is_rejected(cuda, qcu_lib, oracle):
    L = (8, 8, 8, 8)
    b = oracle.full_spinor_random(L, 4)
    b[0, 3, 1, 2] = np.nan
    with qcu_lib.Context(L) as c:
        c.generate_gauge(1, 0.3)
        with pytest.raises(qcu_lib.QcuError) as e:
            c.invert(dev(np.zeros_like(b)), dev(b), kappa=0.12)
        assert e.value.code == qcu_lib.QCU_ERR_INVALID_ARG


def test_allocation_failure_is_reported(cuda, qcu_lib, oracle):
    L = (8, 8, 8, 8)
    b = oracle.full_spinor_random(L, 4)
    q = qcu_lib
    with q.Context(L) as c:
        c.generate_gauge(1, 0.3)
        q.lib().qcuDebugFailAllocAfter(3)
        try:
            with pytest.raises(q.QcuError) as e:
                c.invert(dev(np.zeros_like(b)), dev(b), kappa=0.12, csw=1.0)
            assert e.value.code == q.QCU_ERR_OUT_OF_MEMORY
        finally:
            q.lib().qcuDebugFailAllocAfter(-1)
        # the context stays usable
        x = dev(np.zeros_like(b))
        rep = c.invert(x, dev(b), kappa=0.12, csw=1.0)[0]
        assert rep["converged"]


def test_iteration_cap_reports_not_converged(cuda, qcu_lib, oracle):
    """A cap far below the iterations needed: every RHS stops at the cap with
    status NOT_CONVERGED, the returned x is the FP64-checked iterate (its
    reported true residual matches the oracle's), and the call raises only
    when asked to."""
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 12, 0.4)
    bs = np.stack([oracle.full_spinor_random(L, 30 + r) for r in range(3)])
    with qcu_lib.Context(L) as c:
        c.load_gauge(dev(U))
        xb = dev(np.zeros_like(bs))
        reps = c.invert(xb, dev(bs), nrhs=3, kappas=[0.125, 0.13, 0.135], csw=1.0, tol=1e-10, maxiter=7,
                        precision="half", raise_on_fail=False)
        xs = host(xb, bs.shape)
        for r, k in enumerate([0.125, 0.13, 0.135]):
            rep = reps[r]
            assert not rep["converged"] and rep["status"] == qcu_lib.QCU_ERR_NOT_CONVERGED
            assert 7 <= rep["iterations"] <= 8
            res = true_residual(oracle, xs[r], bs[r], U, L, k, 1.0)
            assert 1e-10 < res < 1.0
            assert abs(res - rep["true_residual"]) < 1e-6 * res
        with pytest.raises(qcu_lib.QcuError) as e:
            c.invert(dev(np.zeros_like(bs[0])), dev(bs[0]), kappa=0.13, csw=1.0, maxiter=5)
        assert e.value.code == qcu_lib.QCU_ERR_NOT_CONVERGED


def test_zero_source_converges_at_once(cuda, qcu_lib, oracle):
    L = (8, 8, 8, 8)
    b = np.zeros((2, 2048, 4, 3), complex)
    with qcu_lib.Context(L) as c:
        c.generate_gauge(3, 0.4)
        x = dev(np.ones_like(b))
        rep = c.invert(x, dev(b), kappa=0.13, csw=1.0)[0]
        assert rep["converged"] and rep["iterations"] == 0
        assert np.abs(host(x, b.shape)).max() == 0.0


def test_kernel_launches_are_counted(cuda, qcu_lib):
    with qcu_lib.Context((8, 8, 8, 8)) as c:
        c.generate_gauge(1, 0.3)
        n0 = c.launches
        ms, nbytes = c.bench_stencil("half", 1, 1, 5)
        assert c.launches > n0 and ms > 0 and nbytes > 0


def test_repeated_solves_reuse_the_first_solves_step_plan(cuda, qcu_lib, oracle):
    """Successive solves of one context start from the convergence rate the
    engine measured before. A finished column must not leave a no-progress
    rate behind: that made every solve after the first open with two
    64-iteration chunks, mostly masked (2.4x the kernels at delta 1.2e-2)."""
    L = (8, 8, 8, 8)
    b = oracle.full_spinor_random(L, 21)
    with qcu_lib.Context(L) as c:
        c.generate_gauge(4, 0.4)
        counts = []
        for _ in range(3):
            x = dev(np.zeros_like(b))
            n0 = c.launches
            rep = c.invert(x, dev(b), kappa=0.13, csw=1.0, tol=1e-10, precision="half", delta=0.012)[0]
            assert rep["converged"]
            counts.append(c.launches - n0)
        assert counts[1] == counts[2], counts
        assert counts[1] <= 1.1 * counts[0], counts


def test_solve_report_carries_time_and_bytes(cuda, qcu_lib, oracle):
    """Every report of a qcuInvert call carries the call's device time and
    GB/s and the RHS's own algorithmic bytes (positive, and growing with the
    iterations it took)."""
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 5, 0.4)
    bs = np.stack([oracle.full_spinor_random(L, 30 + r) for r in range(3)])
    with qcu_lib.Context(L) as c:
        c.load_gauge(dev(U))
        xb = dev(np.zeros_like(bs))
        reps = c.invert(xb, dev(bs), nrhs=3, kappas=[0.125, 0.13, 0.1375], csw=1.0, tol=1e-10, precision="half")
    secs = {r["seconds"] for r in reps}
    assert len(secs) == 1 and secs.pop() > 0
    total = sum(r["gbytes"] for r in reps)
    assert all(r["gbytes"] > 0 for r in reps)
    assert abs(reps[0]["gbytes_per_s"] * reps[0]["seconds"] - total) < 1e-9 * max(total, 1)
    # more iterations, more bytes
    order = sorted(reps, key=lambda r: r["iterations"])
    assert order[0]["gbytes"] <= order[-1]["gbytes"]
