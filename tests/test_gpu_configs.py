"""Parity at the benchmarked sizes, not only at toy lattices.

Every case uses the bench's own workloads (seeded SU(3) links exp(i eps H),
generated on the GPU by the library's counter-based generator and exported to
the host, so the oracle sees identical inputs):

  * 16^3x32 Wilson-clover, kappa 0.1375, c_sw 1, eps 0.4, antiperiodic t
    (the headline solve), in 16-bit mixed precision and in FP64: the solution
    against the oracle's FP64 Schur solve, and the oracle's true residual;
  * 24^3x48, 12 point sources spanning the four kappas of the multi-RHS
    batch, one batched mixed-precision solve: every column's true residual
    recomputed by the oracle;
  * 32^3x64 (eps 0.5): the FP64 hop (dslashQcu, both parities) and
    fullDslashQcu against the oracle at 1e-12, and the large mixed-precision
    solve (kappa 0.1370) with its true residual recomputed by the oracle.

Tolerances: 1e-12 relative for the FP64 operators; solves must reach a true
residual below 1e-10 by the oracle's FP64 operator; two solutions of the same
system to 1e-10 agree to 1e-8 relative (the system's condition number times
the residual bounds their difference; measured 6e-11 at 16^3x32).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAUGE_SEED, SOURCE_SEED = 20241, 7
BC_T = -1.0


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda")


def rel(a, b):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def close(a, b, tol):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    return np.linalg.norm(a - b) <= tol * np.linalg.norm(b) and np.abs(a - b).max() <= tol * np.abs(b).max()


def gauge_of(ctx, seed, eps):
    ctx.generate_gauge(seed, eps)
    V = ctx.volume
    U = np.zeros((4, 2, V // 2, 3, 3), complex)
    ctx.export_gauge(U)
    return U


def oracle_residual(oracle, x, b, U, L, kappa, csw, C=None):
    if C is None:
        C = oracle.clover_build(U, L, kappa * csw)
    return np.linalg.norm(b - oracle.apply_full(x, U, C, L, kappa, BC_T)) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["half", "double"])
def test_headline_solve_16x16x16x32_matches_oracle(cuda, qcu_lib, oracle, prec):
    import torch
    L, kappa, csw = (16, 16, 16, 32), 0.1375, 1.0
    with qcu_lib.Context(L) as c:
        U = gauge_of(c, GAUGE_SEED, 0.4)
        V = c.volume
        bt = torch.empty(V * 12, dtype=torch.complex128, device="cuda")
        c.generate_spinor(bt, 1, SOURCE_SEED)
        x = torch.zeros_like(bt)
        rep = c.invert(x, bt, kappa=kappa, csw=csw, bc_t=BC_T, tol=1e-10, precision=prec)[0]
        b = bt.cpu().numpy().reshape(2, V // 2, 4, 3)
        xh = x.cpu().numpy().reshape(b.shape)
    assert rep["converged"], rep
    assert oracle_residual(oracle, xh, b, U, L, kappa, csw) < 1e-10
    xo, it, res = oracle.solve_schur(b, U, L, kappa, csw, BC_T, 1e-10)
    assert res < 1e-10
    assert rel(xh, xo) < 1e-8


def test_multi_rhs_24x24x24x48_residuals_by_oracle(cuda, qcu_lib, oracle):
    """12 point sources (3 spin-colour components x 4 kappas) at one site of
    the 24^3x48 lattice, one batched solve; each column checked on its own."""
    import torch
    L, csw = (24, 24, 24, 48), 1.0
    kappas = (0.1360, 0.1365, 0.1370, 0.1375)
    comps = (0, 5, 11)
    with qcu_lib.Context(L) as c:
        U = gauge_of(c, GAUGE_SEED, 0.4)
        V = c.volume
        site = 12345
        b = torch.zeros(len(kappas) * len(comps), 2, V // 2, 12, dtype=torch.complex128, device="cuda")
        kap = []
        for j, k in enumerate(kappas):
            for i, comp in enumerate(comps):
                b[j * len(comps) + i, 0, site, comp] = 1.0
                kap.append(k)
        b = b.reshape(len(kap), -1).contiguous()
        x = torch.zeros_like(b)
        reps = c.invert(x, b, nrhs=len(kap), kappas=kap, csw=csw, bc_t=BC_T, tol=1e-10, precision="half")
        assert all(r["converged"] for r in reps), reps
        for j, k in enumerate(kappas):
            C = oracle.clover_build(U, L, k * csw)
            for i in range(len(comps)):
                r = j * len(comps) + i
                xr = x[r].cpu().numpy().reshape(2, V // 2, 4, 3)
                br = b[r].cpu().numpy().reshape(2, V // 2, 4, 3)
                res = oracle_residual(oracle, xr, br, U, L, k, csw, C)
                assert res < 1e-10, (r, k, res, reps[r])


@pytest.fixture(scope="module")
def large(cuda, qcu_lib):
    """The 32^3x64 gauge field (eps 0.5) and a Gaussian full spinor."""
    import torch
    L = (32, 32, 32, 64)
    with qcu_lib.Context(L) as c:
        U = gauge_of(c, GAUGE_SEED, 0.5)
        V = c.volume
        psi = torch.empty(V * 12, dtype=torch.complex128, device="cuda")
        c.generate_spinor(psi, 1, SOURCE_SEED)
        psi_h = psi.cpu().numpy().reshape(2, V // 2, 4, 3)
    return dict(L=L, U=U, psi=psi_h, V=V)


def test_fp64_operators_32x32x32x64_match_oracle(large, qcu_lib, oracle):
    q, L, U, psi, V = qcu_lib, large["L"], large["U"], large["psi"], large["V"]
    p = q.param(L)
    dU = dev(U)
    q.initGridSize((1, 1, 1, 1), p, dU)
    q.loadQcuGauge(dU, p)
    Dp = []
    for par in (0, 1):
        out = dev(np.zeros((V // 2, 4, 3), complex))
        q.dslashQcu(out, dev(psi[1 - par]), dU, p, par)
        ref = oracle.dslash(np.ascontiguousarray(psi[1 - par]), U, L, par)
        assert close(out.cpu().numpy().reshape(ref.shape), ref, 1e-12), par
        Dp.append(ref)
    out = dev(np.zeros_like(psi))
    q.fullDslashQcu(out, dev(psi), dU, p, 0)
    C = oracle.clover_build(U, L, 1.0)
    Ap = np.stack([oracle.clover_apply(np.ascontiguousarray(psi[par]), np.ascontiguousarray(C[par]))
                   for par in (0, 1)])
    assert close(out.cpu().numpy().reshape(psi.shape), Ap - np.stack(Dp), 1e-12)


def test_large_solve_32x32x32x64_residual_by_oracle(large, qcu_lib, oracle):
    import torch
    L, U, psi, V = large["L"], large["U"], large["psi"], large["V"]
    kappa, csw = 0.1370, 1.0
    with qcu_lib.Context(L) as c:
        c.load_gauge(dev(U))
        x = torch.zeros(V * 12, dtype=torch.complex128, device="cuda")
        rep = c.invert(x, dev(psi), kappa=kappa, csw=csw, bc_t=BC_T, tol=1e-10, precision="half")[0]
        xh = x.cpu().numpy().reshape(psi.shape)
    assert rep["converged"], rep
    assert oracle_residual(oracle, xh, psi, U, L, kappa, csw) < 1e-10
