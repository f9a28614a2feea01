"""The compact 16-bit operator (16-bit spinors, 16-bit 12-real links, 16-bit
clover with a per-site norm) on its single-RHS kernel family: paired decode of
links and clover, third link row rebuilt in the stencil, block-paired
epilogues.

Checked for every epilogue the solver uses, with D and D^dag:
  * against the generic compact kernel (the batched family, here run on two
    copies of the same column) on the same fields: the two differ only in the
    association of FP32 sums, so the stored 16-bit fields agree to within
    two steps of the 16-bit grid (6e-5 of each site's largest component);
  * against the FP64 oracle on inputs quantised by the 16-bit spinor storage:
    to 5e-4 of each site's largest component (the links' and the clover's own
    16-bit rounding comes on top of the spinors').
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CPRE, XPAY, CX, CPOST, OUT2, NORM, CGXR = 1, 2, 4, 8, 16, 32, 64
EPILOGUES = [0, CPRE, XPAY, XPAY | CX, XPAY | CPOST, CPRE | XPAY, CPRE | XPAY | NORM, CPRE | XPAY | OUT2,
             CPRE | XPAY | OUT2 | NORM, XPAY | NORM]
LATTICES = [(8, 8, 8, 8), (6, 4, 4, 2)]
CSW, COEF = 0.1375, -0.018


def half(L):
    return L[0] * L[1] * L[2] * L[3] // 2


@pytest.fixture(scope="module", params=LATTICES, ids=lambda L: "x".join(map(str, L)))
def ctx(request, cuda, qcu_lib, oracle):
    L = request.param
    U = oracle.gauge_random(L, 9, 0.4)
    c = qcu_lib.Context(L)
    c.load_gauge(U)
    c.set_half_operator(False)
    yield c, U, L
    c.close()


def site_err(got, ref):
    return float((np.abs(got - ref).max(axis=(-2, -1)) / np.abs(ref).max(axis=(-2, -1))).max())


def quantised(c, v):
    z = np.zeros_like(v)
    n = len(v)
    return c.debug_stencil("half", 0, XPAY, z, [0.0] * n, [0.0] * n, x=v, out=np.zeros_like(v))["out"]


def launch(c, epi, dag, f, nrhs, **kw):
    """One launch on nrhs copies of column 0 (nrhs 1: the single-RHS family)."""
    rep = lambda a: None if a is None else np.repeat(a[:1], nrhs, axis=0)  # noqa: E731
    return c.debug_stencil("half", dag, epi, rep(f["in"]), [CSW] * nrhs, [COEF] * nrhs,
                           x=rep(f["x"]) if epi & (XPAY | CGXR) else None,
                           out=rep(f["out"]), out2=rep(f["out2"]) if epi & OUT2 else None,
                           pvec=rep(f.get("p")) if epi & CGXR else None,
                           xacc=rep(f.get("xa")) if epi & CGXR else None,
                           racc=rep(f.get("ra")) if epi & CGXR else None,
                           alpha=[0.7] * nrhs if epi & CGXR else None, **kw)


def fields(c, oracle, L, seed):
    names = ("in", "x", "out", "out2", "p", "xa", "ra")
    return {n: quantised(c, oracle.spinor_random(half(L), seed + k)[None]) for k, n in enumerate(names)}


@pytest.mark.parametrize("dag", [0, 1])
@pytest.mark.parametrize("epi", EPILOGUES)
def test_single_rhs_compact_family_against_generic_and_oracle(ctx, oracle, epi, dag):
    c, U, L = ctx
    f = fields(c, oracle, L, 31 * (epi + 1) + dag)
    a = launch(c, epi, dag, f, 1)
    b = launch(c, epi, dag, f, 2)
    assert site_err(a["out"][0], b["out"][0]) < 6e-5
    if epi & OUT2:
        assert site_err(a["out2"][0], b["out2"][0]) < 6e-5
    if epi & NORM:
        assert abs(a["norms"][0] / b["norms"][0] - 1) < 1e-5
    # FP64 oracle on the same (quantised) spinors
    Ci = oracle.clover_invert(oracle.clover_build(U, L, CSW))[0]
    t = oracle.dslash(f["in"][0], U, L, 0, dag, -1.0)
    if epi & CPRE:
        t = oracle.clover_apply(t, np.ascontiguousarray(Ci))
    y = t
    if epi & XPAY:
        xv = oracle.clover_apply(f["x"][0], np.ascontiguousarray(Ci)) if epi & CX else f["x"][0]
        y = xv + COEF * t
        if epi & CPOST:
            y = oracle.clover_apply(y, np.ascontiguousarray(Ci))
    assert site_err(a["out"][0], y) < 5e-4
    if epi & OUT2:
        assert site_err(a["out2"][0], oracle.clover_apply(y, np.ascontiguousarray(Ci))) < 5e-4
    if epi & NORM:
        assert abs(a["norms"][0] / np.vdot(y, y).real - 1) < 1e-3


@pytest.mark.parametrize("dag", [0, 1])
def test_single_rhs_compact_cg_update(ctx, oracle, dag):
    """x += alpha p, r -= alpha z with z = x_in + coef D in (the CG's last
    stencil), single-RHS compact kernel against the generic one and FP64."""
    c, U, L = ctx
    f = fields(c, oracle, L, 4242 + dag)
    a = launch(c, XPAY | CGXR, dag, f, 1)
    b = launch(c, XPAY | CGXR, dag, f, 2)
    for k in ("xacc", "racc"):
        assert site_err(a[k][0], b[k][0]) < 6e-5
    z = f["x"][0] + COEF * oracle.dslash(f["in"][0], U, L, 0, dag, -1.0)
    xr = f["xa"][0] + 0.7 * f["p"][0]
    rr = f["ra"][0] - 0.7 * z
    assert site_err(a["xacc"][0], xr) < 1e-4
    assert site_err(a["racc"][0], rr) < 5e-4
    assert abs(a["norms"][0] / np.vdot(rr, rr).real - 1) < 1e-3
