"""Batched 16-bit stencils: the RHS-paired kernels (two right-hand sides per
thread in the lanes of paired FP32 instructions) against the kernels with one
RHS per thread, and both against the CPU operator.

Per lane the paired kernels do the same roundings in the same order, so every
stored 16-bit field must be bit-identical between the two families, for every
epilogue the solver uses, with a batch that has an odd RHS count, an inactive
column, a column without clover and two clover fields, so that pairs are
uniform, mixed (clover next to Wilson) and half-empty. Only the per-RHS norms
may differ, in the last bits (their block sums group sites differently).
Against the FP64 oracle the tolerance is that of 16-bit storage: 2e-4 of the
largest component, on inputs quantised the same way.

The paired kernels that stage the t neighbours' words (stage 1), or the z and
t neighbours' (stage 2), in shared memory store the same bits as well."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CPRE, XPAY, CX, CPOST, OUT2, NORM, CGXR = 1, 2, 4, 8, 16, 32, 64
EPILOGUES = [0, CPRE, XPAY, XPAY | CX, XPAY | CPOST, CPRE | XPAY, CPRE | XPAY | NORM, CPRE | XPAY | OUT2,
             CPRE | XPAY | OUT2 | NORM, XPAY | NORM]
LATTICES = [(8, 8, 8, 8), (6, 4, 4, 2)]  # the second: half volume 96, not a multiple of 32
CSW = [0.13, 0.13, 0.0, 0.1375, 0.1375]  # kappa*c_sw per RHS; 0 = no clover term
COEF = [-0.017, -0.019, -0.016, -0.018, -0.015]
ACTIVE = [1, 1, 1, 0, 1]


def half(L):
    return L[0] * L[1] * L[2] * L[3] // 2


@pytest.fixture(scope="module", params=LATTICES, ids=lambda L: "x".join(map(str, L)))
def ctx(request, cuda, qcu_lib, oracle):
    L = request.param
    U = oracle.gauge_random(L, 7, 0.4)
    c = qcu_lib.Context(L)
    c.load_gauge(U)
    yield c, U, L
    c.close()


def spinors(oracle, L, seed, n=len(CSW)):
    return np.stack([oracle.spinor_random(half(L), seed + r) for r in range(n)])


def run(c, epi, dag, pairs, fields, **kw):
    return c.debug_stencil("half", dag, epi, fields["in"], CSW, COEF, active=ACTIVE,
                           x=fields["x"] if epi & XPAY else None, out=fields["out"].copy(),
                           out2=fields["out2"].copy() if epi & OUT2 else None, rhs_pairs=pairs, **kw)


@pytest.mark.parametrize("stage", [0, 1, 2])
@pytest.mark.parametrize("dag", [0, 1])
@pytest.mark.parametrize("epi", EPILOGUES)
def test_paired_kernels_store_the_same_bits(ctx, oracle, qcu_lib, epi, dag, stage):
    c, U, L = ctx
    f = dict(zip(("in", "x", "out", "out2"), (spinors(oracle, L, 100 * k) for k in range(1, 5))))
    qcu_lib.lib().qcuDebugSetPairStage(stage)
    try:
        a = run(c, epi, dag, 1, f)
    finally:
        qcu_lib.lib().qcuDebugSetPairStage(-1)
    b = run(c, epi, dag, 0, f)
    assert np.array_equal(a["out"], b["out"])
    if epi & OUT2:
        assert np.array_equal(a["out2"], b["out2"])
    if epi & NORM:
        act = np.array(ACTIVE, bool)
        assert np.allclose(a["norms"][act], b["norms"][act], rtol=1e-12, atol=0)
        assert np.all(a["norms"][~act] == 0) and np.all(b["norms"][~act] == 0)


def quantised(c, oracle, L, v):
    """v after the round trip through 16-bit storage: the launch out = x + 0 D 0
    stores x as it is."""
    z = np.zeros_like(v)
    r = c.debug_stencil("half", 0, XPAY, z, [0.0] * len(v), [0.0] * len(v), x=v, out=np.zeros_like(v), rhs_pairs=1)
    return r["out"]


@pytest.mark.parametrize("dag", [0, 1])
def test_fused_cg_stencil_matches_the_oracle(ctx, oracle, dag):
    """y = x + coef A^-1 D in, second output A^-1 y, norm |y|^2 (the CG's
    fused half-step) against FP64 on the same quantised inputs."""
    c, U, L = ctx
    inp, x = quantised(c, oracle, L, spinors(oracle, L, 500)), quantised(c, oracle, L, spinors(oracle, L, 600))
    out0, out20 = spinors(oracle, L, 700), spinors(oracle, L, 800)
    epi = CPRE | XPAY | OUT2 | NORM
    r = c.debug_stencil("half", dag, epi, inp, CSW, COEF, active=ACTIVE, x=x, out=out0.copy(), out2=out20.copy(),
                        rhs_pairs=1)
    clov = {k: oracle.clover_invert(oracle.clover_build(U, L, k)) for k in set(CSW) if k > 0}
    errs = {}
    for j in range(len(CSW)):
        if not ACTIVE[j]:
            continue
        t = oracle.dslash(inp[j], U, L, 0, dag, -1.0)
        if CSW[j] > 0:
            t = oracle.clover_apply(t, np.ascontiguousarray(clov[CSW[j]][0]))
        y = x[j] + COEF[j] * t
        y2 = oracle.clover_apply(y, np.ascontiguousarray(clov[CSW[j]][0])) if CSW[j] > 0 else y
        for name, got, ref in (("out", r["out"][j], y), ("out2", r["out2"][j], y2)):
            errs[(j, name)] = float((np.abs(got - ref).max(axis=(1, 2)) / np.abs(ref).max(axis=(1, 2))).max())
        errs[(j, "norm")] = abs(r["norms"][j] / np.vdot(y, y).real - 1)
    assert max(errs.values()) < 2e-4, errs
    # the inactive column is not written
    inactive = [j for j in range(len(CSW)) if not ACTIVE[j]]
    b = run(c, epi, dag, 0, dict(**{"in": inp, "x": x, "out": out0, "out2": out20}))
    for j in inactive:
        assert np.array_equal(r["out"][j], b["out"][j])


@pytest.mark.parametrize("dag", [0, 1])
def test_fused_cg_update_matches_between_families_and_fp64(ctx, oracle, dag):
    """x += alpha p, r -= alpha z with z = x_in + coef D in (the CG's last
    stencil): bit-identical between the families; against FP64 on the same
    quantised inputs within the precision of the accumulators' storage
    (16-bit with a site norm: 5e-5 of each site's largest component)."""
    c, U, L = ctx
    inp, xin, p, xa, ra = (quantised(c, oracle, L, spinors(oracle, L, s)) for s in (900, 1000, 1100, 1200, 1300))
    alpha = [0.5, 0.7, 0.9, 1.1, 1.3]
    res = []
    for pairs in (1, 0):
        res.append(c.debug_stencil("half", dag, XPAY | CGXR, inp, CSW, COEF, active=ACTIVE, x=xin, pvec=p,
                                   xacc=xa.copy(), racc=ra.copy(), alpha=alpha, rhs_pairs=pairs))
    a, b = res
    assert np.array_equal(a["xacc"], b["xacc"]) and np.array_equal(a["racc"], b["racc"])
    act = np.array(ACTIVE, bool)
    assert np.allclose(a["norms"][act], b["norms"][act], rtol=1e-12, atol=0)
    for j in range(len(CSW)):
        if not ACTIVE[j]:
            continue
        z = xin[j] + COEF[j] * oracle.dslash(inp[j], U, L, 0, dag, -1.0)
        xr = xa[j] + alpha[j] * p[j]
        rr = ra[j] - alpha[j] * z
        for got, ref in ((a["xacc"][j], xr), (a["racc"][j], rr)):
            err = np.abs(got - ref).max(axis=(1, 2)) / np.abs(ref).max(axis=(1, 2))
            assert err.max() < 5e-5, (j, err.max())
        # the norm is of r before it is stored
        assert abs(a["norms"][j] - np.vdot(rr, rr).real) < 1e-4 * a["norms"][j]
