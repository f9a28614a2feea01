"""GPU parity of every operator entry point against the CPU oracle.

FP64 tolerance: 1e-12 relative (norm-wise and entry-wise) for the hopping
term and every composition; operators that go through the clover inverse at
the reference normalisation (kappa*c_sw = 1, where blocks can be indefinite and
ill-conditioned) are compared at 1e-10 - the library factors with LDL^H, the
reference and the oracle with Gauss-Jordan elimination.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL_INV = 1e-10
LATTICES = [(8, 8, 8, 8), (6, 4, 4, 2)]  # the second has a half volume not a multiple of 32


def close(a, b, tol):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) <= tol * nb and np.abs(a - b).max() <= tol * np.abs(b).max()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda")


def host(t, shape):
    return t.cpu().numpy().reshape(shape)


@pytest.fixture(scope="module", params=LATTICES, ids=lambda L: "x".join(map(str, L)))
def setup(request, cuda, qcu_lib, oracle):
    L = request.param
    U = oracle.gauge_random(L, 2024, 0.3)
    psi = oracle.full_spinor_random(L, 11)
    C = oracle.clover_build(U, L, 1.0)
    Ci = oracle.clover_invert(C)
    q = qcu_lib
    p = q.param(L)
    dU = dev(U)
    q.initGridSize((1, 1, 1, 1), p, dU)
    q.loadQcuGauge(dU, p)
    return dict(L=L, U=U, psi=psi, C=C, Ci=Ci, q=q, p=p, dU=dU)


def test_dslashQcu(setup, oracle):
    s = setup
    L, Vh = s["L"], s["psi"].shape[1]
    for par in (0, 1):
        inp = dev(s["psi"][1 - par])
        out = dev(np.zeros((Vh, 4, 3), complex))
        s["q"].dslashQcu(out, inp, s["dU"], s["p"], par)
        ref = oracle.dslash(np.ascontiguousarray(s["psi"][1 - par]), s["U"], L, par)
        assert close(host(out, ref.shape), ref, TOL)


@pytest.mark.parametrize("dag", [0, 1])
def test_fullDslashQcu(setup, oracle, dag):
    s = setup
    out = dev(np.zeros_like(s["psi"]))
    s["q"].fullDslashQcu(out, dev(s["psi"]), s["dU"], s["p"], dag)
    ref = oracle.full_dslash_ref(s["psi"], s["U"], s["C"], s["Ci"], s["L"], dag)
    assert close(host(out, ref.shape), ref, TOL_INV)
    # (A - D) without the A A^-1 round trip of the reference
    Dp = np.stack([oracle.dslash(np.ascontiguousarray(s["psi"][1 - p]), s["U"], s["L"], p, dag) for p in (0, 1)])
    Ap = np.stack([oracle.clover_apply(np.ascontiguousarray(s["psi"][p]), np.ascontiguousarray(s["C"][p])) for p in (0, 1)])
    assert close(host(out, ref.shape), Ap - Dp, TOL)


def test_invertCloverDslash_is_in_place(setup, oracle):
    s = setup
    t = dev(s["psi"])
    other = dev(np.zeros_like(s["psi"]))
    s["q"].invertCloverDslash(t, other, s["dU"], s["p"], 0)  # `in` ignored, as in the reference
    ref = oracle.invert_clover_ref(s["psi"], s["Ci"], s["L"])
    assert close(host(t, ref.shape), ref, TOL_INV)


def test_preCloverDslash(setup, oracle):
    s = setup
    t = dev(s["psi"])
    s["q"].preCloverDslash(t, t, s["dU"], s["p"])
    ref = np.stack([oracle.clover_apply(np.ascontiguousarray(s["psi"][p]), np.ascontiguousarray(s["C"][p])) for p in (0, 1)])
    assert close(host(t, ref.shape), ref, TOL)


@pytest.mark.parametrize("dag", [0, 1])
def test_one_round_compositions(setup, oracle, dag):
    s = setup
    q, L = s["q"], s["L"]
    out = dev(np.zeros_like(s["psi"]))
    q.newFullCloverDslashOneRound(out, dev(s["psi"]), s["dU"], s["p"], dag)
    assert close(host(out, s["psi"].shape), oracle.new_full_ref(s["psi"], s["U"], s["Ci"], L, dag), TOL_INV)
    q.cloverDslashOneRound(out, dev(s["psi"]), s["dU"], s["p"], dag)
    ref = np.stack([oracle.clover_apply(oracle.dslash(np.ascontiguousarray(s["psi"][1 - p]), s["U"], L, p, dag),
                                        np.ascontiguousarray(s["Ci"][p])) for p in (0, 1)])
    assert close(host(out, ref.shape), ref, TOL_INV)


def test_MmV_one_round(setup, oracle):
    s = setup
    out = dev(np.zeros_like(s["psi"]))
    tmp = dev(np.zeros_like(s["psi"]))
    s["q"].MmV_one_round(out, dev(s["psi"]), s["dU"], s["p"], tmp)
    ref = oracle.mmv_ref(s["psi"], s["U"], s["Ci"], s["L"])
    assert close(host(out, ref.shape), ref, TOL_INV)
    assert close(host(tmp, ref.shape), oracle.new_full_ref(s["psi"], s["U"], s["Ci"], s["L"], 0), TOL_INV)


def test_reference_cg_flow_matches_oracle(cuda, qcu_lib, oracle):
    """cg_inverter on a pure-gauge field (where the reference's CG converges):
    same solution and the same iteration count as the oracle's restatement."""
    L = (8, 8, 8, 8)
    U = oracle.gauge_pure(L, 7)
    b = oracle.full_spinor_random(L, 11)
    q = qcu_lib
    p = q.param(L)
    dU = dev(U)
    q.initGridSize((1, 1, 1, 1), p, dU)
    x = dev(np.zeros_like(b))
    it, conv = q.cg_inverter_ref(dev(b), x, dU, p)
    xr, itr, convr = oracle.cg_inverter_ref(b, U, L, 0)
    assert conv and convr and abs(it - itr) <= 1
    assert close(host(x, b.shape), xr, 1e-9)
    # the legacy entry point gives the same x
    x2 = dev(np.zeros_like(b))
    q.cg_inverter(dev(b), x2, dU, p)
    assert close(host(x2, b.shape), xr, 1e-9)


@pytest.fixture(scope="module")
def ctx8(cuda, qcu_lib, oracle):
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 99, 0.4)
    c = qcu_lib.Context(L)
    c.load_gauge(dev(U))
    yield c, U, L
    c.close()


@pytest.mark.parametrize("bc", [1.0, -1.0])
@pytest.mark.parametrize("dag", [0, 1])
def test_context_dslash_with_time_boundary(ctx8, oracle, bc, dag):
    c, U, L = ctx8
    x = oracle.spinor_random(2048, 3)
    out = dev(np.zeros_like(x))
    c.dslash(out, dev(x), 0, dag, bc)
    assert close(host(out, x.shape), oracle.dslash(x, U, L, 0, dag, bc), TOL)


@pytest.mark.parametrize("inverse", [False, True])
def test_context_clover(ctx8, oracle, inverse):
    c, U, L = ctx8
    psi = oracle.full_spinor_random(L, 4)
    C = oracle.clover_build(U, L, 0.1375)
    M = oracle.clover_invert(C) if inverse else C
    out = dev(np.zeros_like(psi))
    c.apply_clover(out, dev(psi), 0.1375, inverse)
    ref = np.stack([oracle.clover_apply(np.ascontiguousarray(psi[p]), np.ascontiguousarray(M[p])) for p in (0, 1)])
    assert close(host(out, psi.shape), ref, TOL)


@pytest.mark.parametrize("dag", [0, 1])
def test_context_operator(ctx8, oracle, dag):
    c, U, L = ctx8
    psi = oracle.full_spinor_random(L, 5)
    kappa, csw = 0.1375, 1.0
    C = oracle.clover_build(U, L, kappa * csw)
    out = dev(np.zeros_like(psi))
    c.apply_operator(out, dev(psi), kappa, csw, -1.0, dag)
    assert close(host(out, psi.shape), oracle.apply_full(psi, U, C, L, kappa, -1.0, dag), TOL)


def test_generators_match_oracle(cuda, qcu_lib, oracle):
    L = (8, 8, 8, 8)
    with qcu_lib.Context(L) as c:
        c.generate_gauge(31, 0.4)
        g = dev(np.zeros((4, 2, 2048, 3, 3), complex))
        c.export_gauge(g)
        assert close(host(g, (4, 2, 2048, 3, 3)), oracle.gauge_random(L, 31, 0.4), 1e-13)
        s = dev(np.zeros((2, 2, 2048, 4, 3), complex))
        c.generate_spinor(s, 2, 40)
        got = host(s, (2, 2, 2048, 4, 3))
        assert close(got[0], oracle.full_spinor_random(L, 40), 1e-14)
        assert close(got[1], oracle.full_spinor_random(L, 41), 1e-14)


def test_host_pointers_are_staged(cuda, qcu_lib, oracle):
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 5, 0.3)
    with qcu_lib.Context(L) as c:
        c.load_gauge(U)  # numpy (host) array
        x = oracle.spinor_random(2048, 6)
        out = np.zeros_like(x)
        c.dslash(out, x, 1, 0, 1.0)
        assert close(out, oracle.dslash(x, U, L, 1), TOL)


@pytest.mark.parametrize("L", LATTICES, ids=lambda L: "x".join(map(str, L)))
def test_storage_shifts_match_the_oracle(cuda, qcu_lib, oracle, L):
    """shiftVectorStorage / shiftGaugeStorage (the reference's AoS <-> SoA
    shifts) against the oracle's restatement: the transposes bit for bit, the
    rebuilt third row of the links to rounding. The second lattice's half
    volume (96) is not a multiple of the kernels' 128-site tile."""
    nh = L[0] * L[1] * L[2] * L[3] // 2
    psi = oracle.spinor_random(nh, 17)
    soa = dev(np.zeros(24 * nh))
    qcu_lib.shiftVectorStorage(soa, dev(psi), 0, L)
    assert np.array_equal(host(soa, (24, nh)), oracle.shift_vector_storage(psi, 0))
    back = dev(np.zeros_like(psi))
    qcu_lib.shiftVectorStorage(back, soa, 1, L)
    assert np.array_equal(host(back, psi.shape), psi)
    U = oracle.gauge_random(L, 23, 0.4)
    g = dev(np.zeros(8 * 12 * nh))
    qcu_lib.shiftGaugeStorage(g, dev(U), 0, L)
    ref = oracle.shift_gauge_storage(U, 0)
    assert np.array_equal(host(g, ref.shape), ref)
    Ub = dev(np.zeros_like(U))
    qcu_lib.shiftGaugeStorage(Ub, g, 1, L)
    got = host(Ub, U.shape)
    assert np.array_equal(got[..., :2, :], U[..., :2, :])
    assert close(got, oracle.shift_gauge_storage(ref, 1), 1e-14)


def test_storage_shifts_reject_host_pointers(cuda, qcu_lib, oracle):
    L = (4, 4, 4, 4)
    psi = oracle.spinor_random(128, 1)
    with pytest.raises(qcu_lib.QcuError) as e:
        qcu_lib.shiftVectorStorage(np.zeros(24 * 128), psi, 0, L)
    assert e.value.code == qcu_lib.QCU_ERR_INVALID_ARG
