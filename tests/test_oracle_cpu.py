"""Known-answer and structural checks of the CPU oracle (no GPU).

These pin properties any correct restatement of the reference must have,
independently of the reference's own outputs (which test_oracle_golden.py
compares against): exact adjointness of the dagger flag, gauge covariance,
the free-field spectrum, a trivial clover for pure-gauge fields, clover
Hermiticity and inverse, and convergence of the solvers.
"""
import numpy as np
import pytest

L8 = (8, 8, 8, 8)
L4 = (4, 4, 4, 4)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_gauge_field_is_su3(oracle):
    U = oracle.gauge_random(L4, 5, 0.4).reshape(-1, 3, 3)
    eye = np.eye(3)
    assert np.abs(U @ U.conj().transpose(0, 2, 1) - eye).max() < 1e-13
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-13


def test_generators_are_deterministic(oracle):
    a = oracle.gauge_random(L4, 9, 0.3)
    b = oracle.gauge_random(L4, 9, 0.3)
    assert np.array_equal(a, b)
    s1 = oracle.spinor_random(100, 3)
    s2 = oracle.spinor_random(100, 3)
    assert np.array_equal(s1, s2)
    # complex Gaussian with unit variance per real component
    s = oracle.spinor_random(20000, 4).view(np.float64)
    assert abs(s.mean()) < 0.01 and abs(s.std() - 1) < 0.01


@pytest.mark.parametrize("bc", [1.0, -1.0])
@pytest.mark.parametrize("parity", [0, 1])
def test_dagger_flag_is_the_adjoint(oracle, bc, parity):
    Vh = 4096 // 2
    U = oracle.gauge_random(L8, 1234, 0.3)
    x = oracle.spinor_random(Vh, 7)
    y = oracle.spinor_random(Vh, 8)
    Dx = oracle.dslash(x, U, L8, parity, 0, bc)
    Ddy = oracle.dslash(y, U, L8, 1 - parity, 1, bc)
    lhs, rhs = oracle.cdot(y, Dx), oracle.cdot(Ddy, x)
    assert abs(lhs - rhs) < 1e-13 * abs(lhs)


def test_gauge_covariance(oracle):
    U = oracle.gauge_random(L8, 1234, 0.3)
    g = oracle.su3_field(L8, 99)
    Ug = oracle.gauge_transform(U, g, L8)
    psi = oracle.full_spinor_random(L8, 5)
    psig = oracle.spinor_transform(psi, g, L8)
    for p in (0, 1):
        a = oracle.dslash(np.ascontiguousarray(psig[1 - p]), Ug, L8, p)
        full = np.zeros_like(psi)
        full[p] = oracle.dslash(np.ascontiguousarray(psi[1 - p]), U, L8, p)
        assert rel(a, oracle.spinor_transform(full, g, L8)[p]) < 1e-14
    # the clover term is covariant too
    C, Cg = oracle.clover_build(U, L8), oracle.clover_build(Ug, L8)
    a = np.stack([oracle.clover_apply(np.ascontiguousarray(psig[p]), np.ascontiguousarray(Cg[p])) for p in (0, 1)])
    b = np.stack([oracle.clover_apply(np.ascontiguousarray(psi[p]), np.ascontiguousarray(C[p])) for p in (0, 1)])
    assert rel(a, oracle.spinor_transform(np.ascontiguousarray(b), g, L8)) < 1e-13


def test_free_field_plane_wave(oracle):
    """U = 1: D acting on a plane wave e^{ipx} chi gives
    sum_mu [2 cos p_mu - 2 i gamma_mu sin p_mu] chi, so |D psi|^2 = (4 sum_mu sin^2 p_mu + (2 sum cos p_mu)^2)|psi|^2
    for a spinor chi; check the norm identity for one momentum."""
    L = L4
    U = oracle.gauge_unit(L)
    n = np.array([1, 0, 2, 1])
    p = 2 * np.pi * n / np.array(L)
    Vh = 128
    chi = np.zeros((4, 3), complex)
    chi[0, 0] = 1.0
    full = np.zeros((2, Vh, 4, 3), complex)
    for par in (0, 1):
        for s in range(Vh):
            xh = s % 2; r = s // 2; y = r % 4; r //= 4; z = r % 4; t = r // 4
            x = 2 * xh + ((y + z + t + par) & 1)
            full[par, s] = np.exp(1j * np.dot(p, [x, y, z, t])) * chi
    out = np.stack([oracle.dslash(np.ascontiguousarray(full[1 - par]), U, L, par) for par in (0, 1)])
    expect = (2 * np.cos(p).sum()) ** 2 + 4 * (np.sin(p) ** 2).sum()
    assert abs(np.vdot(out, out).real / np.vdot(full, full).real - expect) < 1e-12


def test_clover_trivial_on_pure_gauge(oracle):
    C = oracle.clover_build(oracle.gauge_pure(L8, 3), L8, 1.0)
    assert np.abs(C.reshape(-1, 6, 6) - np.eye(6)).max() < 1e-14


def test_clover_hermitian_and_inverse(oracle):
    C = oracle.clover_build(oracle.gauge_random(L8, 1234, 0.3), L8, 1.0)
    B = C.reshape(-1, 6, 6)
    assert np.abs(B - B.conj().transpose(0, 2, 1)).max() < 1e-15
    Ci = oracle.clover_invert(C).reshape(-1, 6, 6)
    assert np.abs(B @ Ci - np.eye(6)).max() < 1e-10
    # linear in csw: A(c) - 1 = c (A(1) - 1)
    C2 = oracle.clover_build(oracle.gauge_random(L8, 1234, 0.3), L8, 0.25).reshape(-1, 6, 6)
    assert np.abs((C2 - np.eye(6)) - 0.25 * (B - np.eye(6))).max() < 1e-15


def test_schur_operator_adjoint(oracle):
    U = oracle.gauge_random(L8, 77, 0.4)
    Ci = oracle.clover_invert(oracle.clover_build(U, L8, 0.13 * 1.0))
    x = oracle.spinor_random(2048, 1)
    y = oracle.spinor_random(2048, 2)
    Mx = oracle.schur_apply(x, U, Ci, L8, 0.13, -1.0, 0)
    Mdy = oracle.schur_apply(y, U, Ci, L8, 0.13, -1.0, 1)
    assert abs(oracle.cdot(y, Mx) - oracle.cdot(Mdy, x)) < 1e-12 * abs(oracle.cdot(y, Mx))


def test_schur_solve_reaches_true_residual(oracle):
    """Config 1 of the build: 8^3x8 Wilson, kappa = 0.12, antiperiodic t,
    eps = 0.3, source on even sites only."""
    L = (8, 8, 8, 8)
    U = oracle.gauge_random(L, 1, 0.3)
    b = oracle.full_spinor_random(L, 2)
    b[1] = 0
    x, it, res = oracle.solve_schur(b, U, L, 0.12, 0.0, -1.0, 1e-10)
    assert res < 1e-10 and it > 0
    C = oracle.clover_build(U, L, 0.0)
    r = b - oracle.apply_full(x, U, C, L, 0.12, -1.0)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10


def test_reference_cg_flow_on_pure_gauge(oracle):
    """On a pure-gauge field A = 1 and the reference's pseudo-normal operator
    is Hermitian, so its CG converges and solves (A - D) x = b."""
    U = oracle.gauge_pure(L8, 3)
    b = oracle.full_spinor_random(L8, 11)
    x, it, conv = oracle.cg_inverter_ref(b, U, L8, 2000)
    assert conv and 10 < it < 2000
    C = oracle.clover_build(U, L8, 1.0)
    Ci = oracle.clover_invert(C)
    assert rel(oracle.full_dslash_ref(x, U, C, Ci, L8, 0), b) < 1e-12


def test_storage_shift_restatement_follows_the_reference_indexing(oracle):
    """The oracle's storage shifts against element loops written with the
    reference's index formulas (src/qcu_shift_storage.cu:75-161): spinor
    dst[i*nh + s] = src[s*24 + i]; gauge dst[((2*mu+p)*12 + j)*nh + s] =
    src[((2*mu+p)*nh + s)*18 + j] for the first 12 reals of each link."""
    import numpy as np
    L = (4, 2, 2, 2)
    nh = 16
    psi = oracle.spinor_random(nh, 3)
    soa = oracle.shift_vector_storage(psi, 0)
    flat = psi.reshape(-1).view(np.float64)
    for s in range(nh):
        for i in range(24):
            assert soa[i, s] == flat[s * 24 + i]
    assert np.array_equal(oracle.shift_vector_storage(soa, 1), psi)
    U = oracle.gauge_random(L, 5, 0.4)
    g = oracle.shift_gauge_storage(U, 0)
    gf = U.reshape(-1).view(np.float64)
    for mp in range(8):
        for s in range(nh):
            for j in range(12):
                assert g[mp // 2, mp % 2, j, s] == gf[(mp * nh + s) * 18 + j]
    back = oracle.shift_gauge_storage(g, 1)
    assert np.array_equal(back[..., :2, :], U[..., :2, :])
    assert np.abs(back - U).max() < 1e-13  # the rebuilt row of an SU(3) link
