"""Size-independent properties of the GPU operators at the largest benchmarked
lattice, 32^3x64 (seeded links exp(i eps H), eps 0.5, antiperiodic t), checked
on the GPU's own outputs, so they hold where the oracle is too slow to follow:

  * the FP64 hop and its dagger flag are adjoint: <y, D x> = <D^dag y, x>,
    both output parities, to 1e-12 relative;
  * the FP64 Wilson-clover operator M = A - kappa D and its dagger flag are
    adjoint (M^dag = g5 M g5) to 1e-12 relative;
  * the FP64 hop is linear: D(a x + b y) = a D x + b D y to 1e-13;
  * the 16-bit hop, in both storages (FP32 links and clover; 16-bit links and
    clover), stays within the bound of 16-bit storage of the FP64 hop: largest
    component error below 2e-4 of the largest component (input and output each
    carry 1/32767 of their site's largest component).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = (32, 32, 32, 64)
GAUGE_SEED, EPS, BC_T = 20241, 0.5, -1.0


@pytest.fixture(scope="module")
def big(cuda, qcu_lib):
    import torch
    c = qcu_lib.Context(L)
    c.generate_gauge(GAUGE_SEED, EPS)
    V = c.volume
    x = torch.empty(V * 12, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    c.generate_spinor(x, 1, 31)
    c.generate_spinor(y, 1, 32)
    yield c, x.view(2, -1), y.view(2, -1)
    c.close()


def rel_gap(a, b):
    return abs(a - b) / max(abs(a), abs(b))


@pytest.mark.parametrize("parity", [0, 1])
def test_fp64_hop_dagger_is_the_adjoint(big, parity):
    import torch
    c, x, y = big
    dx = torch.zeros_like(x[0])
    c.dslash(dx, x[1 - parity].clone(), parity, 0, BC_T)  # D_{p,1-p} x
    ddy = torch.zeros_like(y[0])
    c.dslash(ddy, y[parity].clone(), 1 - parity, 1, BC_T)  # D^dag_{1-p,p} y
    lhs = torch.vdot(y[parity], dx).item()
    rhs = torch.vdot(ddy, x[1 - parity]).item()
    assert rel_gap(lhs, rhs) < 1e-12, (lhs, rhs)


def test_fp64_operator_dagger_is_the_adjoint(big):
    import torch
    c, x, y = big
    mx = torch.zeros_like(x)
    c.apply_operator(mx.view(-1), x.reshape(-1).clone(), 0.137, 1.0, BC_T, 0)
    mdy = torch.zeros_like(y)
    c.apply_operator(mdy.view(-1), y.reshape(-1).clone(), 0.137, 1.0, BC_T, 1)
    lhs = torch.vdot(y.reshape(-1), mx.reshape(-1)).item()
    rhs = torch.vdot(mdy.reshape(-1), x.reshape(-1)).item()
    assert rel_gap(lhs, rhs) < 1e-12, (lhs, rhs)


def test_fp64_hop_is_linear(big):
    import torch
    c, x, y = big
    a, b = 0.7 - 0.2j, -1.3 + 0.4j

    def hop(v):
        out = torch.zeros_like(v)
        c.dslash(out, v.clone(), 0, 0, BC_T)
        return out

    lhs = hop(a * x[1] + b * y[1])
    rhs = a * hop(x[1]) + b * hop(y[1])
    assert (torch.linalg.vector_norm(lhs - rhs) / torch.linalg.vector_norm(rhs)).item() < 1e-13


@pytest.mark.parametrize("fast_links", [True, False])
def test_16bit_hop_within_the_16bit_bound_of_fp64(big, fast_links):
    import torch
    c, x, _ = big
    ref = torch.zeros_like(x[0])
    c.dslash(ref, x[1].clone(), 0, 0, BC_T)
    ref = ref.cpu().numpy().reshape(1, -1, 4, 3)
    inp = x[1].cpu().numpy().reshape(1, -1, 4, 3)
    c.set_half_operator(fast_links)
    try:
        r = c.debug_stencil("half", 0, 0, inp, [0.0], [0.0], out=np.zeros_like(inp))
    finally:
        c.set_half_operator(None)
    err = np.abs(r["out"] - ref).max() / np.abs(ref).max()
    assert err < 2e-4, err
