"""Direct parity with the UNMODIFIED reference library on the same GPU.

The reference (compiled from its own sources into oracle/_ref/ by
oracle/Makefile) runs in a subprocess per gauge field, because its clover
term is process-global and it exits on errors. Same seeded inputs through the
library's drop-in entry points; FP64 agreement at 1e-12 relative for the
hopping term and 1e-10 for compositions that use A^-1 at kappa*c_sw = 1.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda")


def host(t, shape):
    return t.cpu().numpy().reshape(shape)


def rel(a, b):
    return np.linalg.norm(np.asarray(a).reshape(-1) - np.asarray(b).reshape(-1)) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def ref_out(cuda, oracle):
    from oracle import ref_runner
    if not os.path.exists(oracle.REF_LIB_PATH):
        pytest.skip("reference library not built (oracle/Makefile ref)")
    d, _ = ref_runner.run(L, "random:2024:0.3", ["dslash", "full", "invert", "pre", "newfull", "round", "mmv"], 11)
    return d


@pytest.fixture(scope="module")
def ours(cuda, qcu_lib, oracle):
    q = qcu_lib
    U = oracle.gauge_random(L, 2024, 0.3)
    psi = oracle.full_spinor_random(L, 11)
    p = q.param(L)
    dU = dev(U)
    q.initGridSize((1, 1, 1, 1), p, dU)
    q.loadQcuGauge(dU, p)
    out = {}
    Vh = psi.shape[1]
    for par in (0, 1):
        o = dev(np.zeros((Vh, 4, 3), complex))
        q.dslashQcu(o, dev(psi[1 - par]), dU, p, par)
        out[f"dslash_p{par}"] = host(o, (-1,))
    for d in (0, 1):
        o = dev(np.zeros_like(psi))
        q.fullDslashQcu(o, dev(psi), dU, p, d)
        out[f"full_d{d}"] = host(o, (-1,))
        q.newFullCloverDslashOneRound(o, dev(psi), dU, p, d)
        out[f"newfull_d{d}"] = host(o, (-1,))
        q.cloverDslashOneRound(o, dev(psi), dU, p, d)
        out[f"round_d{d}"] = host(o, (-1,))
    t = dev(psi)
    q.invertCloverDslash(t, t, dU, p, 0)
    out["invert"] = host(t, (-1,))
    t = dev(psi)
    q.preCloverDslash(t, t, dU, p)
    out["pre"] = host(t, (-1,))
    o, tmp = dev(np.zeros_like(psi)), dev(np.zeros_like(psi))
    q.MmV_one_round(o, dev(psi), dU, p, tmp)
    out["mmv"] = host(o, (-1,))
    return out


@pytest.mark.parametrize("name,tol", [("dslash_p0", 1e-12), ("dslash_p1", 1e-12), ("pre", 1e-12),
                                      ("full_d0", 1e-10), ("full_d1", 1e-10), ("invert", 1e-10),
                                      ("newfull_d0", 1e-10), ("newfull_d1", 1e-10), ("round_d0", 1e-10),
                                      ("round_d1", 1e-10), ("mmv", 1e-10)])
def test_matches_reference_library(ref_out, ours, name, tol):
    assert rel(ours[name], ref_out[name]) < tol


def test_reference_cg_matches(cuda, qcu_lib, oracle):
    from oracle import ref_runner
    if not os.path.exists(oracle.REF_LIB_PATH):
        pytest.skip("reference library not built")
    d, _ = ref_runner.run(L, "pure:7", ["cg"], 11)
    assert bool(d["cg_converged"])
    q = qcu_lib
    U = oracle.gauge_pure(L, 7)
    b = oracle.full_spinor_random(L, 11)
    p = q.param(L)
    dU = dev(U)
    q.initGridSize((1, 1, 1, 1), p, dU)
    x = dev(np.zeros_like(b))
    it, conv = q.cg_inverter_ref(dev(b), x, dU, p)
    assert conv and abs(it - int(d["cg_iterations"])) <= 1
    assert rel(host(x, (-1,)), d["cg_x"]) < 1e-9
