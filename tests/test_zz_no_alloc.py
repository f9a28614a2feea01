"""qcuDslashNoAlloc through the C ABI against qcuDslash (GPU).

qcuDslashNoAlloc serves callers that must not allocate device memory during a
call - a framework that already holds the GPU's memory in its own pool, or a
loop that cannot take the implicit synchronisation of cudaMalloc/cudaFree. It
stages its fields in a fixed scratch array compiled into the library instead
of allocating them as qcuDslash does on first use. This file is collected last
(its name sorts after every other test) and stands alone: it creates its own
context, so it passes in a fresh process and after the other tests.

Two calls in a row, each with different arguments, must agree with qcuDslash
on the same inputs to the FP64 tolerance of the other stencil tests (1e-12
relative); a lattice beyond the scratch's stated maximum is refused.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_no_alloc_dslash_matches_qcuDslash_twice(cuda, qcu_lib):
    import torch

    q = qcu_lib
    L = (8, 8, 8, 8)
    Vh = 8 * 8 * 8 * 8 // 2
    c = q.Context(L)
    try:
        c.generate_gauge(2024, 0.4)
        src = torch.zeros(2 * Vh * 12, dtype=torch.complex128, device="cuda")
        c.generate_spinor(src, 1, 77)
        for parity, dagger, bc in ((0, 0, -1.0), (1, 1, 1.0)):
            inp = src[(1 - parity) * Vh * 12:(2 - parity) * Vh * 12].clone()
            ref = torch.zeros(Vh * 12, dtype=torch.complex128, device="cuda")
            got = torch.full((Vh * 12,), complex(7.0, -3.0), dtype=torch.complex128, device="cuda")
            c.dslash(ref, inp, parity, dagger, bc)  # the existing entry point
            code = q.lib().qcuDslashNoAlloc(c._h, ctypes.c_void_p(got.data_ptr()), ctypes.c_void_p(inp.data_ptr()),
                                            parity, dagger, ctypes.c_double(bc))
            assert code == q.QCU_SUCCESS, q.last_error()
            r, g = ref.cpu().numpy(), got.cpu().numpy()
            assert np.isfinite(g).all()
            assert rel(g, r) < TOL and np.abs(g - r).max() <= TOL * np.abs(r).max()
    finally:
        c.close()


def test_no_alloc_dslash_refuses_lattices_beyond_its_scratch(cuda, qcu_lib):
    import torch

    q = qcu_lib
    with q.Context((16, 16, 16, 16)) as c:  # half volume 32768 > 16384
        c.generate_gauge(1, 0.3)
        buf = torch.zeros(32768 * 12, dtype=torch.complex128, device="cuda")
        code = q.lib().qcuDslashNoAlloc(c._h, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()), 0, 0,
                                        ctypes.c_double(1.0))
        assert code == q.QCU_ERR_INVALID_ARG
        assert "16384" in q.last_error()[1]
