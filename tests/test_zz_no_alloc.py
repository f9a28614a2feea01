"""qcuDslashNoAlloc through the C ABI against qcuDslash and the oracle (GPU).

qcuDslashNoAlloc serves callers that must not allocate device memory during a
call - a framework that already holds the GPU's memory in its own pool, or a
loop that cannot take the implicit synchronisation of cudaMalloc/cudaFree. It
stages its fields in a fixed scratch array compiled into the library instead
of allocating them as qcuDslash does on first use. This file is collected last
(its name sorts after every other test) and stands alone: it creates its own
contexts, so it passes in a fresh process and after the other tests.

Checked here:
  * two calls in a row, each with different arguments, agree with qcuDslash
    and with the CPU oracle on the same inputs to the FP64 tolerance of the
    other stencil tests (1e-12 relative);
  * on a fresh context, before any qcuDslash, calls succeed with the
    library's allocator armed to fail its next allocation, and leave the
    device's free memory unchanged;
  * a lattice beyond the scratch's stated maximum, and device memory of no GPU
    (a host buffer), are refused.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def no_alloc(q, c, out, inp, parity, dagger, bc):
    return q.lib().qcuDslashNoAlloc(c._h, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(inp.data_ptr()), parity,
                                    dagger, ctypes.c_double(bc))


def test_no_alloc_dslash_matches_qcuDslash_twice(cuda, qcu_lib, oracle):
    import torch

    q = qcu_lib
    L = (8, 8, 8, 8)
    Vh = 8 * 8 * 8 * 8 // 2
    c = q.Context(L)
    try:
        c.generate_gauge(2024, 0.4)
        U = np.zeros((4, 2, Vh, 3, 3), complex)
        c.export_gauge(U)
        src = torch.zeros(2 * Vh * 12, dtype=torch.complex128, device="cuda")
        c.generate_spinor(src, 1, 77)
        for parity, dagger, bc in ((0, 0, -1.0), (1, 1, 1.0)):
            inp = src[(1 - parity) * Vh * 12:(2 - parity) * Vh * 12].clone()
            ref = torch.zeros(Vh * 12, dtype=torch.complex128, device="cuda")
            got = torch.full((Vh * 12,), complex(7.0, -3.0), dtype=torch.complex128, device="cuda")
            c.dslash(ref, inp, parity, dagger, bc)  # the existing entry point
            code = no_alloc(q, c, got, inp, parity, dagger, bc)
            assert code == q.QCU_SUCCESS, q.last_error()
            r, g = ref.cpu().numpy(), got.cpu().numpy()
            assert np.isfinite(g).all()
            assert rel(g, r) < TOL and np.abs(g - r).max() <= TOL * np.abs(r).max()
            o = oracle.dslash(inp.cpu().numpy().reshape(Vh, 4, 3), U, L, parity, dagger, bc).reshape(-1)
            assert rel(g, o) < TOL and np.abs(g - o).max() <= TOL * np.abs(o).max()
    finally:
        c.close()


def test_no_alloc_dslash_allocates_nothing_on_a_fresh_context(cuda, qcu_lib, oracle):
    import torch

    q = qcu_lib
    L = (8, 8, 8, 16)
    Vh = 8 * 8 * 8 * 16 // 2
    c = q.Context(L)
    try:
        c.generate_gauge(99, 0.3)
        U = np.zeros((4, 2, Vh, 3, 3), complex)
        c.export_gauge(U)
        full = torch.zeros(2 * Vh * 12, dtype=torch.complex128, device="cuda")
        c.generate_spinor(full, 1, 5)  # one full spinor; its odd half is the input
        src = full[Vh * 12:].clone()
        outs = [torch.zeros(Vh * 12, dtype=torch.complex128, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()
        cases = ((0, 0, -1.0), (1, 1, 1.0), (0, 1, -1.0))
        for (parity, dagger, bc), out in zip(cases, outs):
            free0 = torch.cuda.mem_get_info()[0]
            q.lib().qcuDebugFailAllocAfter(0)  # the library's next allocation would fail
            try:
                code = no_alloc(q, c, out, src, parity, dagger, bc)
            finally:
                q.lib().qcuDebugFailAllocAfter(-1)
            torch.cuda.synchronize()
            assert code == q.QCU_SUCCESS, q.last_error()
            assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
            o = oracle.dslash(src.cpu().numpy().reshape(Vh, 4, 3), U, L, parity, dagger, bc).reshape(-1)
            g = out.cpu().numpy()
            assert rel(g, o) < TOL and np.abs(g - o).max() <= TOL * np.abs(o).max()
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


def test_no_alloc_dslash_refuses_host_memory(cuda, qcu_lib):
    import torch

    q = qcu_lib
    Vh = 8 * 8 * 8 * 8 // 2
    with q.Context((8, 8, 8, 8)) as c:
        c.generate_gauge(1, 0.3)
        d = torch.zeros(Vh * 12, dtype=torch.complex128, device="cuda")
        h = torch.zeros(Vh * 12, dtype=torch.complex128)
        assert no_alloc(q, c, d, h, 0, 0, 1.0) == q.QCU_ERR_INVALID_ARG
        assert no_alloc(q, c, h, d, 0, 0, 1.0) == q.QCU_ERR_INVALID_ARG
