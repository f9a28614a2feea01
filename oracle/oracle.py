"""ctypes wrapper for the CPU oracle (liboracle.so) - TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this module; the product library never does. All arrays are
numpy complex128 in the reference's AoS layouts (see qcu_oracle.h):

    gauge       (4, 2, Vh, 3, 3)
    half spinor (Vh, 4, 3)
    full spinor (2, Vh, 4, 3)
    clover      (2, Vh, 2, 6, 6)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libqcu_ref.so")
# the reference's sources (its cg_inverter/ directory), needed only to build
# _ref/libqcu_ref.so; by default a checkout beside this repository
REF_SRC_DIR = os.environ.get("QCU_REFERENCE_DIR",
                             os.path.join(os.path.dirname(HERE), "..", "reference", "cg_inverter"))

_lib = None


def build(ref: bool = False) -> None:
    """Compile the oracle (and, if asked and the reference sources exist, the
    reference library) with oracle/Makefile."""
    targets = ["oracle"]
    if ref and os.path.isdir(REF_SRC_DIR):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={os.path.abspath(REF_SRC_DIR)}"] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I4 = ctypes.POINTER(ctypes.c_int)
        i, d, u64, sz = ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_size_t
        sig = {
            "orc_gauge_random": (None, [P, I4, u64, d]),
            "orc_gauge_unit": (None, [P, I4]),
            "orc_gauge_pure": (None, [P, I4, u64]),
            "orc_gauge_transform": (None, [P, P, P, I4]),
            "orc_su3_random_field": (None, [P, I4, u64]),
            "orc_spinor_random": (None, [P, sz, u64]),
            "orc_spinor_transform": (None, [P, P, P, I4]),
            "orc_dslash": (None, [P, P, P, I4, i, i, d]),
            "orc_clover_build": (None, [P, P, I4, d]),
            "orc_clover_invert": (i, [P, P, sz]),
            "orc_clover_apply": (None, [P, P, sz]),
            "orc_cdot": (None, [P, P, sz, P]),
            "orc_full_dslash_ref": (None, [P, P, P, P, P, I4, i]),
            "orc_new_full_ref": (None, [P, P, P, P, I4, i]),
            "orc_mmv_ref": (None, [P, P, P, P, I4]),
            "orc_invert_clover_ref": (None, [P, P, I4]),
            "orc_cg_inverter_ref": (i, [P, P, P, I4, i, ctypes.POINTER(ctypes.c_int)]),
            "orc_apply_full": (None, [P, P, P, P, I4, d, d, i]),
            "orc_solve_schur": (i, [P, P, P, I4, d, d, d, d, i, ctypes.POINTER(ctypes.c_double)]),
            "orc_solve_schur_cl": (i, [P, P, P, P, P, I4, d, d, d, i, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_int)]),
            "orc_schur_apply": (None, [P, P, P, P, I4, d, d, i]),
            "orc_num_threads": (i, []),
            "orc_set_num_threads": (None, [i]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _L(L):
    return (ctypes.c_int * 4)(*[int(v) for v in L])


def volume(L):
    return int(L[0]) * int(L[1]) * int(L[2]) * int(L[3])


def gauge_random(L, seed: int, eps: float) -> np.ndarray:
    Vh = volume(L) // 2
    g = np.empty((4, 2, Vh, 3, 3), np.complex128)
    lib().orc_gauge_random(_p(g), _L(L), seed, eps)
    return g


def gauge_unit(L) -> np.ndarray:
    Vh = volume(L) // 2
    g = np.empty((4, 2, Vh, 3, 3), np.complex128)
    lib().orc_gauge_unit(_p(g), _L(L))
    return g


def gauge_pure(L, seed: int) -> np.ndarray:
    Vh = volume(L) // 2
    g = np.empty((4, 2, Vh, 3, 3), np.complex128)
    lib().orc_gauge_pure(_p(g), _L(L), seed)
    return g


def su3_field(L, seed: int) -> np.ndarray:
    Vh = volume(L) // 2
    g = np.empty((2, Vh, 3, 3), np.complex128)
    lib().orc_su3_random_field(_p(g), _L(L), seed)
    return g


def gauge_transform(gauge, gfield, L) -> np.ndarray:
    out = np.empty_like(gauge)
    lib().orc_gauge_transform(_p(out), _p(gauge), _p(gfield), _L(L))
    return out


def spinor_transform(psi, gfield, L) -> np.ndarray:
    out = np.empty_like(psi)
    lib().orc_spinor_transform(_p(out), _p(psi), _p(gfield), _L(L))
    return out


def spinor_random(nsites: int, seed: int) -> np.ndarray:
    s = np.empty((nsites, 4, 3), np.complex128)
    lib().orc_spinor_random(_p(s), nsites, seed)
    return s


def full_spinor_random(L, seed: int) -> np.ndarray:
    Vh = volume(L) // 2
    return spinor_random(2 * Vh, seed).reshape(2, Vh, 4, 3)


def shift_vector_storage(src, direction: int) -> np.ndarray:
    """The reference's spinor storage shift for one parity block
    (src/qcu_shift_storage.cu:75-118): direction 0 takes the AoS half spinor
    [site][4][3] complex to the SoA [24][site] doubles (component index
    2*(spin*3 + colour) + re/im), direction 1 back."""
    if direction == 0:
        a = np.ascontiguousarray(src, dtype=np.complex128).reshape(-1, 12)
        return np.ascontiguousarray(a.view(np.float64).reshape(-1, 24).T)
    a = np.ascontiguousarray(np.asarray(src, dtype=np.float64).reshape(24, -1).T)
    return a.view(np.complex128).reshape(-1, 4, 3)


def shift_gauge_storage(src, direction: int) -> np.ndarray:
    """The reference's gauge storage shift (src/qcu_shift_storage.cu:123-161):
    direction 0 takes [4][2][site][3][3] complex to [4][2][12][site] doubles,
    the first two rows of each link (index 2*(row*3 + col) + re/im). Direction
    1 (which the reference leaves undone) goes back and rebuilds the third row
    as conj(row0 x row1) (src/qcu_clover_dslash.cu:11-16)."""
    if direction == 0:
        a = np.ascontiguousarray(src, dtype=np.complex128)
        nh = a.shape[2]
        two = a[:, :, :, :2, :].reshape(4, 2, nh, 6)
        return np.ascontiguousarray(two.view(np.float64).reshape(4, 2, nh, 12).transpose(0, 1, 3, 2))
    a = np.asarray(src, dtype=np.float64)
    nh = a.shape[3]
    two = np.ascontiguousarray(a.transpose(0, 1, 3, 2)).view(np.complex128).reshape(4, 2, nh, 2, 3)
    U = np.empty((4, 2, nh, 3, 3), np.complex128)
    U[..., :2, :] = two
    r0, r1 = two[..., 0, :], two[..., 1, :]
    U[..., 2, 0] = np.conj(r0[..., 1] * r1[..., 2] - r0[..., 2] * r1[..., 1])
    U[..., 2, 1] = np.conj(r0[..., 2] * r1[..., 0] - r0[..., 0] * r1[..., 2])
    U[..., 2, 2] = np.conj(r0[..., 0] * r1[..., 1] - r0[..., 1] * r1[..., 0])
    return U


def dslash(in_half, gauge, L, parity: int, dagger: int = 0, bc_t: float = 1.0) -> np.ndarray:
    out = np.empty_like(in_half)
    lib().orc_dslash(_p(out), _p(np.ascontiguousarray(in_half)), _p(gauge), _L(L), parity, dagger, bc_t)
    return out


def clover_build(gauge, L, csw: float = 1.0) -> np.ndarray:
    Vh = volume(L) // 2
    c = np.empty((2, Vh, 2, 6, 6), np.complex128)
    lib().orc_clover_build(_p(c), _p(gauge), _L(L), csw)
    return c


def clover_invert(clover) -> np.ndarray:
    inv = np.empty_like(clover)
    bad = lib().orc_clover_invert(_p(inv), _p(clover), clover.size // 72)
    if bad:
        raise ArithmeticError(f"{bad} singular clover blocks")
    return inv


def clover_apply(psi_half, mat_half) -> np.ndarray:
    out = np.ascontiguousarray(psi_half).copy()
    lib().orc_clover_apply(_p(out), _p(np.ascontiguousarray(mat_half)), out.size // 12)
    return out


def cdot(x, y) -> complex:
    o = np.zeros(2)
    lib().orc_cdot(_p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(y)), x.size, _p(o))
    return complex(o[0], o[1])


def full_dslash_ref(inp, gauge, clover, cinv, L, dagger: int) -> np.ndarray:
    out = np.empty_like(inp)
    lib().orc_full_dslash_ref(_p(out), _p(inp), _p(gauge), _p(clover), _p(cinv), _L(L), dagger)
    return out


def new_full_ref(inp, gauge, cinv, L, dagger: int) -> np.ndarray:
    out = np.empty_like(inp)
    lib().orc_new_full_ref(_p(out), _p(inp), _p(gauge), _p(cinv), _L(L), dagger)
    return out


def mmv_ref(inp, gauge, cinv, L) -> np.ndarray:
    out = np.empty_like(inp)
    lib().orc_mmv_ref(_p(out), _p(inp), _p(gauge), _p(cinv), _L(L))
    return out


def invert_clover_ref(out, cinv, L) -> np.ndarray:
    res = np.ascontiguousarray(out).copy()
    lib().orc_invert_clover_ref(_p(res), _p(cinv), _L(L))
    return res


def cg_inverter_ref(b, gauge, L, maxiter: int = 0):
    x = np.empty_like(b)
    conv = ctypes.c_int(0)
    it = lib().orc_cg_inverter_ref(_p(x), _p(b), _p(gauge), _L(L), maxiter, ctypes.byref(conv))
    return x, it, bool(conv.value)


def apply_full(inp, gauge, clover, L, kappa, bc_t=-1.0, dagger=0) -> np.ndarray:
    out = np.empty_like(inp)
    lib().orc_apply_full(_p(out), _p(inp), _p(gauge), _p(clover), _L(L), kappa, bc_t, dagger)
    return out


def schur_apply(inp, gauge, cinv, L, kappa, bc_t=-1.0, dagger=0) -> np.ndarray:
    out = np.empty_like(inp)
    lib().orc_schur_apply(_p(out), _p(np.ascontiguousarray(inp)), _p(gauge), _p(cinv), _L(L), kappa, bc_t, dagger)
    return out


def solve_schur(b, gauge, L, kappa, csw, bc_t=-1.0, tol=1e-10, maxiter=100000):
    x = np.empty_like(b)
    res = ctypes.c_double(0)
    it = lib().orc_solve_schur(_p(x), _p(b), _p(gauge), _L(L), kappa, csw, bc_t, tol, maxiter, ctypes.byref(res))
    return x, it, res.value


def solve_schur_cl(b, gauge, clover, cinv, L, kappa, bc_t=-1.0, tol=1e-10, maxiter=100000):
    """solve_schur with a prebuilt clover A (clover_build at kappa*c_sw) and its
    inverse; returns (x, iterations, true residual, true-residual checks)."""
    x = np.empty_like(b)
    res = ctypes.c_double(0)
    chk = ctypes.c_int(0)
    it = lib().orc_solve_schur_cl(_p(x), _p(b), _p(gauge), _p(clover), _p(cinv), _L(L), kappa, bc_t, tol, maxiter,
                                  ctypes.byref(res), ctypes.byref(chk))
    return x, it, res.value, chk.value


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())
