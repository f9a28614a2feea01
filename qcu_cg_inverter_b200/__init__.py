"""qcu_cg_inverter_b200 - B200-native Wilson-clover Dslash, clover and CG.

Python binding of ``libqcu_b200.so`` (built in-tree by ``build.py``). The C
ABI in ``include/qcu.h`` is a drop-in for the reference's ``qcu`` entry points
(YellowBicycleee/Qcu_Cg_Inverter, cg_inverter/include/qcu.h:1-25); this module
mirrors it with the same function names and argument meaning, so a ctypes
front-end written for the reference calls this library the same way. Field
arguments are CUDA tensors (complex128, reference AoS layouts) or raw device
pointers (int).

There is no CPU fallback: importing works without a GPU, but every compute
call goes through the CUDA library and fails loudly if it is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.environ.get("QCU_B200_LIB", os.path.join(HERE, "libqcu_b200.so"))

QCU_SUCCESS = 0
QCU_ERR_INVALID_ARG = 1
QCU_ERR_CUDA = 2
QCU_ERR_NOT_CONVERGED = 3
QCU_ERR_OUT_OF_MEMORY = 4
QCU_ERR_TIMEOUT = 5
QCU_ERR_NOT_INITIALIZED = 6
QCU_ERR_UNSUPPORTED = 7
QCU_ERR_BREAKDOWN = 8
QCU_ERR_SINGULAR_CLOVER = 9
QCU_ERR_BUSY = 10

PREC_DOUBLE, PREC_SINGLE, PREC_HALF = 0, 1, 2
_PREC = {"double": 0, "single": 1, "half": 2, 0: 0, 1: 1, 2: 2}


class QcuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"qcu error {code}: {msg}")
        self.code = code


class QcuParam(ctypes.Structure):
    """reference: include/qcu.h:7-9"""
    _fields_ = [("lattice_size", ctypes.c_int * 4)]


class QcuGrid(ctypes.Structure):
    """reference: include/qcu.h:11-13"""
    _fields_ = [("grid_size", ctypes.c_int * 4)]


class SolveParams(ctypes.Structure):
    _fields_ = [("kappa", ctypes.c_double), ("csw", ctypes.c_double), ("bc_t", ctypes.c_double),
                ("tol", ctypes.c_double), ("maxiter", ctypes.c_int), ("precision", ctypes.c_int),
                ("delta", ctypes.c_double), ("use_graphs", ctypes.c_int), ("autotune", ctypes.c_int)]


class ServerParams(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("tol", ctypes.c_double), ("maxiter", ctypes.c_int),
                ("bc_t", ctypes.c_double), ("delta", ctypes.c_double), ("columns", ctypes.c_int),
                ("clover_slots", ctypes.c_int), ("device_budget", ctypes.c_longlong), ("autotune", ctypes.c_int),
                ("max_chunk", ctypes.c_int)]


class SolveReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("reliable_updates", ctypes.c_int), ("converged", ctypes.c_int),
                ("status", ctypes.c_int), ("true_residual", ctypes.c_double), ("kappa", ctypes.c_double),
                ("gbytes", ctypes.c_double), ("seconds", ctypes.c_double), ("gbytes_per_s", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# host transport callbacks (include/qcu_b200.h qcu_exchange_fn, qcu_allreduce_fn)
_EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_size_t)
_ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int)

_lib = None


def build_library(force: bool = False) -> str:
    """Compiles libqcu_b200.so in-tree (see build.py)."""
    import importlib
    return importlib.import_module(__name__ + ".build").build(force=force)


def lib():
    """Loads libqcu_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m qcu_cg_inverter_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        PP = ctypes.POINTER(QcuParam)
        ll = ctypes.c_longlong
        sig = {
            "initGridSize": (None, [ctypes.POINTER(QcuGrid), PP, P, P, P]),
            "dslashQcu": (None, [P, P, P, PP, i]),
            "fullDslashQcu": (None, [P, P, P, PP, i]),
            "cg_inverter": (None, [P, P, P, PP]),
            "loadQcuGauge": (None, [P, PP]),
            "invertCloverDslash": (None, [P, P, P, PP, i]),
            "qcu_last_error": (i, []),
            "qcu_last_error_string": (ctypes.c_char_p, []),
            "qcuCloverDslashOneRound": (i, [P, P, P, PP, i]),
            "qcuFullCloverDslashOneRound": (i, [P, P, P, PP, i]),
            "qcuNewFullCloverDslashOneRound": (i, [P, P, P, PP, i]),
            "qcuMmVOneRound": (i, [P, P, P, PP, P]),
            "qcuPreCloverDslash": (i, [P, P, P, PP, i]),
            "qcuCgInverterRef": (i, [P, P, P, PP, ctypes.POINTER(i), ctypes.POINTER(i)]),
            "qcuSolveParamsDefault": (None, [ctypes.POINTER(SolveParams)]),
            "qcuContextCreate": (i, [ctypes.POINTER(P), ctypes.POINTER(i), i]),
            "qcuContextDestroy": (i, [P]),
            "qcuContextSetStream": (i, [P, P]),
            "qcuContextGetStream": (P, [P]),
            "qcuContextSetShape": (i, [P, i, i]),
            "qcuContextSetHalfOperator": (i, [P, i]),
            "qcuContextHalfOperator": (i, [P, i]),
            "qcuContextDeviceBytes": (ll, [P]),
            "qcuContextLaunchCount": (ll, [P]),
            "qcuLoadGauge": (i, [P, P]),
            "qcuGenerateGauge": (i, [P, ctypes.c_ulonglong, d]),
            "qcuExportGauge": (i, [P, P]),
            "qcuGenerateSpinor": (i, [P, P, i, ctypes.c_ulonglong]),
            "qcuDslash": (i, [P, P, P, i, i, d]),
            "qcuDslashNoAlloc": (i, [P, P, P, i, i, d]),
            "qcuApplyClover": (i, [P, P, P, d, i]),
            "qcuApplyOperator": (i, [P, P, P, d, d, d, i]),
            "qcuInvert": (i, [P, P, P, i, ctypes.POINTER(d), ctypes.POINTER(SolveParams),
                              ctypes.POINTER(SolveReport)]),
            "qcuBenchStencil": (i, [P, i, i, i, i, ctypes.POINTER(d), ctypes.POINTER(d)]),
            "qcuDebugFailAllocAfter": (None, [ll]),
            "qcuDebugSetPairStage": (None, [ctypes.c_int]),
            "qcuShiftVectorStorage": (i, [P, P, i, i, i, i, i]),
            "qcuShiftGaugeStorage": (i, [P, P, i, i, i, i, i]),
            "qcuDebugStencil": (i, [P, i, i, i, i, ctypes.POINTER(d), ctypes.POINTER(d), ctypes.POINTER(d),
                                    ctypes.POINTER(i), P, P, P, P, P, P, P, ctypes.POINTER(d), i]),
            "qcuAutotune": (i, [P, i, i, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(d)]),
            "qcuServerParamsDefault": (None, [ctypes.POINTER(ServerParams)]),
            "qcuServerCreate": (i, [ctypes.POINTER(P), i, ctypes.POINTER(ServerParams)]),
            "qcuServerDestroy": (i, [P]),
            "qcuServerAddConfig": (i, [P, ctypes.POINTER(i), ctypes.c_ulonglong, d, ctypes.POINTER(i)]),
            "qcuServerPrepare": (i, [P, i]),
            "qcuServerSubmit": (i, [P, i, d, d, i, P, P, ctypes.POINTER(ll)]),
            "qcuServerPoll": (i, [P, ctypes.POINTER(i)]),
            "qcuServerQuery": (i, [P, ll, ctypes.POINTER(i), ctypes.POINTER(d), ctypes.POINTER(SolveReport)]),
            "qcuServerRelease": (i, [P, ll]),
            "qcuServerRunTrace": (i, [P, i, ctypes.POINTER(d), ctypes.POINTER(i), ctypes.POINTER(d),
                                      ctypes.POINTER(d), ctypes.POINTER(i), ctypes.POINTER(P), ctypes.POINTER(P),
                                      ctypes.POINTER(d), ctypes.POINTER(SolveReport)]),
            "qcuServerPending": (i, [P]),
            "qcuServerDeviceBytes": (ll, [P]),
            "qcuHostAlloc": (P, [ll]),
            "qcuSlabGeometry": (i, [ctypes.POINTER(i), i, i, ctypes.POINTER(i)]),
            "qcuCommNcclUniqueId": (i, [P, i]),
            "qcuCommCreateNccl": (i, [ctypes.POINTER(P), P, i, i, i]),
            "qcuCommCreateHost": (i, [ctypes.POINTER(P), i, i, _EXCHANGE_FN, _ALLREDUCE_FN, P]),
            "qcuCommDestroy": (i, [P]),
            "qcuContextCreateSlab": (i, [ctypes.POINTER(P), ctypes.POINTER(i), P, i]),
            "qcuHostFree": (None, [P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    L = lib()
    return L.qcu_last_error(), (L.qcu_last_error_string() or b"").decode()


def _check(code: int):
    if code != QCU_SUCCESS:
        c, m = last_error()
        raise QcuError(code, m)


def _ptr(x):
    """Device (or host) address of a torch tensor, numpy array or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    if hasattr(x, "data_ptr"):
        assert x.is_contiguous(), "field tensors must be contiguous"
        return ctypes.c_void_p(x.data_ptr())
    if hasattr(x, "ctypes"):
        assert x.flags["C_CONTIGUOUS"]
        return ctypes.c_void_p(x.ctypes.data)
    raise TypeError(f"cannot take the address of {type(x)}")


def param(lattice) -> QcuParam:
    p = QcuParam()
    for k in range(4):
        p.lattice_size[k] = int(lattice[k])
    return p


# ---------------------------------------------------------------------------
# the reference interface (include/qcu.h), same names and argument meaning
# ---------------------------------------------------------------------------
def initGridSize(grid, p: QcuParam, gauge, fermion_in=None, fermion_out=None) -> None:
    """reference: src/qcu_communicator.cu:1630. grid must be (1,1,1,1)."""
    g = QcuGrid()
    for k in range(4):
        g.grid_size[k] = int(grid[k])
    lib().initGridSize(ctypes.byref(g), ctypes.byref(p), _ptr(gauge), _ptr(fermion_in), _ptr(fermion_out))
    _check(lib().qcu_last_error())


def loadQcuGauge(gauge, p: QcuParam) -> None:
    """reference: src/dslash.cu:27"""
    lib().loadQcuGauge(_ptr(gauge), ctypes.byref(p))
    _check(lib().qcu_last_error())


def dslashQcu(fermion_out, fermion_in, gauge, p: QcuParam, parity: int) -> None:
    """reference: src/dslash.cu:62 - out(parity) = D in(1-parity)"""
    lib().dslashQcu(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(p), int(parity))
    _check(lib().qcu_last_error())


def fullDslashQcu(fermion_out, fermion_in, gauge, p: QcuParam, dagger_flag: int) -> None:
    """reference: src/dslash.cu:78 - out = (A - D^(dag)) in"""
    lib().fullDslashQcu(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(p), int(dagger_flag))
    _check(lib().qcu_last_error())


def cg_inverter(b_vector, x_vector, gauge, p: QcuParam) -> None:
    """reference: src/cg_inverter.cu:260 (its CG flow, same stopping rule)"""
    lib().cg_inverter(_ptr(b_vector), _ptr(x_vector), _ptr(gauge), ctypes.byref(p))
    code = lib().qcu_last_error()
    if code not in (QCU_SUCCESS, QCU_ERR_NOT_CONVERGED):
        _check(code)


def invertCloverDslash(fermion_out, fermion_in, gauge, p: QcuParam, invert_flag: int = 0) -> None:
    """reference: src/qcu_clover_dslash.cu:902 - A^-1 applied in place to out"""
    lib().invertCloverDslash(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(p), int(invert_flag))
    _check(lib().qcu_last_error())


def cloverDslashOneRound(out, inp, gauge, p, invert_flag):
    _check(lib().qcuCloverDslashOneRound(_ptr(out), _ptr(inp), _ptr(gauge), ctypes.byref(p), int(invert_flag)))


def fullCloverDslashOneRound(out, inp, gauge, p, invert_flag):
    _check(lib().qcuFullCloverDslashOneRound(_ptr(out), _ptr(inp), _ptr(gauge), ctypes.byref(p), int(invert_flag)))


def newFullCloverDslashOneRound(out, inp, gauge, p, invert_flag):
    _check(lib().qcuNewFullCloverDslashOneRound(_ptr(out), _ptr(inp), _ptr(gauge), ctypes.byref(p),
                                                int(invert_flag)))


def MmV_one_round(out, inp, gauge, p, temp):
    _check(lib().qcuMmVOneRound(_ptr(out), _ptr(inp), _ptr(gauge), ctypes.byref(p), _ptr(temp)))


def preCloverDslash(out, inp, gauge, p, invert_flag=0):
    _check(lib().qcuPreCloverDslash(_ptr(out), _ptr(inp), _ptr(gauge), ctypes.byref(p), int(invert_flag)))


def shiftVectorStorage(dst, src, direction: int, lattice) -> None:
    """reference: src/qcu_shift_storage.cu:166 - one parity block of a spinor,
    AoS [V/2][24] <-> SoA [24][V/2] (direction 0 = to SoA); device memory."""
    _check(lib().qcuShiftVectorStorage(_ptr(dst), _ptr(src), int(direction), *[int(v) for v in lattice]))


def shiftGaugeStorage(dst, src, direction: int, lattice) -> None:
    """reference: src/qcu_shift_storage.cu:183 - gauge AoS [4][2][V/2][3][3] <->
    SoA [4][2][12][V/2] (direction 0 = to SoA; 1 rebuilds the third row)."""
    _check(lib().qcuShiftGaugeStorage(_ptr(dst), _ptr(src), int(direction), *[int(v) for v in lattice]))


def save_fields(path, lattice, gauge=None, spinors=None, **meta) -> None:
    """Writes fields in the reference's AoS layouts to one .npz file for
    reproducible fixtures: the lattice extents, an optional gauge field
    ([4][2][V/2][3][3] complex), optional spinors ([n][2][V/2][4][3] or one
    [2][V/2][4][3]) and scalar metadata (seed, eps, kappa, ...). Torch tensors
    are copied to the host."""
    import numpy as np

    def host(a):
        if a is None:
            return None
        if hasattr(a, "detach"):
            a = a.detach().cpu().numpy()
        return np.ascontiguousarray(a, dtype=np.complex128)

    L = np.asarray([int(v) for v in lattice], dtype=np.int64)
    if L.shape != (4,) or L.min() <= 0 or L[0] % 2:
        raise ValueError("lattice must be four positive extents with Lx even")
    vh = int(np.prod(L)) // 2
    arrays = {"lattice": L}
    g = host(gauge)
    if g is not None:
        if g.size != 4 * 2 * vh * 9:
            raise ValueError("gauge field does not match the lattice")
        arrays["gauge"] = g.reshape(4, 2, vh, 3, 3)
    sp = host(spinors)
    if sp is not None:
        if sp.size % (2 * vh * 12):
            raise ValueError("spinors do not match the lattice")
        arrays["spinors"] = sp.reshape(-1, 2, vh, 4, 3)
    for k, v in meta.items():
        arrays["meta_" + k] = np.asarray(v)
    np.savez_compressed(path, **arrays)


def load_fields(path):
    """Reads a file written by save_fields: (lattice, gauge or None, spinors or
    None, metadata dict)."""
    import numpy as np
    with np.load(path) as f:
        lattice = tuple(int(v) for v in f["lattice"])
        gauge = f["gauge"] if "gauge" in f else None
        spinors = f["spinors"] if "spinors" in f else None
        meta = {k[5:]: f[k][()] for k in f.files if k.startswith("meta_")}
    return lattice, gauge, spinors, meta


def cg_inverter_ref(b_vector, x_vector, gauge, p):
    """The reference CG flow with (iterations, converged) returned."""
    it, conv = ctypes.c_int(0), ctypes.c_int(0)
    code = lib().qcuCgInverterRef(_ptr(b_vector), _ptr(x_vector), _ptr(gauge), ctypes.byref(p), ctypes.byref(it),
                                  ctypes.byref(conv))
    if code not in (QCU_SUCCESS, QCU_ERR_NOT_CONVERGED):
        _check(code)
    return it.value, bool(conv.value)


# ---------------------------------------------------------------------------
# context-based API
# ---------------------------------------------------------------------------
def solve_params(**kw) -> SolveParams:
    sp = SolveParams()
    lib().qcuSolveParamsDefault(ctypes.byref(sp))
    for k, v in kw.items():
        if k == "precision":
            v = _PREC[v]
        setattr(sp, k, v)
    return sp


class Context:
    """One lattice on one GPU: resident gauge field, clover bank, solver."""

    def __init__(self, lattice, device: int = 0):
        self.lattice = tuple(int(v) for v in lattice)
        self._h = ctypes.c_void_p()
        L4 = (ctypes.c_int * 4)(*self.lattice)
        _check(lib().qcuContextCreate(ctypes.byref(self._h), L4, int(device)))

    def close(self):
        if self._h:
            lib().qcuContextDestroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def volume(self) -> int:
        L = self.lattice
        return L[0] * L[1] * L[2] * L[3]

    def _after_torch(self, *fields):
        """Orders the context's stream after torch's current stream when a
        field is a CUDA tensor: the kernels that produced it, or that still
        read an output buffer, may be pending there (the library's stream
        does not wait for the default stream by itself)."""
        for x in fields:
            if getattr(x, "is_cuda", False):
                import torch
                s = torch.cuda.current_stream(x.device)
                _check(lib().qcuContextSetStream(self._h, ctypes.c_void_p(s.cuda_stream)))
                return

    def load_gauge(self, gauge):
        self._after_torch(gauge)
        _check(lib().qcuLoadGauge(self._h, _ptr(gauge)))

    def generate_gauge(self, seed: int, eps: float):
        _check(lib().qcuGenerateGauge(self._h, int(seed), float(eps)))

    def export_gauge(self, out):
        self._after_torch(out)
        _check(lib().qcuExportGauge(self._h, _ptr(out)))

    def generate_spinor(self, out, nrhs: int, seed: int):
        self._after_torch(out)
        _check(lib().qcuGenerateSpinor(self._h, _ptr(out), int(nrhs), int(seed)))

    def dslash(self, out, inp, parity: int, dagger: int = 0, bc_t: float = 1.0):
        self._after_torch(inp, out)
        _check(lib().qcuDslash(self._h, _ptr(out), _ptr(inp), int(parity), int(dagger), float(bc_t)))

    def apply_clover(self, out, inp, csw_eff: float, inverse: bool):
        self._after_torch(inp, out)
        _check(lib().qcuApplyClover(self._h, _ptr(out), _ptr(inp), float(csw_eff), int(bool(inverse))))

    def apply_operator(self, out, inp, kappa: float, csw: float, bc_t: float = -1.0, dagger: int = 0):
        self._after_torch(inp, out)
        _check(lib().qcuApplyOperator(self._h, _ptr(out), _ptr(inp), float(kappa), float(csw), float(bc_t),
                                      int(dagger)))

    def invert(self, x, b, nrhs: int = 1, kappas=None, raise_on_fail: bool = True, **kw):
        sp = solve_params(**kw)
        self._after_torch(b, x)
        reps = (SolveReport * nrhs)()
        karr = None
        if kappas is not None:
            karr = (ctypes.c_double * nrhs)(*[float(k) for k in kappas])
        code = lib().qcuInvert(self._h, _ptr(x), _ptr(b), int(nrhs), karr, ctypes.byref(sp), reps)
        if code != QCU_SUCCESS and (raise_on_fail or code not in (QCU_ERR_NOT_CONVERGED, QCU_ERR_BREAKDOWN)):
            _check(code)
        return [r.as_dict() for r in reps]

    def bench_stencil(self, precision, variant: int, nrhs: int = 1, iters: int = 20):
        ms, nbytes = ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().qcuBenchStencil(self._h, _PREC[precision], int(variant), int(nrhs), int(iters),
                                     ctypes.byref(ms), ctypes.byref(nbytes)))
        return ms.value, nbytes.value

    def debug_stencil(self, precision, dagger: int, epi: int, inp, csw_eff, coef, active=None, x=None,
                      out=None, out2=None, pvec=None, xacc=None, racc=None, alpha=None, rhs_pairs: int = -1):
        """One batched stencil launch (epilogue flags `epi`) on fields converted
        from the FP64 AoS arrays given (numpy, nrhs x Vh x 4 x 3 complex, parity
        0 output); out/out2/xacc/racc are updated in place. rhs_pairs picks the
        kernel family of the fast 16-bit operator (1 paired, 0 one RHS per
        thread, -1 as built). Returns the per-RHS norms of the launch."""
        import numpy as np
        nrhs = len(csw_eff)
        arr = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.complex128)
        inp, x, out, out2, pvec, xacc, racc = map(arr, (inp, x, out, out2, pvec, xacc, racc))
        ptr = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
        dv = lambda v: None if v is None else (ctypes.c_double * nrhs)(*[float(t) for t in v])
        act = None if active is None else (ctypes.c_int * nrhs)(*[int(bool(t)) for t in active])
        norms = (ctypes.c_double * nrhs)()
        _check(lib().qcuDebugStencil(self._h, _PREC[precision], int(dagger), int(epi), nrhs, dv(csw_eff), dv(coef),
                                     dv(alpha), act, ptr(inp), ptr(x), ptr(pvec), ptr(out), ptr(out2), ptr(xacc),
                                     ptr(racc), norms, int(rhs_pairs)))
        return dict(out=out, out2=out2, xacc=xacc, racc=racc, norms=np.array(list(norms)))

    def set_shape(self, rhs_lanes: int, site_lanes: int):
        """Thread-block shape (RHS lanes x site lanes) of single-RHS kernels."""
        _check(lib().qcuContextSetShape(self._h, int(rhs_lanes), int(site_lanes)))

    def set_half_operator(self, fast_links):
        """16-bit solver storage: FP32 links/clover (True), 16-bit (False), or
        chosen per solve by lattice size and RHS count (None, the default)."""
        _check(lib().qcuContextSetHalfOperator(self._h, -1 if fast_links is None else int(bool(fast_links))))

    def half_storage(self, nrhs: int = 1) -> str:
        """'fast' (FP32 links and clover) or 'compact' (16-bit): what a 16-bit
        solve of nrhs right-hand sides uses on this context."""
        v = lib().qcuContextHalfOperator(self._h, int(nrhs))
        if v < 0:
            _check(-v)
        return "fast" if v == 1 else "compact"

    def autotune(self, precision, nrhs: int = 1):
        """Times every launch shape for (precision, nrhs); returns (Rb, Sb, ms)."""
        rb, sb, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
        _check(lib().qcuAutotune(self._h, _PREC[precision], int(nrhs), ctypes.byref(rb), ctypes.byref(sb),
                                 ctypes.byref(ms)))
        return rb.value, sb.value, ms.value

    @property
    def stream(self) -> int:
        """Address of the context's cudaStream_t (wrap with torch.cuda.ExternalStream)."""
        return int(lib().qcuContextGetStream(self._h) or 0)

    @property
    def launches(self) -> int:
        return int(lib().qcuContextLaunchCount(self._h))

    @property
    def device_bytes(self) -> int:
        return int(lib().qcuContextDeviceBytes(self._h))


# ---------------------------------------------------------------------------
# request server
# ---------------------------------------------------------------------------
def server_params(**kw) -> ServerParams:
    sp = ServerParams()
    lib().qcuServerParamsDefault(ctypes.byref(sp))
    for k, v in kw.items():
        if k == "precision":
            v = _PREC[v]
        setattr(sp, k, v)
    return sp


class PinnedBuffer:
    """Page-locked host memory (qcuHostAlloc) viewed as a numpy complex128 array."""

    def __init__(self, nbytes: int):
        import numpy as np
        self.nbytes = int(nbytes)
        addr = lib().qcuHostAlloc(self.nbytes)
        if not addr:
            raise QcuError(QCU_ERR_OUT_OF_MEMORY, f"cannot pin {self.nbytes} host bytes")
        self.addr = int(addr)
        buf = (ctypes.c_char * self.nbytes).from_address(self.addr)
        self.array = np.frombuffer(buf, dtype=np.complex128)

    def free(self):
        if self.addr:
            self.array = None
            lib().qcuHostFree(ctypes.c_void_p(self.addr))
            self.addr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop over resident gauge configurations
    (qcuServer* in include/qcu_b200.h)."""

    def __init__(self, device: int = 0, **kw):
        self._h = ctypes.c_void_p()
        self.params = server_params(**kw)
        _check(lib().qcuServerCreate(ctypes.byref(self._h), int(device), ctypes.byref(self.params)))
        self.lattices = []

    def close(self):
        if self._h:
            lib().qcuServerDestroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_config(self, lattice, seed: int, eps: float) -> int:
        cid = ctypes.c_int(0)
        L4 = (ctypes.c_int * 4)(*[int(v) for v in lattice])
        _check(lib().qcuServerAddConfig(self._h, L4, int(seed), float(eps), ctypes.byref(cid)))
        self.lattices.append(tuple(int(v) for v in lattice))
        return cid.value

    def prepare(self, config_id: int):
        _check(lib().qcuServerPrepare(self._h, int(config_id)))

    def submit(self, config_id: int, kappa: float, csw: float, nrhs: int, b, x) -> int:
        t = ctypes.c_longlong(0)
        _check(lib().qcuServerSubmit(self._h, int(config_id), float(kappa), float(csw), int(nrhs), _ptr(b), _ptr(x),
                                     ctypes.byref(t)))
        return t.value

    def poll(self) -> int:
        n = ctypes.c_int(0)
        _check(lib().qcuServerPoll(self._h, ctypes.byref(n)))
        return n.value

    def query(self, ticket: int, nrhs: int):
        """(finished, latency_s, reports, status) of a request."""
        fin, lat = ctypes.c_int(0), ctypes.c_double(0)
        reps = (SolveReport * nrhs)()
        code = lib().qcuServerQuery(self._h, int(ticket), ctypes.byref(fin), ctypes.byref(lat), reps)
        if code == QCU_ERR_INVALID_ARG and not fin.value:
            _check(code)
        return bool(fin.value), lat.value, [r.as_dict() for r in reps], code

    def release(self, ticket: int):
        _check(lib().qcuServerRelease(self._h, int(ticket)))

    def wait(self, ticket: int, nrhs: int, timeout_s: float = 600.0):
        import time
        t0 = time.monotonic()
        while True:
            fin, lat, reps, code = self.query(ticket, nrhs)
            if fin:
                return lat, reps, code
            if time.monotonic() - t0 > timeout_s:
                raise QcuError(QCU_ERR_TIMEOUT, f"request {ticket} did not finish in {timeout_s} s")
            self.poll()

    def run_trace(self, arrival_s, config_id, kappa, csw, nrhs, b, x, raise_on_fail: bool = True):
        """Runs a timed trace; returns (latency_s list, per-request report lists, status)."""
        n = len(arrival_s)
        D = ctypes.c_double * n
        I = ctypes.c_int * n
        Pv = ctypes.c_void_p * n
        lat = D()
        tot = int(sum(nrhs))
        reps = (SolveReport * max(tot, 1))()
        code = lib().qcuServerRunTrace(self._h, n, D(*arrival_s), I(*config_id), D(*kappa), D(*csw), I(*nrhs),
                                       Pv(*[_ptr(v).value for v in b]), Pv(*[_ptr(v).value for v in x]), lat, reps)
        if code != QCU_SUCCESS and raise_on_fail:
            _check(code)
        out, k = [], 0
        for m in nrhs:
            out.append([reps[k + j].as_dict() for j in range(m)])
            k += m
        return list(lat), out, code

    @property
    def pending(self) -> int:
        return int(lib().qcuServerPending(self._h))

    @property
    def device_bytes(self) -> int:
        return int(lib().qcuServerDeviceBytes(self._h))


# ---------------------------------------------------------------------------
# domain decomposition along t (include/qcu_b200.h, "domain decomposition")
# ---------------------------------------------------------------------------
def slab_geometry(lattice, nranks: int, rank: int) -> dict:
    """The t-slab of `rank` of a lattice split over nranks ranks (host
    arithmetic, no GPU): first global slice, local time extent, sites per
    slice, local half volume and the first sites of the two ghost slices."""
    L4 = (ctypes.c_int * 4)(*[int(v) for v in lattice])
    out = (ctypes.c_int * 6)()
    _check(lib().qcuSlabGeometry(L4, int(nranks), int(rank), out))
    return dict(zip(("t0", "lt", "face", "vh", "ghost_fwd", "ghost_bwd"), list(out)))


def _host_view(addr: int, nbytes: int):
    import numpy as np
    return np.ctypeslib.as_array((ctypes.c_ubyte * nbytes).from_address(addr))


def dist_transport():
    """The host transport's two callables over the default torch.distributed
    process group (CPU tensors, e.g. gloo): each rank sends its first slices
    to rank - 1 and its last ones to rank + 1 (tags tell the two streams
    apart when both neighbours are the same rank), and sums in place."""
    import torch
    import torch.distributed as dist
    rank, n = dist.get_rank(), dist.get_world_size()
    lo, hi = (rank - 1) % n, (rank + 1) % n

    def exchange(send_lo, send_hi, recv_lo, recv_hi):
        if n == 1:
            recv_hi[:] = send_lo
            recv_lo[:] = send_hi
            return
        t = [torch.from_numpy(a) for a in (send_lo, send_hi, recv_lo, recv_hi)]
        reqs = [dist.isend(t[0], lo, tag=1), dist.irecv(t[3], hi, tag=1),
                dist.isend(t[1], hi, tag=2), dist.irecv(t[2], lo, tag=2)]
        for r in reqs:
            r.wait()

    def allreduce(values):
        dist.all_reduce(torch.from_numpy(values))

    return exchange, allreduce


class Comm:
    """A communicator of the t-slab decomposition: NCCL (device buffers, the
    context's stream, capturable by CUDA graphs) or a host transport driven by
    two Python callables (the reference's host-staged exchange):

        exchange(send_lo, send_hi, recv_lo, recv_hi)  # numpy uint8 views
        allreduce(values)                             # numpy float64 view, summed in place

    send_lo goes to rank - 1 (its recv_hi), send_hi to rank + 1 (its recv_lo)."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        self._keep = ()
        self.nranks = self.rank = 0

    @staticmethod
    def nccl_unique_id() -> bytes:
        buf = (ctypes.c_ubyte * 128)()
        _check(lib().qcuCommNcclUniqueId(ctypes.cast(buf, ctypes.c_void_p), 128))
        return bytes(buf)

    @classmethod
    def nccl(cls, uid: bytes, nranks: int, rank: int, device: int = 0) -> "Comm":
        c = cls()
        buf = (ctypes.c_ubyte * 128).from_buffer_copy(uid)
        _check(lib().qcuCommCreateNccl(ctypes.byref(c._h), ctypes.cast(buf, ctypes.c_void_p), int(nranks), int(rank),
                                       int(device)))
        c.nranks, c.rank = int(nranks), int(rank)
        return c

    @classmethod
    def host(cls, nranks: int, rank: int, exchange=None, allreduce=None) -> "Comm":
        c = cls()

        def xfn(user, slo, shi, rlo, rhi, nbytes):
            try:
                exchange(_host_view(slo, nbytes), _host_view(shi, nbytes), _host_view(rlo, nbytes),
                         _host_view(rhi, nbytes))
                return 0
            except Exception:  # reported to the library as a failed exchange
                return 1

        def rfn(user, values, n):
            try:
                import numpy as np
                allreduce(np.ctypeslib.as_array(values, shape=(n,)))
                return 0
            except Exception:
                return 1

        cx = _EXCHANGE_FN(xfn) if exchange else _EXCHANGE_FN()
        cr = _ALLREDUCE_FN(rfn) if allreduce else _ALLREDUCE_FN()
        _check(lib().qcuCommCreateHost(ctypes.byref(c._h), int(nranks), int(rank), cx, cr, None))
        c._keep = (cx, cr)  # the callbacks must outlive the communicator
        c.nranks, c.rank = int(nranks), int(rank)
        return c

    @classmethod
    def torch_distributed(cls, device: int = 0) -> "Comm":
        """From the default torch.distributed process group: NCCL between the
        GPUs when the group's backend is nccl (the unique id travels through
        a broadcast), else the host transport over the group (gloo)."""
        import torch
        import torch.distributed as dist
        rank, n = dist.get_rank(), dist.get_world_size()
        if dist.get_backend() == "nccl":
            obj = [cls.nccl_unique_id() if rank == 0 else None]
            dist.broadcast_object_list(obj, src=0)
            return cls.nccl(obj[0], n, rank, device)
        exchange, allreduce = dist_transport()
        return cls.host(n, rank, exchange, allreduce)

    def close(self):
        if self._h:
            lib().qcuCommDestroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SlabContext(Context):
    """The slab of this rank of a lattice decomposed along t. Same methods as
    Context, on the rank's local fields (slices t0 .. t0 + lt - 1 of every
    global field, reference AoS layouts of the local lattice); every rank
    makes the same calls in the same order."""

    def __init__(self, lattice, comm: Comm, device: int = 0):
        geo = slab_geometry(lattice, comm.nranks, comm.rank)
        self.global_lattice = tuple(int(v) for v in lattice)
        self.lattice = self.global_lattice[:3] + (geo["lt"],)
        self.t0 = geo["t0"]
        self.comm = comm  # kept alive with the context
        self._h = ctypes.c_void_p()
        L4 = (ctypes.c_int * 4)(*self.global_lattice)
        _check(lib().qcuContextCreateSlab(ctypes.byref(self._h), L4, comm._h, int(device)))
