"""The C-ABI library without a GPU: it loads, exports every symbol the public
headers declare (also the reference's C++ symbol names), and its host-side
argument checks report errors instead of exiting. No compute call is made."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", "qcu.h"), os.path.join(ROOT, "include", "qcu_b200.h")]


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src, flags=re.M):
            name = m.group(1)
            if m.group(0).lstrip().startswith("typedef"):  # function-pointer types, not functions
                continue
            if name not in ("typedef", "struct"):
                names.append(name)
    return sorted(set(names))


def exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_headers_declare_the_reference_interface():
    names = declared_functions()
    for ref_name in ("initGridSize", "dslashQcu", "fullDslashQcu", "cg_inverter", "loadQcuGauge", "invertCloverDslash"):
        assert ref_name in names


def test_library_exports_every_declared_symbol(qcu_lib):
    syms = exported(qcu_lib.LIB_PATH)
    missing = [n for n in declared_functions() if n not in syms]
    assert not missing, missing


def test_library_exports_reference_cxx_names(qcu_lib):
    syms = exported(qcu_lib.LIB_PATH)
    for m in ("_Z18invertCloverDslashPvS_S_P10QcuParam_si", "_Z15preCloverDslashPvS_S_P10QcuParam_si",
              "_Z20cloverDslashOneRoundPvS_S_P10QcuParam_si", "_Z24fullCloverDslashOneRoundPvS_S_P10QcuParam_si",
              "_Z27newFullCloverDslashOneRoundPvS_S_P10QcuParam_si", "_Z13MmV_one_roundPvS_S_P10QcuParam_sS_",
              "_Z18shiftVectorStoragePvS_iiiii", "_Z17shiftGaugeStoragePvS_iiiii"):
        assert m in syms


def test_library_loads_and_binds(qcu_lib):
    L = qcu_lib.lib()
    assert isinstance(L, ctypes.CDLL)


def test_solve_param_defaults(qcu_lib):
    sp = qcu_lib.solve_params()
    assert sp.tol == 1e-10 and sp.bc_t == -1.0 and sp.precision == qcu_lib.PREC_HALF and sp.delta == 0.0
    assert sp.use_graphs == 1 and sp.autotune == 1


def test_multi_rank_grid_is_rejected_without_exit(qcu_lib):
    with pytest.raises(qcu_lib.QcuError) as e:
        qcu_lib.initGridSize((2, 1, 1, 1), qcu_lib.param((8, 8, 8, 8)), None)
    assert e.value.code == qcu_lib.QCU_ERR_UNSUPPORTED


def test_calls_before_init_report_not_initialized(qcu_lib):
    # no initGridSize in this process: every legacy entry returns early with a status
    code = qcu_lib.lib().qcuPreCloverDslash(None, None, None, None, 0)
    assert code == qcu_lib.QCU_ERR_NOT_INITIALIZED
    assert qcu_lib.last_error()[0] == qcu_lib.QCU_ERR_NOT_INITIALIZED


@pytest.mark.parametrize("lattice", [(7, 8, 8, 8), (8, 0, 8, 8), (8, 8, -2, 8), (128, 128, 128, 256)],
                         ids=["odd-Lx", "zero-extent", "negative-extent", "beyond-32-bit-fields"])
def test_bad_lattice_rejected(qcu_lib, lattice):
    """Rejected before any device call: odd Lx, empty or negative extents, and
    a half volume whose 12-chunk spinor field would pass 2^30 chunks."""
    h = ctypes.c_void_p()
    L4 = (ctypes.c_int * 4)(*lattice)
    assert qcu_lib.lib().qcuContextCreate(ctypes.byref(h), L4, 0) == qcu_lib.QCU_ERR_INVALID_ARG
    assert not h.value


def test_server_param_defaults(qcu_lib):
    sp = qcu_lib.server_params()
    assert sp.precision == qcu_lib.PREC_HALF and sp.tol == 1e-10 and sp.maxiter == 20000 and sp.bc_t == -1.0
    assert sp.columns == 16 and sp.clover_slots == 8 and sp.device_budget == 0 and sp.autotune == 1
    assert sp.max_chunk == 8


def test_server_entry_points_are_declared(qcu_lib):
    names = declared_functions()
    for n in ("qcuServerCreate", "qcuServerSubmit", "qcuServerPoll", "qcuServerQuery", "qcuServerRunTrace",
              "qcuServerDestroy", "qcuHostAlloc"):
        assert n in names


def test_field_dumps_round_trip(qcu_lib, oracle, tmp_path):
    import numpy as np
    L = (4, 4, 2, 2)
    U = oracle.gauge_random(L, 9, 0.3)
    psi = np.stack([oracle.full_spinor_random(L, 40 + r) for r in range(3)])
    f = tmp_path / "fields.npz"
    qcu_lib.save_fields(f, L, gauge=U, spinors=psi, seed=9, eps=0.3)
    L2, U2, psi2, meta = qcu_lib.load_fields(f)
    assert L2 == L and np.array_equal(U2, U) and np.array_equal(psi2, psi)
    assert meta == {"seed": 9, "eps": 0.3}
    with pytest.raises(ValueError):
        qcu_lib.save_fields(f, L, gauge=U[:, :, :1])
