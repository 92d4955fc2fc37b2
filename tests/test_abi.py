"""The C ABI library: builds, loads, exports every declared symbol, validates
arguments and reports the absence of a GPU as an error (no CPU fallback).
None of these tests needs a GPU."""
import ctypes as C
import subprocess

import pytest

from densecrf_ho_b200 import _lib


def _has_gpu():
    try:
        return subprocess.run(["nvidia-smi", "-L"], capture_output=True, timeout=20).returncode == 0
    except Exception:
        return False


def test_library_exports_every_header_symbol():
    names = _lib.header_functions()
    assert len(names) >= 30
    L = _lib.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib._build.LIB], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(names) <= exported


def test_version_and_defaults():
    L = _lib.lib()
    assert b"sm_100a" in L.dcrf_version()
    p = _lib.LPParams.default()
    # LP_inf_params() defaults, src/densecrf.cpp:287-302
    assert (p.prox_max_iter, p.fw_max_iter, p.qp_max_iter, p.best_int) == (10, 10, 1000, 1)
    assert abs(p.prox_reg_const - 1e-2) < 1e-9 and p.qp_tol == 1e3 and p.dual_gap_tol == 1e3


def test_argument_errors_before_device():
    L = _lib.lib()
    h = C.c_void_p()
    assert L.dcrf_model_create(None, 4, 4, 21) == 1
    assert L.dcrf_model_create(C.byref(h), 0, 4, 21) == 1
    assert L.dcrf_model_create(C.byref(h), 4, 4, 65) == 1
    assert b"invalid model size" in L.dcrf_last_error()
    assert L.dcrf_lattice_create(None) == 1
    assert L.dcrf_model_info(None, None, None, None) == 1
    # every model entry point checks its handle before touching the device
    for fn, nargs in (("dcrf_model_pairwise_apply_bf", 5), ("dcrf_model_pairwise_apply_upper_minus_lower_bf", 5),
                      ("dcrf_model_pairwise_apply_upper_minus_lower_bf_ord", 6),
                      ("dcrf_model_pairwise_apply_upper_minus_lower_dc", 5),
                      ("dcrf_model_pairwise_kernel_gradient", 6), ("dcrf_model_pairwise_apply_ord_restricted", 8)):
        assert getattr(L, fn)(*([None] + [0] * (nargs - 1))) == 1, fn
        assert b"invalid model handle" in L.dcrf_last_error(), fn


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly():
    L = _lib.lib()
    h = C.c_void_p()
    assert L.dcrf_model_create(C.byref(h), 8, 8, 21) == 2  # DCRF_E_CUDA
    assert b"CUDA" in L.dcrf_last_error()
    assert L.dcrf_lattice_create(C.byref(h)) == 2
    from densecrf_ho_b200 import DCRFError, Permutohedral
    with pytest.raises(DCRFError):
        Permutohedral()
