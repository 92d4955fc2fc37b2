"""Loads ``libdcrf_cuda.so`` (building it with nvcc if it is missing or stale)
and declares the C ABI of ``include/dcrf.h`` for ctypes."""
from __future__ import annotations

import ctypes as C
import os
import re
import threading

from . import build as _build

STATUS = {0: "DCRF_OK", 1: "DCRF_E_ARG", 2: "DCRF_E_CUDA", 3: "DCRF_E_RANGE", 4: "DCRF_E_STATE",
          5: "DCRF_E_NOMEM", 6: "DCRF_E_NUMERIC", 7: "DCRF_E_TIMEOUT"}


class DCRFError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class LPParams(C.Structure):
    """``dcrf_lp_params`` = LP_inf_params (include/densecrf.h:43-69)."""
    _fields_ = [("prox_reg_const", C.c_float), ("dual_gap_tol", C.c_float),
                ("prox_energy_tol", C.c_float), ("prox_max_iter", C.c_int),
                ("fw_max_iter", C.c_int), ("qp_max_iter", C.c_int), ("qp_tol", C.c_float),
                ("qp_const", C.c_float), ("best_int", C.c_int), ("accel_prox", C.c_int),
                ("work_set_size", C.c_int), ("approx_fw_iter", C.c_int),
                ("less_confident_percent", C.c_float), ("confidence_tol", C.c_float)]

    @classmethod
    def default(cls):
        p = cls()
        lib().dcrf_lp_params_default(C.byref(p))
        return p

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("inner_iters", C.c_int), ("gamma_iters", C.c_int),
                ("energy", C.c_double)]


_lock = threading.Lock()
_lib = None


def header_functions():
    """Names of the functions declared in include/dcrf.h."""
    src = open(os.path.join(_build.INCLUDE, "dcrf.h")).read()
    return sorted(set(re.findall(r"\b(dcrf_[a-z0-9_]+)\s*\(", src)))


def lib():
    global _lib
    with _lock:
        if _lib is None:
            path = _build.build()
            L = C.CDLL(path)
            for name in header_functions():
                fn = getattr(L, name)
                if name == "dcrf_last_error" or name == "dcrf_version":
                    fn.restype = C.c_char_p
                    fn.argtypes = []
                elif name == "dcrf_lp_params_default":
                    fn.restype = None
                elif name == "dcrf_kernel_launches":
                    fn.restype = C.c_ulonglong
                    fn.argtypes = []
                else:
                    fn.restype = C.c_int
            _lib = L
    return _lib


def check(code):
    if code != 0:
        raise DCRFError(code, lib().dcrf_last_error().decode(errors="replace"))
