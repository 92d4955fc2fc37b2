"""ctypes bindings for the CPU oracles -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` /
``--impl reference`` legs import this module.  It exposes

* :class:`Oracle` -- our C restatement (``oracle/liboracle.so``, built from
  ``dcrf_oracle.c``; rebuilt with gcc on first use if missing), and
* :class:`Reference` -- the unmodified densecrf_ho compiled from its own sources
  (``oracle/_ref/libdcrf_ref.so``, built here by ``oracle/Makefile``; absent on
  machines without the reference tree, in which case :func:`reference_available`
  is False).

Both take and return numpy arrays in the reference's memory order:
``[N][L]`` float32 for label matrices, ``[N][d]`` for features.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdcrf_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i16p = np.ctypeslib.ndpointer(np.int16, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

LP_DEFAULTS = dict(prox_reg_const=1e-2, dual_gap_tol=1e3, prox_energy_tol=1e3, prox_max_iter=10,
                   fw_max_iter=10, qp_max_iter=1000, qp_tol=1e3, qp_const=1e-16, best_int=1,
                   accel_prox=1, work_set_size=10, approx_fw_iter=10,
                   less_confident_percent=0.0, confidence_tol=0.95)
"""``LP_inf_params()`` defaults (src/densecrf.cpp:287-302)."""


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


class _OrcLP(C.Structure):
    _fields_ = [("prox_reg_const", C.c_float), ("dual_gap_tol", C.c_float),
                ("prox_energy_tol", C.c_float), ("prox_max_iter", C.c_int),
                ("fw_max_iter", C.c_int), ("qp_max_iter", C.c_int), ("qp_tol", C.c_float),
                ("qp_const", C.c_float), ("best_int", C.c_int), ("accel_prox", C.c_int),
                ("work_set_size", C.c_int), ("approx_fw_iter", C.c_int),
                ("less_confident_percent", C.c_float), ("confidence_tol", C.c_float)]


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        src = os.path.join(HERE, "dcrf_oracle.c")
        if (not os.path.exists(ORACLE_SO)) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
            _build_oracle()
        L = C.CDLL(ORACLE_SO)
        vp = C.c_void_p
        L.orc_lattice_new.restype = vp
        L.orc_lattice_new.argtypes = [_f32p, C.c_int, C.c_int]
        L.orc_lattice_free.argtypes = [vp]
        L.orc_lattice_M.argtypes = [vp]
        L.orc_lattice_export.argtypes = [vp, _i32p, _i32p, _f32p, _i16p, _i32p]
        L.orc_lattice_compute.argtypes = [vp, _f32p, _f32p, C.c_int, C.c_int]
        L.orc_lattice_compute_f64.argtypes = [vp, _f64p, _f64p, C.c_int, C.c_int]
        L.orc_lattice_compute_ord.argtypes = [vp, _f32p, _f32p, C.c_int]
        L.orc_lattice_gradient.argtypes = [vp, _f32p, _f32p, _f32p, C.c_int]
        L.orc_model_new.restype = vp
        L.orc_model_new.argtypes = [C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_model_free.argtypes = [vp]
        L.orc_model_add_features.argtypes = [vp, _f32p, C.c_int, C.c_float]
        L.orc_model_add_gaussian.argtypes = [vp, C.c_float, C.c_float, C.c_float]
        L.orc_model_add_bilateral.argtypes = [vp] + [C.c_float] * 5 + [_u8p, C.c_float]
        L.orc_model_set_cliques.argtypes = [vp, C.c_int, _i32p, _i32p, _f32p, _f32p]
        L.orc_model_lattice_M.argtypes = [vp, C.c_int]
        L.orc_unary_init.argtypes = [vp, _f32p]
        L.orc_apply.argtypes = [vp, C.c_int, C.c_int, _f32p, _f32p]
        L.orc_apply_ord.argtypes = [vp, C.c_int, _f32p, _f32p]
        L.orc_qp.argtypes = [vp, _f32p, _f32p, C.c_int, C.c_void_p]
        L.orc_lp.argtypes = [vp, _f32p, _f32p, C.POINTER(_OrcLP), C.POINTER(C.c_int)]
        L.orc_current_map.argtypes = [vp, _f32p, _i16p]
        for fn in ("orc_energy_true", "orc_energy_ho"):
            getattr(L, fn).restype = C.c_double
            getattr(L, fn).argtypes = [vp, _i16p]
        for fn in ("orc_energy_lp", "orc_lr_qp_value"):
            getattr(L, fn).restype = C.c_double
            getattr(L, fn).argtypes = [vp, _f32p]
        L.orc_last_error.restype = C.c_char_p
        _olib = L
    return _olib


_rlib = None


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _rlib
    if _rlib is None:
        if not reference_available():
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref)")
        L = C.CDLL(REF_SO)
        vp = C.c_void_p
        L.refl_new.restype = vp
        L.refl_new.argtypes = [_f32p, C.c_int, C.c_int]
        L.refl_free.argtypes = [vp]
        L.refl_M.argtypes = [vp]
        L.refl_export.argtypes = [vp, _i32p, _i32p, _f32p, _i32p]
        L.refl_compute.argtypes = [vp, _f32p, _f32p, C.c_int, C.c_int]
        L.refl_compute_ord.argtypes = [vp, _f32p, _f32p, C.c_int]
        L.refl_gradient.argtypes = [vp, _f32p, _f32p, _f32p, C.c_int]
        L.refm_new.restype = vp
        L.refm_new.argtypes = [C.c_int, C.c_int, C.c_int, _f32p]
        L.refm_kernel_gradient.argtypes = [vp, C.c_int, _f32p, _f32p, _f32p]
        L.refm_parameters.argtypes = [vp, C.c_int, _f32p]
        L.refm_unary_energy.argtypes = [vp, np.ctypeslib.ndpointer(np.int16, flags="C_CONTIGUOUS"), _f32p]
        L.refm_pairwise_energy.argtypes = [vp, np.ctypeslib.ndpointer(np.int16, flags="C_CONTIGUOUS"), C.c_int,
                                           _f32p]
        L.refm_max_rounding.argtypes = [vp, _f32p, _f32p]
        L.refm_lr_qp_diag.argtypes = [vp, _f32p, _f32p]
        L.refm_lr_qp_diag.restype = C.c_double
        L.refm_energy_qp_ho.argtypes = [vp, _f32p]
        L.refm_energy_qp_ho.restype = C.c_double
        L.refm_add_features_kernel.argtypes = [vp, _f32p, C.c_int, C.c_float, C.c_int, C.c_int]
        L.refm_kernel_parameters.argtypes = [vp, C.c_int, _f32p]
        L.refm_set_kernel_parameters.argtypes = [vp, C.c_int, _f32p, C.c_int]
        L.refl_compute_ord_restricted.argtypes = [vp, _f32p, _f32p, _i32p, C.c_int, vp, C.c_int, C.c_int]
        L.refm_apply_ord_restricted.argtypes = [vp, C.c_int, _f32p, _f32p, _i32p, C.c_int, vp, C.c_int]
        L.refm_set_unary_logistic.argtypes = [vp, _f32p, _f32p, C.c_int]
        L.refm_unary_get.argtypes = [vp, _f32p]
        L.refm_unary_gradient.argtypes = [vp, _f32p, _f32p]
        L.refm_add_gaussian_compat.argtypes = [vp, C.c_float, C.c_float, C.c_int, _f32p]
        L.refm_add_bilateral_compat.argtypes = [vp] + [C.c_float] * 5 + [_u8p, C.c_int, _f32p]
        L.refm_weight_gradient.argtypes = [vp, C.c_int, _f32p, _f32p, _f32p]
        L.refm_free.argtypes = [vp]
        L.refm_add_gaussian.argtypes = [vp, C.c_float, C.c_float, C.c_float]
        L.refm_add_bilateral.argtypes = [vp] + [C.c_float] * 5 + [_u8p, C.c_float]
        L.refm_add_features.argtypes = [vp, _f32p, C.c_int, C.c_float]
        L.refm_add_superpixel.argtypes = [vp, _u8p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float]
        L.refm_num_cliques.argtypes = [vp]
        L.refm_clique_total.argtypes = [vp]
        L.refm_get_cliques.argtypes = [vp, _i32p, _i32p, _f32p, _f32p]
        L.refm_set_cliques.argtypes = [vp, C.c_int, _i32p, _i32p, _f32p, _f32p]
        L.refm_unary_init.argtypes = [vp, _f32p]
        L.refm_apply.argtypes = [vp, C.c_int, C.c_int, _f32p, _f32p]
        L.refm_apply_ord.argtypes = [vp, C.c_int, _f32p, _f32p]
        L.refm_qp.argtypes = [vp, _f32p, _f32p]
        L.refm_qp_fixed.argtypes = [vp, _f32p, _f32p, C.c_int, C.c_void_p]
        L.refm_lp.argtypes = ([vp, _f32p, _f32p] + [C.c_float] * 3 + [C.c_int] * 3 +
                              [C.c_float] * 2 + [C.c_int] * 4 + [C.c_float] * 2)
        L.refm_current_map.argtypes = [vp, _f32p, _i16p]
        for fn in ("refm_energy_true", "refm_energy_ho"):
            getattr(L, fn).restype = C.c_double
            getattr(L, fn).argtypes = [vp, _i16p]
        for fn in ("refm_energy_lp", "refm_lr_qp_value"):
            getattr(L, fn).restype = C.c_double
            getattr(L, fn).argtypes = [vp, _f32p]
        L.refm_apply_bf.argtypes = [vp, C.c_int, C.c_int, _f32p, _f32p]
        L.refm_apply_sorted.argtypes = [vp, C.c_int, C.c_int, C.c_int, _f32p, _i32p, vp]
        L.refms_filter.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, C.c_float, _f32p]
        L.refms_segment.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _i32p]
        L.ref_last_error.restype = C.c_char_p
        _rlib = L
    return _rlib


class _Lattice:
    def __init__(self, lib, pfx, f):
        f = _c(f, np.float32)
        self.N, self.d = f.shape
        self._lib, self._p = lib, pfx
        self._h = getattr(lib, pfx + "_new")(f, self.d, self.N)

    def __del__(self):
        try:
            getattr(self._lib, self._p + "_free")(self._h)
        except Exception:
            pass

    @property
    def M(self):
        return getattr(self._lib, self._p + "_M")(self._h)

    def compute(self, x, reverse=False):
        x = _c(x, np.float32)
        out = np.empty_like(x)
        getattr(self._lib, self._p + "_compute")(self._h, out, x, x.shape[1], int(reverse))
        return out

    def compute_ord(self, x):
        x = _c(x, np.float32)
        out = np.empty_like(x)
        getattr(self._lib, self._p + "_compute_ord")(self._h, out, x, x.shape[1])
        return out


class OracleLattice(_Lattice):
    """Restated ``Permutohedral`` (init / compute / compute_upper_minus_lower_ord)."""

    def __init__(self, f):
        super().__init__(oracle_lib(), "orc_lattice", f)

    def export(self):
        d1, N, M = self.d + 1, self.N, self.M
        off = np.empty(N * d1, np.int32)
        rk = np.empty(N * d1, np.int32)
        by = np.empty(N * d1, np.float32)
        keys = np.empty(max(M * self.d, 1), np.int16)
        nbr = np.empty(max(2 * d1 * M, 1), np.int32)
        self._lib.orc_lattice_export(self._h, off, rk, by, keys, nbr)
        return dict(offset=off, rank=rk, bary=by, keys=keys[:M * self.d],
                    nbr=nbr[:2 * d1 * M], M=M)

    def gradient(self, a, b):
        """df [N][d] = d(a^T K b)/d(features) (restated Permutohedral::gradient)."""
        a = _c(a, np.float32)
        b = _c(b, np.float32)
        df = np.empty((self.N, self.d), np.float32)
        self._lib.orc_lattice_gradient(self._h, df, a, b, a.shape[1])
        return df

    def compute_f64(self, x, reverse=False):
        x = _c(x, np.float64)
        out = np.empty_like(x)
        self._lib.orc_lattice_compute_f64(self._h, out, x, x.shape[1], int(reverse))
        return out


class ReferenceLattice(_Lattice):
    """The reference's own ``Permutohedral``."""

    def __init__(self, f):
        super().__init__(ref_lib(), "refl", f)

    def export(self):
        d1, N, M = self.d + 1, self.N, self.M
        off = np.empty(N * d1, np.int32)
        rk = np.empty(N * d1, np.int32)
        by = np.empty(N * d1, np.float32)
        nbr = np.empty(max(2 * d1 * M, 1), np.int32)
        self._lib.refl_export(self._h, off, rk, by, nbr)
        return dict(offset=off, rank=rk, bary=by, nbr=nbr[:2 * d1 * M], M=M)

    def compute_ord_restricted(self, rQ, pI, Q, store):
        """compute_upper_minus_lower_ord_restricted(rout, rQ, pI, Q, store)
        on a zeroed rout [nP][L]."""
        pI = _c(pI, np.int32)
        rQ = _c(rQ, np.float32).reshape(len(pI), -1)
        L = rQ.shape[1]
        out = np.zeros((len(pI), L), np.float32)
        q = None if Q is None else _c(Q, np.float32)
        self._lib.refl_compute_ord_restricted(self._h, out, rQ, pI, len(pI),
                                              None if q is None else q.ctypes.data_as(C.c_void_p), L, int(store))
        return out

    def gradient(self, a, b):
        """df [N][d] = d(a^T K b)/d(features) (Permutohedral::gradient)."""
        a = _c(a, np.float32)
        b = _c(b, np.float32)
        df = np.empty((self.N, self.d), np.float32)
        self._lib.refl_gradient(self._h, df, a, b, a.shape[1])
        return df


class _Model:
    pfx = ""

    def __init__(self, lib, W, H, L, unary):
        self._lib, self.W, self.H, self.L, self.N = lib, W, H, L, W * H
        self._h = getattr(lib, self.pfx + "_new")(W, H, L, _c(unary, np.float32))
        self.nterms = 0

    def _fn(self, name):
        return getattr(self._lib, self.pfx + "_" + name)

    def __del__(self):
        try:
            self._fn("free")(self._h)
        except Exception:
            pass

    def add_gaussian(self, sx, sy, w):
        self._fn("add_gaussian")(self._h, sx, sy, w)
        self.nterms += 1

    def add_bilateral(self, sx, sy, sr, sg, sb, rgb, w):
        self._fn("add_bilateral")(self._h, sx, sy, sr, sg, sb, _c(rgb, np.uint8), w)
        self.nterms += 1

    def add_features(self, f, w):
        f = _c(f, np.float32)
        self._fn("add_features")(self._h, f, f.shape[1], w)
        self.nterms += 1

    def set_cliques(self, offsets, idx, expw, constants):
        offsets = _c(offsets, np.int32)
        self._fn("set_cliques")(self._h, len(offsets) - 1, offsets, _c(idx, np.int32),
                                _c(expw, np.float32), _c(constants, np.float32))

    def _new(self):
        return np.empty((self.N, self.L), np.float32)

    def unary_init(self):
        q = self._new()
        self._fn("unary_init")(self._h, q)
        return q

    def apply(self, k, x, nonorm=False):
        out = self._new()
        self._fn("apply")(self._h, k, int(nonorm), out, _c(x, np.float32))
        return out

    def current_map(self, Q):
        lab = np.empty(self.N, np.int16)
        self._fn("current_map")(self._h, _c(Q, np.float32), lab)
        return lab

    def energy_true(self, lab):
        return self._fn("energy_true")(self._h, _c(lab, np.int16))

    def energy_ho(self, lab):
        return self._fn("energy_ho")(self._h, _c(lab, np.int16))

    def energy_lp(self, Q):
        return self._fn("energy_lp")(self._h, _c(Q, np.float32))

    def lr_qp_value(self, Q):
        return self._fn("lr_qp_value")(self._h, _c(Q, np.float32))

    def kernel_gradient(self, k, b, Q):
        """pairwise_[k]->kernelGradient(b, Q): d (DIAG_KERNEL) or d x d
        (FULL_KERNEL) floats (reference model only)."""
        out = np.zeros(256, np.float32)
        n = self._lib.refm_kernel_gradient(self._h, k, _c(b, np.float32), _c(Q, np.float32), out)
        return out[:n]

    def unary_energy(self, lab):
        out = np.zeros(self.N, np.float32)
        self._lib.refm_unary_energy(self._h, _c(lab, np.int16), out)
        return out

    def pairwise_energy(self, lab, term=-1):
        out = np.zeros(self.N, np.float32)
        self._lib.refm_pairwise_energy(self._h, _c(lab, np.int16), term, out)
        return out

    def max_rounding(self, Q):
        out = self._new()
        self._lib.refm_max_rounding(self._h, _c(Q, np.float32), out)
        return out

    def energy_qp_ho(self, Q):
        """compute_energy_higher_order(Q) (z of the last QP; reference model only)."""
        return self._lib.refm_energy_qp_ho(self._h, _c(Q, np.float32))

    def lr_qp_value_diag(self, Q, dd):
        return self._lib.refm_lr_qp_diag(self._h, _c(Q, np.float32), _c(dd, np.float32))

    def add_features_kernel(self, f, w, ktype, ntype):
        """addPairwiseEnergy(f, Potts(w), ktype, ntype) (reference model only)."""
        f = _c(f, np.float32)
        self._lib.refm_add_features_kernel(self._h, f, f.shape[1], w, ktype, ntype)
        self.nterms += 1

    def kernel_parameters(self, k):
        out = np.zeros(64, np.float32)
        n = self._lib.refm_kernel_parameters(self._h, k, out)
        return out[:n]

    def set_kernel_parameters(self, k, p):
        p = _c(p, np.float32).reshape(-1)
        self._lib.refm_set_kernel_parameters(self._h, k, p, p.size)

    def set_unary_logistic(self, w, f):
        """setUnaryEnergy(new LogisticUnaryEnergy(W, f)): w [L][F] (row-major
        numpy, i.e. W), f [N][F] (reference model only)."""
        w = np.asarray(w, np.float32)
        self._lib.refm_set_unary_logistic(self._h, _c(w.T, np.float32), _c(f, np.float32), w.shape[1])

    def unary_get(self):
        out = self._new()
        self._lib.refm_unary_get(self._h, out)
        return out

    def unary_gradient(self, b, F):
        """unary_->gradient(b) = b f^T as [L][F] (reference model only)."""
        out = np.zeros(self.L * F, np.float32)
        n = self._lib.refm_unary_gradient(self._h, _c(b, np.float32), out)
        return out[:n].reshape(F, self.L).T

    def parameters(self, k):
        """pairwise_[k]->parameters() (reference model only)."""
        out = np.zeros(self.L * (self.L + 1) // 2 + 1, np.float32)
        n = self._lib.refm_parameters(self._h, k, out)
        return out[:n]

    def weight_gradient(self, k, b, Q):
        """pairwise_[k]->gradient(b, Q): the compatibility's gradient (reference model only)."""
        out = np.zeros(self.L * (self.L + 1) // 2 + 16, np.float32)
        n = self._lib.refm_weight_gradient(self._h, k, _c(b, np.float32), _c(Q, np.float32), out)
        return out[:n]


class OracleModel(_Model):
    """Restated ``DenseCRF2D`` with Potts terms."""
    pfx = "orc_model"

    def __init__(self, W, H, L, unary):
        super().__init__(oracle_lib(), W, H, L, unary)

    def _fn(self, name):
        lib = self._lib
        return getattr(lib, "orc_model_" + name) if hasattr(lib, "orc_model_" + name) \
            else getattr(lib, "orc_" + name)

    def lattice_M(self, k):
        return self._lib.orc_model_lattice_M(self._h, k)

    def apply_ord(self, k, x):
        out = self._new()
        if self._lib.orc_apply_ord(self._h, k, out, _c(x, np.float32)) != 0:
            raise RuntimeError(self._lib.orc_last_error().decode())
        return out

    def qp(self, init, fixed_iters=0):
        out = self._new()
        en = np.zeros(max(fixed_iters, 1) + 4096, np.float64)
        it = self._lib.orc_qp(self._h, _c(init, np.float32), out, fixed_iters,
                              en.ctypes.data_as(C.c_void_p))
        return out, it, en[:it]

    def lp(self, init, **params):
        p = dict(LP_DEFAULTS)
        p.update(params)
        s = _OrcLP(**p)
        out = self._new()
        nit = C.c_int(0)
        if self._lib.orc_lp(self._h, _c(init, np.float32), out, C.byref(s), C.byref(nit)) != 0:
            raise RuntimeError(self._lib.orc_last_error().decode())
        return out, nit.value


class ReferenceModel(_Model):
    """The reference's own ``DenseCRF2D`` (Potts terms)."""
    pfx = "refm"

    def __init__(self, W, H, L, unary):
        super().__init__(ref_lib(), W, H, L, unary)

    def add_superpixel(self, rgb, spatial, rng, min_region, constant, normaliser):
        buf = _c(rgb, np.uint8).copy()
        return self._lib.refm_add_superpixel(self._h, buf, spatial, rng, min_region, constant,
                                             normaliser)

    def add_gaussian_compat(self, sx, sy, kind, params):
        """addPairwiseGaussian with a Diagonal (kind 1, L weights) or Matrix
        (kind 2, L x L, column-major) compatibility."""
        self._lib.refm_add_gaussian_compat(self._h, sx, sy, kind, _c(params, np.float32))
        self.nterms += 1

    def add_bilateral_compat(self, sx, sy, sr, sg, sb, rgb, kind, params):
        self._lib.refm_add_bilateral_compat(self._h, sx, sy, sr, sg, sb, _c(rgb, np.uint8), kind,
                                            _c(params, np.float32))
        self.nterms += 1

    def get_cliques(self):
        R = self._lib.refm_num_cliques(self._h)
        T = self._lib.refm_clique_total(self._h)
        off = np.empty(R + 1, np.int32)
        idx = np.empty(max(T, 1), np.int32)
        ex = np.empty(max(R, 1), np.float32)
        cs = np.empty(max(R, 1), np.float32)
        self._lib.refm_get_cliques(self._h, off, idx, ex, cs)
        return off, idx[:T], ex[:R], cs[:R]

    def apply_ord_restricted(self, k, rQ, pI, Q, store):
        """pairwise_[k]->apply_upper_minus_lower_ord_restricted(rout, rQ, pI, Q, store)."""
        pI = _c(pI, np.int32)
        rQ = _c(rQ, np.float32).reshape(len(pI), self.L)
        out = np.zeros((len(pI), self.L), np.float32)
        q = None if Q is None else _c(Q, np.float32)
        self._lib.refm_apply_ord_restricted(self._h, k, out, rQ, pI, len(pI),
                                            None if q is None else q.ctypes.data_as(C.c_void_p), int(store))
        return out

    def apply_ord(self, k, x):
        out = self._new()
        if self._lib.refm_apply_ord(self._h, k, out, _c(x, np.float32)) != 0:
            raise RuntimeError(self._lib.ref_last_error().decode())
        return out

    def apply_bf(self, k, Q, nonorm=False):
        """pairwise_[k] (or no_norm_pairwise_[k])->apply_bf(out, Q)."""
        out = self._new()
        self._lib.refm_apply_bf(self._h, k, int(nonorm), out, _c(Q, np.float32))
        return out

    def _sorted(self, kind, k, ind, Q, nonorm):
        out = self._new()
        q = None if Q is None else _c(Q, np.float32)
        self._lib.refm_apply_sorted(self._h, k, int(nonorm), kind, out, _c(ind, np.int32),
                                    None if q is None else q.ctypes.data_as(C.c_void_p))
        return out

    def apply_upper_minus_lower_bf(self, k, ind, nonorm=False):
        return self._sorted(0, k, ind, None, nonorm)

    def apply_upper_minus_lower_bf_ord(self, k, ind, Q, nonorm=False):
        return self._sorted(1, k, ind, Q, nonorm)

    def apply_upper_minus_lower_dc(self, k, ind, nonorm=False):
        return self._sorted(2, k, ind, None, nonorm)

    def qp(self, init, fixed_iters=0):
        out = self._new()
        if fixed_iters <= 0:
            self._lib.refm_qp(self._h, _c(init, np.float32), out)
            return out, None, None
        en = np.zeros(fixed_iters, np.float64)
        it = self._lib.refm_qp_fixed(self._h, _c(init, np.float32), out, fixed_iters,
                                     en.ctypes.data_as(C.c_void_p))
        return out, it, en[:it]

    def lp(self, init, **params):
        p = dict(LP_DEFAULTS)
        p.update(params)
        out = self._new()
        rc = self._lib.refm_lp(self._h, _c(init, np.float32), out, p["prox_reg_const"],
                               p["dual_gap_tol"], p["prox_energy_tol"], p["prox_max_iter"],
                               p["fw_max_iter"], p["qp_max_iter"], p["qp_tol"], p["qp_const"],
                               p["best_int"], p["accel_prox"], p["work_set_size"],
                               p["approx_fw_iter"], p["less_confident_percent"],
                               p["confidence_tol"])
        if rc != 0:
            raise RuntimeError(self._lib.ref_last_error().decode())
        return out, None


def ref_meanshift_filter(rgb, W, H, spatial, rng):
    """EDISON's filtered L*u*v* image (reference, Filter NO_SPEEDUP)."""
    out = np.zeros((W * H, 3), np.float32)
    ref_lib().refms_filter(_c(rgb, np.uint8).copy(), W, H, spatial, C.c_float(rng), out)
    return out


def ref_meanshift_segment(rgb, W, H, spatial, rng, min_region):
    """EDISON's region labels (reference, Segment NO_SPEEDUP) and count."""
    lab = np.zeros(W * H, np.int32)
    n = ref_lib().refms_segment(_c(rgb, np.uint8).copy(), W, H, spatial, C.c_float(rng), min_region, lab)
    return lab, n


def build_model(cls, img, gaussian=(3.0, 3.0), bilateral=(50.0, 15.0, 5.0)):
    """Gaussian + bilateral Potts model of ``src/example_inference.cpp:39-42``."""
    m = cls(img["W"], img["H"], img["L"], img["unary"])
    m.add_gaussian(gaussian[0], gaussian[0], gaussian[1])
    s, c, w = bilateral
    m.add_bilateral(s, s, c, c, c, img["rgb"], w)
    return m


class RestrictedOrd:
    """numpy float32 restatement of the restricted ordered filter,
    ``seqCompute_upper_minus_lower_ord_restricted``
    (src/permutohedral.cpp:702-900), from a lattice's exported tables
    (offset, barycentric, blur neighbours); the stored splat and vertex set of
    the last store call are kept between calls as the reference keeps them.

    Bins follow addSplitArray / sliceSplitArray (:548-589): lower bin
    min(floor(q*10 in float), 9), upper bin max(floor((q - 1e-9)*10 in double), 0).
    """

    def __init__(self, ex, d):
        self.d, self.M = d, int(ex["M"])
        d1 = d + 1
        self.N = len(ex["offset"]) // d1
        self.off = np.asarray(ex["offset"]).reshape(self.N, d1)
        self.bary = np.asarray(ex["bary"], np.float32).reshape(self.N, d1)
        self.nbr = np.asarray(ex["nbr"]).reshape(d1, self.M, 2)
        self.stored = None
        self.active = None

    @staticmethod
    def _bins(q, upper):
        q = np.asarray(q, np.float32)
        if upper:
            return np.maximum(np.floor((q.astype(np.float64) - 1e-9) * 10.0).astype(np.int64), 0)
        return np.minimum(np.floor(q * np.float32(10)).astype(np.int64), 9)

    def _splat(self, vals, i, q, upper):
        c = self._bins(q, upper)[:, None]
        b = np.arange(10)[None, :]
        mask = b >= c if upper else b <= c
        for j in range(self.d + 1):
            o = self.off[i, j] + 1
            vals[o] = vals[o] + np.where(mask, self.bary[i, j], np.float32(0))

    def compute(self, rQ, pI, Q, store):
        rQ = np.asarray(rQ, np.float32)
        pI = [int(i) for i in pI]
        L, M, d = rQ.shape[1], self.M, self.d
        alpha = np.float32(1) / (np.float32(1) + np.float32(2.0 ** -d))
        out = np.zeros((len(pI), L), np.float32)
        inside = set(pI)
        if store:
            self.stored = {}
            act, seen = [], set()
            for i in pI:
                for j in range(d + 1):
                    o = int(self.off[i, j])
                    if o not in seen:
                        seen.add(o)
                        act.append(o)
            self.active = np.array(act, np.int64)
        for upper in (False, True):
            if store:
                vals = np.zeros((M + 2, L, 10), np.float32)
                for i in range(self.N):
                    if i not in inside:
                        self._splat(vals, i, Q[i], upper)
                self.stored[upper] = vals.copy()
            else:
                vals = self.stored[upper].copy()
            for ii, i in enumerate(pI):
                self._splat(vals, i, rQ[ii], upper)
            new = np.zeros_like(vals)
            a = self.active
            for j in range(d + 1):
                if len(a):
                    n = self.nbr[j, a]
                    new[a + 1] = vals[a + 1] + np.float32(0.5) * (vals[n[:, 0] + 1] + vals[n[:, 1] + 1])
                vals, new = new, vals
            for ii, i in enumerate(pI):
                c = self._bins(rQ[ii], upper)
                for j in range(d + 1):
                    o = self.off[i, j] + 1
                    w = self.bary[i, j]
                    coef = np.float32(w) * alpha if upper else np.float32(-w) * alpha
                    out[ii] = out[ii] + vals[o, np.arange(L), c] * coef
        return out


# ----------------------------------------------- exact and D&C filters ----

def sqnorm_eigen(diff):
    """``VectorXf::squaredNorm()`` in Eigen 3.2's SSE2 order (Redux.h,
    LinearVectorizedTraversal from an aligned start; predux of
    SSE/PacketMath.h) over the last axis of float32 ``diff``: squares in
    float32; fewer than 4 summed left to right; else 4-lane packets (a second
    accumulator from 8 on), reduced as (p0 + p2) + (p1 + p3), then the tail."""
    s = (diff * diff).astype(np.float32)
    d = s.shape[-1]
    al = d & ~3
    if al == 0:
        r = s[..., 0]
        for i in range(1, d):
            r = (r + s[..., i]).astype(np.float32)
        return r
    p = s[..., 0:4]
    if al > 4:
        q = s[..., 4:8]
        al2 = d & ~7
        for idx in range(8, al2, 8):
            p = (p + s[..., idx:idx + 4]).astype(np.float32)
            q = (q + s[..., idx + 4:idx + 8]).astype(np.float32)
        p = (p + q).astype(np.float32)
        if al > al2:
            p = (p + s[..., al2:al2 + 4]).astype(np.float32)
    r = ((p[..., 0] + p[..., 2]).astype(np.float32) + (p[..., 1] + p[..., 3]).astype(np.float32)).astype(np.float32)
    for i in range(al, d):
        r = (r + s[..., i]).astype(np.float32)
    return r


def _kmat(fa, fb):
    """exp(-|f_a - f_b|^2) in float64 for all pairs (rows of fa, rows of fb),
    the norm in float32 as the reference forms it (src/pairwise.cpp:315)."""
    diff = (fa[:, None, :] - fb[None, :, :]).astype(np.float32)
    return np.exp(-sqnorm_eigen(diff).astype(np.float64))


def compat_apply(raw, kind, params):
    """LabelCompatibility::apply (src/labelcompatibility.cpp): Potts (kind 0,
    params = w): -w v; Diagonal (1, L weights): w_l v; Matrix (2, the
    symmetrised L x L, column-major): W v summed over m in order."""
    raw = raw.astype(np.float32)
    if kind == 0:
        return (np.float32(-params) * raw).astype(np.float32)
    if kind == 1:
        return (np.asarray(params, np.float32)[None, :] * raw).astype(np.float32)
    W = np.asarray(params, np.float32).reshape(raw.shape[1], raw.shape[1]).T  # W[l, m]
    out = (W[None, :, 0] * raw[:, 0:1]).astype(np.float32)
    for m in range(1, raw.shape[1]):
        out = (out + (W[None, :, m] * raw[:, m:m + 1]).astype(np.float32)).astype(np.float32)
    return out


def bf_apply(feat, Q):
    """``apply_bf`` before the compatibility (src/pairwise.cpp:368-380):
    out(l, c) = sum_b k(c, b) Q(l, b), each product in double added to the
    float out in b order."""
    feat = np.asarray(feat, np.float32)
    Q = np.asarray(Q, np.float32)
    K = _kmat(feat, feat)  # [c, b]
    acc = np.zeros(Q.shape, np.float32)
    for b in range(feat.shape[0]):
        acc = (acc.astype(np.float64) + K[:, b:b + 1] * Q[b][None, :].astype(np.float64)).astype(np.float32)
    return acc


def bf_sorted(feat, ind, Q=None):
    """``apply_upper_minus_lower_bf`` (Q None, src/pairwise.cpp:301-332) or
    ``apply_upper_minus_lower_bf_ord`` (:333-367) before the compatibility;
    ind [N][L]; out in sorted positions."""
    feat = np.asarray(feat, np.float32)
    ind = np.asarray(ind)
    N, L = ind.shape
    out = np.zeros((N, L), np.float32)
    for l in range(L):
        sf = feat[ind[:, l]]
        K = _kmat(sf, sf)
        acc = np.zeros(N, np.float32)
        if Q is None:
            up = np.triu(np.ones((N, N), bool), 1)  # b > c
            lo = up.T
        else:
            qs = np.asarray(Q, np.float32)[ind[:, l], l]
            up = ~(qs[None, :] > qs[:, None])
            lo = ~(qs[None, :] < qs[:, None])
        for sign, mask in ((1.0, up), (-1.0, lo)):
            for b in range(N):
                m = mask[:, b]
                acc[m] = (acc[m].astype(np.float64) + sign * K[m, b]).astype(np.float32)
        out[:, l] = acc
    return out


def _dc_cross(out, ex, lo, ml, mh, hi):
    """``seqCompute_upper_minus_lower_dc`` (src/permutohedral.cpp:902-997) on
    one lattice's exported tables (offset, bary [N][d+1], nbr [d+1][M][2])."""
    off, bary, nbr, d = ex["offset"], ex["bary"], ex["nbr"], ex["d"]
    d1 = d + 1
    act = []
    seen = set()
    for rng in (range(mh, hi), range(lo, ml)):
        for i in rng:
            for j in range(d1):
                o = int(off[i, j])
                if o not in seen:
                    seen.add(o)
                    act.append(o)
    alpha = np.float32(1.0) / np.float32(1.0 + 2.0 ** -d)
    half = np.float32(0.5)
    for splat_rng, slice_rng, sign in ((range(mh, hi), range(lo, ml), 1), (range(lo, ml), range(mh, hi), -1)):
        vals = {}
        for i in splat_rng:
            for j in range(d1):
                o = int(off[i, j])
                vals[o] = np.float32(vals.get(o, np.float32(0.0)) + bary[i, j])
        for j in range(d1):
            new = {}
            for v in act:
                n1, n2 = int(nbr[j, v, 0]), int(nbr[j, v, 1])
                s = np.float32(vals.get(n1, np.float32(0.0)) + vals.get(n2, np.float32(0.0)))
                new[v] = np.float32(vals.get(v, np.float32(0.0)) + half * s)
            vals = new
        for i in slice_rng:
            for j in range(d1):
                t = np.float32(np.float32(bary[i, j] * vals[int(off[i, j])]) * alpha)
                out[i] = np.float32(out[i] + t) if sign > 0 else np.float32(out[i] - t)


def _dc_slice(out, sf, ex, lo, hi):
    """``apply_upper_minus_lower_sorted_slice`` (src/pairwise.cpp:262-300)."""
    size = hi - lo
    if size <= 30:
        alpha = 1.0 / 0.6
        K = _kmat(sf[lo:hi], sf[lo:hi])
        for c in range(lo, hi):
            for b in range(lo, c):
                out[c] = np.float32(np.float64(out[c]) - K[c - lo, b - lo] * alpha)
        for c in range(lo, hi):
            for b in range(c + 1, hi):
                out[c] = np.float32(np.float64(out[c]) + K[c - lo, b - lo] * alpha)
        return
    ml = lo + size // 2
    mh = ml if size % 2 == 0 else ml + 1
    _dc_slice(out, sf, ex, lo, mh)
    _dc_slice(out, sf, ex, ml, hi)
    _dc_cross(out, ex, lo, ml, mh, hi)


def dc_sorted(feat, ind, lattice_cls=None):
    """``apply_upper_minus_lower_dc`` before the compatibility
    (src/pairwise.cpp:241-260): per label a lattice of the sorted features
    (``lattice_cls``: :class:`OracleLattice` by default) and the recursion."""
    feat = np.asarray(feat, np.float32)
    ind = np.asarray(ind)
    N, L = ind.shape
    d = feat.shape[1]
    out = np.zeros((N, L), np.float32)
    lat_cls = lattice_cls or OracleLattice
    for l in range(L):
        sf = np.ascontiguousarray(feat[ind[:, l]])
        lat = lat_cls(sf)
        e = lat.export()
        M = lat.M
        ex = {"offset": np.asarray(e["offset"]).reshape(N, d + 1), "bary": np.asarray(e["bary"]).reshape(N, d + 1),
              "nbr": np.asarray(e["nbr"]).reshape(d + 1, M, 2), "d": d}
        col = np.zeros(N, np.float32)
        _dc_slice(col, sf, ex, 0, N)
        out[:, l] = col
    return out


# ------------------------------------------------------ kernel gradient ----

def kernel_gradient_diag(f, kparams, ntype, b, Q, w):
    """``PairwisePotential::kernelGradient(b, Q)`` of a DIAG_KERNEL term with a
    Potts compatibility (src/pairwise.cpp:402-407): lbl = -w Q; the lattice
    on the scaled features diag(kparams) f (``setParameters``, :155-161) and
    its norm n (``initLattice``, :40-57: 1/sqrt(K1 + 1e-20) symmetric, else
    1/(K1 + 1e-20), in double); ``featureGradient(b, lbl)`` (:95-122) with
    G = the restated ``Permutohedral::gradient`` for NormalizationType
    ``ntype`` (0 none, 1 before, 2 after, 3 symmetric); then
    ``(f o fg).rowwise().sum()`` (:174) over the original features, a float
    sum left to right over the pixels as Eigen's row reduction runs it.
    f [N][d], b and Q [N][L]; float32 throughout as the reference."""
    f = np.asarray(f, np.float32)
    a = np.asarray(b, np.float32)
    Q = np.asarray(Q, np.float32)
    N = f.shape[0]
    lat = OracleLattice(np.ascontiguousarray((f * np.asarray(kparams, np.float32)[None, :]).astype(np.float32)))
    lbl = (np.float32(-w) * Q).astype(np.float32)
    c = lat.compute(np.ones((N, 1), np.float32))[:, 0].astype(np.float64)
    n = (1.0 / np.sqrt(c + 1e-20) if ntype == 3 else 1.0 / (c + 1e-20)).astype(np.float32)

    def G(x, y):
        return lat.gradient(np.ascontiguousarray(x, np.float32), np.ascontiguousarray(y, np.float32))

    def col(x, s):  # x * s.asDiagonal()
        return (x * s[:, None]).astype(np.float32)

    ones = np.ones_like(a)
    nn = (n * n).astype(np.float32)
    if ntype == 0:
        fg = G(a, lbl)
    elif ntype == 3:
        fa = lat.compute(col(a, n), True)
        fb = lat.compute(col(lbl, n))
        n3 = (nn * n).astype(np.float32)
        X = col((np.float32(0.5) * ((a * fb).astype(np.float32) + (fa * lbl).astype(np.float32))).astype(np.float32),
                n3)
        fg = (-G(X, ones) + G(col(a, n), col(lbl, n))).astype(np.float32)
    elif ntype == 2:
        X = col((a * lat.compute(lbl)).astype(np.float32), nn)
        fg = (-G(X, ones) + G(col(a, n), lbl)).astype(np.float32)
    else:
        X = col((lat.compute(a, True) * lbl).astype(np.float32), nn)
        fg = (-G(X, ones) + G(a, col(lbl, n))).astype(np.float32)
    t = (f * fg).astype(np.float32)
    out = t[0].copy()
    for i in range(1, N):
        out = (out + t[i]).astype(np.float32)
    return out


def eigen_sum(x):
    """``ArrayXf::sum()`` of a contiguous float32 array as Eigen 3.2 reduces it
    with SSE2 (Redux.h, LinearVectorizedTraversal from an aligned start): two
    4-lane accumulators over 8-element steps, added lane-wise, one more
    packet if a whole one is left, ``(p0 + p2) + (p1 + p3)``, then the tail
    left to right (fewer than 4 elements: left to right)."""
    s = np.asarray(x, np.float32).reshape(-1)
    S = s.size
    al = (S // 4) * 4
    if al == 0:
        r = s[0]
        for i in range(1, S):
            r = np.float32(r + s[i])
        return r
    p0 = s[0:4].copy()
    if al > 4:
        p1 = s[4:8].copy()
        al2 = (S // 8) * 8
        for idx in range(8, al2, 8):
            p0 = (p0 + s[idx:idx + 4]).astype(np.float32)
            p1 = (p1 + s[idx + 4:idx + 8]).astype(np.float32)
        p0 = (p0 + p1).astype(np.float32)
        if al > al2:
            p0 = (p0 + s[al2:al2 + 4]).astype(np.float32)
    r = np.float32(np.float32(p0[0] + p0[2]) + np.float32(p0[1] + p0[3]))
    for i in range(al, S):
        r = np.float32(r + s[i])
    return r


def weight_gradient_potts(f, b, Q, diagonal=False):
    """``PairwisePotential::gradient(b, Q)`` of a term with the default
    DIAG_KERNEL / NORMALIZE_SYMMETRIC kernel (src/pairwise.cpp:390-395):
    fq = n K(n Q) on the restated lattice (``DenseKernel::filter``), then the
    compatibility's gradient (src/labelcompatibility.cpp:72-76, 94-96):
    Potts ``-(b o fq).sum()`` in Eigen's vectorised order; with ``diagonal``
    ``(b o fq).rowwise().sum()``, per label a float sum over the pixels left
    to right (a row of a column-major array has no packet access).
    f [N][d], b and Q [N][L]."""
    f = np.asarray(f, np.float32)
    b = np.asarray(b, np.float32)
    Q = np.asarray(Q, np.float32)
    lat = OracleLattice(np.ascontiguousarray(f))
    N = f.shape[0]
    c = lat.compute(np.ones((N, 1), np.float32))[:, 0].astype(np.float64)
    n = (1.0 / np.sqrt(c + 1e-20)).astype(np.float32)
    fq = (lat.compute((Q * n[:, None]).astype(np.float32)) * n[:, None]).astype(np.float32)
    t = (b * fq).astype(np.float32)
    if diagonal:
        out = t[0].copy()
        for i in range(1, N):
            out = (out + t[i]).astype(np.float32)
        return out
    return np.float32(-eigen_sum(t))


# ------------------------------------------------ per-pixel energies ----

def unary_energy(U, lab):
    """``DenseCRF::unaryEnergy(l)`` (src/densecrf.cpp:887-899): U(l_i, i), 0
    where l_i is off the label range.  U [N][L], lab [N] int."""
    U = np.asarray(U, np.float32)
    lab = np.asarray(lab)
    L = U.shape[1]
    ok = (lab >= 0) & (lab < L)
    r = np.zeros(U.shape[0], np.float32)
    r[ok] = U[np.nonzero(ok)[0], lab[ok]]
    return r


def pairwise_energy_true(model, lab, term=-1):
    """``DenseCRF::pairwise_energy_true(l, term)`` (:902-927) on a model with
    ``apply(k, x, nonorm)``: the unnormalised Potts twin applied to
    Q = [l_i != j], r_i = -Q'(l_i, i) (0 off the label range); term -1 adds
    the terms in order to a zero vector."""
    lab = np.asarray(lab)
    N, L = lab.shape[0], model.L
    if term == -1:
        r = np.zeros(N, np.float32)
        for k in range(model.nterms):
            r = (r + pairwise_energy_true(model, lab, k)).astype(np.float32)
        return r
    Q = np.ones((N, L), np.float32)
    ok = (lab >= 0) & (lab < L)
    Q[np.nonzero(ok)[0], lab[ok]] = 0.0
    out = model.apply(term, Q, nonorm=True)
    r = np.zeros(N, np.float32)
    r[ok] = -out[np.nonzero(ok)[0], lab[ok]]
    return r


def max_rounding(Q):
    """``DenseCRF::max_rounding`` (:832-840): one-hot at each pixel's first
    maximum (``maxCoeff``)."""
    Q = np.asarray(Q, np.float32)
    out = np.zeros_like(Q)
    out[np.arange(Q.shape[0]), np.argmax(Q, axis=1)] = 1.0
    return out


def eigen_sum_d(x):
    """``ArrayXd::sum()`` in Eigen 3.2's SSE2 order: as :func:`eigen_sum` with
    2-lane packets (two accumulators over 4-element steps, predux p0 + p1)."""
    s = np.asarray(x, np.float64).reshape(-1)
    S = s.size
    al = (S // 2) * 2
    if al == 0:
        return float(s[0])
    p0 = s[0:2].copy()
    if al > 2:
        p1 = s[2:4].copy()
        al2 = (S // 4) * 4
        for idx in range(4, al2, 4):
            p0 = p0 + s[idx:idx + 2]
            p1 = p1 + s[idx + 2:idx + 4]
        p0 = p0 + p1
        if al > al2:
            p0 = p0 + s[al2:al2 + 2]
    r = p0[0] + p0[1]
    for i in range(al, S):
        r = r + s[i]
    return float(r)


def dot_product(a, b):
    """``dotProduct(M1, M2, tmp)`` (src/eigen_utils.cpp:68-74): both cast to
    double, multiplied element-wise (exactly), summed in Eigen's order."""
    return eigen_sum_d(np.asarray(a, np.float32).astype(np.float64) * np.asarray(b, np.float32).astype(np.float64))


def lr_qp_value_diag(model, U, Q, dd):
    """``DenseCRF::compute_LR_QP_value(Q, diag_dom)`` (src/densecrf.cpp:940-957)
    on a model with ``apply(k, x)``: U.Q - dd.Q + sum_k Q.apply_k(Q) +
    Q.(dd o Q), each a :func:`dot_product`, accumulated in double in that
    order."""
    Q = np.asarray(Q, np.float32)
    dd = np.asarray(dd, np.float32)
    e = 0.0
    e += dot_product(U, Q)
    e -= dot_product(dd, Q)
    for k in range(model.nterms):
        e += dot_product(Q, model.apply(k, Q))
    e += dot_product(Q, (dd * Q).astype(np.float32))
    return e
