"""densecrf_ho_b200 -- B200-native dense-CRF inference, a drop-in for the hot
path of densecrf_ho.

The product is the C ABI ``libdcrf_cuda.so`` (``include/dcrf.h``) and the C++
shim with the reference's class API (``densecrf_ho_b200/cpp``).  This module is
a thin ctypes mirror of the same classes, used by the test-suite, the
benchmark and Python callers:

* :class:`Permutohedral` -- ``init`` / ``compute`` /
  ``compute_upper_minus_lower_ord`` (include/permutohedral.h:50-88);
* :class:`DenseCRF2D` -- ``setUnaryEnergy``, ``addPairwiseGaussian``,
  ``addPairwiseBilateral``, ``addPairwiseEnergy``, cliques, ``unary_init``,
  ``qp_inference_super_pixels_non_convex``, ``lp_inference_prox_super_pixels``,
  ``currentMap`` and the energies (include/densecrf.h:73-194).

Arrays use the reference's memory order: label matrices ``[N, L]`` float32
(Eigen column-major L x N), features ``[N, d]``.  There is no CPU fallback:
without the CUDA library or a GPU every call raises :class:`DCRFError`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import DCRFError, LPParams, SolveStats, lib, check

__all__ = ["Permutohedral", "DenseCRF2D", "LPParams", "SolveStats", "DCRFError", "lib"]

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


class Permutohedral:
    """Device permutohedral lattice (class Permutohedral)."""

    def __init__(self):
        self._h = C.c_void_p()
        check(lib().dcrf_lattice_create(C.byref(self._h)))
        self.N = self.d = self.M = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().dcrf_lattice_destroy(h)
            except Exception:
                pass

    def init(self, features):
        f = _f32(features)
        N, d = f.shape
        check(lib().dcrf_lattice_init(self._h, f.ctypes.data_as(C.c_void_p), d, N))
        M = C.c_int()
        check(lib().dcrf_lattice_info(self._h, C.byref(M), None, None))
        self.N, self.d, self.M = N, d, M.value
        return self

    def compute(self, inp, reverse=False):
        x = _f32(inp)
        if x.ndim == 1:
            x = x.reshape(-1, 1)
        out = np.empty_like(x)
        check(lib().dcrf_lattice_compute(self._h, out.ctypes.data_as(C.c_void_p),
                                         x.ctypes.data_as(C.c_void_p), x.shape[1], int(reverse)))
        return out

    def filter_shape(self):
        """Launch shapes of the 21-label plain filter: (splat warps per block,
        blur threads, slice pixels per tile, splat form)."""
        shp = (C.c_int * 4)()
        check(lib().dcrf_lattice_filter_shape(self._h, shp))
        return tuple(shp)

    def set_filter_shape(self, shape):
        """Pins the launch shapes (no autotuning for this lattice)."""
        shp = (C.c_int * 4)(*[int(x) for x in shape])
        check(lib().dcrf_lattice_set_filter_shape(self._h, shp))
        return self

    def compute_upper_minus_lower_ord(self, Q):
        x = _f32(Q)
        out = np.empty_like(x)
        check(lib().dcrf_lattice_compute_ord(self._h, out.ctypes.data_as(C.c_void_p),
                                             x.ctypes.data_as(C.c_void_p), x.shape[1]))
        return out

    def compute_upper_minus_lower_ord_restricted(self, rQ, pI, Q=None, store=True):
        """``compute_upper_minus_lower_ord_restricted(rout, rQ, pI, Q, store)``:
        the ordered filter at the pixels pI (strictly ascending) with values
        rQ [len(pI), L]; the other pixels splat Q [N, L] (store) or the splat
        kept by the last store call (store=False)."""
        pi = np.ascontiguousarray(pI, np.int32).reshape(-1)
        x = _f32(rQ)
        L = x.shape[1] if x.ndim == 2 else _f32(Q).shape[1]
        x = x.reshape(pi.size, L)
        out = np.zeros((pi.size, L), np.float32)
        q = _f32(Q) if store else None
        check(lib().dcrf_lattice_compute_ord_restricted(
            self._h, out.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
            pi.ctypes.data_as(C.c_void_p), int(pi.size), None if q is None else q.ctypes.data_as(C.c_void_p),
            int(L), int(bool(store))))
        return out

    def gradient(self, a, b):
        """``df [N, d]`` = d(a^T K b) / d(features) (``Permutohedral::gradient``)."""
        a, b = _f32(a), _f32(b)
        if a.ndim == 1:
            a, b = a.reshape(-1, 1), b.reshape(-1, 1)
        df = np.empty((self.N, self.d), np.float32)
        check(lib().dcrf_lattice_gradient(self._h, df.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p),
                                          b.ctypes.data_as(C.c_void_p), a.shape[1]))
        return df

    def export(self):
        d1, N, M, d = self.d + 1, self.N, self.M, self.d
        off = np.empty(N * d1, np.int32)
        rk = np.empty(N * d1, np.int32)
        by = np.empty(N * d1, np.float32)
        keys = np.empty(max(M * d, 1), np.int16)
        nbr = np.empty(max(2 * d1 * M, 1), np.int32)
        check(lib().dcrf_lattice_export(self._h, off.ctypes.data_as(C.c_void_p),
                                        rk.ctypes.data_as(C.c_void_p), by.ctypes.data_as(C.c_void_p),
                                        keys.ctypes.data_as(C.c_void_p), nbr.ctypes.data_as(C.c_void_p)))
        return dict(offset=off, rank=rk, bary=by, keys=keys[:M * d], nbr=nbr[:2 * d1 * M], M=M)


class DenseCRF2D:
    """Device dense CRF over a W x H grid with L labels (class DenseCRF2D)."""

    def __init__(self, W, H, L):
        self.W, self.H, self.L, self.N = W, H, L, W * H
        self._h = C.c_void_p()
        check(lib().dcrf_model_create(C.byref(self._h), W, H, L))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().dcrf_model_destroy(h)
            except Exception:
                pass

    @property
    def handle(self):
        return self._h

    def _mat(self, a):
        return _f32(a, (self.N, self.L))

    def _new(self):
        return np.empty((self.N, self.L), np.float32)

    # -- set-up ---------------------------------------------------------
    def setUnaryEnergy(self, unary):
        u = self._mat(unary)
        check(lib().dcrf_model_set_unary(self._h, u.ctypes.data_as(C.c_void_p)))

    def setUnaryEnergyLogistic(self, weights, features):
        """``setUnaryEnergy(new LogisticUnaryEnergy(W, f))``: weights W [L][F],
        features f [N][F]; the unary is W f."""
        w = np.asarray(weights, np.float32)
        if w.ndim != 2 or w.shape[0] != self.L:
            raise DCRFError(1, "weights must be L x F")
        F = w.shape[1]
        f = _f32(features, (self.N, F))
        wc = np.ascontiguousarray(w.T)  # column-major W
        check(lib().dcrf_model_set_unary_logistic(self._h, wc.ctypes.data_as(C.c_void_p),
                                                  f.ctypes.data_as(C.c_void_p), F))

    def getUnaryEnergy(self):
        """``getUnaryEnergy()->get()``: the unary [N, L] in use."""
        out = self._new()
        check(lib().dcrf_model_get_unary(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def unary_parameters(self):
        """``unary_->parameters()`` as W [L][F] (empty for a constant unary)."""
        n = C.c_int(0)
        check(lib().dcrf_model_unary_parameters(self._h, None, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        check(lib().dcrf_model_unary_parameters(self._h, out.ctypes.data_as(C.c_void_p), None))
        return out.reshape(-1, self.L).T if n.value else out

    def unary_set_parameters(self, weights):
        """``unary_->setParameters(W)``, W [L][F]; the unary is recomputed."""
        w = np.ascontiguousarray(np.asarray(weights, np.float32).T)
        if w.size != self.unary_parameters().size:
            raise DCRFError(1, "wrong number of unary parameters")
        check(lib().dcrf_model_unary_set_parameters(self._h, w.ctypes.data_as(C.c_void_p)))

    def unary_gradient(self, b):
        """``unary_->gradient(b)`` = b f^T as [L][F] (empty for a constant unary)."""
        bb = self._mat(b)
        n = C.c_int(0)
        check(lib().dcrf_model_unary_gradient(self._h, bb.ctypes.data_as(C.c_void_p), None, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        if n.value:
            check(lib().dcrf_model_unary_gradient(self._h, bb.ctypes.data_as(C.c_void_p),
                                                  out.ctypes.data_as(C.c_void_p), None))
            return out.reshape(-1, self.L).T
        return out

    def addPairwiseGaussian(self, sx, sy, w):
        check(lib().dcrf_model_add_gaussian(self._h, C.c_float(sx), C.c_float(sy), C.c_float(w)))

    def addPairwiseBilateral(self, sx, sy, sr, sg, sb, rgb, w):
        im = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1)
        if im.size != 3 * self.N:
            raise DCRFError(1, "rgb must hold W*H*3 bytes")
        check(lib().dcrf_model_add_bilateral(self._h, *(C.c_float(v) for v in (sx, sy, sr, sg, sb)),
                                             im.ctypes.data_as(C.c_void_p), C.c_float(w)))

    def addPairwiseEnergy(self, features, w):
        f = _f32(features)
        check(lib().dcrf_model_add_pairwise(self._h, f.ctypes.data_as(C.c_void_p), f.shape[1],
                                            C.c_float(w)))

    CONST_KERNEL, DIAG_KERNEL, FULL_KERNEL = 0, 1, 2
    NO_NORMALIZATION, NORMALIZE_BEFORE, NORMALIZE_AFTER, NORMALIZE_SYMMETRIC = 0, 1, 2, 3

    def unaryEnergy(self, labels):
        """``unaryEnergy(l)``: the per-pixel unary energy of a labelling."""
        lab = np.ascontiguousarray(labels, np.int16).reshape(-1)
        out = np.zeros(self.N, np.float32)
        check(lib().dcrf_model_unary_energy(self._h, lab.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
        return out

    def pairwise_energy_true(self, labels, term=-1):
        """``pairwise_energy_true(l, term)``: per-pixel pairwise energy (term -1: all)."""
        lab = np.ascontiguousarray(labels, np.int16).reshape(-1)
        out = np.zeros(self.N, np.float32)
        check(lib().dcrf_model_pairwise_energy(self._h, lab.ctypes.data_as(C.c_void_p), int(term),
                                               out.ctypes.data_as(C.c_void_p)))
        return out

    def max_rounding(self, Q):
        """``max_rounding(Q)``: one-hot at each pixel's first maximum."""
        x = self._mat(Q)
        out = self._new()
        check(lib().dcrf_model_max_rounding(self._h, x.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
        return out

    def compute_energy_higher_order(self, Q):
        """``compute_energy_higher_order(Q)``, with the clique variables of the last QP."""
        x = self._mat(Q)
        e = C.c_double()
        check(lib().dcrf_model_energy_higher_order(self._h, x.ctypes.data_as(C.c_void_p), C.byref(e)))
        return e.value

    def compute_LR_QP_value_diag(self, Q, diag_dom):
        """``compute_LR_QP_value(Q, diag_dom)``."""
        x, d = self._mat(Q), self._mat(diag_dom)
        e = C.c_double()
        check(lib().dcrf_model_lr_qp_value_diag(self._h, x.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p),
                                                C.byref(e)))
        return e.value

    def setKernel(self, k, ktype=1, ntype=3):
        """Term k's KernelType and NormalizationType (addPairwiseEnergy's last
        two arguments; the defaults are DIAG_KERNEL, NORMALIZE_SYMMETRIC)."""
        check(lib().dcrf_model_set_kernel(self._h, int(k), int(ktype), int(ntype)))

    def pairwise_kernel_parameters(self, k):
        """``pairwise_[k]->kernelParameters()``."""
        n = C.c_int(0)
        check(lib().dcrf_model_pairwise_kernel_parameters(self._h, int(k), None, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        if n.value:
            check(lib().dcrf_model_pairwise_kernel_parameters(self._h, int(k), out.ctypes.data_as(C.c_void_p),
                                                              None))
        return out

    def pairwise_set_kernel_parameters(self, k, p):
        """``pairwise_[k]->setKernelParameters(p)``: rebuilds the term's lattice
        on the scaled (DIAG) or transformed (FULL, p column-major) features."""
        p = np.ascontiguousarray(p, np.float32).reshape(-1)
        if p.size != self.pairwise_kernel_parameters(k).size:
            raise DCRFError(1, "wrong number of kernel parameters")
        check(lib().dcrf_model_pairwise_set_kernel_parameters(self._h, int(k), p.ctypes.data_as(C.c_void_p)))

    def setCompatibility(self, k, diagonal=None, matrix=None, potts=None):
        """Label compatibility of term k: ``diagonal`` (L weights,
        DiagonalCompatibility), ``matrix`` (L x L, MatrixCompatibility, used as
        0.5 (m + m^T)) or ``potts`` (the weight)."""
        if diagonal is not None:
            kind, p = 1, np.ascontiguousarray(diagonal, np.float32).reshape(-1)
            if p.size != self.L:
                raise DCRFError(1, "diagonal needs L weights")
        elif matrix is not None:
            m = np.asarray(matrix, np.float32)
            if m.shape != (self.L, self.L):
                raise DCRFError(1, "matrix must be L x L")
            kind, p = 2, np.ascontiguousarray(m.T).reshape(-1)  # column-major, as Eigen stores it
        else:
            kind, p = 0, np.array([potts], np.float32)
        check(lib().dcrf_model_set_compat(self._h, int(k), kind, p.ctypes.data_as(C.c_void_p)))

    def setCliques(self, offsets, idx, exp_weight, constants):
        offsets = np.ascontiguousarray(offsets, np.int32)
        idx = np.ascontiguousarray(idx, np.int32)
        ew = np.ascontiguousarray(exp_weight, np.float32)
        cs = np.ascontiguousarray(constants, np.float32)
        R = len(offsets) - 1
        check(lib().dcrf_model_set_cliques(self._h, R, offsets.ctypes.data_as(C.c_void_p),
                                           idx.ctypes.data_as(C.c_void_p) if idx.size else None,
                                           ew.ctypes.data_as(C.c_void_p), cs.ctypes.data_as(C.c_void_p)))

    def info(self):
        n, N, L = C.c_int(), C.c_int(), C.c_int()
        check(lib().dcrf_model_info(self._h, C.byref(n), C.byref(N), C.byref(L)))
        return n.value

    def lattice_size(self, k):
        M = C.c_int()
        check(lib().dcrf_model_lattice_size(self._h, k, C.byref(M)))
        return M.value

    # -- inference ------------------------------------------------------
    def unary_init(self):
        q = self._new()
        check(lib().dcrf_model_unary_init(self._h, q.ctypes.data_as(C.c_void_p)))
        return q

    def pairwise_apply(self, k, Q, nonorm=False):
        x = self._mat(Q)
        out = self._new()
        check(lib().dcrf_model_pairwise_apply(self._h, k, int(nonorm), out.ctypes.data_as(C.c_void_p),
                                              x.ctypes.data_as(C.c_void_p)))
        return out

    def pairwise_apply_upper_minus_lower_ord(self, k, Q):
        x = self._mat(Q)
        out = self._new()
        check(lib().dcrf_model_pairwise_apply_ord(self._h, k, out.ctypes.data_as(C.c_void_p),
                                                  x.ctypes.data_as(C.c_void_p)))
        return out

    def pairwise_apply_upper_minus_lower_ord_restricted(self, k, rQ, pI, Q=None, store=True):
        """``pairwise_[k]->apply_upper_minus_lower_ord_restricted(rout, rQ, pI,
        Q, store)``: rQ, rout [len(pI), L]; Q [N, L] read on a store call."""
        pi = np.ascontiguousarray(pI, np.int32).reshape(-1)
        x = _f32(rQ).reshape(pi.size, self.L)
        out = np.zeros((pi.size, self.L), np.float32)
        q = self._mat(Q) if store else None
        check(lib().dcrf_model_pairwise_apply_ord_restricted(
            self._h, int(k), out.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
            pi.ctypes.data_as(C.c_void_p), int(pi.size), None if q is None else q.ctypes.data_as(C.c_void_p),
            int(bool(store))))
        return out

    def pairwise_apply_bf(self, k, Q, nonorm=False):
        """``pairwise_[k]->apply_bf(out, Q)`` (``no_norm_pairwise_[k]`` with
        nonorm): the exact Gaussian filter, O(N^2) per label."""
        q = self._mat(Q)
        out = self._new()
        check(lib().dcrf_model_pairwise_apply_bf(self._h, int(k), int(bool(nonorm)), out.ctypes.data_as(C.c_void_p),
                                                 q.ctypes.data_as(C.c_void_p)))
        return out

    def _sorted(self, fn, k, ind, Q, nonorm):
        i = np.ascontiguousarray(ind, np.int32).reshape(self.N, self.L)
        out = self._new()
        args = [self._h, int(k), int(bool(nonorm)), out.ctypes.data_as(C.c_void_p), i.ctypes.data_as(C.c_void_p)]
        if Q is not None:
            q = self._mat(Q)
            args.append(q.ctypes.data_as(C.c_void_p))
        check(getattr(lib(), fn)(*args))
        return out

    def pairwise_apply_upper_minus_lower_bf(self, k, ind, nonorm=False):
        """``apply_upper_minus_lower_bf(out, ind)``: ind [N, L], ind[c, l] the
        pixel at sorted position c for label l; out in sorted positions."""
        return self._sorted("dcrf_model_pairwise_apply_upper_minus_lower_bf", k, ind, None, nonorm)

    def pairwise_apply_upper_minus_lower_bf_ord(self, k, ind, Q, nonorm=False):
        """``apply_upper_minus_lower_bf_ord(out, ind, Q)``."""
        return self._sorted("dcrf_model_pairwise_apply_upper_minus_lower_bf_ord", k, ind, Q, nonorm)

    def pairwise_apply_upper_minus_lower_dc(self, k, ind, nonorm=False):
        """``apply_upper_minus_lower_dc(out, ind)``: the divide-and-conquer
        ordered filter on lattices of the sorted features."""
        return self._sorted("dcrf_model_pairwise_apply_upper_minus_lower_dc", k, ind, None, nonorm)

    def qp_inference_super_pixels_non_convex(self, init, max_iter=0, stats=False):
        x = self._mat(init)
        out = self._new()
        p = C.c_int(max_iter)
        st = SolveStats()
        check(lib().dcrf_model_qp(self._h, x.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                                  C.byref(p), C.byref(st)))
        return (out, st) if stats else out

    def addSuperPixel(self, rgb, spatial_radius, range_radius, min_region_count, constant, normaliser):
        """``DenseCRF2D::addSuperPixel`` (src/densecrf.cpp:193-251): mean-shift
        regions of ``rgb`` (EDISON's segmentation, the mode search on the GPU)
        appended as cliques; returns the number of regions added."""
        im = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1)
        if im.size != 3 * self.N:
            raise DCRFError(1, "rgb must hold 3 bytes per pixel")
        n = C.c_int()
        check(lib().dcrf_model_add_superpixel(self._h, im.ctypes.data_as(C.c_void_p), int(spatial_radius),
                                              int(range_radius), int(min_region_count), C.c_float(constant),
                                              C.c_float(normaliser), C.byref(n)))
        return n.value

    def getCliques(self):
        """The cliques the model holds: ``(offsets, idx, exp_weight, constants)``."""
        R, T = C.c_int(), C.c_int()
        check(lib().dcrf_model_clique_info(self._h, C.byref(R), C.byref(T)))
        off = np.zeros(R.value + 1, np.int32)
        idx = np.zeros(max(T.value, 1), np.int32)
        ew = np.zeros(max(R.value, 1), np.float32)
        cs = np.zeros(max(R.value, 1), np.float32)
        check(lib().dcrf_model_get_cliques(self._h, off.ctypes.data_as(C.c_void_p), idx.ctypes.data_as(C.c_void_p),
                                           ew.ctypes.data_as(C.c_void_p), cs.ctypes.data_as(C.c_void_p)))
        return off, idx[:T.value], ew[:R.value], cs[:R.value]

    def lp_inference_prox_super_pixels(self, init, params=None, stats=False, **kw):
        x = self._mat(init)
        out = self._new()
        p = params if params is not None else LPParams.default()
        for k, v in kw.items():
            setattr(p, k, v)
        st = SolveStats()
        check(lib().dcrf_model_lp(self._h, x.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                                  C.byref(p), C.byref(st)))
        return (out, st) if stats else out

    def currentMap(self, Q):
        x = self._mat(Q)
        lab = np.empty(self.N, np.int16)
        check(lib().dcrf_model_current_map(self._h, x.ctypes.data_as(C.c_void_p),
                                           lab.ctypes.data_as(C.c_void_p)))
        return lab

    def _energy_l(self, fn, labels):
        lab = np.ascontiguousarray(labels, np.int16)
        e = C.c_double()
        check(fn(self._h, lab.ctypes.data_as(C.c_void_p), C.byref(e)))
        return e.value

    def assignment_energy_true(self, labels):
        return self._energy_l(lib().dcrf_model_energy_true, labels)

    def assignment_energy_higher_order(self, labels):
        return self._energy_l(lib().dcrf_model_energy_ho, labels)

    def compute_energy_LP_higher_order(self, Q):
        x = self._mat(Q)
        e = C.c_double()
        check(lib().dcrf_model_energy_lp(self._h, x.ctypes.data_as(C.c_void_p), C.byref(e)))
        return e.value

    def compute_LR_QP_value(self, Q):
        x = self._mat(Q)
        e = C.c_double()
        check(lib().dcrf_model_lr_qp_value(self._h, x.ctypes.data_as(C.c_void_p), C.byref(e)))
        return e.value


class DenseCRF2DBatch:
    """Several images of different sizes solved together (``dcrf_batch_*``).

    Images share the label count and the pairwise parameters; pixel arrays
    are the images' ``[W_i*H_i, ...]`` arrays stacked in order.  Each image's
    QP result equals :meth:`DenseCRF2D.qp_inference_super_pixels_non_convex`
    of that image alone.
    """

    def __init__(self, sizes, L):
        self.sizes = [(int(w), int(h)) for w, h in sizes]
        self.L = int(L)
        w = (C.c_int * len(self.sizes))(*[s[0] for s in self.sizes])
        h = (C.c_int * len(self.sizes))(*[s[1] for s in self.sizes])
        self._h = C.c_void_p()
        check(lib().dcrf_batch_create(C.byref(self._h), len(self.sizes), w, h, self.L))
        n = C.c_int64()
        off = (C.c_int64 * (len(self.sizes) + 1))()
        check(lib().dcrf_batch_info(self._h, C.byref(n), off))
        self.N = n.value
        self.offsets = np.array(off[:], np.int64)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().dcrf_batch_destroy(h)
            except Exception:
                pass

    def _mat(self, a):
        return _f32(a, (self.N, self.L))

    def _new(self):
        return np.empty((self.N, self.L), np.float32)

    def split(self, a):
        """The per-image pieces of a stacked ``[N, ...]`` array."""
        return [a[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.sizes))]

    def setUnaryEnergy(self, unary):
        u = self._mat(unary)
        check(lib().dcrf_batch_set_unary(self._h, u.ctypes.data_as(C.c_void_p)))

    def addPairwiseGaussian(self, sx, sy, w):
        check(lib().dcrf_batch_add_gaussian(self._h, C.c_float(sx), C.c_float(sy), C.c_float(w)))

    def addPairwiseBilateral(self, sx, sy, sr, sg, sb, rgb, w):
        im = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1)
        if im.size != 3 * self.N:
            raise DCRFError(1, "rgb must hold 3 bytes per pixel of every image")
        check(lib().dcrf_batch_add_bilateral(self._h, *(C.c_float(v) for v in (sx, sy, sr, sg, sb)),
                                             im.ctypes.data_as(C.c_void_p), C.c_float(w)))

    def unary_init(self):
        q = self._new()
        check(lib().dcrf_batch_unary_init(self._h, q.ctypes.data_as(C.c_void_p)))
        return q

    def qp_inference_super_pixels_non_convex(self, init, max_iter=0, stats=False):
        x = self._mat(init)
        out = self._new()
        p = C.c_int(max_iter)
        st = (SolveStats * len(self.sizes))()
        check(lib().dcrf_batch_qp(self._h, x.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                                  C.byref(p), st))
        return (out, list(st)) if stats else out

    def pairwise_apply(self, k, x):
        """``pairwise_[k]->apply(out, x)`` of every image at once, over the
        term's concatenated lattice (each image's rows equal its own
        ``DenseCRF2D.pairwise_apply``)."""
        xx = self._mat(x)
        out = self._new()
        check(lib().dcrf_batch_pairwise_apply(self._h, int(k), out.ctypes.data_as(C.c_void_p),
                                              xx.ctypes.data_as(C.c_void_p)))
        return out

    def filter_shape(self, k):
        """Term k's launch shapes (see Permutohedral.filter_shape)."""
        shp = (C.c_int * 4)()
        check(lib().dcrf_batch_filter_shape(self._h, int(k), shp))
        return tuple(shp)

    def set_filter_shape(self, k, shape):
        """Pins term k's launch shapes (no autotuning for its lattice)."""
        shp = (C.c_int * 4)(*[int(x) for x in shape])
        check(lib().dcrf_batch_set_filter_shape(self._h, int(k), shp))

    def lattice_size(self, k):
        """Vertex count of term k's concatenated lattice."""
        m = C.c_int64()
        check(lib().dcrf_batch_lattice_size(self._h, int(k), C.byref(m)))
        return m.value

    # -- differentiation (unrolled mean-field) --------------------------
    def n_terms(self):
        n = C.c_int()
        check(lib().dcrf_batch_terms(self._h, C.byref(n)))
        return n.value

    def set_weight(self, k, w):
        check(lib().dcrf_batch_set_weight(self._h, int(k), C.c_float(w)))

    def set_checkpointing(self, every=1, recompute_lattice=False):
        """Keep every ``every``-th mean-field iterate (the backward pass
        recomputes the others); release the lattices between the passes and
        rebuild them when ``recompute_lattice``."""
        check(lib().dcrf_batch_set_checkpointing(self._h, int(every), int(bool(recompute_lattice))))

    def meanfield_state_bytes(self, iterations):
        n = C.c_uint64()
        check(lib().dcrf_batch_meanfield_state_bytes(self._h, int(iterations), C.byref(n)))
        return n.value

    def meanfield(self, iterations):
        """Q_T of ``iterations`` mean-field steps (Q_0 .. Q_T are kept for
        :meth:`meanfield_backward`)."""
        out = self._new()
        check(lib().dcrf_batch_meanfield(self._h, int(iterations), out.ctypes.data_as(C.c_void_p)))
        return out

    def meanfield_backward(self, grad_Q):
        """``(dL/dU, dL/dw)`` for ``grad_Q = dL/dQ_T`` of the last :meth:`meanfield`."""
        g = self._mat(grad_Q)
        gu = self._new()
        gw = np.zeros(max(self.n_terms(), 1), np.float64)
        check(lib().dcrf_batch_meanfield_backward(self._h, g.ctypes.data_as(C.c_void_p),
                                                  gu.ctypes.data_as(C.c_void_p), gw.ctypes.data_as(C.c_void_p)))
        return gu, gw[:self.n_terms()]


__all__.append("DenseCRF2DBatch")


def _pairwise_kernel_gradient(self, k, b, Q):
    """``pairwise_[k]->kernelGradient(b, Q)``: gradient of the term's kernel
    parameters (DIAG_KERNEL d feature scales, FULL_KERNEL the d x d matrix
    column-major, CONST_KERNEL none)."""
    bb, qq = self._mat(b), self._mat(Q)
    d = C.c_int()
    check(lib().dcrf_model_pairwise_kernel_gradient(self._h, int(k), None, None, None, C.byref(d)))
    out = np.zeros(max(d.value, 1), np.float32)
    check(lib().dcrf_model_pairwise_kernel_gradient(self._h, int(k), bb.ctypes.data_as(C.c_void_p),
                                                    qq.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                                                    C.byref(d)))
    return out[:d.value]


def _pairwise_parameters(self, k):
    """``pairwise_[k]->parameters()``: Potts [w], Diagonal [w_l], Matrix the
    upper triangle of the symmetric matrix by column."""
    n = C.c_int(0)
    check(lib().dcrf_model_pairwise_parameters(self._h, int(k), None, C.byref(n)))
    out = np.zeros(n.value, np.float32)
    check(lib().dcrf_model_pairwise_parameters(self._h, int(k), out.ctypes.data_as(C.c_void_p), None))
    return out


def _pairwise_set_parameters(self, k, v):
    """``pairwise_[k]->setParameters(v)``, v as ``parameters()`` returns it."""
    v = np.ascontiguousarray(v, np.float32).reshape(-1)
    if v.size != self.pairwise_parameters(k).size:
        raise DCRFError(1, "wrong number of compatibility parameters")
    check(lib().dcrf_model_pairwise_set_parameters(self._h, int(k), v.ctypes.data_as(C.c_void_p)))


def _pairwise_gradient(self, k, b, Q):
    """``pairwise_[k]->gradient(b, Q)``: gradient of the term's compatibility
    parameters (the layout of ``parameters()``)."""
    bb, qq = self._mat(b), self._mat(Q)
    out = np.zeros(self.pairwise_parameters(k).size, np.float32)
    check(lib().dcrf_model_pairwise_gradient(self._h, int(k), bb.ctypes.data_as(C.c_void_p),
                                             qq.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
    return out


DenseCRF2D.pairwise_parameters = _pairwise_parameters
DenseCRF2D.pairwise_set_parameters = _pairwise_set_parameters
DenseCRF2D.pairwise_kernel_gradient = _pairwise_kernel_gradient
DenseCRF2D.pairwise_gradient = _pairwise_gradient


def set_device_memory_limit(nbytes):
    """Budget (bytes, 0 = none) on the device memory the library holds for
    live models, lattices and batches; a request beyond it raises a
    DCRFError with DCRF_E_NOMEM before any device call."""
    check(lib().dcrf_set_device_memory_limit(C.c_uint64(int(nbytes))))


def device_memory_stats():
    """``(in_use, cached, mallocs)``: bytes held by live objects, bytes kept
    in the library's cache of freed blocks, cudaMalloc calls made so far."""
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check(lib().dcrf_device_memory_stats(C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


__all__ += ["set_device_memory_limit", "device_memory_stats"]


def meanshift_segment(rgb, W, H, spatial_radius, range_radius, min_region_count):
    """EDISON's mean-shift segmentation (the step addSuperPixel runs):
    ``(labels int32 [W*H], n_regions)``."""
    im = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1)
    if im.size != 3 * W * H:
        raise DCRFError(1, "rgb must hold 3 bytes per pixel")
    lab = np.empty(W * H, np.int32)
    n = C.c_int()
    check(lib().dcrf_meanshift_segment(im.ctypes.data_as(C.c_void_p), int(W), int(H), int(spatial_radius),
                                       C.c_float(range_radius), int(min_region_count),
                                       lab.ctypes.data_as(C.c_void_p), C.byref(n)))
    return lab, n.value


def meanshift_regions(filtered, W, H, range_radius, min_region_count):
    """The region steps alone (host, no GPU) from a filtered L*u*v* image
    ``[W*H, 3]``: ``(labels, n_regions)``."""
    f = np.ascontiguousarray(filtered, dtype=np.float32).reshape(-1)
    if f.size != 3 * W * H:
        raise DCRFError(1, "filtered must hold 3 floats per pixel")
    lab = np.empty(W * H, np.int32)
    n = C.c_int()
    check(lib().dcrf_meanshift_regions(f.ctypes.data_as(C.c_void_p), int(W), int(H), C.c_float(range_radius),
                                       int(min_region_count), lab.ctypes.data_as(C.c_void_p), C.byref(n)))
    return lab, n.value


__all__ += ["meanshift_segment", "meanshift_regions"]
