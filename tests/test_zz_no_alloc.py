"""dcrf_lattice_compute_noalloc: the lattice filter for callers that may not
allocate device memory during a call (hosts that give out all GPU memory from
their own pool, or run under a fixed budget in a latency-critical loop).  Its
scratch is a fixed device array instead of cudaMalloc'd buffers.

Called through the C ABI; checked against the allocating entry point
dcrf_lattice_compute_dev, bit for bit (the tolerance of every lattice-filter
test here), on two calls in a row -- the second one reuses the array that the
first one left behind, on a different lattice and label count.  Collected last
so that a failure here cannot stop the rest of a run that stops at the first
failure.
"""
import ctypes as C

import numpy as np
import pytest

from densecrf_ho_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _lattice(L_, f):
    h = C.c_void_p()
    _lib.check(L_.dcrf_lattice_create(C.byref(h)))
    f = np.ascontiguousarray(f, np.float32)
    _lib.check(L_.dcrf_lattice_init(h, f.ctypes.data_as(C.c_void_p), f.shape[1], f.shape[0]))
    return h


def _both(L_, h, x, reverse):
    import torch
    xd = torch.from_numpy(x).cuda()
    ref = torch.empty_like(xd)
    out = torch.full_like(xd, float("nan"))
    torch.cuda.synchronize()
    _lib.check(L_.dcrf_lattice_compute_dev(h, C.c_void_p(ref.data_ptr()), C.c_void_p(xd.data_ptr()),
                                           x.shape[1], int(reverse)))
    _lib.check(L_.dcrf_lattice_compute_noalloc(h, C.c_void_p(out.data_ptr()), C.c_void_p(xd.data_ptr()),
                                               x.shape[1], int(reverse)))
    torch.cuda.synchronize()
    return ref.cpu().numpy(), out.cpu().numpy()


def test_noalloc_matches_allocating_filter_twice_in_a_row():
    L_ = _lib.lib()
    W, H = 160, 120
    img = synth.make_image(W, H, 21, 9)
    lat_b = _lattice(L_, synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"]))
    lat_g = _lattice(L_, synth.gaussian_features(W, H, 3, 3))
    try:
        rng = np.random.default_rng(3)
        x21 = rng.standard_normal((W * H, 21)).astype(np.float32)
        ref, out = _both(L_, lat_b, x21, False)
        assert np.array_equal(ref, out)
        x5 = rng.random((W * H, 5)).astype(np.float32)  # second call: other lattice, other L
        ref, out = _both(L_, lat_g, x5, True)
        assert np.array_equal(ref, out)
    finally:
        L_.dcrf_lattice_destroy(lat_b)
        L_.dcrf_lattice_destroy(lat_g)


def test_noalloc_rejects_sizes_beyond_the_fixed_scratch():
    import torch
    L_ = _lib.lib()
    W, H = 64, 48
    h = _lattice(L_, synth.gaussian_features(W, H, 1.0, 1.0))
    try:
        M = C.c_int()
        _lib.check(L_.dcrf_lattice_info(h, C.byref(M), None, None))
        L = (8 << 20) // (2 * (M.value + 1)) + 1  # one label more than fits
        x = torch.zeros((W * H, L), device="cuda")
        rc = L_.dcrf_lattice_compute_noalloc(h, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), L, 0)
        assert rc == 1  # DCRF_E_ARG
        assert b"exceeds the fixed scratch" in L_.dcrf_last_error()
    finally:
        L_.dcrf_lattice_destroy(h)
