"""dcrf_lattice_compute_noalloc: the lattice filter for callers that may not
allocate device memory during a call (hosts that give out all GPU memory from
their own pool, or run under a fixed budget in a latency-critical loop).  Its
scratch is a fixed device array instead of cudaMalloc'd buffers.

Called through the C ABI; checked against the allocating entry point
dcrf_lattice_compute_dev and against the CPU oracle, bit for bit (the
tolerance of every lattice-filter test here), on two calls in a row -- the
second one reuses the array that the first one left behind, on a different
lattice and label count -- and first on fresh lattices with one and two
labels (the double-precision blur of the reference's seqCompute).  Around
each call the library's allocation counters, and the device's free memory,
must not move.  Collected last so that a failure here cannot stop the rest
of a run that stops at the first failure.
"""
import ctypes as C

import numpy as np
import pytest

from densecrf_ho_b200 import _lib, device_memory_stats, synth

pytestmark = pytest.mark.gpu


def _lattice(L_, f):
    h = C.c_void_p()
    _lib.check(L_.dcrf_lattice_create(C.byref(h)))
    f = np.ascontiguousarray(f, np.float32)
    _lib.check(L_.dcrf_lattice_init(h, f.ctypes.data_as(C.c_void_p), f.shape[1], f.shape[0]))
    return h


def _noalloc(L_, h, out, xd, L, reverse):
    """One no-alloc call; returns (library counters, device free bytes) before
    and after it, the device synchronised on both sides."""
    import torch
    torch.cuda.synchronize()
    s0, f0 = device_memory_stats(), torch.cuda.mem_get_info()[0]
    _lib.check(L_.dcrf_lattice_compute_noalloc(h, C.c_void_p(out.data_ptr()), C.c_void_p(xd.data_ptr()), L,
                                               int(reverse)))
    torch.cuda.synchronize()
    return (s0, f0), (device_memory_stats(), torch.cuda.mem_get_info()[0])


def _both(L_, h, x, reverse):
    import torch
    xd = torch.from_numpy(x).cuda()
    ref = torch.empty_like(xd)
    out = torch.full_like(xd, float("nan"))
    torch.cuda.synchronize()
    _lib.check(L_.dcrf_lattice_compute_dev(h, C.c_void_p(ref.data_ptr()), C.c_void_p(xd.data_ptr()),
                                           x.shape[1], int(reverse)))
    before, after = _noalloc(L_, h, out, xd, x.shape[1], reverse)
    assert before[0] == after[0], "the no-alloc call changed the library's device allocations"
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


@pytest.mark.parametrize("L", [1, 2])
def test_noalloc_first_on_a_fresh_lattice_small_label_counts(L, oracle_mod):
    """L <= 2 takes the reference's seqCompute arithmetic (double-precision
    blur, (w v) alpha slice).  The no-alloc call comes first on a fresh
    lattice; the allocating filter and the oracle are checked against it
    afterwards, and a repeated call leaves the device's free memory as it was."""
    import torch
    L_ = _lib.lib()
    W, H = 61, 47
    img = synth.make_image(W, H, 21, 20 + L)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    h = _lattice(L_, f)
    try:
        x = np.random.default_rng(L).random((W * H, L)).astype(np.float32)
        xd = torch.from_numpy(x).cuda()
        out = torch.full_like(xd, float("nan"))
        before, after = _noalloc(L_, h, out, xd, L, False)
        assert before[0] == after[0], "the no-alloc call changed the library's device allocations"
        got = out.cpu().numpy()
        assert np.array_equal(got, oracle_mod.OracleLattice(f).compute(x))
        ref = torch.empty_like(xd)
        _lib.check(L_.dcrf_lattice_compute_dev(h, C.c_void_p(ref.data_ptr()), C.c_void_p(xd.data_ptr()), L, 0))
        torch.cuda.synchronize()
        assert np.array_equal(ref.cpu().numpy(), got)
        # every kernel of the call is loaded by now: the repeat must not take
        # a byte of device memory
        out2 = torch.full_like(xd, float("nan"))
        before, after = _noalloc(L_, h, out2, xd, L, False)
        assert before == after, (before, after)
        assert np.array_equal(out2.cpu().numpy(), got)
    finally:
        L_.dcrf_lattice_destroy(h)


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
