"""CUDA lattice vs the oracle and the reference's golden vectors.

Lattice tables (vertex count M, offsets, ranks, barycentric weights, keys,
neighbours) and filter outputs are required to be BIT-EXACT: the CUDA path
reproduces the reference's float operation order and the splat gathers in
the order the reference's scatter accumulates.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden, golden_names
from densecrf_ho_b200 import Permutohedral, check, lib, synth

pytestmark = pytest.mark.gpu


def _eq(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("name", golden_names("lattice_"))
def test_lattice_matches_reference_golden(name):
    g = golden(name)
    for t in ("g", "b"):
        lat = Permutohedral().init(g[f"{t}_f"])
        ex = lat.export()
        assert ex["M"] == int(g[f"{t}_M"])
        for k in ("offset", "rank", "bary", "nbr"):
            assert _eq(ex[k], g[f"{t}_{k}"]), (name, t, k)
        assert _eq(lat.compute(g["x"]), g[f"{t}_compute"])
        assert _eq(lat.compute(g["x"], reverse=True), g[f"{t}_compute_rev"])
        assert _eq(lat.compute(g["x1"]), g[f"{t}_compute_l1"])
        assert _eq(lat.compute_upper_minus_lower_ord(g["x"]), g[f"{t}_ord"])


CASES = [(1, 1), (3, 1), (5, 3), (17, 13), (64, 48), (97, 61), (160, 120)]


@pytest.mark.parametrize("W,H", CASES)
@pytest.mark.parametrize("kind", ["gauss", "bilat"])
def test_lattice_tables_bit_exact(W, H, kind, oracle_mod):
    img = synth.make_image(W, H, 21, W * 31 + H)
    f = (synth.gaussian_features(W, H, 3, 3) if kind == "gauss"
         else synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"]))
    a = Permutohedral().init(f).export()
    b = oracle_mod.OracleLattice(f).export()
    assert a["M"] == b["M"]
    for k in ("offset", "rank", "bary", "keys", "nbr"):
        assert _eq(a[k], b[k]), k


@pytest.mark.parametrize("d", [1, 3, 4, 7, 9])
def test_lattice_other_dimensions(d, oracle_mod):
    rng = np.random.default_rng(d)
    N = 1001
    f = (rng.random((N, d)) * 6).astype(np.float32)
    lat = Permutohedral().init(f)
    a, b = lat.export(), oracle_mod.OracleLattice(f).export()
    assert a["M"] == b["M"]
    for k in ("offset", "rank", "bary", "keys", "nbr"):
        assert _eq(a[k], b[k]), k
    x = rng.random((N, 5)).astype(np.float32)
    assert _eq(lat.compute(x), oracle_mod.OracleLattice(f).compute(x))


@pytest.mark.parametrize("L", [1, 2, 3, 21, 33])
def test_filter_bit_exact(L, oracle_mod):
    W, H = 80, 60
    img = synth.make_image(W, H, 21, 7)
    for f in (synth.gaussian_features(W, H, 3, 3),
              synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])):
        lat, orc = Permutohedral().init(f), oracle_mod.OracleLattice(f)
        x = np.random.default_rng(L).standard_normal((W * H, L)).astype(np.float32)
        assert _eq(lat.compute(x), orc.compute(x))
        assert _eq(lat.compute(x, reverse=True), orc.compute(x, True))
        q = np.random.default_rng(L + 1).random((W * H, L)).astype(np.float32)
        q[::7] = 0.0
        q[::11] = 1.0
        assert _eq(lat.compute_upper_minus_lower_ord(q), orc.compute_ord(q))


@pytest.mark.parametrize("L", [60, 130, 200])
def test_ordered_filter_wide_labels(L, oracle_mod):
    """The long-list ordered splat splits a vertex's 20 L bin chains over a
    block whose shape depends on L (opt-in shared memory above 48 KB) and
    falls back to a warp per list past 160 labels."""
    W, H = 72, 54
    img = synth.make_image(W, H, 21, 9)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    lat, orc = Permutohedral().init(f), oracle_mod.OracleLattice(f)
    q = np.random.default_rng(L).random((W * H, L)).astype(np.float32)
    q[::5] = 1.0
    q[::13] = 0.0
    assert _eq(lat.compute_upper_minus_lower_ord(q), orc.compute_ord(q))


@pytest.mark.parametrize("L", [5, 21])
def test_ordered_filter_huge_lists(L, oracle_mod):
    """A coarse lattice whose splat lists run to thousands of entries: the
    longest lists are shared by several blocks, the rest take one each."""
    W, H = 128, 96
    img = synth.make_image(W, H, 21, 9)
    f = synth.bilateral_features(W, H, 500, 500, 100, 100, 100, img["rgb"])
    lat, orc = Permutohedral().init(f), oracle_mod.OracleLattice(f)
    q = np.random.default_rng(L).random((W * H, L)).astype(np.float32)
    q[::3] = np.float32(0.3)  # exact multiples of 0.1: lower and upper bins differ
    assert _eq(lat.compute_upper_minus_lower_ord(q), orc.compute_ord(q))
    x = np.random.default_rng(L + 5).standard_normal((W * H, L)).astype(np.float32)
    assert _eq(lat.compute(x), orc.compute(x))


# Every launch shape the autotuner can choose for the 21-label plain filter:
# (splat warps per block, blur threads, slice pixels per tile, splat form).
FILTER_SHAPES = [(4, 256, 128, 0), (2, 128, 64, 1), (8, 512, 256, 1), (2, 256, 128, 2), (8, 128, 64, 2),
                 (4, 512, 256, 3), (4, 128, 128, 4), (4, 256, 128, 5)]


@pytest.mark.parametrize("shape", FILTER_SHAPES)
def test_filter_every_launch_shape_bit_exact(shape, oracle_mod):
    """Each pinned shape on lattices with short (<= 64 entries), long and
    huge (> 1024) splat lists, both blur orders: bit-equal to the oracle."""
    W, H = 160, 120
    img = synth.make_image(W, H, 21, 5)
    feats = (synth.gaussian_features(W, H, 3, 3),
             synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"]),
             synth.bilateral_features(W, H, 300, 300, 60, 60, 60, img["rgb"]))
    x = np.random.default_rng(17).standard_normal((W * H, 21)).astype(np.float32)
    for f in feats:
        lat, orc = Permutohedral().init(f).set_filter_shape(shape), oracle_mod.OracleLattice(f)
        assert lat.filter_shape() == tuple(shape)
        assert _eq(lat.compute(x), orc.compute(x))
        assert _eq(lat.compute(x, reverse=True), orc.compute(x, True))
    n = C.c_ulonglong(99)
    check(lib().dcrf_device_wait_timeouts(C.byref(n)))
    assert n.value == 0


@pytest.mark.parametrize("form", [3, 5])
def test_staged_splat_ragged_end_and_unaligned_input(form, oracle_mod):
    """The staged splat forms at an odd pixel count (84 N not a multiple of
    16: the bulk copy of the last pixel's run would pass the end of the input
    and takes plain loads instead) and with an input pointer that is not
    16-byte aligned (the bulk-copy form falls back to the tiled one)."""
    import torch
    W, H = 161, 119
    img = synth.make_image(W, H, 21, 8)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    lat, orc = Permutohedral().init(f).set_filter_shape((4, 256, 128, form)), oracle_mod.OracleLattice(f)
    x = np.random.default_rng(23).standard_normal((W * H, 21)).astype(np.float32)
    ref = orc.compute(x)
    assert _eq(lat.compute(x), ref)
    buf = torch.empty(W * H * 21 + 1, device="cuda")
    buf[1:] = torch.from_numpy(x.ravel()).cuda()  # 4 bytes past a 16-byte boundary
    out = torch.empty(W * H * 21, device="cuda")
    check(lib().dcrf_lattice_compute_dev(lat._h, C.c_void_p(out.data_ptr()), C.c_void_p(buf[1:].data_ptr()),
                                         21, 0))
    torch.cuda.synchronize()
    assert _eq(out.cpu().numpy().reshape(W * H, 21), ref)


def test_filter_error_vs_fp64_oracle(oracle_mod):
    """Relative error of the FP32 filter against the FP64 lattice oracle."""
    W, H = 160, 120
    img = synth.make_image(W, H, 21, 3)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    x = np.random.default_rng(0).random((W * H, 21)).astype(np.float32)
    out = Permutohedral().init(f).compute(x)
    ref64 = oracle_mod.OracleLattice(f).compute_f64(x.astype(np.float64))
    rel = np.linalg.norm(out - ref64) / np.linalg.norm(ref64)
    assert rel < 1e-6, rel


def test_full_size_properties(oracle_mod):
    """640x480: M and the tables of both lattices match the oracle; the filter
    is linear (K(a x + y) = a K x + K y to float accuracy) and deterministic."""
    W, H = 640, 480
    img = synth.make_image(W, H, 21, 1)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    lat = Permutohedral().init(f)
    a, b = lat.export(), oracle_mod.OracleLattice(f).export()
    assert a["M"] == b["M"]
    for k in ("offset", "bary", "nbr"):
        assert _eq(a[k], b[k])
    rng = np.random.default_rng(2)
    x = rng.random((W * H, 21)).astype(np.float32)
    y = rng.random((W * H, 21)).astype(np.float32)
    kx, ky, kxy = lat.compute(x), lat.compute(y), lat.compute(2 * x + y)
    assert np.linalg.norm(kxy - (2 * kx + ky)) / np.linalg.norm(kxy) < 1e-6
    assert _eq(lat.compute(x), kx)


@pytest.mark.parametrize("name", golden_names("gradient_"))
def test_feature_gradient_matches_reference(name):
    """Permutohedral::gradient, bit for bit, against the reference's own
    values (tests/golden/make_gradient_golden.py)."""
    g = golden(name)
    lat = Permutohedral().init(g["f"])
    assert _eq(lat.gradient(g["a"], g["b"]), g["df"])


def test_restricted_ord_matches_reference_golden():
    """compute_upper_minus_lower_ord_restricted and the pairwise terms'
    apply_upper_minus_lower_ord_restricted, bit for bit against the
    reference's own outputs (tests/golden/make_restricted_golden.py): a store
    call, a reuse call with new values, and a reuse call on a smaller pixel
    set whose blur still covers the first call's vertices."""
    from densecrf_ho_b200 import DenseCRF2D
    g = golden("restricted_32x24.npz")
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    Q, pI = g["Q"], g["pI"]
    for name in ("g", "b"):
        lat = Permutohedral().init(g[f"{name}_f"])
        assert _eq(lat.compute_upper_minus_lower_ord_restricted(Q[pI], pI, Q, True), g[f"{name}_out1"])
        assert _eq(lat.compute_upper_minus_lower_ord_restricted(g["rQ2"], pI, None, False), g[f"{name}_out2"])
        assert _eq(lat.compute_upper_minus_lower_ord_restricted(g["rQ3"], g["pI3"], None, False),
                   g[f"{name}_out3"])
    img = synth.make_image(W, H, L, int(g["seed"]))
    m = DenseCRF2D(W, H, L)
    m.setUnaryEnergy(img["unary"])
    m.addPairwiseGaussian(3.0, 3.0, 3.0)
    m.addPairwiseBilateral(50.0, 50.0, 15.0, 15.0, 15.0, img["rgb"], 5.0)
    for k in range(2):
        f = m.pairwise_apply_upper_minus_lower_ord_restricted
        assert _eq(f(k, Q[pI], pI, Q, True), g[f"m{k}_out1"])
        assert _eq(f(k, g["rQ2"], pI, None, False), g[f"m{k}_out2"])
        assert _eq(f(k, g["rQ3"], g["pI3"], None, False), g[f"m{k}_out3"])


@pytest.mark.parametrize("L", [1, 5])
def test_restricted_ord_vs_restatement(L, oracle_mod):
    """Against the numpy restatement on the C oracle's tables: a larger
    bilateral lattice, an empty pixel set, and the full pixel set, where
    every vertex is active and the restricted filter is the ordered filter."""
    W, H = 97, 61
    N = W * H
    img = synth.make_image(W, H, 21, 4)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    rng = np.random.default_rng(L)
    Q = rng.random((N, L)).astype(np.float32)
    Q[::7] = np.float32(0.3)
    lat = Permutohedral().init(f)
    ref = oracle_mod.RestrictedOrd(oracle_mod.OracleLattice(f).export(), 5)
    pI = np.sort(rng.choice(N, N // 3, replace=False)).astype(np.int32)
    rQ = rng.random((len(pI), L)).astype(np.float32)
    assert _eq(lat.compute_upper_minus_lower_ord_restricted(rQ, pI, Q, True), ref.compute(rQ, pI, Q, True))
    rQ2 = rng.random((len(pI), L)).astype(np.float32)
    assert _eq(lat.compute_upper_minus_lower_ord_restricted(rQ2, pI, None, False),
               ref.compute(rQ2, pI, None, False))
    empty = np.zeros(0, np.int32)
    assert lat.compute_upper_minus_lower_ord_restricted(np.zeros((0, L), np.float32), empty, Q, True).shape == (0, L)
    allp = np.arange(N, dtype=np.int32)
    full = lat.compute_upper_minus_lower_ord_restricted(Q, allp, Q, True)
    assert _eq(full, lat.compute_upper_minus_lower_ord(Q))


def test_restricted_ord_errors():
    from densecrf_ho_b200 import DCRFError
    W, H, L = 16, 12, 3
    lat = Permutohedral().init(synth.gaussian_features(W, H, 3, 3))
    Q = np.full((W * H, L), 0.5, np.float32)
    pI = np.array([3, 9, 40], np.int32)
    with pytest.raises(DCRFError):   # nothing stored yet
        lat.compute_upper_minus_lower_ord_restricted(Q[pI], pI, None, False)
    with pytest.raises(DCRFError):   # not ascending
        lat.compute_upper_minus_lower_ord_restricted(Q[pI], pI[::-1].copy(), Q, True)
    with pytest.raises(DCRFError):   # out of [0, 1]
        lat.compute_upper_minus_lower_ord_restricted(Q[pI] + 1, pI, Q, True)
    lat.compute_upper_minus_lower_ord_restricted(Q[pI], pI, Q, True)
    with pytest.raises(DCRFError):   # stored for another label count
        lat.compute_upper_minus_lower_ord_restricted(np.zeros((3, 2), np.float32), pI, None, False)
