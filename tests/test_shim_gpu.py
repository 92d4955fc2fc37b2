"""The drop-in C++ API (densecrf_ho_b200/cpp/densecrf.h: DenseCRF2D,
Permutohedral, PairwisePotential, LP_inf_params with the reference's names)
gives the same results as the C ABI called from Python.

The self-test binary is compiled with g++ against Eigen by
``__graft_entry__.build()``; it runs the example's model
(src/example_inference.cpp:39-63 settings) through the C++ classes and
writes raw float outputs, which must equal the Python path bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

from densecrf_ho_b200 import DenseCRF2D, LPParams, Permutohedral, synth
from densecrf_ho_b200.build import SHIM_BIN

pytestmark = pytest.mark.gpu


def _need_shim():
    if not os.path.exists(SHIM_BIN):
        pytest.skip("shim_selftest not built (it needs Eigen headers at build time)")


def test_cpp_shim_matches_c_abi(tmp_path):
    _need_shim()
    W, H, L = 61, 43, 21
    img = synth.make_image(W, H, L, 5)
    rgb, unary = img["rgb"], img["unary"]
    (tmp_path / "rgb.u8").write_bytes(np.ascontiguousarray(rgb, np.uint8).tobytes())
    (tmp_path / "unary.f32").write_bytes(np.ascontiguousarray(unary, np.float32).tobytes())
    prefix = str(tmp_path / "out")
    r = subprocess.run([SHIM_BIN, str(W), str(H), str(L), str(tmp_path / "rgb.u8"),
                        str(tmp_path / "unary.f32"), prefix], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = dict(l.split(" ", 1) for l in r.stdout.strip().splitlines())

    def load(ext):
        return np.fromfile(prefix + "." + ext, np.float32).reshape(W * H, L)

    m = DenseCRF2D(W, H, L)
    m.setUnaryEnergy(unary)
    m.addPairwiseGaussian(3.0, 3.0, 3.0)
    m.addPairwiseBilateral(50.0, 50.0, 15.0, 15.0, 15.0, rgb, 5.0)
    Q = m.unary_init()
    assert np.array_equal(load("init"), Q)
    qp = m.qp_inference_super_pixels_non_convex(Q)
    assert np.array_equal(load("qp"), qp)
    p = LPParams.default()
    p.prox_energy_tol = p.dual_gap_tol
    p.prox_max_iter = 3
    p.fw_max_iter = 3
    lp = m.lp_inference_prox_super_pixels(Q, p)
    assert np.array_equal(load("lp"), lp)
    assert float(lines["qp_energy"]) == pytest.approx(m.assignment_energy_true(m.currentMap(qp)), rel=1e-9)
    assert float(lines["lp_energy"]) == pytest.approx(m.assignment_energy_true(m.currentMap(lp)), rel=1e-9)

    jj, ii = np.mgrid[0:H, 0:W]
    F = np.stack([ii.reshape(-1) / np.float32(3), jj.reshape(-1) / np.float32(3)], 1).astype(np.float32)
    lat = Permutohedral().init(F)
    assert int(lines["lattice_M"]) == lat.M
    assert np.array_equal(load("filt"), lat.compute(Q))
    pw = DenseCRF2D(W * H, 1, L)
    pw.addPairwiseEnergy(F, 3.0)
    assert np.array_equal(load("pw"), pw.pairwise_apply(0, Q))
    ind = np.argsort(-Q, axis=0, kind="stable").astype(np.int32)
    assert np.array_equal(load("dc"), pw.pairwise_apply_upper_minus_lower_dc(0, ind))

    assert lines["range_error"] == "Value out of bounds"
    assert lines["kernel_error"] == "ok"

    dg = -(2.0 + np.float32(0.1) * np.arange(L, dtype=np.float32))
    a, b = np.mgrid[0:L, 0:L]
    mt = np.where(a == b, np.float32(-5.0), np.float32(0.1) * (a + 2 * b).astype(np.float32) / np.float32(L))
    m2 = DenseCRF2D(W, H, L)
    m2.setUnaryEnergy(unary)
    m2.addPairwiseGaussian(3.0, 3.0, 1.0)
    m2.addPairwiseBilateral(50.0, 50.0, 15.0, 15.0, 15.0, rgb, 1.0)
    m2.setCompatibility(0, diagonal=dg.astype(np.float32))
    m2.setCompatibility(1, matrix=mt.astype(np.float32))
    qpc = m2.qp_inference_super_pixels_non_convex(m2.unary_init())
    assert np.array_equal(load("qpc"), qpc)
    assert float(lines["compat_energy"]) == pytest.approx(m2.assignment_energy_true(m2.currentMap(qpc)), rel=1e-9)
