"""The headless example program (densecrf_ho_b200/cpp/example_inference):
its readers against fixtures made with the reference's own ProbImage codec,
and its solves against the Python C-ABI path on the same inputs.

The binary is compiled with g++ against Eigen by __graft_entry__.build()."""
import hashlib
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN
from densecrf_ho_b200.build import CLI_BIN

FIX = os.path.join(GOLDEN, "cli_48x32")


def _need_cli():
    if not os.path.exists(CLI_BIN):
        pytest.skip("example_inference not built (it needs Eigen headers at build time)")


def _run(args, env=None, timeout=300):
    return subprocess.run([CLI_BIN] + args, capture_output=True, text=True, timeout=timeout,
                          env={**os.environ, **(env or {})})


def test_unary_decoder_matches_reference_codec(tmp_path):
    _need_cli()
    rec = json.load(open(FIX + ".json"))
    r = _run(["--dump-unary", FIX + ".c_unary", str(tmp_path / "u.f32")])
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == [str(rec["W"]), str(rec["H"]), str(rec["D"])]
    assert hashlib.sha256((tmp_path / "u.f32").read_bytes()).hexdigest() == rec["unary_sha256"]


def _bmp24_topdown(path, rgb, W, H):
    row = (W * 3 + 3) & ~3
    px = rgb.reshape(H, W, 3)[:, :, ::-1]
    data = b"".join(px[j].tobytes() + b"\0" * (row - 3 * W) for j in range(H))
    info = struct.pack("<IiiHHIIiiII", 40, W, -H, 1, 24, 0, len(data), 2835, 2835, 0, 0)
    with open(path, "wb") as f:
        f.write(b"BM" + struct.pack("<IHHI", 54 + len(data), 0, 0, 54) + info + data)


def test_bmp_reader(tmp_path):
    _need_cli()
    rec = json.load(open(FIX + ".json"))
    r = _run(["--dump-image", FIX + ".bmp", str(tmp_path / "a.u8")])
    assert r.returncode == 0, r.stderr
    assert hashlib.sha256((tmp_path / "a.u8").read_bytes()).hexdigest() == rec["rgb_sha256"]
    rgb = np.random.default_rng(0).integers(0, 256, 7 * 5 * 3).astype(np.uint8)  # odd width: padded rows
    _bmp24_topdown(tmp_path / "b.bmp", rgb, 7, 5)
    r = _run(["--dump-image", str(tmp_path / "b.bmp"), str(tmp_path / "b.u8")])
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.fromfile(tmp_path / "b.u8", np.uint8), rgb)
    (tmp_path / "bad.bmp").write_bytes(b"XX" + b"\0" * 60)
    assert _run(["--dump-image", str(tmp_path / "bad.bmp"), str(tmp_path / "c.u8")]).returncode == 1


def _pgm(path):
    b = open(path, "rb").read()
    parts = b.split(b"\n", 3)
    assert parts[0] == b"P5"
    return np.frombuffer(parts[3], np.uint8)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["unary", "qp", "lp"])
def test_cli_matches_python_api(method, tmp_path):
    _need_cli()
    from densecrf_ho_b200 import DenseCRF2D, LPParams
    rec = json.load(open(FIX + ".json"))
    W, H, D = rec["W"], rec["H"], rec["D"]
    env = {"DCRF_IMAGE": FIX + ".bmp", "DCRF_UNARY": FIX + ".c_unary", "DCRF_OUTPUT": str(tmp_path / "seg.pgm")}
    r = _run([method], env)
    assert r.returncode == 0, r.stderr
    line = [l for l in r.stdout.splitlines() if l.startswith("# method: ")][-1]
    name, energy = line[len("# method: "):].split("\t")
    assert name == method
    _run(["--dump-unary", FIX + ".c_unary", str(tmp_path / "u.f32")])
    _run(["--dump-image", FIX + ".bmp", str(tmp_path / "i.u8")])
    U = np.fromfile(tmp_path / "u.f32", np.float32).reshape(W * H, D)
    rgb = np.fromfile(tmp_path / "i.u8", np.uint8)
    m = DenseCRF2D(W, H, D)
    m.setUnaryEnergy(U)
    m.addPairwiseGaussian(2.0, 2.0, 3.0)  # the program's defaults
    m.addPairwiseBilateral(30.0, 30.0, 8.0, 8.0, 8.0, rgb, 2.0)
    Q = m.unary_init()
    if method == "qp":
        Q = m.qp_inference_super_pixels_non_convex(Q)
    elif method == "lp":
        prm = LPParams.default()
        prm.prox_energy_tol = prm.dual_gap_tol
        Q = m.lp_inference_prox_super_pixels(Q, prm)
    lab = m.currentMap(Q)
    assert np.array_equal(_pgm(tmp_path / "seg.pgm"), lab.astype(np.uint8))
    assert float(energy) == pytest.approx(m.assignment_energy_true(lab), rel=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["qp_sp", "lp_sp"])
def test_cli_higher_order_methods_match_python_api(method, tmp_path):
    """qp_sp / lp_sp: the program adds addSuperPixel(img, 8, 4, 100, 50, 1000)
    cliques (the engine's mean-shift) as the reference's does; its labels and
    reported energy equal the same solve through the Python API."""
    _need_cli()
    from densecrf_ho_b200 import DenseCRF2D, LPParams
    rec = json.load(open(FIX + ".json"))
    W, H, D = rec["W"], rec["H"], rec["D"]
    env = {"DCRF_IMAGE": FIX + ".bmp", "DCRF_UNARY": FIX + ".c_unary", "DCRF_OUTPUT": str(tmp_path / "seg.pgm")}
    r = _run([method, "3", "5", "30", "5", "10"], env)
    assert r.returncode == 0, r.stderr
    assert "Running tests on" in r.stdout
    line = [l for l in r.stdout.splitlines() if l.startswith("# method: ")][-1]
    energy = float(line.split("\t")[1])
    _run(["--dump-unary", FIX + ".c_unary", str(tmp_path / "u.f32")])
    _run(["--dump-image", FIX + ".bmp", str(tmp_path / "i.u8")])
    U = np.fromfile(tmp_path / "u.f32", np.float32).reshape(W * H, D)
    rgb = np.fromfile(tmp_path / "i.u8", np.uint8)
    m = DenseCRF2D(W, H, D)
    m.setUnaryEnergy(U)
    m.addPairwiseGaussian(3.0, 3.0, 5.0)
    m.addPairwiseBilateral(30.0, 30.0, 5.0, 5.0, 5.0, rgb, 10.0)
    Q = m.unary_init()
    assert m.addSuperPixel(rgb, 8, 4, 100, 50.0, 1000.0) >= 1
    if method == "qp_sp":
        Q = m.qp_inference_super_pixels_non_convex(Q)
    else:
        prm = LPParams.default()
        prm.prox_energy_tol = prm.dual_gap_tol
        Q = m.lp_inference_prox_super_pixels(Q, prm)
    lab = m.currentMap(Q)
    assert np.array_equal(_pgm(tmp_path / "seg.pgm"), lab.astype(np.uint8))
    ref = m.assignment_energy_higher_order(lab) if method == "qp_sp" else m.assignment_energy_true(lab)
    assert energy == pytest.approx(ref, rel=1e-5)
