"""The CPU oracle (our C restatement) pinned against the reference.

Every check is bit-exact (``np.array_equal``): the restatement follows the
reference's float operation order, including Eigen's SSE2 reduction order and
its packet exp in ``unary_init``.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import golden, golden_names
from densecrf_ho_b200 import synth

LAT = golden_names("lattice_")
MOD = golden_names("model_")


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("name", LAT)
def test_lattice_pinned_to_golden(name, oracle_mod):
    g = golden(name)
    for t in ("g", "b"):
        lat = oracle_mod.OracleLattice(g[f"{t}_f"])
        ex = lat.export()
        assert ex["M"] == int(g[f"{t}_M"])
        for k in ("offset", "rank", "bary", "nbr"):
            assert _bits_equal(ex[k], g[f"{t}_{k}"]), (name, t, k)
        assert _bits_equal(lat.compute(g["x"]), g[f"{t}_compute"])
        assert _bits_equal(lat.compute(g["x"], True), g[f"{t}_compute_rev"])
        assert _bits_equal(lat.compute(g["x1"]), g[f"{t}_compute_l1"])
        assert _bits_equal(lat.compute_ord(g["x"]), g[f"{t}_ord"])


def _oracle_model(O, g):
    img = dict(W=int(g["W"]), H=int(g["H"]), L=21, rgb=g["rgb"], unary=g["unary"])
    m = O.build_model(O.OracleModel, img)
    if "cl_off" in g:
        m.set_cliques(g["cl_off"], g["cl_idx"], g["cl_exp"], g["cl_const"])
    return m


@pytest.mark.parametrize("name", MOD)
def test_model_pinned_to_golden(name, oracle_mod):
    g = golden(name)
    m = _oracle_model(oracle_mod, g)
    Q = g["unary_init"]  # the reference's own initialisation
    assert _bits_equal(m.unary_init(), Q)
    rq = (Q - Q.min()) / (Q - Q.min()).max()
    for k in range(2):
        assert _bits_equal(m.apply(k, Q), g[f"apply{k}"])
        assert _bits_equal(m.apply(k, Q, True), g[f"apply{k}_nonorm"])
        assert _bits_equal(m.apply_ord(k, rq), g[f"ord{k}"])
    lab = m.current_map(Q)
    assert _bits_equal(lab, g["map"])
    assert m.energy_true(lab) == float(g["e_true"])
    assert m.energy_ho(lab) == float(g["e_ho"])
    assert m.energy_lp(Q) == float(g["e_lp"])
    assert m.lr_qp_value(Q) == float(g["e_lrqp"])
    assert _bits_equal(m.qp(Q)[0], g["qp"])
    q100, it, en = m.qp(Q, 100)
    assert it == int(g["qp100_iters"])
    assert _bits_equal(q100, g["qp100"])
    assert _bits_equal(en, g["qp100_energies"])
    out, _ = m.lp(Q, prox_max_iter=4, fw_max_iter=4)
    assert _bits_equal(out, g["lp"])


def test_oracle_f64_filter_close_to_f32(oracle_mod):
    """The FP64 lattice oracle agrees with the FP32 filter to float accuracy."""
    W, H = 40, 30
    img = synth.make_image(W, H, 21, 5)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    lat = oracle_mod.OracleLattice(f)
    x = np.random.default_rng(1).random((W * H, 21)).astype(np.float32)
    a = lat.compute(x)
    b = lat.compute_f64(x.astype(np.float64))
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-5


@pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).reference_available()")
@pytest.mark.parametrize("W,H,seed", [(37, 23, 1), (64, 48, 2), (33, 31, 3)])
def test_oracle_matches_reference_live(W, H, seed, oracle_mod):
    """Fresh seeded cases against the compiled reference (this container only)."""
    O = oracle_mod
    img = synth.make_image(W, H, 21, seed)
    for f in (synth.gaussian_features(W, H, 3, 3),
              synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])):
        a, b = O.OracleLattice(f).export(), O.ReferenceLattice(f).export()
        assert a["M"] == b["M"]
        for k in ("offset", "rank", "bary", "nbr"):
            assert np.array_equal(a[k], b[k])
    mo = O.build_model(O.OracleModel, img)
    mr = O.build_model(O.ReferenceModel, img)
    Q = mr.unary_init()
    assert np.array_equal(mo.qp(Q)[0], mr.qp(Q)[0])
    assert np.array_equal(mo.lp(Q, prox_max_iter=3, fw_max_iter=3)[0],
                          mr.lp(Q, prox_max_iter=3, fw_max_iter=3)[0])


def test_apply_ord_rejects_out_of_range(oracle_mod):
    """apply_upper_minus_lower_ord throws "Value out of bounds" outside [0, 1]."""
    img = synth.make_image(16, 12, 21, 0)
    m = oracle_mod.build_model(oracle_mod.OracleModel, img)
    bad = np.full((16 * 12, 21), 0.5, np.float32)
    bad[3, 4] = 1.5
    with pytest.raises(RuntimeError, match="Value out of bounds"):
        m.apply_ord(0, bad)


def test_restricted_restatement_pinned_to_golden(oracle_mod):
    """The numpy restatement of the restricted ordered filter on the C
    oracle's lattice tables reproduces the reference's own outputs
    (tests/golden/make_restricted_golden.py) bit for bit: store call, reuse
    call, reuse call on a smaller pixel set; and the pairwise terms' Potts
    compatibility on top."""
    g = golden("restricted_32x24.npz")
    for name, d, w in (("g", 2, 3.0), ("b", 5, 5.0)):
        r = oracle_mod.RestrictedOrd(oracle_mod.OracleLattice(g[f"{name}_f"]).export(), d)
        o1 = r.compute(g["Q"][g["pI"]], g["pI"], g["Q"], True)
        o2 = r.compute(g["rQ2"], g["pI"], None, False)
        o3 = r.compute(g["rQ3"], g["pI3"], None, False)
        for o, key in ((o1, "out1"), (o2, "out2"), (o3, "out3")):
            assert np.array_equal(o, g[f"{name}_{key}"]), (name, key)
            k = 0 if name == "g" else 1
            assert np.array_equal(np.float32(-w) * o, g[f"m{k}_{key}"]), (name, key)


@pytest.mark.parametrize("name", golden_names("gradient_"))
def test_lattice_gradient_pinned_to_golden(name, oracle_mod):
    """The restated Permutohedral::gradient (src/permutohedral.cpp:1095-1178)
    against the reference's own values (tests/golden/make_gradient_golden.py)."""
    g = golden(name)
    df = oracle_mod.OracleLattice(g["f"]).gradient(g["a"], g["b"])
    assert _bits_equal(df, g["df"]), name


def test_kernel_gradient_pinned_to_golden(oracle_mod):
    """The restated DIAG_KERNEL kernelGradient for every NormalizationType (the
    Gaussian term with its scales set) and the bilateral term after
    setKernelParameters, bit for bit against the reference's own values
    (tests/golden/make_kernel_golden.py)."""
    g = golden("kernel_24x18_L5.npz")
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    fg = synth.gaussian_features(W, H, 3.0, 3.0)
    for t in range(4):
        r = oracle_mod.kernel_gradient_diag(fg, g["kg_kdiag"], t, g["b"], g[f"kg_1{t}_unary_init"], 3.0)
        assert _bits_equal(r, g[f"kg_1{t}"]), t
    img = synth.make_image(W, H, L, int(g["seed"]))
    fb = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    r = oracle_mod.kernel_gradient_diag(fb, g["kparam"], 3, g["b"], g["kparam_unary_init"], 5.0)
    assert _bits_equal(r, g["kparam_kgrad1"])


def test_weight_gradient_pinned_to_golden(oracle_mod):
    """The restated Potts weight gradient (PairwisePotential::gradient) of both
    terms of the example model, bit for bit against the reference's own
    values (tests/golden/make_gradient_golden.py)."""
    g = golden("mgrad_24x18_L5.npz")
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    img = synth.make_image(W, H, L, int(g["seed"]))
    feats = (synth.gaussian_features(W, H, 3.0, 3.0), synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"]))
    for k, f in enumerate(feats):
        r = oracle_mod.weight_gradient_potts(f, g["b"], g["Q"])
        assert _bits_equal(np.float32(r), g[f"wgrad{k}"][0]), k
    # DiagonalCompatibility terms (tests/golden/make_compat_golden.py)
    g = golden("compat_diag_24x18_L5.npz")
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    img = synth.make_image(W, H, L, int(g["seed"]))
    feats = (synth.gaussian_features(W, H, 3.0, 3.0), synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"]))
    for k, f in enumerate(feats):
        r = oracle_mod.weight_gradient_potts(f, g["b"], g["unary_init"], diagonal=True)
        assert _bits_equal(r, g[f"wgrad{k}"]), k


def test_per_pixel_energies_pinned_to_golden(oracle_mod):
    """unaryEnergy, pairwise_energy_true (each term and all) and max_rounding
    restated on the C oracle's model, bit for bit against the reference's own
    values (tests/golden/make_energy_golden.py)."""
    O = oracle_mod
    g = golden("energies_24x18.npz")
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    img = synth.make_image(W, H, L, int(g["seed"]))
    m = O.build_model(O.OracleModel, img)
    lab = g["lab"]
    assert _bits_equal(O.unary_energy(img["unary"], lab), g["unary_e"])
    assert _bits_equal(O.pairwise_energy_true(m, lab, 0), g["pw0"])
    assert _bits_equal(O.pairwise_energy_true(m, lab, 1), g["pw1"])
    assert _bits_equal(O.pairwise_energy_true(m, lab, -1), g["pw_all"])
    assert _bits_equal(O.max_rounding(g["Q"]), g["maxround"])
    # compute_LR_QP_value(Q, diag_dom): double sums in Eigen's packet order
    assert O.lr_qp_value_diag(m, img["unary"], g["Q"], g["dd"]) == float(g["lrqp_dd"])


@pytest.mark.parametrize("record,W,H,L", [("qp_320x240_seed1.json", 320, 240, 21),
                                          ("lp_640x480_seed2.json", 640, 480, 21)])
def test_unary_init_of_the_benchmark_images_pinned(record, W, H, L, oracle_mod):
    """The restated expAndNormalize (Eigen's packet exp over the aligned
    packets, libm expf over the tail, the packet-order sum) gives the very
    bytes the reference started its recorded full-size solves from."""
    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, record)) as f:
        rec = json.load(f)
    img = synth.make_image(W, H, L, rec["seed"])
    Q = oracle_mod.build_model(oracle_mod.OracleModel, img).unary_init()
    assert hashlib.sha256(Q.tobytes()).hexdigest() == rec["init_sha256"]
