"""Generates the golden vectors in this directory from the UNMODIFIED reference.

The reference ships no tests or expected values, so its outputs on seeded
synthetic inputs are the golden vectors.  This script needs
``oracle/_ref/libdcrf_ref.so`` (``make -C oracle ref``, which compiles the
reference's own sources); the fixtures it writes are committed so that the
tests can check against them where the reference tree is absent.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

LATTICE_CASES = [(23, 17, 11), (32, 24, 12), (41, 9, 13)]   # N % 4 = 3, 0, 1
MODEL_CASES = [(24, 18, 21), (27, 15, 22)]                  # N % 4 = 0, 1
HO_CASE = (40, 30, 23)
LP_SMALL = dict(prox_max_iter=4, fw_max_iter=4)


def lattice_fixture(W, H, seed):
    img = synth.make_image(W, H, 21, seed)
    rng = np.random.default_rng(seed)
    out = dict(W=W, H=H, rgb=img["rgb"])
    x = rng.random((W * H, 21)).astype(np.float32)
    x1 = rng.random((W * H, 1)).astype(np.float32)
    out["x"], out["x1"] = x, x1
    for name, f in (("g", synth.gaussian_features(W, H, 3.0, 3.0)),
                    ("b", synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"]))):
        lat = O.ReferenceLattice(f)
        ex = lat.export()
        for k in ("offset", "rank", "bary", "nbr"):
            out[f"{name}_{k}"] = ex[k]
        out[f"{name}_M"] = np.int64(ex["M"])
        out[f"{name}_f"] = f
        out[f"{name}_compute"] = lat.compute(x)
        out[f"{name}_compute_rev"] = lat.compute(x, True)
        out[f"{name}_compute_l1"] = lat.compute(x1)
        out[f"{name}_ord"] = lat.compute_ord(x)
    return out


def model_fixture(W, H, seed, cliques=None):
    img = synth.make_image(W, H, 21, seed)
    m = O.build_model(O.ReferenceModel, img)
    out = dict(W=W, H=H, rgb=img["rgb"], unary=img["unary"])
    if cliques is not None:
        off, idx, ex, cs = cliques
        m.set_cliques(off, idx, ex, cs)
        out.update(cl_off=off, cl_idx=idx, cl_exp=ex, cl_const=cs)
    Q = m.unary_init()
    out["unary_init"] = Q
    rq = (Q - Q.min()) / (Q - Q.min()).max()
    for k in range(2):
        out[f"apply{k}"] = m.apply(k, Q)
        out[f"apply{k}_nonorm"] = m.apply(k, Q, True)
        out[f"ord{k}"] = m.apply_ord(k, rq)
    lab = m.current_map(Q)
    out["map"] = lab
    out["e_true"] = np.float64(m.energy_true(lab))
    out["e_ho"] = np.float64(m.energy_ho(lab))
    out["e_lp"] = np.float64(m.energy_lp(Q))
    out["e_lrqp"] = np.float64(m.lr_qp_value(Q))
    out["qp"] = m.qp(Q)[0]
    qf, it, en = m.qp(Q, 100)
    out["qp100"], out["qp100_iters"], out["qp100_energies"] = qf, np.int64(it), en
    out["lp"] = m.lp(Q, **LP_SMALL)[0]
    return out


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    for W, H, s in LATTICE_CASES:
        np.savez_compressed(os.path.join(HERE, f"lattice_{W}x{H}.npz"), **lattice_fixture(W, H, s))
    for W, H, s in MODEL_CASES:
        np.savez_compressed(os.path.join(HERE, f"model_{W}x{H}.npz"), **model_fixture(W, H, s))
    # Higher-order cliques from the reference's own mean-shift (spatial 8 and
    # 16, range 8, min region 20) with the CLI's default weights 50 / 1000 so
    # the clique terms are non-zero (src/example_inference.cpp:48, 120).
    W, H, s = HO_CASE
    img = synth.make_image(W, H, 21, s)
    ref = O.build_model(O.ReferenceModel, img)
    for sr in (8, 16):
        ref.add_superpixel(img["rgb"], sr, 8, 20, 50.0, 1000.0)
    cl = ref.get_cliques()
    np.savez_compressed(os.path.join(HERE, f"model_ho_{W}x{H}.npz"), **model_fixture(W, H, s, cl))
    print("written:", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
