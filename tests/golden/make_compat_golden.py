"""Golden vectors of the non-Potts label compatibilities
(include/labelcompatibility.h, src/labelcompatibility.cpp:79-129) from the
reference itself (oracle/_ref, built from its sources): a 24x18, 5-label
Gaussian + bilateral model whose terms carry a DiagonalCompatibility (case
"diag") or a MatrixCompatibility (case "matrix"), with the pairwise apply
(normalised and the unnormalised Potts twin), the ordered apply, the energies
fixed-iteration QP / short LP solves, parameters() and the compatibility and
kernel gradients.

Run: python tests/golden/make_compat_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

W, H, L, SEED = 24, 18, 5, 5
QP_ITERS = 20
LP_SMALL = dict(prox_max_iter=3, fw_max_iter=4)


def compat_params(case):
    """Term 0 (Gaussian) and term 1 (bilateral) parameters, as the reference's
    constructors take them (matrices column-major)."""
    rng = np.random.default_rng(len(case))
    if case == "diag":
        return [np.float32(-3.0) * (1 + rng.random(L, np.float32)),
                np.float32(-5.0) * (1 + rng.random(L, np.float32))]
    out = []
    for w in (3.0, 5.0):
        m = rng.random((L, L), np.float32)      # asymmetric: the constructor symmetrises
        np.fill_diagonal(m, -w)
        out.append(np.asfortranarray(m).T.reshape(-1).copy())   # column-major
    return out


def fixture(case):
    img = synth.make_image(W, H, L, SEED)
    kind = 1 if case == "diag" else 2
    p0, p1 = compat_params(case)
    m = O.ReferenceModel(W, H, L, img["unary"])
    m.add_gaussian_compat(3.0, 3.0, kind, p0)
    m.add_bilateral_compat(50.0, 50.0, 15.0, 15.0, 15.0, img["rgb"], kind, p1)
    out = dict(W=W, H=H, L=L, seed=SEED, kind=kind, p0=p0, p1=p1)
    Q = m.unary_init()
    out["unary_init"] = Q
    rq = (Q - Q.min()) / (Q - Q.min()).max()
    for k in range(2):
        out[f"apply{k}"] = m.apply(k, Q)
        out[f"apply{k}_nonorm"] = m.apply(k, Q, True)
        out[f"ord{k}"] = m.apply_ord(k, rq)
    rng = np.random.default_rng(9)
    b = rng.standard_normal((W * H, L)).astype(np.float32)
    out["b"] = b
    for k in range(2):
        out[f"params{k}"] = m.parameters(k)
        out[f"kgrad{k}"] = m.kernel_gradient(k, b, Q)
        out[f"wgrad{k}"] = m.weight_gradient(k, b, Q)
    lab = m.current_map(Q)
    out["map"] = lab
    out["e_true"] = np.float64(m.energy_true(lab))
    out["e_lp"] = np.float64(m.energy_lp(Q))
    out["e_lrqp"] = np.float64(m.lr_qp_value(Q))
    qf, it, en = m.qp(Q, QP_ITERS)
    out["qp"], out["qp_iters"], out["qp_energies"] = qf, np.int64(it), en
    out["lp"] = m.lp(Q, **LP_SMALL)[0]
    return out


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    for case in ("diag", "matrix"):
        g = fixture(case)
        np.savez_compressed(os.path.join(HERE, f"compat_{case}_{W}x{H}_L{L}.npz"), **g)
        print(case, "qp iters", int(g["qp_iters"]), "e_true", float(g["e_true"]),
              "lp range", float(g["lp"].min()), float(g["lp"].max()))


if __name__ == "__main__":
    main()
