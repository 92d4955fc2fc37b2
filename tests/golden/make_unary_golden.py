"""Golden vectors of LogisticUnaryEnergy (include/unary.h:48-57,
src/unary.cpp:47-70) from the reference itself (oracle/_ref, built from its
sources): a 24x18, 5-label model whose unary is W f with W [L][F] and
per-pixel features f [N][F] (colour, position, a constant and noise), with
get(), unary_init, gradient(b) and a fixed-iteration QP.

Run: python tests/golden/make_unary_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

W, H, L, F, SEED = 24, 18, 5, 8, 6


def features(img):
    rng = np.random.default_rng(SEED)
    jj, ii = np.mgrid[0:H, 0:W]
    rgb = img["rgb"].reshape(-1, 3).astype(np.float32) / np.float32(255)
    cols = [rgb, (ii.reshape(-1, 1) / W).astype(np.float32), (jj.reshape(-1, 1) / H).astype(np.float32),
            np.ones((W * H, 1), np.float32), rng.standard_normal((W * H, F - 6)).astype(np.float32)]
    return np.ascontiguousarray(np.concatenate(cols, 1), np.float32)


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    img = synth.make_image(W, H, L, SEED)
    f = features(img)
    rng = np.random.default_rng(SEED + 1)
    w = (rng.standard_normal((L, F)) * 2).astype(np.float32)
    m = O.build_model(O.ReferenceModel, img)
    m.set_unary_logistic(w, f)
    b = rng.standard_normal((W * H, L)).astype(np.float32)
    Q = m.unary_init()
    out = dict(W=W, H=H, L=L, F=F, seed=SEED, w=w, f=f, b=b, unary=m.unary_get(), unary_init=Q,
               ugrad=m.unary_gradient(b, F))
    qf, it, en = m.qp(Q, 20)
    out["qp"], out["qp_iters"], out["qp_energies"] = qf, np.int64(it), en
    np.savez_compressed(os.path.join(HERE, f"unary_logistic_{W}x{H}_L{L}.npz"), **out)
    print("qp iters", it, "grad max", float(np.abs(out["ugrad"]).max()))


if __name__ == "__main__":
    main()
