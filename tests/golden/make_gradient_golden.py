"""Golden vectors of Permutohedral::gradient (src/permutohedral.cpp:1095-1178),
computed by the reference itself (oracle/_ref, built from its sources):
for each case the features f, the two inputs a, b and df = d(a^T K b)/df.
Run: python tests/golden/make_gradient_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cases():
    img = synth.make_image(23, 17, 21, 11)
    yield "gauss_23x17_L3", synth.gaussian_features(23, 17, 3, 3), 3
    yield "bilat_23x17_L21", synth.bilateral_features(23, 17, 50, 50, 15, 15, 15, img["rgb"]), 21
    rng = np.random.default_rng(4)
    yield "rand_d3_N301_L1", (rng.random((301, 3)) * 5).astype(np.float32), 1
    yield "rand_d1_N64_L2", (rng.random((64, 1)) * 9).astype(np.float32), 2


def main():
    for name, f, L in cases():
        rng = np.random.default_rng(len(name))
        a = rng.standard_normal((f.shape[0], L)).astype(np.float32)
        b = rng.standard_normal((f.shape[0], L)).astype(np.float32)
        df = O.ReferenceLattice(f).gradient(a, b)
        np.savez_compressed(os.path.join(HERE, f"gradient_{name}.npz"), f=f, a=a, b=b, df=df)
        print(name, f.shape, L, float(np.abs(df).max()))


if __name__ == "__main__":
    main()


def model_case():
    """pairwise_[k]->kernelGradient(b, Q) and ->gradient(b, Q) of the example's
    Gaussian + bilateral model, from the reference itself."""
    img = synth.make_image(24, 18, 5, 3)
    m = O.build_model(O.ReferenceModel, img)
    rng = np.random.default_rng(0)
    b = rng.standard_normal((24 * 18, 5)).astype(np.float32)
    Q = rng.random((24 * 18, 5)).astype(np.float32)
    out = dict(W=24, H=18, L=5, seed=3, b=b, Q=Q)
    for k in range(2):
        out[f"kgrad{k}"] = m.kernel_gradient(k, b, Q)
        out[f"wgrad{k}"] = m.weight_gradient(k, b, Q)
    np.savez_compressed(os.path.join(HERE, "mgrad_24x18_L5.npz"), **out)
    print("model", {k: v for k, v in out.items() if "grad" in k})


if __name__ == "__main__":
    model_case()
