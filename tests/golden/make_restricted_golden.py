"""Golden vectors of the restricted ordered filter
(Permutohedral::compute_upper_minus_lower_ord_restricted,
src/permutohedral.cpp:702-900, and
PairwisePotential::apply_upper_minus_lower_ord_restricted,
src/pairwise.cpp:229-240) from the reference itself (oracle/_ref, built from
its sources).  For a Gaussian (d = 2) and a bilateral (d = 5) lattice of a
32x24 image, three calls in a row: a store call on a pixel subset pI, a
reuse call with new values at pI, and a reuse call on a smaller subset
(whose blur still runs over the first call's vertex set).  The same three
calls through both pairwise terms of the example model.

Run: python tests/golden/make_restricted_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

W, H, L, SEED = 32, 24, 21, 8


def calls(rng, N):
    Q = rng.random((N, L)).astype(np.float32)
    Q[::9] = np.float32(0.5)  # exact bin boundaries
    pI = np.sort(rng.choice(N, N // 5, replace=False)).astype(np.int32)
    rQ2 = rng.random((len(pI), L)).astype(np.float32)
    sub = np.sort(rng.choice(len(pI), len(pI) // 2, replace=False))
    return Q, pI, rQ2, pI[sub].astype(np.int32), rQ2[sub]


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    img = synth.make_image(W, H, L, SEED)
    rng = np.random.default_rng(SEED)
    Q, pI, rQ2, pI3, rQ3 = calls(rng, W * H)
    out = dict(W=W, H=H, L=L, seed=SEED, Q=Q, pI=pI, rQ2=rQ2, pI3=pI3, rQ3=rQ3)
    for name, f in (("g", synth.gaussian_features(W, H, 3.0, 3.0)),
                    ("b", synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"]))):
        lat = O.ReferenceLattice(f)
        out[f"{name}_f"] = f
        out[f"{name}_out1"] = lat.compute_ord_restricted(Q[pI], pI, Q, True)
        out[f"{name}_out2"] = lat.compute_ord_restricted(rQ2, pI, None, False)
        out[f"{name}_out3"] = lat.compute_ord_restricted(rQ3, pI3, None, False)
    m = O.build_model(O.ReferenceModel, img)
    for k in range(2):
        out[f"m{k}_out1"] = m.apply_ord_restricted(k, Q[pI], pI, Q, True)
        out[f"m{k}_out2"] = m.apply_ord_restricted(k, rQ2, pI, None, False)
        out[f"m{k}_out3"] = m.apply_ord_restricted(k, rQ3, pI3, None, False)
    np.savez_compressed(os.path.join(HERE, f"restricted_{W}x{H}.npz"), **out)
    print({k: float(np.abs(v).max()) for k, v in out.items() if "out" in k})


if __name__ == "__main__":
    main()
