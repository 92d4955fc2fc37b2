"""Golden vectors of PairwisePotential's exact and divide-and-conquer filters
(apply_bf, apply_upper_minus_lower_bf, apply_upper_minus_lower_bf_ord,
apply_upper_minus_lower_dc; src/pairwise.cpp:241-380,
src/permutohedral.cpp:902-997) from the reference itself (oracle/_ref, built
from its sources).

* "potts": the 23x17 (N = 391, so the halvings of the divide-and-conquer
  filter are odd and even) 3-label Gaussian + bilateral example model, Q on
  a 1/8 grid so that the ordered variant meets ties, ind = the positions
  sorted by decreasing Q (stable).
* "diag": the same terms with DiagonalCompatibility, for the compatibility
  after the filter and the Potts twin (nonorm).
* "feat8": one term on random 8-dimensional features (the two-packet order
  of the squared distance), 12x10, 2 labels;
* "feat3" on 5x4 (N = 20: the divide-and-conquer filter is one block of
  pairs) and on 31x1 (N = 31: one odd halving into two blocks sharing the
  middle position);
* "dims": apply_bf on 8x5 random features of every dimension d = 1..16 (the
  squared distance's packet order for each), 2 labels.

Run: python tests/golden/make_bruteforce_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

SEED = 11


def inputs(rng, N, L):
    Q = (rng.integers(0, 9, (N, L)) / 8.0).astype(np.float32)
    ind = np.argsort(-Q, axis=0, kind="stable").astype(np.int32)
    return Q, ind


def run_terms(m, nterms, Q, ind, out, nonorm=False):
    sfx = "_nonorm" if nonorm else ""
    for k in range(nterms):
        out[f"bf{k}{sfx}"] = m.apply_bf(k, Q, nonorm)
        out[f"bfs{k}{sfx}"] = m.apply_upper_minus_lower_bf(k, ind, nonorm)
        out[f"bfo{k}{sfx}"] = m.apply_upper_minus_lower_bf_ord(k, ind, Q, nonorm)
        out[f"dc{k}{sfx}"] = m.apply_upper_minus_lower_dc(k, ind, nonorm)


def image_case(case, W, H, L):
    img = synth.make_image(W, H, L, SEED)
    rng = np.random.default_rng(SEED)
    Q, ind = inputs(rng, W * H, L)
    out = dict(W=W, H=H, L=L, seed=SEED, Q=Q, ind=ind)
    if case == "potts":
        m = O.build_model(O.ReferenceModel, img)
    else:
        p0 = np.float32(-3.0) * (1 + rng.random(L, np.float32))
        p1 = np.float32(-5.0) * (1 + rng.random(L, np.float32))
        out["p0"], out["p1"] = p0, p1
        m = O.ReferenceModel(W, H, L, img["unary"])
        m.add_gaussian_compat(3.0, 3.0, 1, p0)
        m.add_bilateral_compat(50.0, 50.0, 15.0, 15.0, 15.0, img["rgb"], 1, p1)
    run_terms(m, 2, Q, ind, out)
    if case == "diag":
        run_terms(m, 2, Q, ind, out, nonorm=True)
    return out


def feature_case(W, H, L, d):
    rng = np.random.default_rng(SEED + d)
    N = W * H
    f = (rng.random((N, d)) * 2.0).astype(np.float32)
    U = rng.random((N, L)).astype(np.float32)
    Q, ind = inputs(rng, N, L)
    m = O.ReferenceModel(W, H, L, U)
    m.add_features(f, 2.5)
    out = dict(W=W, H=H, L=L, f=f, U=U, w=np.float32(2.5), Q=Q, ind=ind)
    run_terms(m, 1, Q, ind, out)
    return out


def dims_case(W=8, H=5, L=2):
    rng = np.random.default_rng(SEED + 100)
    N = W * H
    U = rng.random((N, L)).astype(np.float32)
    Q = rng.random((N, L)).astype(np.float32)
    out = dict(W=W, H=H, L=L, U=U, Q=Q)
    for d in range(1, 17):
        f = (rng.random((N, d)) * 1.5).astype(np.float32)
        m = O.ReferenceModel(W, H, L, U)
        m.add_features(f, 2.0)
        out[f"f{d}"] = f
        out[f"bf_d{d}"] = m.apply_bf(0, Q)
    return out


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    cases = {"potts_23x17_L3": image_case("potts", 23, 17, 3),
             "diag_23x17_L3": image_case("diag", 23, 17, 3),
             "feat8_12x10_L2": feature_case(12, 10, 2, 8),
             "feat3_5x4_L2": feature_case(5, 4, 2, 3),
             "feat3_31x1_L3": feature_case(31, 1, 3, 3)}
    np.savez_compressed(os.path.join(HERE, "bfdims_8x5_L2.npz"), **dims_case())
    for name, out in cases.items():
        np.savez_compressed(os.path.join(HERE, f"bruteforce_{name}.npz"), **out)
        print(name, {k: float(np.abs(v).max()) for k, v in out.items() if k[:2] in ("bf", "dc")})


if __name__ == "__main__":
    main()
