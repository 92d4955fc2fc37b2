"""Golden vectors of addSuperPixel's mean-shift segmentation from the
UNMODIFIED reference (oracle/_ref/libdcrf_ref.so: EDISON's msImageProcessor
and DenseCRF2D::addSuperPixel compiled from the reference's sources).

For a few seeded synthetic images: the filtered L*u*v* image of
Filter(spatial, range, NO_SPEEDUP), the region labels of Segment(spatial,
range, min_region, NO_SPEEDUP), and the clique state a model holds after
addSuperPixel at two spatial radii one after the other (the second call's
weights start at an unaligned position of the reference's weight vector).

    python tests/golden/make_meanshift_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = [  # W, H, seed, (spatial, range, min_region) runs, clique weights
    (64, 48, 5, [(8, 8.0, 20), (16, 8.0, 20), (8, 4.0, 100)], (50.0, 1000.0)),
    (53, 41, 9, [(8, 8.0, 20), (4, 6.0, 10)], (3.0, 40.0)),
]


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    for W, H, seed, runs, (c, n) in CASES:
        img = synth.make_image(W, H, 21, seed)
        out = dict(W=W, H=H, seed=seed, rgb=img["rgb"], runs=np.array([[s, r, m] for s, r, m in runs]),
                   constant=c, normaliser=n)
        for k, (s, r, m) in enumerate(runs):
            out[f"filtered{k}"] = O.ref_meanshift_filter(img["rgb"], W, H, s, r)
            out[f"labels{k}"], out[f"count{k}"] = O.ref_meanshift_segment(img["rgb"], W, H, s, r, m)
        ref = O.build_model(O.ReferenceModel, img)
        for s, r, m in runs[:2]:
            ref.add_superpixel(img["rgb"], s, int(r), m, c, n)
        out["cl_off"], out["cl_idx"], out["cl_exp"], out["cl_const"] = ref.get_cliques()
        np.savez_compressed(os.path.join(HERE, f"meanshift_{W}x{H}.npz"), **out)
        print(W, H, [int(out[f"count{k}"]) for k in range(len(runs))], "cliques", len(out["cl_exp"]))


if __name__ == "__main__":
    main()
