"""The host half of addSuperPixel's mean-shift segmentation (8-connected
labelling, transitive closure, pruning: dcrf_meanshift_regions) on the
reference's own filtered images, against the reference's region labels
(tests/golden/make_meanshift_golden.py).  Needs no GPU."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, golden_names
from densecrf_ho_b200 import meanshift_regions, synth

CASES = golden_names("meanshift_")


@pytest.mark.parametrize("name", CASES)
def test_regions_from_reference_filtered_images(name):
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    for k, (s, r, m) in enumerate(g["runs"]):
        lab, n = meanshift_regions(g[f"filtered{k}"], W, H, float(r), int(m))
        assert n == int(g[f"count{k}"]), (name, k)
        assert np.array_equal(lab, g[f"labels{k}"]), (name, k)


def test_regions_of_the_benchmark_image_scale_8(oracle_mod):
    """The config-3 segmentation at spatial radius 8 from the reference's
    filtered 640x480 image: the region map recorded from the reference's
    addSuperPixel (tests/golden/cliques_640x480_seed2.npz)."""
    if not oracle_mod.reference_available():
        pytest.skip("needs the reference's filter (oracle/_ref)")
    z = np.load(os.path.join(GOLDEN, "cliques_640x480_seed2.npz"))
    W, H = int(z["W"]), int(z["H"])
    img = synth.make_image(W, H, 21, 2)
    f = oracle_mod.ref_meanshift_filter(img["rgb"], W, H, 8, 8.0)
    lab, n = meanshift_regions(f, W, H, 8.0, 100)
    assert n == int(z["counts"][0])
    assert np.array_equal(lab, z["regions"][0].astype(np.int32))
