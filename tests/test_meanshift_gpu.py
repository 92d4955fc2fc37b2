"""addSuperPixel (src/densecrf.cpp:193-251) with the engine's own mean-shift
segmentation: the GPU mode search against EDISON's filtered image bit for
bit, the regions against EDISON's labels, and the clique state (pixel lists,
weights, constants) against the reference model's after addSuperPixel --
on the golden images of tests/golden/make_meanshift_golden.py and on the
640x480 benchmark image at the three radii of the benchmark's cliques."""
import ctypes as C
import os
import sys
import time

import numpy as np
import pytest

from conftest import GOLDEN, golden, golden_names
from densecrf_ho_b200 import DenseCRF2D, _lib, meanshift_segment, synth

pytestmark = pytest.mark.gpu

CASES = golden_names("meanshift_")


def _filter(rgb, W, H, s, r):
    out = np.zeros((W * H, 3), np.float32)
    _lib.check(_lib.lib().dcrf_meanshift_filter(np.ascontiguousarray(rgb, np.uint8).ctypes.data_as(C.c_void_p),
                                                W, H, int(s), C.c_float(r), out.ctypes.data_as(C.c_void_p)))
    return out


@pytest.mark.parametrize("name", CASES)
def test_filter_and_regions_vs_reference(name):
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    for k, (s, r, m) in enumerate(g["runs"]):
        f = _filter(g["rgb"], W, H, s, r)
        assert np.array_equal(f, g[f"filtered{k}"]), (name, k, int((f != g[f"filtered{k}"]).sum()))
        lab, n = meanshift_segment(g["rgb"], W, H, int(s), float(r), int(m))
        assert n == int(g[f"count{k}"]) and np.array_equal(lab, g[f"labels{k}"]), (name, k)


@pytest.mark.parametrize("name", CASES)
def test_add_superpixel_cliques_vs_reference(name):
    g = golden(name)
    W, H = int(g["W"]), int(g["H"])
    m = DenseCRF2D(W, H, 21)
    for s, r, mr in g["runs"][:2]:
        m.addSuperPixel(g["rgb"], int(s), int(r), int(mr), float(g["constant"]), float(g["normaliser"]))
    off, idx, ew, cs = m.getCliques()
    assert np.array_equal(off, g["cl_off"]) and np.array_equal(idx, g["cl_idx"])
    assert np.array_equal(ew, g["cl_exp"]) and np.array_equal(cs, g["cl_const"])


def test_benchmark_cliques_640x480_three_radii():
    """The config-3 cliques: addSuperPixel at spatial radii 8, 16, 32, range
    8, min region 100, weights (50, 1000), on the 640x480 benchmark image --
    the same pixel lists and weights the reference's addSuperPixel produced
    (tests/golden/cliques_640x480_seed2.npz)."""
    sys.path.insert(0, GOLDEN)
    from make_config_goldens import load_cliques
    z = np.load(os.path.join(GOLDEN, "cliques_640x480_seed2.npz"))
    W, H = int(z["W"]), int(z["H"])
    img = synth.make_image(W, H, 21, 2)
    m = DenseCRF2D(W, H, 21)
    t = time.perf_counter()
    counts = [m.addSuperPixel(img["rgb"], int(s), 8, 100, 50.0, 1000.0) for s in z["scales"]]
    print(f"three mean-shift segmentations + cliques at 640x480: {time.perf_counter() - t:.3f} s")
    assert counts == [int(c) for c in z["counts"]]
    off, idx, ew, cs = m.getCliques()
    roff, ridx, rew, rcs = load_cliques(50.0, 1000.0)
    assert np.array_equal(off, roff) and np.array_equal(idx, ridx)
    assert np.array_equal(ew, rew) and np.array_equal(cs, rcs)
