"""Batched QP over images of different sizes (dcrf_batch_*) against the
single-image solver, image by image.

The batch runs every image's own single-image solve (the first solve for an
output buffer one image after the other, later ones from several host
threads at once): outputs, step counts and energies must be identical to
single-image solves, bit for bit.
"""
import numpy as np
import pytest

from densecrf_ho_b200 import DCRFError, DenseCRF2D, DenseCRF2DBatch, synth

pytestmark = pytest.mark.gpu

SIZES = [(37, 29), (64, 48), (50, 50), (23, 41), (96, 31)]


def _images(sizes, seed0=11):
    return [synth.make_image(w, h, 21, seed0 + i) for i, (w, h) in enumerate(sizes)]


def _batch(sizes, imgs):
    b = DenseCRF2DBatch(sizes, 21)
    b.setUnaryEnergy(np.concatenate([im["unary"] for im in imgs]))
    b.addPairwiseGaussian(3.0, 3.0, 3.0)
    b.addPairwiseBilateral(50.0, 50.0, 15.0, 15.0, 15.0, np.concatenate([im["rgb"] for im in imgs]), 5.0)
    return b


def _single(w, h, im):
    m = DenseCRF2D(w, h, 21)
    m.setUnaryEnergy(im["unary"])
    m.addPairwiseGaussian(3.0, 3.0, 3.0)
    m.addPairwiseBilateral(50.0, 50.0, 15.0, 15.0, 15.0, im["rgb"], 5.0)
    return m


@pytest.mark.parametrize("max_iter", [0, 7])
def test_batch_qp_equals_single_solves(max_iter):
    imgs = _images(SIZES)
    b = _batch(SIZES, imgs)
    q0 = b.unary_init()
    out, st = b.qp_inference_super_pixels_non_convex(q0, max_iter=max_iter, stats=True)
    for i, ((w, h), im) in enumerate(zip(SIZES, imgs)):
        m = _single(w, h, im)
        qi = m.unary_init()
        assert np.array_equal(b.split(q0)[i], qi)
        o, s = m.qp_inference_super_pixels_non_convex(qi, max_iter=max_iter, stats=True)
        assert np.array_equal(b.split(out)[i], o), i
        assert st[i].iterations == s.iterations
        assert st[i].energy == s.energy


def test_batch_concurrent_solves_equal_single_solves():
    """Twelve images: the first solve runs image after image, the second (same
    output buffer) from several host threads; a weight change sends the next
    solve back to one thread, after which the threads take over again.
    Every solve equals the single-image solves."""
    sizes = [(40 + 7 * i, 30 + 5 * (i % 4)) for i in range(12)]
    imgs = _images(sizes, 70)
    b = _batch(sizes, imgs)
    q0 = b.unary_init()
    singles = [_single(w, h, im) for (w, h), im in zip(sizes, imgs)]
    want = [m.qp_inference_super_pixels_non_convex(b.split(q0)[i]) for i, m in enumerate(singles)]
    for _ in range(3):
        out = b.qp_inference_super_pixels_non_convex(q0)
        for i in range(len(sizes)):
            assert np.array_equal(b.split(out)[i], want[i]), i
    b.set_weight(1, 9.0)
    for m in singles:
        m.pairwise_set_parameters(1, np.array([9.0], np.float32))
    want = [m.qp_inference_super_pixels_non_convex(b.split(q0)[i]) for i, m in enumerate(singles)]
    for _ in range(2):
        out = b.qp_inference_super_pixels_non_convex(q0)
        for i in range(len(sizes)):
            assert np.array_equal(b.split(out)[i], want[i]), i


def test_batch_qp_repeat_is_deterministic():
    """Repeated solves (the later ones concurrent) give the same output."""
    imgs = _images(SIZES[:3], 40)
    b = _batch(SIZES[:3], imgs)
    q0 = b.unary_init()
    a = b.qp_inference_super_pixels_non_convex(q0, max_iter=5)
    c = b.qp_inference_super_pixels_non_convex(q0, max_iter=5)
    d = b.qp_inference_super_pixels_non_convex(q0)
    e = b.qp_inference_super_pixels_non_convex(q0)
    assert np.array_equal(a, c)
    assert np.array_equal(d, e)


def test_batch_single_image_and_errors():
    (w, h), = [(41, 33)]
    im = synth.make_image(w, h, 21, 3)
    b = _batch([(w, h)], [im])
    q0 = b.unary_init()
    m = _single(w, h, im)
    assert np.array_equal(b.qp_inference_super_pixels_non_convex(q0), m.qp_inference_super_pixels_non_convex(q0))
    with pytest.raises(DCRFError) as e:
        DenseCRF2DBatch([(10, 0)], 21)
    assert e.value.code == 1
    nb = DenseCRF2DBatch([(8, 8), (4, 4)], 21)
    with pytest.raises(DCRFError) as e:
        nb.qp_inference_super_pixels_non_convex(np.zeros((80, 21), np.float32))
    assert e.value.code == 4


def test_batch_pairwise_apply_equals_single_applies():
    """PairwisePotential::apply over the concatenated lattice of each term:
    every image's rows equal its own single-image apply, bit for bit."""
    imgs = _images(SIZES, 40)
    b = _batch(SIZES, imgs)
    x = np.random.default_rng(4).random((b.N, 21)).astype(np.float32)
    for k in range(2):
        out = b.pairwise_apply(k, x)
        Ms = 0
        for i, ((w, h), im) in enumerate(zip(SIZES, imgs)):
            m = _single(w, h, im)
            assert np.array_equal(b.split(out)[i], m.pairwise_apply(k, b.split(x)[i])), (k, i)
            Ms += m.lattice_size(k)
        assert b.lattice_size(k) == Ms


@pytest.mark.parametrize("kind", [0, 2, 3, 4, 5])
def test_batch_splat_forms_equal_single_solves(kind):
    """The batched QP (live-image compaction) and the batched apply with each
    splat form pinned on both terms' concatenated lattices: outputs, steps
    and energies equal the single-image solves and applies, bit for bit."""
    imgs = _images(SIZES, 60)
    b = _batch(SIZES, imgs)
    for k in range(2):
        b.set_filter_shape(k, (4, 256, 128, kind))
    q0 = b.unary_init()
    out, st = b.qp_inference_super_pixels_non_convex(q0, max_iter=9, stats=True)
    x = np.random.default_rng(9).random((b.N, 21)).astype(np.float32)
    applied = [b.pairwise_apply(k, x) for k in range(2)]
    for i, ((w, h), im) in enumerate(zip(SIZES, imgs)):
        m = _single(w, h, im)
        o, s = m.qp_inference_super_pixels_non_convex(b.split(q0)[i], max_iter=9, stats=True)
        assert np.array_equal(b.split(out)[i], o), i
        assert st[i].iterations == s.iterations and st[i].energy == s.energy
        for k in range(2):
            assert np.array_equal(b.split(applied[k])[i], m.pairwise_apply(k, b.split(x)[i])), (k, i)
    assert b.filter_shape(0) == (4, 256, 128, kind)
