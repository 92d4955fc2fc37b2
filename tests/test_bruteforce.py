"""PairwisePotential's exact and divide-and-conquer filters (apply_bf,
apply_upper_minus_lower_bf / _bf_ord / _dc; src/pairwise.cpp:241-380,
src/permutohedral.cpp:902-997).

CPU: the numpy restatement in oracle/oracle.py pinned bit for bit to the
reference's own outputs (tests/golden/make_bruteforce_golden.py).
GPU: the CUDA kernels through the C ABI against the same fixtures, and on a
larger image against the restatement.  The kernels carry every sum in the
reference's order: k = exp(-|f_c - f_b|^2) in double (CUDA's exp where the
reference has glibc's), accumulated into float one term at a time.  A one-ulp
difference of the two exps can flip a float rounding, so the bound is: at
least 99 % of the values bit-equal, all within 1e-5 of the largest.
"""
import numpy as np
import pytest

from conftest import golden, golden_names
from densecrf_ho_b200 import DenseCRF2D, synth

NAMES = golden_names("bruteforce_")


def _case_inputs(g):
    """The terms of a fixture: (features, compatibility kind, params)."""
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    if "f" in g:
        return [(g["f"], 0, float(g["w"]))]
    img = synth.make_image(W, H, L, int(g["seed"]))
    fg = synth.gaussian_features(W, H, 3.0, 3.0)
    fb = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    if "p0" in g:
        return [(fg, 1, g["p0"]), (fb, 1, g["p1"])]
    return [(fg, 0, 3.0), (fb, 0, 5.0)]


@pytest.mark.parametrize("name", NAMES)
def test_restatement_pinned_to_reference(name, oracle_mod):
    O = oracle_mod
    g = golden(name)
    Q, ind = g["Q"], g["ind"]
    for k, (f, kind, p) in enumerate(_case_inputs(g)):
        variants = [("", kind, p)]
        if f"bf{k}_nonorm" in g:  # the Potts twin with parameters()(0)
            variants.append(("_nonorm", 0, float(np.asarray(p).reshape(-1)[0])))
        for sfx, kd, pp in variants:
            assert np.array_equal(O.compat_apply(O.bf_apply(f, Q), kd, pp), g[f"bf{k}{sfx}"]), (name, k, sfx)
            assert np.array_equal(O.compat_apply(O.bf_sorted(f, ind), kd, pp), g[f"bfs{k}{sfx}"]), (name, k, sfx)
            assert np.array_equal(O.compat_apply(O.bf_sorted(f, ind, Q), kd, pp), g[f"bfo{k}{sfx}"]), (name, k, sfx)
            assert np.array_equal(O.compat_apply(O.dc_sorted(f, ind), kd, pp), g[f"dc{k}{sfx}"]), (name, k, sfx)


def test_restatement_every_dimension_pinned():
    """apply_bf for d = 1..16 (tests/golden/bfdims_8x5_L2.npz): the squared
    distance's packet order of every dimension, bit for bit."""
    from oracle import oracle as O
    g = golden("bfdims_8x5_L2.npz")
    for d in range(1, 17):
        assert np.array_equal(O.compat_apply(O.bf_apply(g[f"f{d}"], g["Q"]), 0, 2.0), g[f"bf_d{d}"]), d


def test_squared_norm_order_matters():
    """The packet order of the squared distance is not the left-to-right sum:
    on these values the two differ, and the reference's is the packet one."""
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    diff = rng.standard_normal((2000, 5)).astype(np.float32)
    seq = diff[:, 0] * diff[:, 0]
    for i in range(1, 5):
        seq = (seq + diff[:, i] * diff[:, i]).astype(np.float32)
    assert not np.array_equal(O.sqnorm_eigen(diff), seq)


def _close(a, ref):
    a, ref = np.asarray(a), np.asarray(ref)
    eq = np.mean(a.view(np.int32) == ref.view(np.int32))
    err = np.abs(a - ref).max()
    return eq >= 0.99 and err <= 1e-5 * max(np.abs(ref).max(), 1.0), (eq, err)


def _gpu_model(g, terms):
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    m = DenseCRF2D(W, H, L)
    if "U" in g:
        m.setUnaryEnergy(g["U"])
    for k, (f, kind, p) in enumerate(terms):
        if kind == 0:
            m.addPairwiseEnergy(f, float(p))
        else:
            m.addPairwiseEnergy(f, 1.0)
            m.setCompatibility(k, diagonal=p)
    return m


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_against_reference_golden(name):
    g = golden(name)
    terms = _case_inputs(g)
    m = _gpu_model(g, terms)
    Q, ind = g["Q"], g["ind"]
    for k in range(len(terms)):
        for sfx in ("", "_nonorm"):
            if f"bf{k}{sfx}" not in g:
                continue
            nn = sfx != ""
            for key, got in (("bf", m.pairwise_apply_bf(k, Q, nonorm=nn)),
                             ("bfs", m.pairwise_apply_upper_minus_lower_bf(k, ind, nonorm=nn)),
                             ("bfo", m.pairwise_apply_upper_minus_lower_bf_ord(k, ind, Q, nonorm=nn)),
                             ("dc", m.pairwise_apply_upper_minus_lower_dc(k, ind, nonorm=nn))):
                ok, info = _close(got, g[f"{key}{k}{sfx}"])
                assert ok, (name, key, k, sfx, info)


@pytest.mark.gpu
def test_gpu_dc_and_bf_larger_image(oracle_mod):
    """61x47 (N = 2867: a deeper recursion with odd and even halvings), 2
    labels, the bilateral term, against the restatement; ind with repeated
    pixels (the reference takes any ind)."""
    O = oracle_mod
    W, H, L = 61, 47, 2
    N = W * H
    img = synth.make_image(W, H, L, 4)
    f = synth.bilateral_features(W, H, 50, 50, 15, 15, 15, img["rgb"])
    rng = np.random.default_rng(4)
    Q = rng.random((N, L)).astype(np.float32)
    ind = np.argsort(-Q, axis=0, kind="stable").astype(np.int32)
    ind[100:110, 1] = ind[0, 1]
    m = DenseCRF2D(W, H, L)
    m.addPairwiseEnergy(f, 5.0)
    ok, info = _close(m.pairwise_apply_upper_minus_lower_dc(0, ind), O.compat_apply(O.dc_sorted(f, ind), 0, 5.0))
    assert ok, info
    ok, info = _close(m.pairwise_apply_upper_minus_lower_bf(0, ind), O.compat_apply(O.bf_sorted(f, ind), 0, 5.0))
    assert ok, info
    ok, info = _close(m.pairwise_apply_bf(0, Q), O.compat_apply(O.bf_apply(f, Q), 0, 5.0))
    assert ok, info


@pytest.mark.gpu
def test_gpu_sorted_filters_reject_bad_ind():
    from densecrf_ho_b200 import DCRFError
    m = DenseCRF2D(8, 6, 2)
    m.addPairwiseGaussian(3.0, 3.0, 1.0)
    ind = np.zeros((48, 2), np.int32)
    ind[5, 1] = 48
    with pytest.raises(DCRFError):
        m.pairwise_apply_upper_minus_lower_dc(0, ind)
    with pytest.raises(DCRFError):
        m.pairwise_apply_upper_minus_lower_bf(0, ind)


@pytest.mark.gpu
def test_gpu_apply_bf_shared_exp_on_large_images(oracle_mod):
    """256x200 x 21 labels: apply_bf's grid is large enough for one exp per
    pair to serve eight labels (the small images above take one label per
    thread); sampled rows against the restatement, in the reference's order."""
    O = oracle_mod
    W, H, L = 256, 200, 21
    N = W * H
    f = synth.gaussian_features(W, H, 3.0, 3.0)
    Q = np.random.default_rng(6).random((N, L)).astype(np.float32)
    m = DenseCRF2D(W, H, L)
    m.addPairwiseEnergy(f, 3.0)
    got = m.pairwise_apply_bf(0, Q)
    rows = np.random.default_rng(7).choice(N, 12, replace=False)
    K = O._kmat(f[rows], f)  # [rows, b] in double
    acc = np.zeros((len(rows), L), np.float32)
    for b in range(N):
        acc = (acc.astype(np.float64) + K[:, b:b + 1] * Q[b][None, :].astype(np.float64)).astype(np.float32)
    ok, info = _close(got[rows], O.compat_apply(acc, 0, 3.0))
    assert ok, info


@pytest.mark.gpu
def test_gpu_apply_bf_every_dimension():
    """apply_bf for d = 1..16 against the reference (the specialised d = 2, 3,
    5 kernels and the generic one)."""
    g = golden("bfdims_8x5_L2.npz")
    W, H, L = int(g["W"]), int(g["H"]), int(g["L"])
    for d in range(1, 17):
        m = DenseCRF2D(W, H, L)
        m.setUnaryEnergy(g["U"])
        m.addPairwiseEnergy(g[f"f{d}"], 2.0)
        ok, info = _close(m.pairwise_apply_bf(0, g["Q"]), g[f"bf_d{d}"])
        assert ok, (d, info)
