"""The adjoint of unrolled mean-field iterations (dcrf_batch_meanfield /
dcrf_batch_meanfield_backward) against FP64 central finite differences.

The finite differences run an FP64 mean-field on the CPU with the oracle's
FP64 lattice filter on the same lattices (the lattice structure is exact), at
step 1e-6 on 256 random coordinates of the unaries and on each Potts weight.
A torch.autograd.Function over the C ABI (here, in the test harness only)
drives the GPU side.
"""
import ctypes as C

import numpy as np
import pytest

from densecrf_ho_b200 import DenseCRF2DBatch, lib, check, synth

pytestmark = pytest.mark.gpu

GAUSS = (3.0, 3.0)
BILAT = (50.0, 15.0, 5.0)
# Gradient bound against FP64 finite differences: relative per coordinate,
# with coordinates whose finite difference is below ADJOINT_FLOOR of the
# largest measured against that floor instead (an FP32 forward carries
# absolute errors of a few 1e-8 of the largest gradient).
ADJOINT_RTOL = 1e-4
ADJOINT_FLOOR = 1e-2


def _setup(sizes, L, seed):
    imgs = [synth.make_image(w, h, L, seed + i) for i, (w, h) in enumerate(sizes)]
    b = DenseCRF2DBatch(sizes, L)
    U = np.concatenate([im["unary"] for im in imgs])
    b.setUnaryEnergy(U)
    b.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
    b.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1],
                           np.concatenate([im["rgb"] for im in imgs]), BILAT[2])
    return b, U, imgs


class FP64MeanField:
    """Q_{t+1} = softmax(-U + sum_k w_k n_k o K_k(n_k o Q_t)) in FP64 with the
    oracle's FP64 filter, image by image."""

    def __init__(self, sizes, imgs, oracle_mod):
        self.sizes = sizes
        self.terms = []
        for (w, h), im in zip(sizes, imgs):
            lg = oracle_mod.OracleLattice(synth.gaussian_features(w, h, GAUSS[0], GAUSS[0]))
            lb = oracle_mod.OracleLattice(synth.bilateral_features(w, h, BILAT[0], BILAT[0], BILAT[1], BILAT[1],
                                                                   BILAT[1], im["rgb"]))
            per = []
            for lat in (lg, lb):
                n = 1.0 / np.sqrt(lat.compute_f64(np.ones((w * h, 1)))[:, 0] + 1e-20)
                per.append((lat, n))
            self.terms.append(per)
        self.off = np.concatenate([[0], np.cumsum([w * h for w, h in sizes])])

    @staticmethod
    def softmax(a):
        e = np.exp(a - a.max(1, keepdims=True))
        return e / e.sum(1, keepdims=True)

    def run(self, U, weights, T):
        out = []
        for i, per in enumerate(self.terms):
            u = U[self.off[i]:self.off[i + 1]].astype(np.float64)
            q = self.softmax(-u)
            for _ in range(T):
                a = -u.copy()
                for (lat, n), w in zip(per, weights):
                    a += w * n[:, None] * lat.compute_f64(n[:, None] * q)
                q = self.softmax(a)
            out.append(q)
        return np.concatenate(out)


def _torch_meanfield():
    import torch

    class MeanField(torch.autograd.Function):
        @staticmethod
        def forward(ctx, U, batch, T):
            Ls = lib()
            U = U.contiguous()
            check(Ls.dcrf_batch_set_unary_dev(batch._h, C.c_void_p(U.data_ptr())))
            Q = torch.empty_like(U)
            check(Ls.dcrf_batch_meanfield_dev(batch._h, int(T), C.c_void_p(Q.data_ptr())))
            ctx.batch = batch
            return Q

        @staticmethod
        def backward(ctx, gQ):
            Ls = lib()
            gQ = gQ.contiguous()
            gU = torch.empty_like(gQ)
            gw = np.zeros(ctx.batch.n_terms(), np.float64)
            check(Ls.dcrf_batch_meanfield_backward_dev(ctx.batch._h, C.c_void_p(gQ.data_ptr()),
                                                       C.c_void_p(gU.data_ptr()), gw.ctypes.data_as(C.c_void_p)))
            torch.cuda.synchronize()
            ctx.batch.last_grad_w = gw
            return gU, None, None

    return MeanField


def test_meanfield_forward_matches_fp64(oracle_mod):
    sizes = [(26, 19), (21, 17)]
    b, U, imgs = _setup(sizes, 5, 3)
    q = b.meanfield(10)
    ref = FP64MeanField(sizes, imgs, oracle_mod).run(U, [GAUSS[1], BILAT[2]], 10)
    assert np.abs(q - ref).max() < 1e-5


def test_meanfield_gradient_vs_fp64_finite_differences(oracle_mod):
    import torch
    sizes = [(26, 19), (21, 17)]
    L, T = 5, 10
    b, U, imgs = _setup(sizes, L, 3)
    c = np.random.default_rng(0).standard_normal(U.shape)  # loss = sum(c o Q_T)
    Ut = torch.from_numpy(U).cuda().requires_grad_(True)
    Q = _torch_meanfield().apply(Ut, b, T)
    loss = (torch.from_numpy(c).cuda() * Q.double()).sum()
    loss.backward()
    gU = Ut.grad.cpu().numpy().astype(np.float64)
    gw = b.last_grad_w

    ref = FP64MeanField(sizes, imgs, oracle_mod)
    w0 = [GAUSS[1], BILAT[2]]
    f = lambda UU, ww: float((c * ref.run(UU, ww, T)).sum())
    h = 1e-6
    rng = np.random.default_rng(1)
    flat = rng.choice(U.size, 256, replace=False)
    U64 = U.astype(np.float64)
    fd = np.empty(len(flat))
    for j, idx in enumerate(flat):
        Up, Um = U64.copy(), U64.copy()
        Up.flat[idx] += h
        Um.flat[idx] -= h
        fd[j] = (f(Up, w0) - f(Um, w0)) / (2 * h)
    err = np.abs(gU.flat[flat] - fd)
    assert err.max() <= 1e-3 * np.abs(fd).max() + 1e-6, (err.max(), np.abs(fd).max())
    for k in range(2):
        wp, wm = list(w0), list(w0)
        wp[k] += h
        wm[k] -= h
        fdw = (f(U64, wp) - f(U64, wm)) / (2 * h)
        assert abs(gw[k] - fdw) <= 1e-3 * abs(fdw) + 1e-6, (k, gw[k], fdw)


def _fd_at(ref, U64, c, T, w0, flat, h):
    """FP64 central differences of loss = sum(c o Q_T) at the flat unary
    coordinates, each on the image it belongs to alone (the others do not
    move), the two forwards subtracted element by element before the sum.
    The oracle's filter runs outside the GIL, so threads share the work."""
    import concurrent.futures as cf
    import os
    L = U64.shape[1]

    def one(idx):
        i = int(np.searchsorted(ref.off, idx // L, side="right") - 1)
        a, b = ref.off[i], ref.off[i + 1]
        sub = FP64MeanField.__new__(FP64MeanField)
        sub.sizes, sub.terms, sub.off = ref.sizes[i:i + 1], ref.terms[i:i + 1], np.array([0, b - a])
        Up, Um = U64[a:b].copy(), U64[a:b].copy()
        Up.flat[idx - a * L] += h
        Um.flat[idx - a * L] -= h
        return float((c[a:b] * (sub.run(Up, w0, T) - sub.run(Um, w0, T))).sum()) / (2 * h)

    with cf.ThreadPoolExecutor(min(16, os.cpu_count() or 1)) as ex:
        return np.array(list(ex.map(one, flat)))


def test_meanfield_gradient_21_labels_128x128_vs_fp64_finite_differences(oracle_mod):
    """The stated check at a realistic size: 21 labels, a 128x128 image and
    a 26x19 one in the batch, 256 random unary coordinates, FP64 central
    differences with step 1e-6 (forward in FP64 with the oracle's FP64
    filter on the same lattices), and each Potts weight.  The GPU forward is
    FP32; ADJOINT_RTOL / ADJOINT_FLOOR give the bound."""
    import torch
    sizes = [(128, 128), (26, 19)]
    L, T = 21, 10
    b, U, imgs = _setup(sizes, L, 3)
    c = np.random.default_rng(0).standard_normal(U.shape)
    Ut = torch.from_numpy(U).cuda().requires_grad_(True)
    Q = _torch_meanfield().apply(Ut, b, T)
    (torch.from_numpy(c).cuda() * Q.double()).sum().backward()
    gU = Ut.grad.cpu().numpy().astype(np.float64)
    gw = b.last_grad_w
    ref = FP64MeanField(sizes, imgs, oracle_mod)
    w0 = [GAUSS[1], BILAT[2]]
    U64 = U.astype(np.float64)
    flat = np.random.default_rng(1).choice(U.size, 256, replace=False)
    fd = _fd_at(ref, U64, c, T, w0, flat, 1e-6)
    g = gU.flat[flat]
    scale = np.abs(fd).max()
    rel = np.abs(g - fd) / np.maximum(np.abs(fd), ADJOINT_FLOOR * scale)
    print("adjoint vs FD: max rel", rel.max(), "median", np.median(rel), "p99", np.percentile(rel, 99),
          "plain rel max", (np.abs(g - fd) / np.abs(fd)).max(), "max|fd|", scale)
    wrel = []
    for k in range(2):
        wp, wm = list(w0), list(w0)
        wp[k] += 1e-6
        wm[k] -= 1e-6
        fdw = float((c * (ref.run(U64, wp, T) - ref.run(U64, wm, T))).sum()) / 2e-6
        wrel.append(abs(gw[k] - fdw) / abs(fdw))
    print("weights rel", wrel)
    assert rel.max() <= ADJOINT_RTOL, (rel.max(), np.median(rel), scale)
    assert max(wrel) <= ADJOINT_RTOL, wrel


def test_meanfield_directional_derivative_larger_batch():
    """Four 128x96 images, 21 labels: <dL/dU, V> against a central difference
    of the FP32 forward along V, and dL/dw against changed weights."""
    import torch
    sizes = [(128, 96)] * 4
    b, U, _ = _setup(sizes, 21, 7)
    rng = np.random.default_rng(3)
    c = rng.standard_normal(U.shape)
    V = rng.standard_normal(U.shape).astype(np.float32)
    T = 10

    def loss(UU, w=None):
        if w is not None:
            b.set_weight(0, w[0])
            b.set_weight(1, w[1])
        b.setUnaryEnergy(UU)
        return float((c * b.meanfield(T).astype(np.float64)).sum())

    L0 = loss(U)
    gU, gw = b.meanfield_backward(c.astype(np.float32))
    eps = 1e-2
    dd = (loss(U + eps * V) - loss(U - eps * V)) / (2 * eps)
    pred = float((gU.astype(np.float64) * V).sum())
    assert abs(dd - pred) <= 1e-3 * abs(pred), (dd, pred)
    epw = 1e-2
    for k in range(2):
        w = [GAUSS[1], BILAT[2]]
        wp, wm = list(w), list(w)
        wp[k] += epw
        wm[k] -= epw
        fd = (loss(U, wp) - loss(U, wm)) / (2 * epw)
        assert abs(fd - gw[k]) <= 2e-3 * abs(gw[k]), (k, fd, gw[k])
    assert np.isfinite(L0)


@pytest.mark.parametrize("every,recompute", [(3, False), (4, True), (10, True)])
def test_checkpointing_and_lattice_recompute_give_identical_gradients(every, recompute):
    """Keeping every k-th iterate (the backward pass recomputing the rest) and
    rebuilding the lattices between the passes reproduce the all-iterates
    gradients bit for bit: the recomputed values come from the same kernels
    on the same inputs.  The checkpoint memory shrinks as stated."""
    sizes = [(64, 48), (37, 29), (50, 50)]
    T = 10
    b, U, _ = _setup(sizes, 21, 11)
    c = np.random.default_rng(2).standard_normal(U.shape).astype(np.float32)
    q_all = b.meanfield(T)
    gU_all, gw_all = b.meanfield_backward(c)
    full = b.meanfield_state_bytes(T)
    b.set_checkpointing(every, recompute)
    q = b.meanfield(T)
    gU, gw = b.meanfield_backward(c)
    assert np.array_equal(q, q_all)
    assert np.array_equal(gU, gU_all)
    assert np.array_equal(gw, gw_all)
    arr = 4 * b.N * 21
    slots = T // every + 1 + (1 if T % every else 0)
    assert b.meanfield_state_bytes(T) == (slots + min(every - 1, T - 1)) * arr
    assert full == (T + 1) * arr
    # a second forward / backward in the same mode (lattices rebuilt again)
    q2 = b.meanfield(T)
    gU2, _ = b.meanfield_backward(c)
    assert np.array_equal(q2, q_all) and np.array_equal(gU2, gU_all)
