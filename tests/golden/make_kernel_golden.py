"""Golden vectors of DenseKernel's kernel and normalisation types
(include/pairwise.h:33-40, src/pairwise.cpp:32-168) from the reference
itself (oracle/_ref, built from its sources), on a 24x18, 5-label Gaussian +
bilateral model:

* "norm<t>": the Gaussian term added by addPairwiseEnergy with
  NormalizationType t (0 none, 1 before, 2 after): its apply, the
  unnormalised twin's apply, the energies and a fixed-iteration QP;
* "kparam": the default model after setKernelParameters on the bilateral
  term (diagonal scales): the term's apply on the rebuilt lattice, the twin's
  apply (the original features), the energies, a QP and kernelGradient;
* "const": a CONST_KERNEL term (no kernel parameters);
* "kg_<ktype><ntype>": kernelGradient of the Gaussian term as DIAG_KERNEL
  (ktype 1, scales KDIAG set) or FULL_KERNEL (ktype 2, matrix KFULL set) for
  each NormalizationType (0 none, 1 before, 2 after, 3 symmetric).

Run: python tests/golden/make_kernel_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

W, H, L, SEED = 24, 18, 5, 9
KPARAM = np.array([1.3, 0.8, 1.1, 0.9, 1.2], np.float32)
KDIAG = np.array([1.3, 0.7], np.float32)
KFULL = np.array([1.2, 0.3, -0.2, 0.9], np.float32)  # 2 x 2, column-major


def model(img, ktype=1, ntype=3):
    m = O.ReferenceModel(W, H, L, img["unary"])
    m.add_features_kernel(synth.gaussian_features(W, H, 3.0, 3.0), 3.0, ktype, ntype)
    m.add_bilateral(50.0, 50.0, 15.0, 15.0, 15.0, img["rgb"], 5.0)
    return m


def record(m, out, pre, b):
    Q = m.unary_init()
    out[pre + "unary_init"] = Q
    for k in range(2):
        out[f"{pre}apply{k}"] = m.apply(k, Q)
        out[f"{pre}apply{k}_nonorm"] = m.apply(k, Q, True)
    lab = m.current_map(Q)
    out[pre + "e_true"] = np.float64(m.energy_true(lab))
    out[pre + "e_lrqp"] = np.float64(m.lr_qp_value(Q))
    qf, it, en = m.qp(Q, 20)
    out[pre + "qp"], out[pre + "qp_iters"], out[pre + "qp_energies"] = qf, np.int64(it), en
    for k in range(2):
        out[f"{pre}kparams{k}"] = m.kernel_parameters(k)
        try:
            out[f"{pre}kgrad{k}"] = m.kernel_gradient(k, b, Q)
        except Exception:  # noqa: BLE001 -- recorded as absent
            pass


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    img = synth.make_image(W, H, L, SEED)
    b = np.random.default_rng(SEED).standard_normal((W * H, L)).astype(np.float32)
    out = dict(W=W, H=H, L=L, seed=SEED, b=b, kparam=KPARAM, kg_kdiag=KDIAG, kg_kfull=KFULL)
    for t in (0, 1, 2):
        m = model(img, 1, t)
        Q = m.unary_init()
        pre = f"norm{t}_"
        for k in range(2):
            out[f"{pre}apply{k}"] = m.apply(k, Q)
            out[f"{pre}apply{k}_nonorm"] = m.apply(k, Q, True)
        out[pre + "unary_init"] = Q
        out[pre + "e_lrqp"] = np.float64(m.lr_qp_value(Q))
        qf, it, en = m.qp(Q, 20)
        out[pre + "qp"], out[pre + "qp_iters"], out[pre + "qp_energies"] = qf, np.int64(it), en
    m = model(img)
    m.set_kernel_parameters(1, KPARAM)
    record(m, out, "kparam_", b)
    m = model(img, 0, 3)
    out["const_kparams0"] = m.kernel_parameters(0)
    out["const_kgrad0"] = m.kernel_gradient(0, b, m.unary_init())
    for kt, kp in ((1, KDIAG), (2, KFULL)):
        for t in (0, 1, 2, 3):
            m = model(img, kt, t)
            m.set_kernel_parameters(0, kp)
            Q = m.unary_init()
            out[f"kg_{kt}{t}_unary_init"] = Q
            out[f"kg_{kt}{t}"] = m.kernel_gradient(0, b, Q)
    np.savez_compressed(os.path.join(HERE, f"kernel_{W}x{H}_L{L}.npz"), **out)
    print(sorted(k for k in out if "kgrad" in k or "kparams" in k), out["kparam_kgrad1"])


if __name__ == "__main__":
    main()
