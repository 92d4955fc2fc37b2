"""Golden vectors of the reference's per-pixel energies and rounding
(DenseCRF::unaryEnergy, pairwise_energy_true, max_rounding and
compute_LR_QP_value with a diag_dom, src/densecrf.cpp:832-957) from the
reference itself (oracle/_ref, built from its sources), on the example's
Gaussian + bilateral model at 24x18 with 21 labels.

Run: python tests/golden/make_energy_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

W, H, L, SEED = 24, 18, 21, 10


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    img = synth.make_image(W, H, L, SEED)
    m = O.build_model(O.ReferenceModel, img)
    rng = np.random.default_rng(SEED)
    lab = rng.integers(0, L, W * H).astype(np.int16)
    lab[::17] = -1  # off the label range: 0 energy
    Q = rng.random((W * H, L)).astype(np.float32)
    Q[5, 3] = Q[5, 7] = np.float32(2.0)  # a tie: the first maximum wins
    dd = (rng.random((W * H, L)) * 0.5).astype(np.float32)
    out = dict(W=W, H=H, L=L, seed=SEED, lab=lab, Q=Q, dd=dd, unary_e=m.unary_energy(lab),
               pw_all=m.pairwise_energy(lab, -1), pw0=m.pairwise_energy(lab, 0), pw1=m.pairwise_energy(lab, 1),
               maxround=m.max_rounding(Q), lrqp_dd=np.float64(m.lr_qp_value_diag(Q, dd)))
    # compute_energy_higher_order after a QP, with the reference's own
    # mean-shift cliques (spatial 8, range 8, min region 20; weights 50 / 1000)
    mh = O.build_model(O.ReferenceModel, img)
    mh.add_superpixel(img["rgb"], 8, 8, 20, 50.0, 1000.0)
    off, idx, ex, cs = mh.get_cliques()
    Q0 = mh.unary_init()
    qf, it, _ = mh.qp(Q0, 5)
    out.update(cl_off=off, cl_idx=idx, cl_exp=ex, cl_const=cs, ho_unary_init=Q0, ho_qp=qf,
               e_qp_ho_after=np.float64(mh.energy_qp_ho(Q)), e_qp_ho_qp=np.float64(mh.energy_qp_ho(qf)))
    m.qp(m.unary_init(), 5)
    out["e_qp_ho_nocliques"] = np.float64(m.energy_qp_ho(Q))
    np.savez_compressed(os.path.join(HERE, f"energies_{W}x{H}.npz"), **out)
    print({k: float(np.abs(v).sum()) for k, v in out.items() if k not in ("W", "H", "L", "seed")})


if __name__ == "__main__":
    main()
