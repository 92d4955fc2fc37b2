"""Full-size golden checksums: the LP of the benchmark workload.

Runs the bit-exact CPU restatement (oracle/dcrf_oracle.c, itself pinned to the
reference in tests/test_oracle.py) on the 640x480, 21-label synthetic image of
seed 2 with the LP parameters of the benchmark (prox_max_iter=50,
prox_energy_tol=1e3), and records the SHA-256 of the resulting Q (float32
[N][L] bytes), its integer energy and the iteration count.  Takes ~15 minutes
on one core; the GPU test compares its own 1-second solve against it.

    python tests/golden/make_full_size.py
"""
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    W, H, seed = 640, 480, 2
    img = synth.make_image(W, H, 21, seed)
    m = O.build_model(O.OracleModel, img)
    Q = m.unary_init()
    t = time.time()
    out, nit = m.lp(Q, prox_max_iter=50, prox_energy_tol=1e3)
    rec = dict(W=W, H=H, L=21, seed=seed, prox_max_iter=50, prox_energy_tol=1e3, prox_iters=nit,
               init_sha256=hashlib.sha256(Q.tobytes()).hexdigest(),
               q_sha256=hashlib.sha256(out.tobytes()).hexdigest(),
               energy_true=m.energy_true(m.current_map(out)), cpu_seconds=time.time() - t)
    with open(os.path.join(HERE, "lp_640x480_seed2.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(rec)


if __name__ == "__main__":
    main()
