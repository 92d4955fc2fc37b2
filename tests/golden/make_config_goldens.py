"""Full-size golden results of the benchmark configurations, from the UNMODIFIED
reference (``oracle/_ref/libdcrf_ref.so``, compiled from the reference's own
sources by ``make -C oracle ref``).

Each subcommand runs the stock reference on one configuration's seeded
synthetic input and writes a small record (hashes, energies, iteration counts,
CPU seconds; label maps where a test needs them) that the GPU tests compare
against:

  qp320    config 1: ``qp_inference_super_pixels_non_convex`` at 320x240
           (seed 1), with the reference's own stop rule and with the loop body
           run exactly 100 times (``refm_qp_fixed``)        -> qp_320x240_seed1.json
  lp640    config 2: ``lp_inference_prox_super_pixels`` at 640x480 (seed 2),
           prox_max_iter=50, prox_energy_tol=1e3; also times bounded samples of
           the same solve (one proximal iteration of 2 and of 10 Frank-Wolfe
           steps) on the same core, which is what converts the benchmark's
           CPU sample into whole solves                      -> lp_640x480_seed2.json
  cliques  config 3 input: the reference's ``addSuperPixel`` (EDISON
           mean-shift, spatial radii 8 / 16 / 32, range 8, min region 100) on
           the 640x480 seed-2 image, with the CLI's higher-order weights
           (50, 1000) and with (1.0, 0.5)                    -> cliques_640x480_seed2.npz
  ho640    config 3: qp_sp and lp_sp (prox_max_iter=50) on those cliques, for
           one weight setting (``ho640 50 1000`` / ``ho640 1 0.5``)
                                                             -> ho_640x480_seed2_<c>_<n>.npz

    python tests/golden/make_config_goldens.py qp320|lp640|cliques|ho640 [c n]

Every run is single-threaded (the reference's solvers are); lp640 and ho640
take about 15-20 minutes each, the mean-shift about 8.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

os.environ.setdefault("OMP_NUM_THREADS", "1")

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

GAUSS = (3.0, 3.0)
BILAT = (50.0, 15.0, 5.0)
MS_SCALES = (8, 16, 32)
MS_RANGE = 8
MS_MIN_REGION = 100
HO_WEIGHTS = ((50.0, 1000.0), (1.0, 0.5))


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def model(img):
    return O.build_model(O.ReferenceModel, img, gaussian=GAUSS, bilateral=BILAT)


def qp320():
    W, H, seed = 320, 240, 1
    img = synth.make_image(W, H, 21, seed)
    m = model(img)
    Q = m.unary_init()
    t = time.perf_counter()
    q_rule, _, _ = m.qp(Q)
    t_rule = time.perf_counter() - t
    t = time.perf_counter()
    q_fix, it, en = m.qp(Q, 100)
    t_fix = time.perf_counter() - t
    lab_rule, lab_fix = m.current_map(q_rule), m.current_map(q_fix)
    rec = dict(W=W, H=H, L=21, seed=seed, source="reference", init_sha256=sha(Q),
               stop_rule=dict(q_sha256=sha(q_rule), labels_sha256=sha(lab_rule),
                              energy_true=m.energy_true(lab_rule), cpu_seconds=t_rule),
               fixed100=dict(iterations=int(it), q_sha256=sha(q_fix), labels_sha256=sha(lab_fix),
                             energies=[float(e) for e in en], energy_true=m.energy_true(lab_fix),
                             lr_qp_value=m.lr_qp_value(q_fix), cpu_seconds=t_fix))
    with open(os.path.join(HERE, "qp_320x240_seed1.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec)[:400])


def lp640():
    W, H, seed = 640, 480, 2
    img = synth.make_image(W, H, 21, seed)
    m = model(img)
    Q = m.unary_init()
    samples = {}
    for fw in (2, 10):
        ts = []
        for _ in range(3):
            t = time.perf_counter()
            m.lp(Q, prox_max_iter=1, fw_max_iter=fw, prox_energy_tol=1e3)
            ts.append(time.perf_counter() - t)
        samples[f"prox1_fw{fw}_seconds"] = ts
    t = time.perf_counter()
    out, _ = m.lp(Q, prox_max_iter=50, prox_energy_tol=1e3)
    t_full = time.perf_counter() - t
    lab = m.current_map(out)
    rec = dict(W=W, H=H, L=21, seed=seed, prox_max_iter=50, prox_energy_tol=1e3, prox_iters=50,
               source="reference", init_sha256=sha(Q), q_sha256=sha(out), labels_sha256=sha(lab),
               energy_true=m.energy_true(lab), cpu_seconds=t_full, samples=samples,
               cpu=_cpu_name())
    with open(os.path.join(HERE, "lp_640x480_seed2.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


def _cpu_name() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cliques():
    """Region maps of the reference's three mean-shift segmentations, and the
    clique weights addSuperPixel gives them under each HO weight setting."""
    W, H, seed = 640, 480, 2
    img = synth.make_image(W, H, 21, seed)
    out = dict(W=W, H=H, scales=np.array(MS_SCALES), range_radius=MS_RANGE, min_region=MS_MIN_REGION)
    times = []
    for c, n in HO_WEIGHTS:
        m = model(img)
        counts = []
        for sr in MS_SCALES:
            t = time.perf_counter()
            counts.append(m.add_superpixel(img["rgb"], sr, MS_RANGE, MS_MIN_REGION, c, n))
            times.append(time.perf_counter() - t)
        off, idx, ew, cs = m.get_cliques()
        tag = f"{c:g}_{n:g}"
        out[f"exp_{tag}"], out[f"const_{tag}"] = ew, cs
        if "regions" not in out:
            regions = np.full((len(MS_SCALES), W * H), -1, np.int32)
            r0 = 0
            for s, R in enumerate(counts):
                for r in range(R):
                    regions[s, idx[off[r0 + r]:off[r0 + r + 1]]] = r
                r0 += R
            assert (regions >= 0).all(), "a scale's regions do not cover the image"
            out["regions"] = regions.astype(np.uint16)
            out["counts"] = np.array(counts)
            back = cliques_from_regions(out["regions"])
            assert np.array_equal(back[0], off) and np.array_equal(back[1], idx), \
                "region maps do not reproduce the reference's clique lists"
    out["meanshift_seconds"] = np.array(times)
    np.savez_compressed(os.path.join(HERE, "cliques_640x480_seed2.npz"), **out)
    print("cliques:", out["counts"], "pixels per clique",
          np.diff(cliques_from_regions(out["regions"])[0]).min(), "..",
          np.diff(cliques_from_regions(out["regions"])[0]).max(), "seconds", times)


def cliques_from_regions(regions: np.ndarray):
    """``(offsets, idx)`` of the concatenated scales: per scale, per region in
    id order, its pixels in increasing order, which is how addSuperPixel
    fills ``super_pixel_container_`` (src/densecrf.cpp:218-223, 241)."""
    offs, idxs, base = [np.zeros(1, np.int64)], [], 0
    for reg in regions.astype(np.int64):
        order = np.argsort(reg, kind="stable")
        cnt = np.bincount(reg)
        offs.append(base + np.cumsum(cnt))
        base += int(cnt.sum())
        idxs.append(order)
    return np.concatenate(offs).astype(np.int32), np.concatenate(idxs).astype(np.int32)


def load_cliques(c: float, n: float, path=None):
    """The committed config-3 cliques as ``(offsets, idx, exp_weight, constants)``."""
    z = np.load(path or os.path.join(HERE, "cliques_640x480_seed2.npz"))
    off, idx = cliques_from_regions(z["regions"])
    tag = f"{c:g}_{n:g}"
    return off, idx, z[f"exp_{tag}"], z[f"const_{tag}"]


def ho640(c: float, n: float):
    W, H, seed = 640, 480, 2
    img = synth.make_image(W, H, 21, seed)
    m = model(img)
    m.set_cliques(*load_cliques(c, n))
    Q = m.unary_init()
    t = time.perf_counter()
    q_qp, _, _ = m.qp(Q)
    t_qp = time.perf_counter() - t
    t = time.perf_counter()
    q_lp, _ = m.lp(Q, prox_max_iter=50, prox_energy_tol=1e3)
    t_lp = time.perf_counter() - t
    lq, ll = m.current_map(q_qp), m.current_map(q_lp)
    out = dict(W=W, H=H, seed=seed, constant=c, normaliser=n, init_sha256=sha(Q),
               qp_q_sha256=sha(q_qp), qp_labels=lq.astype(np.uint8),
               qp_energy_ho=m.energy_ho(lq), qp_energy_true=m.energy_true(lq), qp_seconds=t_qp,
               lp_q_sha256=sha(q_lp), lp_labels=ll.astype(np.uint8),
               lp_energy_ho=m.energy_ho(ll), lp_energy_lp=m.energy_lp(q_lp),
               lp_energy_true=m.energy_true(ll), lp_seconds=t_lp)
    np.savez_compressed(os.path.join(HERE, f"ho_640x480_seed2_{c:g}_{n:g}.npz"), **out)
    print({k: v for k, v in out.items() if not isinstance(v, np.ndarray)})


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libdcrf_ref.so missing: run `make -C oracle ref` first")
    cmd = sys.argv[1] if len(sys.argv) > 1 else ""
    if cmd == "qp320":
        qp320()
    elif cmd == "lp640":
        lp640()
    elif cmd == "cliques":
        cliques()
    elif cmd == "ho640":
        ho640(float(sys.argv[2]), float(sys.argv[3]))
    else:
        sys.exit(__doc__)


if __name__ == "__main__":
    main()
