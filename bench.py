#!/usr/bin/env python
"""Benchmark of the dense-CRF hot path on B200 (one JSON line on stdout).

Workload (default ``--workload lp``): the proximal LP solve
``lp_inference_prox_super_pixels`` on a 640x480 image with 21 labels, a
Gaussian (sxy=3, w=3) and a bilateral (sxy=50, srgb=15, w=5) Potts term,
LP_inf_params() defaults with prox_max_iter=50 and prox_energy_tol =
dual_gap_tol (as the reference CLI sets it).  Input: seeded synthetic Voronoi
image + unaries (densecrf_ho_b200.synth).  One step = one LP solve.

  value        solves/s with init / output resident in HBM (dcrf_model_lp_dev)
  e2e          solves/s through the host-buffer C-ABI call dcrf_model_lp, i.e.
               with the H2D copy of the initial Q and the D2H copy of the result
               inside every step
  roofline     the LP's dominant operation, the 10-bin ordered lattice filter
               (splat + d+1 blur passes + slice), timed alone with CUDA events on
               the library's stream, against the measured HBM copy bandwidth
  cpu_baseline the reference itself (oracle/_ref, compiled from its sources) on
               the host cores: a bounded sample (one proximal iteration) scaled
               to a full solve

``--impl reference`` times the reference alone, on all usable host cores.
Under torchrun (N > 1) every rank solves its own image (replicas, no
collective on the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from densecrf_ho_b200 import synth  # noqa: E402

L = 21
GAUSS = (3.0, 3.0)                # sxy, w
BILAT = (50.0, 15.0, 5.0)         # sxy, srgb, w
LP_OVERRIDES = dict(prox_max_iter=50, prox_energy_tol=1e3)
ROOFLINE_TRAFFIC = os.path.join(ROOT, "profiles", "roofline_traffic.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", default="640x480")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only-roofline", action="store_true",
                    help="time only the ordered and plain lattice filters (a short command for ncu)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the extra workloads (QP, qp_sp / lp_sp, batch, adjoint): a short command for ncu")
    ap.add_argument("--only-batch", action="store_true",
                    help="time only qp_sp / lp_sp, the 64-image batched QP and the 16-image mean-field adjoint")
    ap.add_argument("--only-batch-qp", action="store_true",
                    help="time only the batched QP, without the sequential comparison (a short command for ncu)")
    ap.add_argument("--only-batch-filter", action="store_true",
                    help="time only the batched lattice filter over the 64-image concatenated lattices")
    ap.add_argument("--splat-form", type=int, default=None,
                    help="pin the 21-label plain filter's splat form (0-5, dcrf_batch_set_filter_shape) in the "
                         "batched filter and batched QP legs instead of autotuning it")
    ap.add_argument("--all-splat-forms", action="store_true",
                    help="with --only-batch-filter: time the batched filter with every splat form pinned")
    ap.add_argument("--only-ho", action="store_true",
                    help="time only qp_sp / lp_sp at 640x480 (no CPU reference)")
    ap.add_argument("--batch-images", type=int, default=64,
                    help="images of the batched workloads (64 = the benchmark; fewer for profiling runs)")
    ap.add_argument("--prox-iters", type=int, default=50,
                    help="prox_max_iter of the solve (50 = the benchmark; smaller for profiling runs)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def replica_seed(seed, rank):
    """Replicas: rank r solves its own image, seeded seed + r."""
    return seed + rank


def max_over_ranks(ms, world):
    """Max of a per-rank time over all ranks (the job's time), on the process
    group's own device (CUDA for NCCL, CPU for gloo)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload_name(W, H):
    return (f"lp_inference_prox_super_pixels {W}x{H} L={L}, Potts gaussian sxy={GAUSS[0]} w={GAUSS[1]} "
            f"+ bilateral sxy={BILAT[0]} srgb={BILAT[1]} w={BILAT[2]}, prox_max_iter=50, "
            f"prox_energy_tol=1e3")


def ord_filter_bytes(N, M, d, Lv=L, R=10):
    """Algorithmic bytes of one 10-bin ordered filter call:
    N (8L + 16(d+1)) + 2 M (8 R L + (d+1) (8 R L + 8))."""
    return N * (8 * Lv + 16 * (d + 1)) + 2 * M * (8 * R * Lv + (d + 1) * (8 * R * Lv + 8))


def filter_bytes(N, M, d, Lv=L):
    """Algorithmic bytes of one splat/blur/slice call:
    N (8L + 16(d+1) + 8) + M (8L + (d+1)(8L + 8))."""
    return N * (8 * Lv + 16 * (d + 1) + 8) + M * (8 * Lv + (d + 1) * (8 * Lv + 8))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------ reference on CPU --
# The reference's LP at the benchmark size takes about a quarter of an hour
# on one core, so the CPU legs time a bounded piece of the same solve -- one
# proximal iteration of REF_SAMPLE_FW Frank-Wolfe steps (prox_max_iter=1),
# from the workload's initial Q -- and convert it to whole solves with the
# ratio of the same two quantities measured by the stock reference on one
# core in one run: tests/golden/lp_640x480_seed2.json holds the full solve's
# CPU seconds and the sample's (written by tests/golden/make_config_goldens.py
# lp640; summary in profiles/reference_lp_640x480_full_solve.md).
REF_SAMPLE_FW = 2
REF_FULL_SOLVE = os.path.join(ROOT, "tests", "golden", "lp_640x480_seed2.json")


def ref_solve_fraction(W, H, seed):
    """(fraction of a full solve one sample is, description) from the
    recorded stock-reference run, or None when none is recorded for W x H."""
    if not os.path.exists(REF_FULL_SOLVE):
        return None
    with open(REF_FULL_SOLVE) as f:
        rec = json.load(f)
    key = f"prox1_fw{REF_SAMPLE_FW}_seconds"
    if (rec.get("W"), rec.get("H"), rec.get("seed")) != (W, H, seed) or rec.get("source") != "reference" \
            or key not in rec.get("samples", {}):
        return None
    t_sample = statistics.median(rec["samples"][key])
    return t_sample / rec["cpu_seconds"], (f"recorded on one core ({rec.get('cpu', '?')}): full solve "
                                           f"{rec['cpu_seconds']:.1f} s ({rec['prox_iters']} proximal x 10 "
                                           f"Frank-Wolfe iterations), sample {t_sample:.2f} s")


def _ref_worker(args):
    """Times `reps` samples of the reference LP on one core: each is
    lp_inference_prox_super_pixels with prox_max_iter=1, fw_max_iter=fw from
    the workload's initial Q.  With a barrier, every sample starts together
    with the other workers'."""
    W, H, seed, fw, reps, barrier = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    use_ref = O.reference_available()
    cls = O.ReferenceModel if use_ref else O.OracleModel
    img = synth.make_image(W, H, L, seed)
    m = O.build_model(cls, img, gaussian=GAUSS, bilateral=BILAT)
    Q = m.unary_init()
    times = []
    for _ in range(reps):
        if barrier is not None:
            barrier.wait()
        t0 = time.perf_counter()
        m.lp(Q, prox_max_iter=1, fw_max_iter=fw, prox_energy_tol=1e3)
        times.append(time.perf_counter() - t0)
    return dict(times=times, kind="reference" if use_ref else "port")


def _ref_batch_worker(args):
    """The stock reference's QP (qp_inference_super_pixels_non_convex, its
    own stop rule) on a share of the batch's images, one core: the models are
    built first, then (after the barrier) the solves are timed together."""
    idx, n, barrier = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    sizes = synth.batch_sizes(n, 4)
    models = []
    for i in idx:
        w, h = sizes[i]
        img = synth.make_image(w, h, L, 1000 + i)
        m = O.build_model(O.ReferenceModel, img, gaussian=GAUSS, bilateral=BILAT)
        models.append((m, m.unary_init()))
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for m, q0 in models:
        m.qp(q0)
    return time.perf_counter() - t0


def cpu_batch_reference(n=64):
    """The batch's images solved by the stock reference as independent
    single-threaded processes over the usable host cores (round robin); the
    wall time of the slowest worker."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    if not O.reference_available():
        return None
    workers = min(usable_cores(), n)
    shares = [list(range(w, n, workers)) for w in range(workers)]
    ctx = mp.get_context("spawn")
    barrier = ctx.Manager().Barrier(workers)
    with ctx.Pool(workers) as pool:
        times = pool.map(_ref_batch_worker, [(sh, n, barrier) for sh in shares])
    wall = max(times)
    return {"images": n, "cores": workers, "kind": "reference", "seconds": wall, "solves_per_s": n / wall,
            "sample": f"all {n} images, the stock reference's QP (its stop rule), {workers} single-threaded "
                      f"processes, round robin; models built before the timed solves"}


def cpu_reference(W, H, seed, workers, fw, reps):
    """Per step: the wall time of `workers` concurrent samples (the slowest
    worker's), so that steps x time is time actually spent."""
    ctx = mp.get_context("spawn")
    if workers == 1:
        res = [_ref_worker((W, H, seed, fw, reps, None))]
    else:
        barrier = ctx.Manager().Barrier(workers)
        with ctx.Pool(workers) as pool:
            res = pool.map(_ref_worker, [(W, H, seed, fw, reps, barrier)] * workers)
    per_step = [max(r["times"][i] for r in res) for i in range(reps)]
    return dict(kind=res[0]["kind"], per_step=per_step)


def cpu_filter_baseline(W, H, img, reps=5):
    """The reference's own lattice calls on one core, on the workload image:
    Permutohedral::init of each term's lattice, Permutohedral::compute with
    L = 21 and PairwisePotential::apply (median of reps), beside the GPU's
    lattice-filter rate."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    if not O.reference_available():
        return None
    N = W * H
    x = np.random.default_rng(0).random((N, L)).astype(np.float32)
    feats = {"gaussian": synth.gaussian_features(W, H, GAUSS[0], GAUSS[0]),
             "bilateral": synth.bilateral_features(W, H, BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1],
                                                   img["rgb"])}
    m = O.build_model(O.ReferenceModel, img, gaussian=GAUSS, bilateral=BILAT)
    out = {"cores": 1, "kind": "reference", "workload": f"{W}x{H}, L={L}"}
    for k, (name, f) in enumerate(feats.items()):
        ti, tc, ta = [], [], []
        for _ in range(reps):
            t0 = time.perf_counter()
            lat = O.ReferenceLattice(f)
            ti.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            lat.compute(x)
            tc.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            m.apply(k, x)
            ta.append(time.perf_counter() - t0)
            del lat
        tcm = statistics.median(tc)
        out[name] = {"init_ms": statistics.median(ti) * 1e3, "compute_ms": tcm * 1e3,
                     "apply_ms": statistics.median(ta) * 1e3, "compute_gpix_label_s": N * L / tcm / 1e9}
    return out


def usable_cores():
    n = os.cpu_count() or 1
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        pass
    avail_gb = 64.0
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable"):
                    avail_gb = int(ln.split()[1]) / 2**20
    except Exception:
        pass
    return max(1, min(n, int(avail_gb / 2.0), 64))


def run_reference(args):
    """The reference's own CPU LP on the host cores (oracle/_ref, compiled from
    its sources), one single-threaded process per usable core, rank 0 only.
    Each step: every worker runs one sample (one proximal iteration of
    REF_SAMPLE_FW Frank-Wolfe steps); ms_per_step is the measured wall time of
    the step, and the solves it is worth come from the recorded stock-reference
    ratio of sample to full solve (ref_solve_fraction)."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    W, H = map(int, args.size.split("x"))
    frac = ref_solve_fraction(W, H, args.seed)
    if frac is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"no stock-reference full solve recorded for {W}x{H} seed {args.seed}"}))
        return
    fraction, recorded = frac
    workers = usable_cores()
    steps = args.steps + args.warmup
    r = cpu_reference(W, H, args.seed, workers, REF_SAMPLE_FW, steps)
    timed = r["per_step"][args.warmup:] or r["per_step"]
    step_s = statistics.mean(timed)
    value = workers * fraction / step_s
    sample = (f"{workers} concurrent single-threaded reference LPs; each step runs one proximal iteration "
              f"({REF_SAMPLE_FW} Frank-Wolfe steps, prox_max_iter=1) from the workload's initial Q on every "
              f"worker, measured {step_s:.2f} s per step; one sample = {fraction:.5f} of a full solve "
              f"({recorded})")
    line = {"metric": "LP solves/s", "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(W, H), "global_batch": workers,
                       "parallelism": f"{workers} host processes",
                       "solve_fraction_per_worker_step": fraction},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers, "kind": r["kind"],
                             "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------ ours --
def measure_filters(W, H, img, reps=20, lp_q=None):
    """Times the ordered filter (the LP's dominant operation) and the plain
    splat/blur/slice filter on the bilateral and Gaussian lattices of the
    workload image, with CUDA events on each lattice's own stream.  The
    ordered filter's input is uniform random Q (its bins spread over all ten
    bins: the slice's least local case); with lp_q (device [N][L]) it is also
    timed on that Q, the LP's own iterate."""
    import torch
    from densecrf_ho_b200 import Permutohedral, lib, check
    Ls = lib()
    N = W * H
    roof = {}
    rq = torch.rand((N, L), device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    ro = torch.empty_like(rq)
    feats = {"bilateral": synth.bilateral_features(W, H, BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1],
                                                   img["rgb"]),
             "gaussian": synth.gaussian_features(W, H, GAUSS[0], GAUSS[0])}
    for name, f in feats.items():
        # Permutohedral::init through the C ABI (host features, so with their
        # upload): warm, median of 5
        Permutohedral().init(f)
        ti = []
        for _ in range(5):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tmp = Permutohedral().init(f)
            torch.cuda.synchronize()
            ti.append((time.perf_counter() - t0) * 1e3)
            del tmp
        lat = Permutohedral().init(f)
        lptr = C.c_void_p()
        check(Ls.dcrf_lattice_stream(lat._h, C.byref(lptr)))
        ls = torch.cuda.ExternalStream(lptr.value)
        run = lambda: check(Ls.dcrf_lattice_compute_ord_dev(lat._h, C.c_void_p(ro.data_ptr()),
                                                            C.c_void_p(rq.data_ptr()), L))
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ls)
        for _ in range(reps):
            run()
        e1.record(ls)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / reps / 1e3
        ab = ord_filter_bytes(N, lat.M, lat.d)
        roof[name] = dict(M=lat.M, d=lat.d, seconds=t, bytes=ab, gbs=ab / t / 1e9, init_ms=statistics.median(ti))
        if lp_q is not None:
            runq = lambda: check(Ls.dcrf_lattice_compute_ord_dev(lat._h, C.c_void_p(ro.data_ptr()),
                                                                 C.c_void_p(lp_q.data_ptr()), L))
            for _ in range(3):
                runq()
            torch.cuda.synchronize()
            e0.record(ls)
            for _ in range(reps):
                runq()
            e1.record(ls)
            torch.cuda.synchronize()
            tq = e0.elapsed_time(e1) / reps / 1e3
            roof[name]["lp_q"] = dict(seconds=tq, gbs=ab / tq / 1e9)
        # plain splat/blur/slice filter: the lattice-filter metric
        x = torch.rand((N, L), device="cuda")
        y = torch.empty_like(x)
        runp = lambda: check(Ls.dcrf_lattice_compute_dev(lat._h, C.c_void_p(y.data_ptr()),
                                                          C.c_void_p(x.data_ptr()), L, 0))
        for _ in range(3):
            runp()
        torch.cuda.synchronize()
        e0.record(ls)
        for _ in range(reps):
            runp()
        e1.record(ls)
        torch.cuda.synchronize()
        tp = e0.elapsed_time(e1) / reps / 1e3
        fb = filter_bytes(N, lat.M, lat.d)
        roof[name].update(filter_seconds=tp, filter_bytes=fb, filter_gbs=fb / tp / 1e9,
                          filter_gpix_label_s=N * L / tp / 1e9)
        del lat
    return roof


def measure_qp(reps=10, cpu=True):
    """Config 1: the plain QP (Frank-Wolfe, up to 100 iterations; it stops earlier
    when the step numerator is exactly zero, as the reference does) on a
    320x240 image.  Device-resident solves/s, the set-up (two lattice builds +
    normalisation) time, and the reference's own CPU time for the same solve."""
    import torch
    from densecrf_ho_b200 import DenseCRF2D, SolveStats, lib, check
    Ls = lib()
    W, H = 320, 240
    img = synth.make_image(W, H, L, 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    crf = DenseCRF2D(W, H, L)
    crf.setUnaryEnergy(img["unary"])
    crf.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
    crf.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"], BILAT[2])
    setup_ms = (time.perf_counter() - t0) * 1e3
    Q0 = crf.unary_init()
    init = torch.from_numpy(Q0).cuda()
    out = torch.empty_like(init)
    p = C.c_int(100)
    st = SolveStats()
    sptr = C.c_void_p()
    check(Ls.dcrf_model_stream(crf.handle, C.byref(sptr)))
    stream = torch.cuda.ExternalStream(sptr.value)
    run = lambda: check(Ls.dcrf_model_qp_dev(crf.handle, C.c_void_p(init.data_ptr()), C.c_void_p(out.data_ptr()),
                                             C.byref(p), C.byref(st)))
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    res = {"workload": "qp_inference_super_pixels_non_convex 320x240 L=21, max_iter=100",
           "solves_per_s": 1e3 / ms, "ms_per_solve": ms, "fw_steps": st.iterations, "setup_ms": setup_ms}
    if cpu:
        sys.path.insert(0, ROOT)
        from oracle import oracle as O
        cls = O.ReferenceModel if O.reference_available() else O.OracleModel
        m = O.build_model(cls, img, gaussian=GAUSS, bilateral=BILAT)
        t0 = time.perf_counter()
        _, it, _ = m.qp(Q0, 100)
        dt = time.perf_counter() - t0
        res["cpu_reference"] = {"seconds_per_solve": dt, "cores": 1, "fw_steps": it,
                                "kind": "reference" if O.reference_available() else "port"}
        res["cpu_vs_gpu"] = dt * 1e3 / ms
    return res


def measure_ho(W=640, H=480, seed=2, cpu=True):
    """Config 3: qp_sp and lp_sp (the QP / LP with sparse superpixel cliques)
    at 640x480.  Cliques: the reference's own addSuperPixel (EDISON mean
    shift at spatial radii 8 / 16 / 32, range 8, min region 100) on the
    benchmark image, recorded by tests/golden/make_config_goldens.py, with
    the HO settings (constant, normaliser) = (1.0, 0.5) and the CLI's
    (50, 1000).  GPU solves/s (device-resident) and the energies; for the
    (50, 1000) setting the reference's own qp_sp on one CPU core and the
    relative energy gap.  Also the engine's own addSuperPixel at the three
    radii (the mean-shift mode search on the GPU) beside the reference's
    recorded CPU seconds, and whether its cliques equal the reference's."""
    import torch
    from densecrf_ho_b200 import DenseCRF2D, LPParams, SolveStats, lib, check
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_config_goldens import load_cliques
    Ls = lib()
    img = synth.make_image(W, H, L, seed)
    z = np.load(os.path.join(ROOT, "tests", "golden", "cliques_640x480_seed2.npz"))
    out = {"workload": f"qp_sp / lp_sp {W}x{H} L={L}, the reference's mean-shift cliques at spatial radii "
                       f"{[int(x) for x in z['scales']]}, range 8, min region 100"}
    # the engine's addSuperPixel, three radii (warm: one run first)
    seg = DenseCRF2D(W, H, L)
    for s_ in z["scales"]:
        seg.addSuperPixel(img["rgb"], int(s_), 8, 100, 50.0, 1000.0)
    t0 = time.perf_counter()
    seg = DenseCRF2D(W, H, L)
    for s_ in z["scales"]:
        seg.addSuperPixel(img["rgb"], int(s_), 8, 100, 50.0, 1000.0)
    t_ms = time.perf_counter() - t0
    so, si, se, sc = seg.getCliques()
    ro, ri, re_, rc = load_cliques(50.0, 1000.0)
    ref_ms_s = float(np.sum(z["meanshift_seconds"][:len(z["scales"])]))
    out["add_superpixel_3_radii"] = {"seconds": t_ms, "cpu_reference_seconds": ref_ms_s, "cores": 1,
                                     "speedup": ref_ms_s / t_ms,
                                     "cliques_equal_reference": bool(np.array_equal(so, ro) and np.array_equal(si, ri)
                                                                     and np.array_equal(se, re_))}
    for const, norm in ((1.0, 0.5), (50.0, 1000.0)):
        off, idx, ew, cs = load_cliques(const, norm)
        crf = DenseCRF2D(W, H, L)
        crf.setUnaryEnergy(img["unary"])
        crf.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
        crf.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"], BILAT[2])
        crf.setCliques(off, idx, ew, cs)
        Q0 = crf.unary_init()
        init = torch.from_numpy(Q0).cuda()
        res = torch.empty_like(init)
        sptr = C.c_void_p()
        check(Ls.dcrf_model_stream(crf.handle, C.byref(sptr)))
        stream = torch.cuda.ExternalStream(sptr.value)
        st = SolveStats()
        params = LPParams.default()
        for k, v in LP_OVERRIDES.items():
            setattr(params, k, v)
        qp = lambda: check(Ls.dcrf_model_qp_dev(crf.handle, C.c_void_p(init.data_ptr()), C.c_void_p(res.data_ptr()),
                                                None, C.byref(st)))
        lp = lambda: check(Ls.dcrf_model_lp_dev(crf.handle, C.c_void_p(init.data_ptr()), C.c_void_p(res.data_ptr()),
                                                C.byref(params), C.byref(st)))
        row = {"cliques": int(len(off) - 1), "clique_pixels": int(off[-1]),
               "exp_weight_range": [float(ew.min()), float(ew.max())]}
        for name, fn, reps in (("qp_sp", qp, 5), ("lp_sp", lp, 1)):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            q = res.cpu().numpy()
            lab = crf.currentMap(q)
            row[name] = {"solves_per_s": 1e3 / ms, "ms_per_solve": ms, "iterations": st.iterations,
                         "energy_true": crf.assignment_energy_true(lab),
                         "energy_higher_order": crf.assignment_energy_higher_order(lab)}
            if name == "qp_sp":
                qp_q = q
        if cpu and const == 50.0:
            sys.path.insert(0, ROOT)
            from oracle import oracle as O
            if O.reference_available():
                m = O.build_model(O.ReferenceModel, img, gaussian=GAUSS, bilateral=BILAT)
                m.set_cliques(off, idx, ew, cs)
                t0 = time.perf_counter()
                rq, _, _ = m.qp(Q0)
                dt = time.perf_counter() - t0
                e_ref = m.energy_ho(m.current_map(rq))
                e_gpu = row["qp_sp"]["energy_higher_order"]
                row["qp_sp"]["cpu_reference"] = {"seconds_per_solve": dt, "cores": 1, "kind": "reference",
                                                 "energy_higher_order": e_ref,
                                                 "energy_rel_gap": abs(e_gpu - e_ref) / abs(e_ref),
                                                 "labels_identical": float(np.mean(m.current_map(rq) ==
                                                                                   crf.currentMap(qp_q)))}
        out[f"ho_{const:g}_{norm:g}"] = row
    return out


def pin_splat_form(b, form):
    """Pins both terms' launch shapes of a batch: the default blur / slice
    shapes with splat form `form` (no autotuning)."""
    for k in range(b.n_terms()):
        b.set_filter_shape(k, (4, 256, 128, int(form)))


SPLAT_FORMS = ("staged", "warp_long", "warp_all", "tiled_all", "staged_long_tiled_short", "bulk_all")


def measure_batch(n=64, max_iter=100, reps=3, sequential=True, splat_form=None):
    """Config 4: the plain QP (as config 1, up to 100 Frank-Wolfe iterations)
    of n images of uneven sizes (H ~ U[240, 500], W ~ U[320, 500], seeded),
    solved as one batch (dcrf_batch_qp_dev: concatenated lattices, per-image
    scalars, the loop replayed as a CUDA graph) and as n sequential
    single-image solves (dcrf_model_qp_dev, every image once per pass), both
    device-resident and timed with CUDA events on the solvers' streams.  The batch's output must equal
    the sequential outputs bit for bit."""
    import torch
    from densecrf_ho_b200 import DenseCRF2D, DenseCRF2DBatch, SolveStats, lib, check
    Ls = lib()
    sizes = synth.batch_sizes(n, 4)
    imgs = [synth.make_image(w, h, L, 1000 + i) for i, (w, h) in enumerate(sizes)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = DenseCRF2DBatch(sizes, L)
    b.setUnaryEnergy(np.concatenate([im["unary"] for im in imgs]))
    b.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
    b.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1],
                           np.concatenate([im["rgb"] for im in imgs]), BILAT[2])
    setup_ms = (time.perf_counter() - t0) * 1e3
    if splat_form is not None:
        pin_splat_form(b, splat_form)
    q0 = b.unary_init()
    init = torch.from_numpy(q0).cuda()
    out = torch.empty_like(init)
    p = C.c_int(max_iter)
    st = (SolveStats * n)()
    sptr = C.c_void_p()
    check(Ls.dcrf_batch_stream(b._h, C.byref(sptr)))
    bstream = torch.cuda.ExternalStream(sptr.value)
    run_b = lambda: check(Ls.dcrf_batch_qp_dev(b._h, C.c_void_p(init.data_ptr()), C.c_void_p(out.data_ptr()),
                                               C.byref(p), st))
    run_b()  # eager first iteration + capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = Ls.dcrf_kernel_launches()
    e0.record(bstream)
    for _ in range(reps):
        run_b()
    e1.record(bstream)
    torch.cuda.synchronize()
    batch_launches = (Ls.dcrf_kernel_launches() - l0) // reps
    batch_ms = e0.elapsed_time(e1) / reps
    steps = [s.iterations for s in st]
    if not sequential:
        return {"images": n, "pixels": int(b.N), "batch_ms": batch_ms, "fw_steps": steps,
                "batch_launches_per_solve": int(batch_launches)}

    # Sequential: every image once after the other, as a caller with one
    # model per image would run them (each solve ends with its host read of
    # the stop flag, so the solves do not overlap); the events bracket the
    # whole pass, on the first and the last model's streams.
    models, same = [], True
    outs = b.split(out)
    inits = b.split(init)
    for i, ((w, h), im) in enumerate(zip(sizes, imgs)):
        m = DenseCRF2D(w, h, L)
        m.setUnaryEnergy(im["unary"])
        m.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
        m.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], im["rgb"], BILAT[2])
        models.append(m)
    mis = [inits[i].contiguous() for i in range(n)]
    mos = [torch.empty_like(x) for x in mis]
    ones = [SolveStats() for _ in range(n)]
    streams = []
    for m in models:
        check(Ls.dcrf_model_stream(m.handle, C.byref(sptr)))
        streams.append(torch.cuda.ExternalStream(sptr.value))

    def run_all():
        for i, m in enumerate(models):
            check(Ls.dcrf_model_qp_dev(m.handle, C.c_void_p(mis[i].data_ptr()), C.c_void_p(mos[i].data_ptr()),
                                       C.byref(p), C.byref(ones[i])))

    run_all()  # eager first iterations + captures
    torch.cuda.synchronize()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(streams[0])
    for _ in range(reps):
        run_all()
    a1.record(streams[-1])
    torch.cuda.synchronize()
    seq_ms = a0.elapsed_time(a1) / reps
    for i in range(n):
        same = same and bool(torch.equal(mos[i], outs[i])) and ones[i].iterations == steps[i]
    return {"workload": f"batched qp_inference_super_pixels_non_convex, {n} images H~U[240,500] W~U[320,500] "
                        f"(seeded), L={L}, max_iter={max_iter}",
            "images": n, "pixels": int(b.N), "batch_ms": batch_ms, "sequential_ms": seq_ms,
            "batch_solves_per_s": n / (batch_ms / 1e3), "sequential_solves_per_s": n / (seq_ms / 1e3),
            "speedup_vs_sequential": seq_ms / batch_ms, "fw_steps_max": max(steps), "fw_steps_min": min(steps),
            "batch_launches_per_solve": int(batch_launches), "setup_ms": setup_ms,
            "outputs_match_sequential": same}


def measure_batch_filter(n=64, reps=10, splat_form=None, all_forms=False):
    """The batched lattice filter: PairwisePotential::apply of each pairwise
    term (normalised Potts filter, pre- and post-scaled by the norm) over the
    term's concatenated lattice of the config-4 batch (n images, H ~ U[240,
    500], W ~ U[320, 500], seeded, about 10 M pixels), device-resident, timed
    with CUDA events on the batch's stream.  The pixel arrays (0.86 GB each)
    are far larger than L2, so no flush is needed between calls.
    Algorithmic bytes: N (8L + 16(d+1) + 8) + M (8L + (d+1)(8L + 8))."""
    import torch
    from densecrf_ho_b200 import DenseCRF2DBatch, lib, check
    Ls = lib()
    sizes = synth.batch_sizes(n, 4)
    imgs = [synth.make_image(w, h, L, 1000 + i) for i, (w, h) in enumerate(sizes)]
    b = DenseCRF2DBatch(sizes, L)
    b.setUnaryEnergy(np.concatenate([im["unary"] for im in imgs]))
    b.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
    b.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1],
                           np.concatenate([im["rgb"] for im in imgs]), BILAT[2])
    N = int(b.N)
    if splat_form is not None:
        pin_splat_form(b, splat_form)
    x = torch.rand((N, L), device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    y = torch.empty_like(x)
    sptr = C.c_void_p()
    check(Ls.dcrf_batch_stream(b._h, C.byref(sptr)))
    bs = torch.cuda.ExternalStream(sptr.value)
    peak, peak_kind = measured_peaks()
    if all_forms:  # every splat form pinned in turn; outputs must not change
        forms = {}
        for k, name in enumerate(("gaussian", "bilateral")):
            ref = None
            for f, fname in enumerate(SPLAT_FORMS):
                b.set_filter_shape(k, (4, 256, 128, f))
                run = lambda: check(Ls.dcrf_batch_pairwise_apply_dev(b._h, k, C.c_void_p(y.data_ptr()),
                                                                     C.c_void_p(x.data_ptr())))
                for _ in range(3):
                    run()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(bs)
                for _ in range(reps):
                    run()
                e1.record(bs)
                torch.cuda.synchronize()
                if ref is None:
                    ref = y.clone()
                forms[f"{name}_{fname}"] = {"ms": e0.elapsed_time(e1) / reps, "same_output": bool(torch.equal(ref, y))}
        return {"images": n, "pixels": N, "forms": forms}
    out = {"workload": f"PairwisePotential::apply over the concatenated lattice of {n} images "
                       f"H~U[240,500] W~U[320,500] (seeded), L={L}, device-resident",
           "images": n, "pixels": N, "peak_gbs": peak, "peak_kind": peak_kind}
    for k, (name, d) in enumerate((("gaussian", 2), ("bilateral", 5))):
        M = b.lattice_size(k)
        run = lambda: check(Ls.dcrf_batch_pairwise_apply_dev(b._h, k, C.c_void_p(y.data_ptr()),
                                                             C.c_void_p(x.data_ptr())))
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = Ls.dcrf_kernel_launches()
        e0.record(bs)
        for _ in range(reps):
            run()
        e1.record(bs)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / reps / 1e3
        fb = filter_bytes(N, M, d)
        shp = (C.c_int * 4)()
        check(Ls.dcrf_batch_filter_shape(b._h, k, shp))
        out[name] = {"M": M, "d": d, "ms": t * 1e3, "bytes": fb, "gbs": fb / t / 1e9, "frac": fb / t / 1e9 / peak,
                     "gpix_label_s": N * L / t / 1e9,
                     "launches_per_call": int((Ls.dcrf_kernel_launches() - l0) // reps),
                     "tuned_shape": {"splat_form": SPLAT_FORMS[shp[3]],
                                     "splat_vertices_per_block": shp[0], "blur_threads": shp[1],
                                     "slice_pixels_per_block": shp[2]}}
    return out


def measure_next_rows(W=640, H=480, seed=2, cpu=True, reps=5):
    """The reference's learning and restricted-filter building blocks, through
    the C ABI with host buffers (so host<->device copies included), on the
    workload image: kernelGradient and gradient of both pairwise terms, the
    LogisticUnaryEnergy gradient, a MatrixCompatibility apply, and the
    restricted ordered filter (a store call and a reuse call on 20 % of the
    pixels).  Beside each, the reference's own CPU code (oracle/_ref, one
    core) on the same inputs at 320x240 (the CPU side is slow at 640x480),
    scaled to 640x480 by the pixel count."""
    from densecrf_ho_b200 import DenseCRF2D, Permutohedral
    O = None
    if cpu:
        from oracle import oracle as O
    out = {"workload": f"{W}x{H} L={L}; CPU reference at 320x240 scaled by the pixel count", "ms": {}}

    def model_for(w, h, cls=None):
        img = synth.make_image(w, h, L, seed)
        if cls is None:
            m = DenseCRF2D(w, h, L)
            m.setUnaryEnergy(img["unary"])
            m.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
            m.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"], BILAT[2])
        else:
            m = cls(w, h, L, img["unary"])
            m.add_gaussian(GAUSS[0], GAUSS[0], GAUSS[1])
            m.add_bilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"], BILAT[2])
        return m, img

    def ops(m, img, w, h, ref):
        rng = np.random.default_rng(0)
        N = w * h
        b = rng.standard_normal((N, L)).astype(np.float32)
        Q = m.unary_init()
        rq = (Q - Q.min()) / (Q - Q.min()).max()
        pI = np.sort(rng.choice(N, N // 5, replace=False)).astype(np.int32)
        f = synth.bilateral_features(w, h, BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"])
        if ref:
            lat = O.ReferenceLattice(f)
            return {
                "kernel_gradient_bilateral": lambda: m.kernel_gradient(1, b, Q),
                "kernel_gradient_gaussian": lambda: m.kernel_gradient(0, b, Q),
                "weight_gradient_bilateral": lambda: m.weight_gradient(1, b, Q),
                "restricted_ord_store": lambda: lat.compute_ord_restricted(rq[pI], pI, rq, True),
                "restricted_ord_reuse": lambda: lat.compute_ord_restricted(rq[pI], pI, None, False),
            }
        lat = Permutohedral().init(f)
        return {
            "kernel_gradient_bilateral": lambda: m.pairwise_kernel_gradient(1, b, Q),
            "kernel_gradient_gaussian": lambda: m.pairwise_kernel_gradient(0, b, Q),
            "weight_gradient_bilateral": lambda: m.pairwise_gradient(1, b, Q),
            "restricted_ord_store": lambda: lat.compute_upper_minus_lower_ord_restricted(rq[pI], pI, rq, True),
            "restricted_ord_reuse": lambda: lat.compute_upper_minus_lower_ord_restricted(rq[pI], pI, None, False),
        }

    m, img = model_for(W, H)
    for name, fn in ops(m, img, W, H, False).items():
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        out["ms"][name] = (time.perf_counter() - t0) / reps * 1e3
    # the compatibility and unary-energy variants on their own models
    mm = np.random.default_rng(1).random((L, L)).astype(np.float32)
    np.fill_diagonal(mm, -5.0)
    m.setCompatibility(1, matrix=mm)
    Q = m.unary_init()
    m.pairwise_apply(1, Q)
    t0 = time.perf_counter()
    for _ in range(reps):
        m.pairwise_apply(1, Q)
    out["ms"]["matrix_compat_apply_bilateral"] = (time.perf_counter() - t0) / reps * 1e3
    F = 8
    wl = np.random.default_rng(2).standard_normal((L, F)).astype(np.float32)
    fl = np.random.default_rng(3).random((W * H, F)).astype(np.float32)
    m.setUnaryEnergyLogistic(wl, fl)
    bb = np.random.default_rng(4).standard_normal((W * H, L)).astype(np.float32)
    m.unary_gradient(bb)
    t0 = time.perf_counter()
    for _ in range(reps):
        m.unary_gradient(bb)
    out["ms"]["logistic_unary_gradient"] = (time.perf_counter() - t0) / reps * 1e3
    del m
    if cpu and O is not None and O.reference_available():
        w, h = 320, 240
        scale = (W * H) / (w * h)
        rm, rimg = model_for(w, h, O.ReferenceModel)
        cpu_ms = {}
        for name, fn in ops(rm, rimg, w, h, True).items():
            t0 = time.perf_counter()
            fn()
            cpu_ms[name] = (time.perf_counter() - t0) * 1e3 * scale
        out["cpu_reference_ms_scaled"] = cpu_ms
        out["cpu_vs_gpu"] = {k: cpu_ms[k] / out["ms"][k] for k in cpu_ms}
    return out


def measure_exact_filters(seed=2, cpu=True, reps=3, bf_size=(48, 40), dc_size=(160, 120)):
    """PairwisePotential's exact filters (apply_bf, apply_upper_minus_lower_bf
    / _bf_ord, O(N^2) per label) on a 48x40 image and the divide-and-conquer
    ordered filter (apply_upper_minus_lower_dc) on a 160x120 one, the
    bilateral term, 21 labels, through the C ABI with host buffers; beside
    each, the reference's own CPU code (oracle/_ref, one core) on the same
    inputs, and the fraction of bit-equal outputs.  These back the
    reference's BRUTE_FORCE energy check and run on no solver path; the sizes
    keep the CPU side to seconds."""
    from densecrf_ho_b200 import DenseCRF2D
    out = {"workload": f"bilateral term, L={L}, ind = positions by decreasing Q; exact filters "
                       f"{bf_size[0]}x{bf_size[1]}, divide-and-conquer {dc_size[0]}x{dc_size[1]}",
           "ms": {}}
    O = None
    if cpu:
        from oracle import oracle as O
        if not O.reference_available():
            O = None
    if O is not None:
        out["cpu_reference_ms"], out["bit_equal_fraction"] = {}, {}
    for (W, H), names in ((bf_size, ("apply_bf", "upper_minus_lower_bf", "upper_minus_lower_bf_ord")),
                          (dc_size, ("upper_minus_lower_dc",))):
        img = synth.make_image(W, H, L, seed)
        N = W * H
        Q = np.random.default_rng(seed).random((N, L)).astype(np.float32)
        ind = np.argsort(-Q, axis=0, kind="stable").astype(np.int32)
        m = DenseCRF2D(W, H, L)
        m.setUnaryEnergy(img["unary"])
        m.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
        m.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"], BILAT[2])
        gpu = {"apply_bf": lambda: m.pairwise_apply_bf(1, Q),
               "upper_minus_lower_bf": lambda: m.pairwise_apply_upper_minus_lower_bf(1, ind),
               "upper_minus_lower_bf_ord": lambda: m.pairwise_apply_upper_minus_lower_bf_ord(1, ind, Q),
               "upper_minus_lower_dc": lambda: m.pairwise_apply_upper_minus_lower_dc(1, ind)}
        res = {}
        for name in names:
            res[name] = gpu[name]()
            t0 = time.perf_counter()
            for _ in range(reps):
                gpu[name]()
            out["ms"][name] = (time.perf_counter() - t0) / reps * 1e3
        del m
        if O is None:
            continue
        rm = O.build_model(O.ReferenceModel, dict(W=W, H=H, L=L, unary=img["unary"], rgb=img["rgb"]),
                           gaussian=GAUSS, bilateral=BILAT)
        ref = {"apply_bf": lambda: rm.apply_bf(1, Q),
               "upper_minus_lower_bf": lambda: rm.apply_upper_minus_lower_bf(1, ind),
               "upper_minus_lower_bf_ord": lambda: rm.apply_upper_minus_lower_bf_ord(1, ind, Q),
               "upper_minus_lower_dc": lambda: rm.apply_upper_minus_lower_dc(1, ind)}
        for name in names:
            t0 = time.perf_counter()
            r = ref[name]()
            out["cpu_reference_ms"][name] = (time.perf_counter() - t0) * 1e3
            out["bit_equal_fraction"][name] = float(np.mean(r.view(np.int32) == res[name].view(np.int32)))
    if O is not None:
        out["cpu_vs_gpu"] = {k: out["cpu_reference_ms"][k] / out["ms"][k] for k in out["cpu_reference_ms"]}
    return out


def measure_adjoint(n=16, size=512, T=10, reps=3):
    """Config 5: unrolled mean-field (T iterations) forward and its hand-written
    adjoint (dcrf_batch_meanfield_dev / _backward_dev) on n size x size images,
    21 labels, gradients with respect to the unaries and both Potts weights;
    device-resident, CUDA events on the batch's stream.  The gradient is
    checked here against a central difference of the FP32 forward along a
    random direction (the FP64 finite-difference check at 256 coordinates is
    tests/test_adjoint_gpu.py)."""
    import torch
    from densecrf_ho_b200 import DenseCRF2DBatch, lib, check
    Ls = lib()
    sizes = [(size, size)] * n
    imgs = [synth.make_image(size, size, L, 2000 + i) for i in range(n)]
    b = DenseCRF2DBatch(sizes, L)
    U = np.concatenate([im["unary"] for im in imgs])
    b.setUnaryEnergy(U)
    b.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
    b.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1],
                           np.concatenate([im["rgb"] for im in imgs]), BILAT[2])
    rng = np.random.default_rng(5)
    c = torch.from_numpy(rng.standard_normal(U.shape).astype(np.float32)).cuda()
    Q = torch.empty_like(c)
    gU = torch.empty_like(c)
    gw = np.zeros(2, np.float64)
    sptr = C.c_void_p()
    check(Ls.dcrf_batch_stream(b._h, C.byref(sptr)))
    st = torch.cuda.ExternalStream(sptr.value)
    fwd = lambda: check(Ls.dcrf_batch_meanfield_dev(b._h, T, C.c_void_p(Q.data_ptr())))
    bwd = lambda: check(Ls.dcrf_batch_meanfield_backward_dev(b._h, C.c_void_p(c.data_ptr()), C.c_void_p(gU.data_ptr()),
                                                             gw.ctypes.data_as(C.c_void_p)))
    fwd()
    bwd()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    tf = tb = 0.0
    for _ in range(reps):
        ev[0].record(st)
        fwd()
        ev[1].record(st)
        bwd()
        ev[2].record(st)
        torch.cuda.synchronize()
        tf += ev[0].elapsed_time(ev[1])
        tb += ev[1].elapsed_time(ev[2])
    tf, tb = tf / reps, tb / reps
    # directional check: <dL/dU, V> vs (L(U + eV) - L(U - eV)) / 2e, L = sum(c o Q_T)
    V = rng.standard_normal(U.shape).astype(np.float32)
    eps = 1e-2
    cd = c.double()

    def loss(UU):
        b.setUnaryEnergy(UU)
        fwd()
        torch.cuda.synchronize()
        return float((cd * Q.double()).sum())

    pred = float((gU.double() * torch.from_numpy(V).cuda().double()).sum())
    dd = (loss(U + eps * V) - loss(U - eps * V)) / (2 * eps)
    b.setUnaryEnergy(U)
    full_bytes = b.meanfield_state_bytes(T)
    # checkpointing: every 5th iterate kept, the rest recomputed in the
    # backward pass, the lattices released after the forward and rebuilt
    b.set_checkpointing(5, True)
    fwd()
    bwd()
    torch.cuda.synchronize()
    tfr = tbr = 0.0
    for _ in range(reps):
        ev[0].record(st)
        fwd()
        ev[1].record(st)
        bwd()
        ev[2].record(st)
        torch.cuda.synchronize()
        tfr += ev[0].elapsed_time(ev[1])
        tbr += ev[1].elapsed_time(ev[2])
    tfr, tbr = tfr / reps, tbr / reps
    ck_bytes = b.meanfield_state_bytes(T)
    b.set_checkpointing(1, False)
    return {"workload": f"unrolled mean-field, {n} images {size}x{size}, L={L}, {T} iterations, forward + adjoint "
                        f"(dL/dU and dL/dw for the Gaussian and bilateral Potts weights)",
            "forward_ms": tf, "backward_ms": tb, "images_per_s": n / ((tf + tb) / 1e3),
            "state_bytes": full_bytes,
            "checkpoint_every_5_lattice_recompute": {"forward_ms": tfr, "backward_ms": tbr,
                                                      "images_per_s": n / ((tfr + tbr) / 1e3),
                                                      "state_bytes": ck_bytes},
            "pixels": n * size * size, "directional_check_rel_err": abs(dd - pred) / abs(pred),
            "fd64_check": adjoint_fd64_check(T=T),
            "grad_w": [float(x) for x in gw]}


def adjoint_fd64_check(T=10, W=48, H=40, coords=16, h=1e-6):
    """The adjoint against FP64 central finite differences on a small image
    (21 labels, `coords` random unary coordinates and both Potts weights):
    the finite differences run an FP64 mean-field on the host with the
    oracle's FP64 lattice filter on the same lattices (the checker only).
    Returns the largest relative error, each coordinate's error measured
    against max(|fd|, 1e-2 max|fd|)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from densecrf_ho_b200 import DenseCRF2DBatch
    img = synth.make_image(W, H, L, 3)
    U = img["unary"].astype(np.float32)
    b = DenseCRF2DBatch([(W, H)], L)
    b.setUnaryEnergy(U)
    b.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
    b.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"], BILAT[2])
    c = np.random.default_rng(0).standard_normal(U.shape)
    b.meanfield(T)
    gU, gw = b.meanfield_backward(c.astype(np.float32))
    lats = []
    for f in (synth.gaussian_features(W, H, GAUSS[0], GAUSS[0]),
              synth.bilateral_features(W, H, BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"])):
        lat = O.OracleLattice(f)
        lats.append((lat, 1.0 / np.sqrt(lat.compute_f64(np.ones((W * H, 1)))[:, 0] + 1e-20)))

    def softmax(a):
        e = np.exp(a - a.max(1, keepdims=True))
        return e / e.sum(1, keepdims=True)

    def run(UU, ws):
        q = softmax(-UU)
        for _ in range(T):
            a = -UU.copy()
            for (lat, nrm), w in zip(lats, ws):
                a += w * nrm[:, None] * lat.compute_f64(nrm[:, None] * q)
            q = softmax(a)
        return float((c * q).sum())

    U64, w0 = U.astype(np.float64), [GAUSS[1], BILAT[2]]
    flat = np.random.default_rng(1).choice(U.size, coords, replace=False)
    fd = np.empty(coords)
    for j, idx in enumerate(flat):
        Up, Um = U64.copy(), U64.copy()
        Up.flat[idx] += h
        Um.flat[idx] -= h
        fd[j] = (run(Up, w0) - run(Um, w0)) / (2 * h)
    rel = np.abs(gU.flat[flat].astype(np.float64) - fd) / np.maximum(np.abs(fd), 1e-2 * np.abs(fd).max())
    wrel = []
    for k in range(2):
        wp, wm = list(w0), list(w0)
        wp[k] += h
        wm[k] -= h
        fdw = (run(U64, wp) - run(U64, wm)) / (2 * h)
        wrel.append(abs(gw[k] - fdw) / abs(fdw))
    return {"image": f"{W}x{H}", "labels": L, "iterations": T, "coordinates": coords, "step": h,
            "unary_max_rel_err": float(rel.max()), "weight_max_rel_err": float(max(wrel))}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from densecrf_ho_b200 import DenseCRF2D, LPParams, Permutohedral, SolveStats, lib, check

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    W, H = map(int, args.size.split("x"))
    N = W * H
    seed = replica_seed(args.seed, rank)
    img = synth.make_image(W, H, L, seed)
    if args.only_roofline:
        print(json.dumps(measure_filters(W, H, img, reps=3)))
        return
    if args.only_batch_filter:
        print(json.dumps(measure_batch_filter(n=args.batch_images, splat_form=args.splat_form,
                                              all_forms=args.all_splat_forms)))
        return
    if args.only_ho:
        print(json.dumps(measure_ho(cpu=False)))
        return
    if args.only_batch_qp:
        print(json.dumps(measure_batch(n=args.batch_images, reps=1, sequential=False, splat_form=args.splat_form)))
        return
    if args.only_batch:
        print(json.dumps(measure_ho()))
        print(json.dumps(measure_batch()))
        print(json.dumps(measure_adjoint()))
        return
    t0 = time.perf_counter()
    crf = DenseCRF2D(W, H, L)
    crf.setUnaryEnergy(img["unary"])
    crf.addPairwiseGaussian(GAUSS[0], GAUSS[0], GAUSS[1])
    crf.addPairwiseBilateral(BILAT[0], BILAT[0], BILAT[1], BILAT[1], BILAT[1], img["rgb"], BILAT[2])
    Q0 = crf.unary_init()
    setup_ms = (time.perf_counter() - t0) * 1e3
    params = LPParams.default()
    for k, v in LP_OVERRIDES.items():
        setattr(params, k, v)
    params.prox_max_iter = args.prox_iters
    Ls = lib()
    sptr = C.c_void_p()
    check(Ls.dcrf_model_stream(crf.handle, C.byref(sptr)))
    stream = torch.cuda.ExternalStream(sptr.value)
    init_d = torch.from_numpy(Q0).cuda()
    out_d = torch.empty_like(init_d)
    st = SolveStats()

    def step_dev():
        check(Ls.dcrf_model_lp_dev(crf.handle, C.c_void_p(init_d.data_ptr()), C.c_void_p(out_d.data_ptr()),
                                   C.byref(params), C.byref(st)))

    for _ in range(args.warmup):
        step_dev()
    torch.cuda.synchronize()

    def timed(fn, k):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return max_over_ranks(e0.elapsed_time(e1), world)

    clocks = ClockSampler(local)
    clocks.start()
    l0 = Ls.dcrf_kernel_launches()
    ms = timed(step_dev, args.steps)
    launches = Ls.dcrf_kernel_launches() - l0
    clk = clocks.stop()
    prox_iters, fw_iters, gamma_iters = st.iterations, st.inner_iters, st.gamma_iters
    value = world * args.steps / (ms / 1e3)

    # e2e: the host-buffer C-ABI call, pinned host input and output.
    init_h = torch.from_numpy(Q0).pin_memory()
    out_h = torch.empty_like(init_h).pin_memory()

    def step_host():
        check(Ls.dcrf_model_lp(crf.handle, C.c_void_p(init_h.data_ptr()), C.c_void_p(out_h.data_ptr()),
                               C.byref(params), C.byref(st)))

    step_host()
    ms_e2e = timed(step_host, args.steps)
    e2e_value = world * args.steps / (ms_e2e / 1e3)
    same = bool(torch.equal(out_h, out_d.cpu()))

    roof = measure_filters(W, H, img, reps=20, lp_q=out_d)
    peak, peak_kind = measured_peaks()
    dom = roof["bilateral"]
    traffic = None
    if os.path.exists(ROOFLINE_TRAFFIC):
        with open(ROOFLINE_TRAFFIC) as f:
            tr = json.load(f)
        traffic = tr.get("ord_filter_bytes_per_call", {}).get(f"{W}x{H}")
    roofline = {"bound": "hbm", "achieved": dom["gbs"], "peak": peak, "unit": "GB/s",
                "frac": dom["gbs"] / peak, "traffic": traffic,
                "kernel": f"ordered lattice filter, bilateral d=5 lattice (M={dom['M']}), {W}x{H}, L={L}",
                "peak_kind": peak_kind,
                "gaussian_d2": {"M": roof["gaussian"]["M"], "gbs": roof["gaussian"]["gbs"],
                                "frac": roof["gaussian"]["gbs"] / peak},
                "on_lp_solution": {"input": "the LP's final Q (bins concentrated at 0 and 9) instead of uniform Q",
                                   "ms": dom["lp_q"]["seconds"] * 1e3, "gbs": dom["lp_q"]["gbs"],
                                   "frac": dom["lp_q"]["gbs"] / peak}}

    line = {"metric": "LP solves/s", "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Voronoi image + -log softmax unaries)",
            "config": {"workload": workload_name(W, H), "global_batch": world,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "solver state ~12 x N x L x 4 B = 310 MB > 126 MB L2; no flush needed",
                       "prox_iters": prox_iters, "fw_iters": fw_iters, "gamma_iters": gamma_iters},
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": N * L * 4,
                    "d2h_bytes_per_step": N * L * 4, "output_matches_device_path": same},
            "clocks": clk, "gpu_launches": int(launches),
            "extra": {"setup_ms": setup_ms,
                      "lattice_filter_gpix_label_s": {k: v["filter_gpix_label_s"] for k, v in roof.items()},
                      "lattice_filter_gbs": {k: v["filter_gbs"] for k, v in roof.items()},
                      "ord_filter_ms": {k: v["seconds"] * 1e3 for k, v in roof.items()},
                      "lattice_init_ms": {k: v["init_ms"] for k, v in roof.items()}}}
    if rank == 0 and world == 1 and not args.no_extra:
        line["extra"]["qp_320x240"] = measure_qp(cpu=not args.no_cpu_baseline)
        line["extra"]["ho_640x480"] = measure_ho(cpu=not args.no_cpu_baseline)
        line["extra"]["batch_filter_64"] = measure_batch_filter()
        line["extra"]["batch_qp_64"] = measure_batch()
        if not args.no_cpu_baseline:
            cb = cpu_batch_reference()
            if cb is not None:
                cb["gpu_batch_vs_cpu"] = line["extra"]["batch_qp_64"]["batch_solves_per_s"] / cb["solves_per_s"]
                line["extra"]["batch_qp_64"]["cpu_reference_all_cores"] = cb
        line["extra"]["adjoint_16x512x512"] = measure_adjoint()
        line["extra"]["next_rows_640x480"] = measure_next_rows(cpu=not args.no_cpu_baseline)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        frac = ref_solve_fraction(W, H, args.seed)
        if frac is not None:
            fraction, recorded = frac
            r = cpu_reference(W, H, args.seed, 1, REF_SAMPLE_FW, 3)
            t = statistics.median(r["per_step"])
            line["cpu_baseline"] = {"value": fraction / t, "unit": "solves/s", "cores": 1, "kind": r["kind"],
                                    "sample": (f"3 samples of the reference LP on 1 core, each one proximal "
                                               f"iteration ({REF_SAMPLE_FW} Frank-Wolfe steps, "
                                               f"prox_max_iter=1), median {t:.2f} s; one sample = "
                                               f"{fraction:.5f} of a full solve ({recorded})")}
        fb = cpu_filter_baseline(W, H, img)
        if fb is not None:
            gpu = line["extra"]["lattice_filter_gpix_label_s"]
            line["cpu_baseline_filter"] = {
                "value": fb["bilateral"]["compute_gpix_label_s"], "unit": "Gpix.label/s", "cores": 1,
                "kind": "reference",
                "sample": f"Permutohedral::compute, bilateral d=5 lattice, {W}x{H}, L={L}, median of 5",
                "detail": fb,
                "gpu_vs_cpu": {k: gpu[k] / fb[k]["compute_gpix_label_s"] for k in ("gaussian", "bilateral")}}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
