#!/usr/bin/env python
"""Benchmark: pairs/s of SIFT extraction + prior-guided matching at 2640x1978.

Workload (one step): 64 synthetic image pairs at 2640x1978 (uint8; seeded blobs + 1/f noise; B =
A warped by a random homography + noise), per-image keypoint caps drawn from U[2000, 16000];
every image goes through the features.sift_gpu sequence (detect with max_kp = 2.2 nfeat, grid
spread, describe, RootSIFT); each pair is then matched by prior-guided matching: predicted
position = true homography + N(0, 15 px), candidates = the 16 nearest keypoints within 40 px
(the pipeline's guided_k), exact squared distances, ratio 0.85, one-to-one filter. A "pair" is
extraction of both images + the match.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fsb|reference]

value  : pairs/s with the images resident in HBM (device-pointer C ABI, fsb_*_d).
e2e    : the same pairs through the public host API (features.sift_gpu_u8 + matching
         guided_from_pred) with host buffers, copies included.
roofline: the pyramid (dominant stage): the step's images through the pyramid stage alone as one
         graph with the extraction graph's images in flight (fsb_pyramid_batch_d), CUDA events on its
         stream; beside it the same for one image at a time on one stream; algorithmic bytes per
         image = H*W + 44 * (sum of octave pixels).
--impl reference: the reference's CPU implementation of the path (OpenCV SIFT as
         features.sift_cpu calls it + the NumPy/cKDTree guided matcher), oracle port, on the host
         cores; one pair per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "pairs/s SIFT+guided match @2640x1978: BF16/FP8+rerank vs FP32, same matches"
H_IMG, W_IMG = 1978, 2640
RADIUS, RATIO, KC = 40.0, 0.85, 16


def _json_num(o):
    """numpy scalars in the JSON line"""
    if hasattr(o, "item"):
        return o.item()
    raise TypeError(type(o).__name__)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="fsb", choices=["fsb", "reference"])
    p.add_argument("--pairs", type=int, default=64)
    p.add_argument("--seed", type=int, default=1000)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--streams", type=int, default=6, help="host threads, each with its own context/stream")
    p.add_argument("--extract", default="graph", choices=["graph", "threads"],
                   help="graph: every image of a step in one sync-free batch (one CUDA graph); threads: "
                        "fsb_sift_features_d per image on --streams host threads")
    p.add_argument("--chains", type=int, default=16, help="images in flight inside the extraction graph")
    p.add_argument("--sweep-pairs", type=int, default=256, help="dense precision sweep: pairs per batch (0: skip)")
    p.add_argument("--sweep-n", type=int, default=16384, help="dense precision sweep: descriptors per image")
    p.add_argument("--plain-pairs", type=int, default=16,
                   help="pairs timed through the plain sequential path (one stream, one pair at a time; 0: skip)")
    p.add_argument("--filter-pairs", type=int, default=64,
                   help="pairs for the learned match filter (3/4 train, 1/4 held out; 0: skip)")
    p.add_argument("--flight-lines", type=int, default=20,
                   help="synthetic flight: lines x frames per line (20: 400 frames; 0: skip)")
    p.add_argument("--flight-train", type=int, default=500,
                   help="synthetic flight: pairs whose candidates train the learned filter (the rest are held out)")
    return p.parse_args()


def config(args, extra=None):
    c = {"workload": "SIFT (sift_gpu sequence) + prior-guided match of %d pairs at %dx%d per GPU per step; "
                     "nfeat U[2000,16000] per image; prior = true homography + N(0,15 px); the %d nearest "
                     "keypoints within %g px, ratio %g" % (args.pairs, W_IMG, H_IMG, KC, RADIUS, RATIO),
         "pairs_per_step_per_gpu": args.pairs, "image": [W_IMG, H_IMG], "radius_px": RADIUS, "kc": KC, "ratio": RATIO,
         "contrast": 0.015, "edge": 12.0, "distances": "exact (uint8 RootSIFT, integer dp4a)",
         "l2": "inputs larger than L2: %d images x %.1f MB per step" % (2 * args.pairs, H_IMG * W_IMG / 1e6),
         "parallelism": "replicas: independent pairs per GPU (weak scaling)"}
    if extra:
        c.update(extra)
    return c


def rank_seed(seed, rank):
    """Seed of a rank's pairs: the ranks are replicas, each extracting and matching its own pairs
    (disjoint seeds for fewer than 100000 pairs per rank); no data-path collective."""
    return seed + 100000 * rank


def max_over_ranks(ms, dist, device):
    """The slowest rank's time (a step of the whole job ends when every rank has finished)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, pairs_per_rank, ms):
    """Whole-job pairs/s: every rank's pairs over the slowest rank's time."""
    return world * pairs_per_rank / (ms / 1000.0)


def gen_pairs(n, seed):
    import multiprocessing as mp
    jobs = [(H_IMG, W_IMG, seed + i) for i in range(n)]
    from fieldstitch_b200 import synth
    workers = max(1, min(len(jobs), (os.cpu_count() or 2) - 1, 32))
    if workers == 1:
        return [synth.flight_pair(j) for j in jobs]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(synth.flight_pair, jobs)


# ------------------------------------------------------------------------------------- clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_id), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = [n for i, n in enumerate(names) if any(r[5 + i].strip() == "Active" for r in rows)]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_smi_id(torch, dev):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:  # noqa: BLE001
        return str(dev)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s)"


def pyramid_bytes(h, w):
    """Algorithmic bytes of one image's pyramid: H*W input + 44 B per octave pixel (DoG 5 x 4 B +
    gradient magnitude and angle 3 x 8 B)."""
    import math
    R, C = 2 * h, 2 * w
    budget = max(1, int(round(math.log2(min(h, w)) - 2)) + 1)
    tot = 0
    for _ in range(budget):
        if min(R, C) < 14:
            break
        tot += R * C
        R, C = (R + 1) // 2, (C + 1) // 2
    return h * w + 44 * tot


def traffic_per_pyramid():
    path = os.path.join(ROOT, "profiles", "pyramid_traffic.json")
    if os.path.exists(path):
        try:
            return json.load(open(path)).get("dram_bytes_per_image_2640x1978")
        except (ValueError, OSError):
            return None
    return None


# ------------------------------------------------------------------------------ CPU reference
def cpu_pair(pair, pidx, seed, cores):
    """One pair through the reference's CPU path (oracle port): features.sift_cpu (OpenCV SIFT) ->
    RootSIFT bytes -> prior-guided matching (NumPy + cKDTree). Returns (matches, seconds)."""
    import cv2

    from fieldstitch_b200 import synth
    from oracle import features_ref, matching_ref
    cv2.setNumThreads(cores)
    a, b, H, na, nb = pair
    t0 = time.perf_counter()
    xa, da, _, _ = features_ref.sift_cpu(a, na)
    xb, db, _, _ = features_ref.sift_cpu(b, nb)
    if da is None or db is None:
        return 0, time.perf_counter() - t0
    ua, ub = features_ref.rootsift_u8(da), features_ref.rootsift_u8(db)
    pred = synth.apply_homography(H, xa) + synth.prior_noise(len(xa), seed + pidx).astype(np.float64)
    q, _ = matching_ref.guided_from_pred(pred, ua, xb.astype(np.float64), ub, (W_IMG, H_IMG), RADIUS, KC, RATIO)
    return len(q), time.perf_counter() - t0


def _pool_task(job):
    """One pair on one process of the CPU pool (one thread per process, as one worker of the
    reference's process pool)."""
    pair, pidx, seed = job
    return cpu_pair(pair, pidx, seed, 1)


def _pool_warm(_):
    import cv2  # noqa: F401
    import scipy.spatial  # noqa: F401

    from oracle import features_ref, matching_ref  # noqa: F401
    return os.getpid()


class CpuPool:
    """The reference's CPU path run the way its pipeline runs pair work: a process pool of one
    worker per host core, one pair per task (app/planesite/pipeline.py:535-536,
    pool.imap(match_pair, pairs)); here each task extracts both images and matches them."""

    def __init__(self, workers):
        import multiprocessing as mp
        self.workers = workers
        self.pool = mp.get_context("spawn").Pool(workers)
        self.pool.map(_pool_warm, range(4 * workers), chunksize=1)   # imports done before timing

    def step(self, pairs, seed):
        """Wall-clock seconds for every pair of `pairs` through the pool."""
        t0 = time.perf_counter()
        self.pool.map(_pool_task, [(p, i, seed) for i, p in enumerate(pairs)], chunksize=1)
        return time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def run_reference(args):
    """The reference's CPU implementation of the path (oracle port) with every host core: one step
    = one pool pass over `cores` pairs of the workload (the same pairs every step)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    pairs = gen_pairs(cores, args.seed)
    pool = CpuPool(cores)
    for _ in range(args.warmup):
        pool.step(pairs, args.seed)
    times = [pool.step(pairs, args.seed) for _ in range(args.steps)]
    pool.close()
    per_step = sum(times) / len(times)
    v = len(pairs) / per_step
    line = {"metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step * 1000.0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": config(args, {"pairs_per_step_per_gpu": len(pairs)}), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port",
                             "sample": "%d pairs per step (2 images 2640x1978 + guided match each) over a pool of "
                                       "%d processes, one thread each, %d steps" % (len(pairs), cores, args.steps)},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line, default=_json_num), flush=True)
    return 0


# ---------------------------------------------------------------------------------- GPU arm
def dense_sweep(args, local):
    """Precision sweep of the exhaustive matcher (_ratio_match_bf + _unique): one batch of
    args.sweep_pairs pairs of args.sweep_n x args.sweep_n SIFT-like uint8 descriptors (30% true
    correspondences with +-4 byte noise), ratio 0.8, per precision FP32 (CUDA cores), BF16 and
    E4M3 (tcgen05). Reports pairs/s of the whole batch call, the tensor-core kernel's own time and
    TFLOP/s, the approximate-vs-exact best-distance error, the rows the certificate sent to the
    exact fallback, and whether every pair's match list equals the FP32 one."""
    import torch

    from fieldstitch_b200 import _lib, matching, synth
    dev = torch.device("cuda", local)
    n, npairs = args.sweep_n, args.sweep_pairs
    A, B = [], []
    for p in range(npairs):
        a, b, _ = synth.synth_descriptors_device(n, n, args.seed + 31 * p, device=local)
        A.append(a)
        B.append(b)
    outs = [(torch.empty(n, dtype=torch.int64, device=dev), torch.empty(n, dtype=torch.int64, device=dev))
            for _ in range(npairs)]
    ref_outs = [(torch.empty(n, dtype=torch.int64, device=dev), torch.empty(n, dtype=torch.int64, device=dev))
                for _ in range(npairs)]
    torch.cuda.synchronize()
    ctx = _lib.context(local)
    ctx.timing(True)
    flops = 2.0 * 128 * n * n * npairs
    peak_bf16 = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_bf16 = float(json.load(f)["bf16_tflops"])
        peak_src = "measured (MEASURED_PEAKS.json bf16_tflops, burst)"
    except (OSError, KeyError, ValueError):
        peak_bf16, peak_src = 1590.0, "fallback 1.59 PFLOP/s"
    peak_fp8, why = fp8_gemm_peak(dev)
    if peak_fp8:
        fp8_src = "measured live: cuBLASLt E4M3 GEMM 8192^3 (torch._scaled_mm)"
    else:
        peak_fp8, fp8_src = 2.0 * peak_bf16, peak_src + " x2 (E4M3 rate; live FP8 GEMM failed: %s)" % why
    out, ref = {}, None
    for prec in ("fp32", "bf16", "fp8"):
        o = ref_outs if prec == "fp32" else outs
        res = matching.ratio_match_bf_batch_d(A, B, 0.8, precision=prec, out=o)   # warm-up
        torch.cuda.synchronize()
        ctx.stage_times()
        steps = 2
        main = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for _ in range(steps):
            res = matching.ratio_match_bf_batch_d(A, B, 0.8, precision=prec, out=o)
        torch.cuda.synchronize()
        e1.record(main)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        st = ctx.stage_times()
        r = {"pairs_per_s": npairs / (ms / 1000.0), "ms_per_batch": ms,
             "matches": int(sum(len(q) for q, _ in res))}
        if prec == "fp32":
            ref = res
            r["distance_error_vs_fp64"] = {"max_abs": 0.0, "note": "integers < 2^24, exact in FP32"}
        else:
            ts = matching.tc_stats(local)
            kms, kn = st["tc_dense"]
            kms = kms / max(kn, 1)
            tfl = flops / (kms / 1000.0) / 1e12 if kms > 0 else None
            pk_t = peak_bf16 if prec == "bf16" else peak_fp8
            r.update({"tc_dense_ms": kms, "tc_dense_tflops": tfl, "peak_tflops": pk_t,
                      "peak_source": peak_src if prec == "bf16" else fp8_src,
                      "frac": tfl / pk_t if tfl else None,
                      "distance_error_vs_fp64": {"max_abs": ts["max_abs_err"], "mean_abs": ts["mean_abs_err"],
                                                 "of": "best squared distance per query row, approximate vs exact"},
                      "fallback_rows": ts["fallback_rows"], "rows": ts["rows"],
                      "identical_to_fp32": all(torch.equal(q, q2) and torch.equal(t, t2)
                                               for (q, t), (q2, t2) in zip(res, ref))})
        out[prec] = r
    ctx.timing(False)
    return {"workload": "%d pairs of %dx%d 128-d uint8 SIFT-like descriptors (30%% true correspondences, +-4 "
                        "byte noise), ratio 0.8, _ratio_match_bf + _unique, one batch call per step" % (npairs, n, n),
            "flops_per_batch_algorithmic": flops, **out,
            "speedup_bf16_vs_fp32": out["fp32"]["ms_per_batch"] / out["bf16"]["ms_per_batch"],
            "speedup_fp8_vs_fp32": out["fp32"]["ms_per_batch"] / out["fp8"]["ms_per_batch"]}


def fp8_gemm_peak(dev):
    """Dense E4M3 tensor-core throughput measured live (no driver-measured figure exists for it):
    cuBLASLt through torch._scaled_mm, 8192^3, per-tensor scales, BF16 out: (TFLOP/s, None) or
    (None, why not)."""
    import torch
    try:
        m = 8192
        g = torch.Generator(device=dev).manual_seed(5)
        a = torch.randn(m, m, device=dev, generator=g).to(torch.float8_e4m3fn)
        b = torch.randn(m, m, device=dev, generator=g).to(torch.float8_e4m3fn).t()   # column-major operand
        one = torch.ones((), device=dev, dtype=torch.float32)
        for _ in range(3):
            torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record()
        for _ in range(reps):
            torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        return 2.0 * m ** 3 / (ms / 1000.0) / 1e12, None
    except Exception as e:   # no FP8 GEMM in this torch / cuBLASLt: the caller falls back
        return None, ("%s: %s" % (type(e).__name__, e)).splitlines()[0][:160]


def learned_filter(args, local, pairs):
    """The learned match filter on synthetic pairs of the workload: labels from the plain pipeline's
    own RANSAC verification; train (GPU kernels) on the first 3/4 of the pairs, evaluate on the
    rest against the same verification (and, for reference, against the true homography):
    precision / recall / F1 of the ratio test vs the filter, the filter stage's throughput (BF16
    inference), and the training time."""
    import torch

    from fieldstitch_b200 import match_filter as MF
    from fieldstitch_b200 import synth
    dev = torch.device("cuda", local)
    sets = []
    for i, (a, b, H, na, nb) in enumerate(pairs):
        sets.append(MF.label_pair(a, b, H, na, nb, synth.prior_noise(16000, args.seed + 7 * i), radius=RADIUS,
                                  kc=KC, ratio=RATIO, device=local))
    ntr = max(1, (3 * len(sets)) // 4)
    train, test = sets[:ntr], sets[ntr:]
    feat = torch.cat([s["feat"][torch.from_numpy(s["has_cand"]).to(dev)] for s in train])
    lab = torch.cat([s["label"][torch.from_numpy(s["has_cand"]).to(dev)] for s in train])
    mf = MF.MatchFilter(device=local)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = mf.fit(feat, lab, epochs=30, batch=8192, lr=2e-3, seed=args.seed)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    acc = {"plain": [0.0, 0.0], "filter": [0.0, 0.0]}   # [true positives, accepted]
    acc_t = {"plain": [0.0, 0.0], "filter": [0.0, 0.0]}
    pos = pos_t = 0.0
    agree = total = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = 0.0
    for s in test:
        lh, lt = s["label_host"], s["label_true"]
        pos += lh.sum()
        pos_t += lt.sum()
        e0.record()
        qm, _ = mf.matches(s["t1"], s["b12"], s["nb"], s["feat"])
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        qm = qm.cpu().numpy()
        for k, q in (("plain", s["q_plain"]), ("filter", qm)):
            acc[k][0] += lh[q].sum()
            acc[k][1] += len(q)
            acc_t[k][0] += lt[q].sum()
            acc_t[k][1] += len(q)
        p32 = mf.predict(s["feat"], bf16=False).cpu().numpy() > 0.5
        p16 = mf.predict(s["feat"], bf16=True).cpu().numpy() > 0.5
        agree += int((p32 == p16).sum())
        total += len(p32)

    def prf(tp_n, p):
        tp, n = float(tp_n[0]), float(tp_n[1])
        p = float(p)
        prec = tp / n if n else 0.0
        rec = tp / p if p else 0.0
        return {"precision": prec, "recall": rec, "f1": 2 * tp / (n + p) if (n + p) else 0.0}

    return {"workload": "%d synthetic pairs at %dx%d (the bench's pairs): %d train / %d held out; features of every "
                        "query's best guided candidate (16 nearest within %g px); labels: the plain pipeline's RANSAC "
                        "homography (cv2, 3 px) maps the candidate within 2 px" % (len(sets), W_IMG, H_IMG, len(train),
                                                                                   len(test), RADIUS),
            "train_correspondences": int(len(lab)), "train_epochs": 30, "train_seconds": train_s,
            "loss_first_last": [float(losses[0]), float(losses[-1])],
            "vs_plain_verification": {"ratio_test": prf(acc["plain"], pos), "mlp_filter": prf(acc["filter"], pos)},
            "vs_true_homography": {"ratio_test": prf(acc_t["plain"], pos_t), "mlp_filter": prf(acc_t["filter"], pos_t)},
            "filter_stage_pairs_per_s": len(test) / (ms / 1000.0) if ms > 0 else None,
            "bf16_fp32_decision_agreement": agree / total if total else None}


def synthetic_flight(args, local):
    """Config 5: a seeded 20000 x 16000 procedural terrain, frames of 2640 x 1978 cropped from it along a
    lawnmower grid (80 % forward / 70 % side overlap, +-3 deg yaw, +-2 % scale; return lines flown at
    180 deg), the reference pipeline's GNSS neighbour pairs (16 nearest within 0.95 x the long
    footprint side, plus the next two frames), prior = true homography + N(0, 15 px).

    Batched path: every frame extracted once (sift_gpu sequence, nfeat 7000, the "accurate" preset)
    on args.streams contexts, the prior projections, then every pair's guided match in one
    fsb_match_guided_batch_d call (a CUDA graph). Plain path: one context, frames then pairs one
    after another (host waits after every call). Both from frames resident in HBM; device events and
    the host clock, the larger. The learned filter is trained on the first pairs' candidates (labels:
    the plain pipeline's RANSAC) and replaces the ratio test on every pair."""
    import ctypes
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from fieldstitch_b200 import _lib, synth
    from fieldstitch_b200 import match_filter as MF
    dev = torch.device("cuda", local)
    h, w = H_IMG, W_IMG
    t0 = time.perf_counter()
    terrain = synth.flight_terrain(args.seed + 5, device=local)
    poses = synth.lawnmower(args.seed + 6, lines=args.flight_lines, per_line=args.flight_lines)
    frames = synth.render_frames(terrain, poses, seed=args.seed + 7)
    del terrain
    torch.cuda.empty_cache()
    pairs = synth.gnss_pairs(poses, sigma=15.0, seed=args.seed + 8)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    n, P, nf = len(poses), len(pairs), 7000
    prm = _lib.SiftParams(0.015, 12.0, 0, 0)

    def Pt(t):
        return ctypes.c_void_p(t.data_ptr())

    xy = torch.empty((n, nf, 2), dtype=torch.float32, device=dev)
    rs = torch.empty((n, nf), dtype=torch.float32, device=dev)
    u8 = torch.empty((n, nf, 128), dtype=torch.uint8, device=dev)
    sz = torch.empty((n, nf), dtype=torch.float32, device=dev)
    an = torch.empty((n, nf), dtype=torch.float32, device=dev)
    oc = torch.empty((n, nf), dtype=torch.int32, device=dev)
    bxy = torch.empty((n, nf, 2), dtype=torch.float64, device=dev)
    pred = torch.empty((P, nf, 2), dtype=torch.float64, device=dev)
    g = torch.Generator(device=dev).manual_seed(args.seed + 9)
    noise = (15.0 * torch.randn((P, nf, 2), generator=g, device=dev)).to(torch.float32)
    q_b = torch.empty((P, nf), dtype=torch.int64, device=dev)
    t_b = torch.empty((P, nf), dtype=torch.int64, device=dev)
    Hs = [np.ascontiguousarray(synth.frame_homography(poses[i], poses[j]).reshape(9)) for i, j in pairs]
    eye = np.eye(3).reshape(9).copy()
    nk = [0] * n
    by_first = [[] for _ in range(n)]
    for p, (i, _) in enumerate(pairs):
        by_first[i].append(p)
    S = args.streams
    ctxs = [_lib.Context(local) for _ in range(S)]
    mctx = _lib.Context(local)
    pool = ThreadPoolExecutor(max_workers=S)

    def extract_frames(k):
        c = ctxs[k]
        L, cnt = c.lib, ctypes.c_int32()
        for i in range(k, n, S):
            _lib.check(L.fsb_sift_features_ex_d(c.handle, Pt(frames[i]), h, w, w, ctypes.byref(prm), nf, Pt(xy[i]),
                                                Pt(rs[i]), None, Pt(u8[i]), Pt(sz[i]), Pt(an[i]), Pt(oc[i]),
                                                ctypes.byref(cnt)), "sift")
            nk[i] = cnt.value
            _lib.check(L.fsb_project_d(c.handle, Pt(xy[i]), nk[i], _lib.ptr(eye), None, Pt(bxy[i])), "proj")
            for p in by_first[i]:
                _lib.check(L.fsb_project_d(c.handle, Pt(xy[i]), nk[i], _lib.ptr(Hs[p]), Pt(noise[p]), Pt(pred[p])),
                           "proj")

    Pv, Iv, Dv = ctypes.c_void_p * P, ctypes.c_int32 * P, ctypes.c_double * P
    counts = Iv()

    def match_all():
        _lib.check(mctx.lib.fsb_match_guided_batch_d(
            mctx.handle, P, Pv(*[pred[p].data_ptr() for p in range(P)]), Pv(*[u8[i].data_ptr() for i, _ in pairs]),
            Iv(*[nk[i] for i, _ in pairs]), Pv(*[bxy[j].data_ptr() for _, j in pairs]),
            Pv(*[u8[j].data_ptr() for _, j in pairs]), Iv(*[nk[j] for _, j in pairs]), Dv(*([float(w)] * P)),
            Dv(*([float(h)] * P)), RADIUS, KC, RATIO, Pv(*[q_b[p].data_ptr() for p in range(P)]),
            Pv(*[t_b[p].data_ptr() for p in range(P)]), counts), "guided batch")

    def batched():
        for f in [pool.submit(extract_frames, k) for k in range(S)]:
            f.result()
        match_all()

    def clocked(fn, streams):
        """(ms, result): device events bracketing every stream, and the host clock; the larger."""
        main = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(main)
        for st in streams:
            st.wait_event(e0)
        out = fn()
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        torch.cuda.synchronize()
        return max(e0.elapsed_time(e1), (time.perf_counter() - w0) * 1000.0), out

    streams = [torch.cuda.ExternalStream(c.stream()) for c in ctxs + [mctx]]
    batched()   # warm-up: workspaces, autotuning of the frame geometry, the match graph's capture
    torch.cuda.synchronize()
    ms_batched, _ = clocked(batched, streams)
    got = [(q_b[p, :counts[p]].clone(), t_b[p, :counts[p]].clone()) for p in range(P)]

    # ---- plain path: one context, one call at a time
    pc = ctxs[0]
    L, cnt = pc.lib, ctypes.c_int32()
    q_p = torch.empty(nf, dtype=torch.int64, device=dev)
    t_p = torch.empty(nf, dtype=torch.int64, device=dev)
    same = [True]

    def plain():
        for i in range(n):
            _lib.check(L.fsb_sift_features_ex_d(pc.handle, Pt(frames[i]), h, w, w, ctypes.byref(prm), nf, Pt(xy[i]),
                                                Pt(rs[i]), None, Pt(u8[i]), Pt(sz[i]), Pt(an[i]), Pt(oc[i]),
                                                ctypes.byref(cnt)), "sift")
            nk[i] = cnt.value
            _lib.check(L.fsb_project_d(pc.handle, Pt(xy[i]), nk[i], _lib.ptr(eye), None, Pt(bxy[i])), "proj")
        for p, (i, j) in enumerate(pairs):
            _lib.check(L.fsb_project_d(pc.handle, Pt(xy[i]), nk[i], _lib.ptr(Hs[p]), Pt(noise[p]), Pt(pred[p])),
                       "proj")
            _lib.check(L.fsb_match_guided_d(pc.handle, Pt(pred[p]), Pt(u8[i]), nk[i], Pt(bxy[j]), Pt(u8[j]), nk[j],
                                            float(w), float(h), RADIUS, KC, RATIO, Pt(q_p), Pt(t_p),
                                            ctypes.byref(cnt)), "guided")
            m = cnt.value
            same[0] = same[0] and m == len(got[p][0]) and torch.equal(q_p[:m], got[p][0]) and \
                torch.equal(t_p[:m], got[p][1])

    ms_plain, _ = clocked(plain, [torch.cuda.ExternalStream(pc.stream())])

    # ---- correctness of the batched matches against the true homographies
    n_match = n_good = pairs_ok = 0
    xy_h = xy.cpu().numpy()
    for p, (i, j) in enumerate(pairs):
        q, t = got[p][0].cpu().numpy(), got[p][1].cpu().numpy()
        if len(q) == 0:
            continue
        proj = synth.apply_homography(Hs[p].reshape(3, 3), xy_h[i][q])
        good = np.linalg.norm(proj - xy_h[j][t], axis=1) < 3.0
        n_match += len(q)
        n_good += int(good.sum())
        pairs_ok += int(good.sum() >= 20)

    # ---- learned filter: trained on the first pairs' candidates, applied to every pair
    def frame_dict(i):
        k = nk[i]
        return {"xy": xy[i, :k], "resp": rs[i, :k], "u8": u8[i, :k], "size": sz[i, :k], "angle": an[i, :k],
                "octave": oc[i, :k]}

    n_train = min(args.flight_train, P)
    feats, labs = [], []
    for p in range(n_train):
        i, j = pairs[p]
        A, B = frame_dict(i), frame_dict(j)
        pr = pred[p, :nk[i]]
        t1, b12 = MF.candidates(pr, A, B, (w, h), RADIUS, KC, local)
        ft = MF.features(t1, b12, pr, A, B, RADIUS, local)
        q, t = MF.accept(t1, b12, nk[j], None, ratio=RATIO, device=local)
        t1h = t1.cpu().numpy()
        lab, _ = MF.ransac_labels(xy_h[i][:nk[i]].astype(np.float64), xy_h[j][:nk[j]].astype(np.float64),
                                  q.cpu().numpy(), t.cpu().numpy(), t1h)
        ok = torch.from_numpy(t1h >= 0).to(dev)
        feats.append(ft[ok])
        labs.append(torch.from_numpy(lab).to(dev)[ok])
    mf = MF.MatchFilter(device=local)
    train_feat, train_lab = torch.cat(feats), torch.cat(labs)
    torch.cuda.synchronize()
    t_fit = time.perf_counter()
    mf.fit(train_feat, train_lab, epochs=30, batch=8192, lr=2e-3, seed=args.seed)
    torch.cuda.synchronize()
    fit_s = time.perf_counter() - t_fit

    acc = {"ratio_test": [0, 0], "mlp_filter": [0, 0]}
    pos = 0

    def filter_all(evaluate):
        nonlocal pos
        for p, (i, j) in enumerate(pairs):
            A, B = frame_dict(i), frame_dict(j)
            pr = pred[p, :nk[i]]
            t1, b12 = MF.candidates(pr, A, B, (w, h), RADIUS, KC, local)
            ft = MF.features(t1, b12, pr, A, B, RADIUS, local)
            qf, tf = mf.matches(t1, b12, nk[j], ft)
            if evaluate and p >= n_train:
                t1h = t1.cpu().numpy()
                okc = t1h >= 0
                truth = np.zeros(nk[i], bool)
                if okc.any():
                    proj = synth.apply_homography(Hs[p].reshape(3, 3), xy_h[i][:nk[i]][okc])
                    truth[okc] = np.linalg.norm(proj - xy_h[j][t1h[okc]], axis=1) < 3.0
                pos += int(truth.sum())
                qr = got[p][0].cpu().numpy()
                for key, qq in (("ratio_test", qr), ("mlp_filter", qf.cpu().numpy())):
                    acc[key][0] += int(truth[qq].sum())
                    acc[key][1] += len(qq)

    filter_all(True)
    ms_filter, _ = clocked(lambda: filter_all(False), [torch.cuda.ExternalStream(_lib.context(local).stream())])

    def prf(k):
        tp, m = acc[k]
        return {"precision": tp / m if m else 0.0, "recall": tp / pos if pos else 0.0,
                "f1": 2 * tp / (m + pos) if (m + pos) else 0.0}

    pool.shutdown()
    for c in ctxs + [mctx]:
        c.close()
    del frames
    torch.cuda.empty_cache()
    return {"workload": "synthetic flight: %d frames %dx%d cropped from a seeded 20000x16000 terrain on a %dx%d "
                        "lawnmower grid (80%%/70%% overlap, +-3 deg yaw, +-2%% scale), %d GNSS neighbour pairs "
                        "(pipeline.py:452-476 rule, 16 neighbours), nfeat 7000, prior = true homography + "
                        "N(0, 15 px), the %d nearest within %g px, ratio %g"
                        % (n, w, h, args.flight_lines, args.flight_lines, P, KC, RADIUS, RATIO),
            "frames": n, "pairs": P, "generate_s": gen_s,
            "batched": {"ms": ms_batched, "pairs_per_s": P / (ms_batched / 1000.0), "streams": S,
                        "path": "frames extracted once on %d contexts + projections + one guided-batch graph" % S},
            "plain_fp32": {"ms": ms_plain, "pairs_per_s": P / (ms_plain / 1000.0),
                           "path": "one context, frames then pairs one call at a time"},
            "batched_over_plain": ms_plain / ms_batched,
            "identical_matches_batched_vs_plain": bool(same[0]),
            "matches": {"total": n_match, "within_3px_of_truth": n_good,
                        "pairs_with_20_correct": pairs_ok, "precision_vs_truth": n_good / n_match if n_match else 0.0},
            "learned_filter": {"train_pairs": n_train, "held_out_pairs": P - n_train,
                               "train_correspondences": int(len(train_lab)), "train_seconds": fit_s,
                               "labels": "the plain pipeline's RANSAC homography (cv2, 3 px) of the ratio-test matches",
                               "vs_true_homography": {"ratio_test": prf("ratio_test"), "mlp_filter": prf("mlp_filter")},
                               "filter_path_ms": ms_filter,
                               "e2e_with_filter_pairs_per_s": P / ((ms_batched + ms_filter) / 1000.0),
                               "path": "per pair: guided candidates, features, BF16 inference, accept (one stream)"},
            "precision": "distances are exact integers (uint8 RootSIFT): FP32, BF16 and FP8 give the same matches; "
                         "the extraction is float32"}


def run_fsb(args):
    import ctypes
    from concurrent.futures import ThreadPoolExecutor

    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pairs = gen_pairs(args.pairs, rank_seed(args.seed, rank))   # before any CUDA work
    cpu_pool = CpuPool(os.cpu_count() or 1) if rank == 0 and world == 1 and not args.no_cpu else None
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    import fieldstitch_b200 as F
    from fieldstitch_b200 import _lib, synth
    dev = torch.device("cuda", local)
    h, w = H_IMG, W_IMG
    nmax = 16000
    # device-resident inputs and per-pair prior errors
    d_img = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _, _, _ in pairs]
    d_noise = [torch.from_numpy(synth.prior_noise(nmax, args.seed + 7 * i)).to(dev) for i in range(len(pairs))]
    eye = np.eye(3).reshape(9).copy()
    Hs = [np.ascontiguousarray(p[2].reshape(9)) for p in pairs]
    prm = _lib.SiftParams(0.015, 12.0, 0, 0)

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    class Worker:
        """One context (stream + workspaces) and its output buffers; runs the pairs i = idx mod n."""

        def __init__(self, idx, n):
            self.items = list(range(idx, len(pairs), n))
            self.ctx = _lib.Context(local)
            self.L = self.ctx.lib
            self.stream = torch.cuda.ExternalStream(self.ctx.stream())
            self.xy = [torch.empty((nmax, 2), dtype=torch.float32, device=dev) for _ in range(2)]
            self.rs = [torch.empty(nmax, dtype=torch.float32, device=dev) for _ in range(2)]
            self.u8 = [torch.empty((nmax, 128), dtype=torch.uint8, device=dev) for _ in range(2)]
            self.pred = torch.empty((nmax, 2), dtype=torch.float64, device=dev)
            self.bxy = torch.empty((nmax, 2), dtype=torch.float64, device=dev)
            self.dq = torch.empty(nmax, dtype=torch.int64, device=dev)
            self.dt = torch.empty(nmax, dtype=torch.int64, device=dev)
            self.n_out = ctypes.c_int32()

        def extract(self, items=None):
            """SIFT of both images and the prior projections of the pairs, into the per-pair buffers
            that the batched guided match reads."""
            L, c, n_out = self.L, self.ctx.handle, self.n_out
            for i in (self.items if items is None else items):
                ia, ib = d_img[i]
                B = pb[i]
                for k, (img, nf) in enumerate(((ia, pairs[i][3]), (ib, pairs[i][4]))):
                    _lib.check(L.fsb_sift_features_d(c, P(img), h, w, w, ctypes.byref(prm), nf, P(B["xy"][k]),
                                                     P(B["rs"][k]), None, P(B["u8"][k]), ctypes.byref(n_out)), "sift")
                    B["n"][k] = n_out.value
                _lib.check(L.fsb_project_d(c, P(B["xy"][0]), B["n"][0], _lib.ptr(Hs[i]), P(d_noise[i]), P(B["pred"])),
                           "proj")
                _lib.check(L.fsb_project_d(c, P(B["xy"][1]), B["n"][1], _lib.ptr(eye), None, P(B["bxy"])), "proj")
            return 0

        def run(self, items=None):
            """The plain per-pair sequence: SIFT A, SIFT B, projections, guided match of this pair."""
            L, c, n_out = self.L, self.ctx.handle, self.n_out
            matches = 0
            for i in (self.items if items is None else items):
                ia, ib = d_img[i]
                n = []
                for k, (img, nf) in enumerate(((ia, pairs[i][3]), (ib, pairs[i][4]))):
                    _lib.check(L.fsb_sift_features_d(c, P(img), h, w, w, ctypes.byref(prm), nf, P(self.xy[k]),
                                                     P(self.rs[k]), None, P(self.u8[k]), ctypes.byref(n_out)), "sift")
                    n.append(n_out.value)
                _lib.check(L.fsb_project_d(c, P(self.xy[0]), n[0], _lib.ptr(Hs[i]), P(d_noise[i]), P(self.pred)),
                           "proj")
                _lib.check(L.fsb_project_d(c, P(self.xy[1]), n[1], _lib.ptr(eye), None, P(self.bxy)), "proj")
                _lib.check(L.fsb_match_guided_d(c, P(self.pred), P(self.u8[0]), n[0], P(self.bxy), P(self.u8[1]), n[1],
                                                float(w), float(h), RADIUS, KC, RATIO, P(self.dq), P(self.dt),
                                                ctypes.byref(n_out)), "guided")
                matches += n_out.value
            return matches

    # per-pair device buffers for the batched match
    pb = [{"xy": [torch.empty((nmax, 2), dtype=torch.float32, device=dev) for _ in range(2)],
           "rs": [torch.empty(nmax, dtype=torch.float32, device=dev) for _ in range(2)],
           "u8": [torch.empty((nmax, 128), dtype=torch.uint8, device=dev) for _ in range(2)],
           "pred": torch.empty((nmax, 2), dtype=torch.float64, device=dev),
           "bxy": torch.empty((nmax, 2), dtype=torch.float64, device=dev),
           "q": torch.empty(nmax, dtype=torch.int64, device=dev), "t": torch.empty(nmax, dtype=torch.int64, device=dev),
           "n": [0, 0]} for _ in pairs]
    workers = [Worker(i, args.streams) for i in range(args.streams)]
    pool = ThreadPoolExecutor(max_workers=args.streams)
    mctx = _lib.Context(local)   # the batched match's context (stream)
    mstream = torch.cuda.ExternalStream(mctx.stream())
    NPs = len(pairs)
    Pv, Iv, Dv = ctypes.c_void_p * NPs, ctypes.c_int32 * NPs, ctypes.c_double * NPs
    m_cnt = Iv()

    def match_batch():
        """Every pair's guided match in one call (one CUDA graph, replayed from the second step)."""
        _lib.check(mctx.lib.fsb_match_guided_batch_d(
            mctx.handle, NPs, Pv(*[b["pred"].data_ptr() for b in pb]), Pv(*[b["u8"][0].data_ptr() for b in pb]),
            Iv(*[b["n"][0] for b in pb]), Pv(*[b["bxy"].data_ptr() for b in pb]),
            Pv(*[b["u8"][1].data_ptr() for b in pb]), Iv(*[b["n"][1] for b in pb]), Dv(*([float(w)] * NPs)),
            Dv(*([float(h)] * NPs)), RADIUS, KC, RATIO, Pv(*[b["q"].data_ptr() for b in pb]),
            Pv(*[b["t"].data_ptr() for b in pb]), m_cnt), "guided batch")
        return sum(m_cnt[i] for i in range(NPs))

    # the step's extraction as one sync-free batch: every image in one fsb_sift_features_batch_d call
    # (one CUDA graph, args.chains images in flight), then every pair's prior projections queued
    # with one call on the match context
    ectx = _lib.Context(local)
    estream = torch.cuda.ExternalStream(ectx.stream())
    NI = 2 * NPs
    Pi, Ii = ctypes.c_void_p * NI, ctypes.c_int32 * NI
    e_imgs = Pi(*[d_img[i][k].data_ptr() for i in range(NPs) for k in range(2)])
    e_nf = Ii(*[pairs[i][3 + k] for i in range(NPs) for k in range(2)])
    e_xy = Pi(*[pb[i]["xy"][k].data_ptr() for i in range(NPs) for k in range(2)])
    e_rs = Pi(*[pb[i]["rs"][k].data_ptr() for i in range(NPs) for k in range(2)])
    e_u8 = Pi(*[pb[i]["u8"][k].data_ptr() for i in range(NPs) for k in range(2)])
    e_dcnt = torch.empty(NI, dtype=torch.int32, device=dev)
    e_hcnt = Ii()
    p_hm = np.ascontiguousarray(np.concatenate([np.concatenate([Hs[i], eye]) for i in range(NPs)]))
    p_off = Pi(*[v for i in range(NPs) for v in (d_noise[i].data_ptr(), None)])
    p_out = Pi(*[v for i in range(NPs) for v in (pb[i]["pred"].data_ptr(), pb[i]["bxy"].data_ptr())])

    def extract_graph():
        _lib.check(ectx.lib.fsb_sift_features_batch_d(ectx.handle, NI, e_imgs, h, w, w, ctypes.byref(prm), e_nf, e_xy,
                                                      e_rs, e_u8, ctypes.c_void_p(e_dcnt.data_ptr()), e_hcnt,
                                                      args.chains), "sift batch")
        for i in range(NPs):
            pb[i]["n"] = [e_hcnt[2 * i], e_hcnt[2 * i + 1]]
        _lib.check(mctx.lib.fsb_project_batch_d(mctx.handle, NI, e_xy, e_hcnt, _lib.ptr(p_hm), p_off, p_out), "proj")

    def one_step():
        if args.extract == "graph":
            extract_graph()
        else:
            for f in [pool.submit(wk.extract) for wk in workers]:
                f.result()
        return match_batch()

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(fn, steps):
        """Device time of `steps` calls of fn: start event on the current stream, every worker
        stream waits on it; every worker stream records its end, the current stream waits on all."""
        main = torch.cuda.current_stream(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(main)
        for wk in workers:
            wk.stream.wait_event(e0)
        mstream.wait_event(e0)
        estream.wait_event(e0)
        out = 0
        for _ in range(steps):
            out += fn()
        for st in [wk.stream for wk in workers] + [mstream, estream]:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, out

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    barrier()
    for c_ in [wk.ctx for wk in workers] + [mctx, ectx]:
        c_.timing(True)
        c_.stage_times()
    clocks = Clocks(gpu_smi_id(torch, local))
    launches0 = _lib.launch_count()
    ms_step, matches = timed(one_step, args.steps)
    clk = clocks.stop()
    launches = _lib.launch_count() - launches0
    stages = {}
    for c_ in [wk.ctx for wk in workers] + [mctx, ectx]:
        for k_, (ms_, n_) in c_.stage_times().items():
            a_, b_ = stages.get(k_, (0.0, 0))
            stages[k_] = (a_ + ms_, b_ + n_)
        c_.timing(False)
    if dist is not None:
        ms_step = max_over_ranks(ms_step, dist, dev)
        barrier()
    value = job_rate(world, args.pairs, ms_step)

    # ---- parity of the timed steps' output (outside the timed region): the last step's batched
    # guided matches of two pairs against the oracle's guided matcher (NumPy / cKDTree, the
    # reference's _guided restated) run on the GPU's own keypoints, descriptors and predictions
    parity = {"pairs": [], "parity_checked": False}
    try:
        from oracle import matching_ref
        torch.cuda.synchronize()
        ok = True
        for i in range(min(2, len(pairs))):
            B = pb[i]
            na_, nb_ = B["n"]
            pred = B["pred"][:na_].cpu().numpy()
            ua = B["u8"][0][:na_].cpu().numpy()
            bxy = B["bxy"][:nb_].cpu().numpy()
            ub = B["u8"][1][:nb_].cpu().numpy()
            n_ = m_cnt[i]
            q_g, t_g = B["q"][:n_].cpu().numpy(), B["t"][:n_].cpu().numpy()
            q_ref, t_ref = matching_ref.guided_from_pred(pred, ua, bxy, ub, (w, h), RADIUS, KC, RATIO, ties="index")
            same = bool(np.array_equal(q_g, q_ref) and np.array_equal(t_g, t_ref))
            q_kd, t_kd = matching_ref.guided_from_pred(pred, ua, bxy, ub, (w, h), RADIUS, KC, RATIO)
            shared = len(set(zip(q_g.tolist(), t_g.tolist())) & set(zip(q_kd.tolist(), t_kd.tolist())))
            ok = ok and same
            parity["pairs"].append({"pair": i, "keypoints": [int(na_), int(nb_)], "matches_gpu": int(n_),
                                    "matches_oracle": int(len(q_ref)), "identical": same,
                                    "matches_oracle_kdtree_ties": int(len(q_kd)), "shared_with_kdtree_ties": shared})
        parity["parity_checked"] = ok
        parity["what"] = ("the batched guided matches of pairs 0 and 1 of the last timed step equal the oracle's "
                          "guided matcher on the same keypoints, descriptors and predictions, equal-distance "
                          "candidates at the kc-th place taken by index as the device does (with cKDTree's own "
                          "order among them the shared count is reported beside)")
    except Exception as e:  # reported in the line, never hidden
        parity["error"] = ("%s: %s" % (type(e).__name__, e))[:200]

    # ---- e2e through the public host API (host buffers, copies inside the timed region)
    e2e = None
    if not args.no_e2e:
        # the step's input images in pinned host memory (numpy views of pinned torch tensors)
        def pinned(x):
            t = torch.empty(x.shape, dtype=torch.uint8, pin_memory=True)
            t.numpy()[...] = x
            return t

        host_t = [(pinned(a), pinned(b)) for a, b, _, _, _ in pairs]
        # the synthetic prior error (GNSS / gimbal stand-in) is input data, drawn before timing
        noise = [synth.prior_noise(nmax, args.seed + 7 * i).astype(np.float64) for i in range(len(pairs))]
        host = [(ta.numpy(), tb.numpy()) for ta, tb in host_t]

        def e2e_pair(i):
            a, b = host[i]
            xa, ua, _ = F.features.sift_gpu_u8(a, pairs[i][3], device=local)
            xb, ub, _ = F.features.sift_gpu_u8(b, pairs[i][4], device=local)
            pr = synth.apply_homography(pairs[i][2], xa) + noise[i][:len(xa)]
            q, _ = F.matching.guided_from_pred(pr, ua, xb.astype(np.float64), ub, (w, h), RADIUS, KC, RATIO,
                                               device=local)
            h2d = a.nbytes + b.nbytes + pr.nbytes + ua.nbytes + 16 * len(xb) + ub.nbytes
            d2h = (len(xa) + len(xb)) * (8 + 4 + 128) + 16 * len(q) + 16
            return h2d, d2h

        def e2e_step_threads():
            res = list(pool.map(e2e_pair, range(len(pairs))))
            return sum(r[0] for r in res), sum(r[1] for r in res)

        x_imgs = [im for a, b in host for im in (a, b)]
        e_nfs = [pairs[i][3 + k] for i in range(len(pairs)) for k in range(2)]
        e_pairs = [(2 * i, 2 * i + 1) for i in range(len(pairs))]
        e_priors = [pairs[i][2] for i in range(len(pairs))]
        e_off = [noise[i].astype(np.float32) for i in range(len(pairs))]

        def e2e_step_batch():
            """frontend.extract_and_match: the step's host images to the device, one graph extracting
            every image, the priors projected on the device, one graph matching every pair, the match
            lists back to the host."""
            res = F.frontend.extract_and_match(x_imgs, e_nfs, e_pairs, e_priors, RADIUS, KC, RATIO, offsets=e_off,
                                               chains=args.chains, device=local)
            h2d = sum(im.nbytes for im in x_imgs) + 16 * len(e_pairs) * max(e_nfs) + 72 * len(e_pairs)
            d2h = sum(16 * len(q) for q, _ in res) + 4 * len(x_imgs)
            return h2d, d2h

        e2e_step = e2e_step_batch if args.extract == "graph" else e2e_step_threads

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        ksteps = max(2, args.steps)
        f0 = time.perf_counter()
        main = torch.cuda.current_stream(dev)
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(main)
        h2d = d2h = 0
        for _ in range(ksteps):
            h2d, d2h = e2e_step()
        # the host API returns only after its results are in host memory, so the device is idle
        # here; the device-side events bracket the whole region on the synchronised device
        torch.cuda.synchronize()
        g1.record(main)
        torch.cuda.synchronize()
        ms_e2e = max(g0.elapsed_time(g1), (time.perf_counter() - f0) * 1000.0) / ksteps
        ms_e2e = max_over_ranks(ms_e2e, dist, dev)
        e2e = {"value": job_rate(world, args.pairs, ms_e2e), "unit": "pairs/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e, "steps": ksteps,
               "api": ("frontend.extract_and_match: host images in, one graph for every image, priors projected "
                       "on the device, one graph for every pair, match lists out" if args.extract == "graph" else
                       "features.sift_gpu_u8 + matching.guided_from_pred, %d host threads" % args.streams),
               "host_inputs": ("images in pinned host memory, the prior homographies and their errors in host "
                               "memory; the features stay on the device between extraction and matching"
                               if args.extract == "graph" else
                               "images in pinned host memory; keypoints / descriptors between the two calls in "
                               "the numpy arrays the API returns")}

    # ---- roofline of the dominant stage (pyramid), in the configuration the extraction graph runs
    # it: the pyramids of the step's images alone as one graph (fsb_pyramid_batch_d, args.chains
    # images in flight), CUDA events on the extraction context's stream around 3 replays
    def pyr_batch():
        _lib.check(ectx.lib.fsb_pyramid_batch_d(ectx.handle, NI, e_imgs, h, w, w, 0, args.chains), "pyramid batch")

    pyr_batch()
    pyr_batch()
    torch.cuda.synchronize()
    pb0, pb1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pyr_reps = 3
    pb0.record(estream)
    for _ in range(pyr_reps):
        pyr_batch()
    pb1.record(estream)
    torch.cuda.synchronize()
    pyr_batch_ms = pb0.elapsed_time(pb1) / (pyr_reps * NI)
    # and one image at a time on one stream (the latency of one image's launch chain; octaves 3-8
    # are launch-latency bound there)
    iso = workers[0]
    iso.run(items=[0])   # the context's first pair sizes its buffers; not timed
    torch.cuda.synchronize()
    iso.ctx.timing(True)
    iso.ctx.stage_times()
    iso.run(items=list(range(min(4, len(pairs)))))
    iso_st = iso.ctx.stage_times()
    iso.ctx.timing(False)
    pk, pk_src = peaks()
    pyr_ms, pyr_n = iso_st["pyramid"]
    per_img_ms = pyr_ms / max(pyr_n, 1)
    alg = pyramid_bytes(h, w)
    achieved = alg / (pyr_batch_ms / 1000.0) / 1e9 if pyr_batch_ms > 0 else None
    ach_one = alg / (per_img_ms / 1000.0) / 1e9 if per_img_ms > 0 else None
    roof = {"bound": "hbm", "kernel": "pyramid of one image (base + per octave the per-layer kernels or the fused "
                                      "layer groups, autotuned)",
            "achieved": achieved, "peak": pk, "peak_source": pk_src, "unit": "GB/s",
            "frac": (achieved / pk) if achieved else None, "traffic": traffic_per_pyramid(),
            "algorithmic_bytes": alg, "ms_per_launch_group": pyr_batch_ms,
            "measured": ("CUDA events on the extraction stream around %d replays of the pyramid stage of the step's "
                         "%d images as one graph (fsb_pyramid_batch_d, %d in flight: the configuration of the "
                         "extraction graph); time per image" % (pyr_reps, NI, args.chains)),
            "one_stream": {"achieved": ach_one, "frac": (ach_one / pk) if ach_one else None,
                           "ms_per_launch_group": per_img_ms,
                           "measured": "CUDA events on the library stream, one image at a time on one stream, "
                                       "%d images (includes the launch-chain latency of octaves 3-8)" % pyr_n}}
    n_iso = max(pyr_n, 1)
    iso_stages = {k: v[0] / n_iso for k, v in iso_st.items() if v[1] > 0}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = os.cpu_count() or 1
        n_cpu = 2
        ts = [cpu_pair(pairs[i], i, args.seed, cores)[1] for i in range(n_cpu)]
        pool_pairs = pairs[:min(len(pairs), cores)]
        pool_s = cpu_pool.step(pool_pairs, args.seed) if cpu_pool is not None else None
        cpu = {"value": len(pool_pairs) / pool_s if pool_s else n_cpu / sum(ts), "unit": "pairs/s", "cores": cores,
               "kind": "port",
               "sample": "%d pairs of the same workload (OpenCV SIFT as features.sift_cpu + NumPy/cKDTree guided "
                         "match) over a pool of %d processes, one thread each, one pair per task (as the "
                         "reference's pipeline pool runs pairs)" % (len(pool_pairs), cores),
               "serial": {"value": n_cpu / sum(ts), "unit": "pairs/s", "threads": cores,
                          "sample": "%d pairs one after another in one process, OpenCV on %d threads" % (n_cpu, cores)}}
        cpu_pool.close()

    # ---- the plain sequential path: one context (one stream), one pair at a time
    plain = None
    if args.plain_pairs > 0:
        wk = workers[0]
        items = list(range(min(args.plain_pairs, len(pairs))))
        wk.run(items[:1])
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(wk.stream)
        wk.run(items)
        p1.record(wk.stream)
        torch.cuda.synchronize()
        ms_plain = p0.elapsed_time(p1)
        plain = {"value": len(items) / (ms_plain / 1000.0), "unit": "pairs/s", "pairs": len(items),
                 "path": "one context / stream, pairs one after another, host waits after every call",
                 "batched_over_plain": value / (len(items) / (ms_plain / 1000.0))}

    sweep = None
    if rank == 0 and args.sweep_pairs > 0:
        sweep = dense_sweep(args, local)
    flight = None
    if rank == 0 and args.flight_lines > 0:
        flight = synthetic_flight(args, local)
    filt = None
    if rank == 0 and args.filter_pairs > 0:
        fp = pairs[:args.filter_pairs]
        if args.filter_pairs > len(pairs):
            fp = pairs + gen_pairs(args.filter_pairs - len(pairs), args.seed + 500000)
        filt = learned_filter(args, local, fp)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": config(args, {"host_streams": args.streams, "extraction": (
                                            "every image of a step in one fsb_sift_features_batch_d call (one CUDA "
                                            "graph, %d images in flight, no host wait inside)" % args.chains
                                            if args.extract == "graph" else
                                            "fsb_sift_features_d per image on %d host threads" % args.streams),
                                        "matching": "every pair of a step in one fsb_match_guided_batch_d call "
                                                    "(one CUDA graph, captured once, replayed each step)"}),
                "clocks": clk, "e2e": e2e, "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
                "parity_checked": parity["parity_checked"], "parity": parity,
                "matches_per_step": matches / args.steps, "plain_single_stream": plain,
                "dense_precision_sweep": sweep, "learned_filter": filt, "synthetic_flight": flight,
                "stages_ms_per_step_summed_over_streams": {k: v[0] / args.steps for k, v in stages.items()},
                "stages_ms_per_image_one_stream": iso_stages}
        print(json.dumps(line, default=_json_num), flush=True)
    pool.shutdown()
    for wk in workers:
        wk.ctx.close()
    mctx.close()
    ectx.close()
    if dist is not None:
        barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_fsb(args)


if __name__ == "__main__":
    sys.exit(main())
