#!/usr/bin/env python
"""Benchmark of CURFIL's random-forest training and prediction hot path on B200.

Headline workload (the batching training configuration): 1000 seeded synthetic RGB-D frames 640x480
(40 Voronoi cells, 40 classes, uint8 colour, uint16 depth with 10% holes), 8000 class-uniform samples
per image (8 M per tree; samplesPerImage 80000 divided over 10 trees as RandomForestImage::train
does), trees to depth 25 breadth-first, 4000 candidate features x 32 thresholds per level,
minSampleCount 1, offsets <= 60, boxes <= 15.

A full tree of this configuration takes about half a minute, so a timed step is ONE LEVEL of the
tree, trained from that level's captured input state exactly as the training loop trains it:
candidate generation, the level-batched split search over all open nodes in one persistent launch,
and routing into the next level's sample lists. The steps cycle through levels 1, 8, 16 and 24 of
tree 0 (1, 128, ~7800 and ~9600 open nodes; 8 M samples each), so every 4 steps cover the four
levels once. The tree itself is trained once before timing (its device time is reported too).
Metric: feature evaluations per second (one evaluation = one (sample, candidate feature) response
binned against all 32 thresholds).

Reported beside it:
- `per_node`: the same four levels with the plain per-node split search (the reference's structure:
  responses to HBM, one block per (threshold, feature), score kernel, host argmax, node by node),
  splits checked identical;
- `e2e`: the same levels through the host-buffer entry points (candidate generation and
  evaluateBestSplits from pinned host samples, splits back to the host);
- `cpu_baseline`: the reference's CPU split search (FeatureEvaluationCPU + calculateScores + argmax,
  restated in the oracle, OpenMP on all host cores) on a bounded sample of the workload;
- `config2` (200 frames, 3 trees depth 20, 2000 x 20), `config1` (16 frames 320x240, one tree, GPU
  and CPU trees compared), `predict` (10-tree forest, 64 frames 640x480: batched, plain per-image,
  CUDA graph from host frames, CPU prediction) and `serving` (Poisson streams of mixed sizes).
Under torchrun every rank trains its own tree (tree id = rank): trees are independent, no collective
on the data path.
"""
import argparse
import json
import os
import queue
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 2026
# headline: the batching training configuration
C3 = dict(images=1000, width=640, height=480, cells=40, classes=40, samples_per_image=80000, trees=10,
          max_depth=25, features=4000, thresholds=32, min_samples=1, box_radius=60, region_size=15)
LEVELS = (1, 8, 16, 24)
# the plain-method full-size configuration (also the training settings of the prediction forest)
C2 = dict(images=200, width=640, height=480, cells=40, classes=40, samples_per_image=4000, trees=3, max_depth=20,
          features=2000, thresholds=20, min_samples=50, box_radius=60, region_size=15)
# the plain-method small configuration: 8 classes, class 0 void (ignored), 500 samples per class and image
C1 = dict(images=16, width=320, height=240, cells=12, classes=8, samples_per_image=3500, trees=1, max_depth=12,
          features=500, thresholds=20, min_samples=1, box_radius=60, region_size=15, predict_images=4)
# batched prediction: 64 frames 640x480 through a 10-tree depth-20 forest trained as in C2
C4 = dict(images=64, trees=10)
# serving: Poisson arrivals of mixed frame sizes (weights 1:2:4:1) at these offered rates
SERVE_RATES = (200, 1000, 4000)
# cf_server_config of the serving runs: one 640x480 frame already fills the GPU, so one frame per batch
# costs no throughput and keeps a frame from waiting for a long batch; smallest frames first (with a
# 20 ms age limit) lets small frames pass queued large ones, and device priorities let their thread
# blocks pass a large frame already running.
SERVE_CONFIG = dict(max_batch_frames=1, pipeline_depth=6, policy=1, max_wait_ms=20.0, device_priority=1)
SERVE_SIZES = ((160, 120, 1), (320, 240, 2), (640, 480, 4), (1280, 960, 1))
# load shedding of the overload run: a request still queued this long after submission is refused
SHED_MS = 3.0
BYTES_DEPTH_EVAL = 64   # 2 boxes x 4 corners x (int32 depth sum + int32 valid count)
BYTES_COLOR_EVAL = 32   # 2 boxes x 4 corners x float32
METRIC = "train feature-evals/s"
CPU_MODEL = None


def cpu_model():
    global CPU_MODEL
    if CPU_MODEL is None:
        CPU_MODEL = "unknown"
        try:
            for ln in open("/proc/cpuinfo"):
                if ln.startswith("model name"):
                    CPU_MODEL = ln.split(":", 1)[1].strip()
                    break
        except OSError:
            pass
    return CPU_MODEL


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def workload_config():
    return {"workload": "batching training: %d RGB-D frames %dx%d, %d classes, %d samples/image (%d per tree), "
                        "depth %d, %d features x %d thresholds, minSampleCount %d; a step = one level of tree "
                        "<rank> (candidate generation + level-batched split search + routing), levels %s in turn" % (
                            C3["images"], C3["width"], C3["height"], C3["classes"],
                            C3["samples_per_image"] // C3["trees"], C3["samples_per_image"] // C3["trees"] * C3["images"],
                            C3["max_depth"], C3["features"], C3["thresholds"], C3["min_samples"],
                            "/".join(map(str, LEVELS))),
            "images": C3["images"], "frame": "%dx%d" % (C3["width"], C3["height"]), "classes": C3["classes"],
            "max_depth": C3["max_depth"], "features": C3["features"], "thresholds": C3["thresholds"],
            "samples_per_tree": C3["samples_per_image"] // C3["trees"] * C3["images"], "levels": list(LEVELS),
            "l2": "inputs larger than L2 (integral images 6.1 GB, 128 MB of samples per level)"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.times = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.times.append(time.perf_counter())

    def between(self, t0, t1):
        """(median SM MHz, fraction of samples with sw_power_cap active) of the samples read in [t0, t1]."""
        sm, cap = [], []
        for t, ln in zip(self.times, self.lines):
            parts = [p.strip() for p in ln.split(",")]
            if t0 <= t <= t1 and len(parts) >= 9:
                try:
                    sm.append(float(parts[1]))
                except ValueError:
                    continue
                cap.append(parts[8].lower() == "active")
        return (statistics.median(sm) if sm else None), (sum(cap) / len(cap) if cap else None)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------------------- CPU baseline
# Everything in this section uses the oracle only (frames, samples, candidates and the timed search),
# so the reference arm loads no product code.
def cpu_sample_inputs(frames, per_image, features, thresholds, seed=SEED, cells=40, classes=40):
    """A bounded sample of the headline workload for the CPU: the first `frames` frames of the same
    generator, class-uniform samples drawn with the device sampler's definition at the workload's
    per-image count, and the root-level candidate table of that sample."""
    from oracle import pyoracle as orc
    rgb, depth, labels = orc.synthetic_frames(seed, frames, 640, 480, cells, classes)
    ods = orc.integral(rgb, depth)
    forest_seed = int(orc.sampler_draws(4711, 0, 0xFFFE, 1)[0])
    rc, s, counter = orc.sample_class_uniform_keys(labels, depth, classes, np.zeros(classes, np.uint8), per_image,
                                                   forest_seed)
    assert rc > 0, "sampling failed"
    level_seed = int(orc.sampler_draws(counter, 0, 0xFFFFFE, 1)[0])
    feats, thr = orc.generate_features(ods, s, level_seed, features, thresholds, 60, 15)
    return ods, s, feats, thr


def cpu_split_search(ods, s, feats, thr, classes, seconds, threads):
    """The reference's CPU split search of one node (per-thread [C][F][T][2] counters, merge, scores,
    thresh-major argmax) on as many of the candidate features as fit in about `seconds`."""
    from oracle import pyoracle as orc
    hist = np.bincount(s["label"], minlength=classes).astype(np.uint32)
    F = feats.shape[1]

    def run(k):
        idx = np.linspace(0, F - 1, k).astype(int)   # keeps the depth/colour mix of the sorted table
        f, t = np.ascontiguousarray(feats[:, idx]), np.ascontiguousarray(thr[:, idx])
        t0 = time.perf_counter()
        counters = orc.histograms(ods, s, f, t, classes, threads=threads)
        orc.best_split(orc.scores(counters, hist))
        return time.perf_counter() - t0

    probe = 4
    dt = run(probe)
    k = int(max(probe, min(F, probe * seconds / max(dt, 1e-6))))
    k = max(2, k - k % 2)
    dt = run(k)
    return len(s) * k / dt, k, dt


def cpu_baseline_train(seconds=15.0, frames=100):
    threads = host_threads()
    per_image = C3["samples_per_image"] // C3["trees"]
    ods, s, feats, thr = cpu_sample_inputs(frames, per_image, C3["features"], C3["thresholds"])
    value, k, dt = cpu_split_search(ods, s, feats, thr, C3["classes"], seconds, threads)
    return {"value": value, "unit": "feature-evals/s", "cores": threads, "kind": "port", "cpu": cpu_model(),
            "sample": "root-node split search on the first %d frames of the workload: %d class-uniform samples x "
                      "%d of %d candidate features x %d thresholds (oracle restatement of FeatureEvaluationCPU + "
                      "calculateScores + argmax, OpenMP, %d threads)" % (frames, len(s), k, C3["features"],
                                                                         C3["thresholds"], threads),
            "seconds": dt}


# ----------------------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU split search (restated in the oracle; the reference itself cannot be built
    here) on bounded samples of the headline workload: one step = the root-node search of the first
    100 frames' samples on a feature subset sized to about 5 s, OpenMP on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = host_threads()
    per_image = C3["samples_per_image"] // C3["trees"]
    ods, s, feats, thr = cpu_sample_inputs(100, per_image, C3["features"], C3["thresholds"])
    vals, secs, ks = [], [], []
    for i in range(args.warmup + args.steps):
        v, k, dt = cpu_split_search(ods, s, feats, thr, C3["classes"], 5.0, threads)
        if i >= args.warmup:
            vals.append(v)
            secs.append(dt)
            ks.append(k)
    evals = sum(v * d for v, d in zip(vals, secs))
    value = evals / sum(secs)
    sample = ("root-node split search on the first 100 frames of the workload: %d class-uniform samples x ~%d of "
              "%d candidate features x %d thresholds per step (oracle restatement of FeatureEvaluationCPU + "
              "calculateScores + argmax, OpenMP, %d threads, %s)" % (len(s), int(statistics.median(ks)), C3["features"],
                                                                     C3["thresholds"], threads, cpu_model()))
    line = {"metric": METRIC, "value": value, "unit": "feature-evals/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(),
            "cpu_baseline": {"value": value, "unit": "feature-evals/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "feature-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference cannot be built here (Boost, TBB, Vigra, cuv::ndarray absent; texture references "
                    "removed in CUDA 12); its CPU path is timed through the oracle restatement, which imports "
                    "nothing from the product library"}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------- helpers
def frames(cfg, seed=SEED, n=None, first=0):
    import curfil_b200 as cf
    return cf.synthetic_frames(seed, n or cfg["images"], cfg["width"], cfg["height"], cfg["cells"], cfg["classes"],
                               first=first)


def train_config(c, **kw):
    import curfil_b200 as cf
    return cf.TrainConfig(random_seed=4711, samples_per_image=c["samples_per_image"], feature_count=c["features"],
                          min_sample_count=c["min_samples"], max_depth=c["max_depth"], box_radius=c["box_radius"],
                          region_size=c["region_size"], thresholds=c["thresholds"], **kw)


def splits_equal(a, b):
    return bool(np.array_equal(a["feature"], b["feature"]) and np.array_equal(a["threshold_index"], b["threshold_index"])
                and np.array_equal(a["threshold"], b["threshold"]) and np.array_equal(a["score"], b["score"]))


def trees_equal(A, B):
    """Node arrays equal (leaves carry NaN thresholds and scores, which compare equal here)."""
    if len(A["left"]) != len(B["left"]):
        return False
    return all(np.array_equal(A[k], B[k], equal_nan=A[k].dtype.kind == "f") for k in A if k in B)


def pinned_copy(arr):
    """`arr` copied into page-locked host memory (torch's pinned allocator), same dtype and shape."""
    import torch
    t = torch.empty(arr.nbytes, dtype=torch.uint8, pin_memory=True)
    out = t.numpy().view(arr.dtype).reshape(arr.shape)
    out[...] = arr
    return out, t


# ----------------------------------------------------------------------------------------- headline
def headline(ctx, stream, local, rank, world, args, barrier, max_over_ranks, sum_over_ranks):
    """Config 3: level snapshots of tree <rank>, K timed level steps, per-node form and host-buffer
    entry points on the same levels."""
    import torch
    import curfil_b200 as cf
    out = {}
    t0 = time.perf_counter()
    rgb, depth, labels = frames(C3, n=args.images)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    cfg = train_config(C3, sampler=1)
    tree_id = rank
    samples, prior, counter = cf.sample_tree_pixels(labels, depth, C3["classes"], cfg, C3["trees"],
                                                    cf.forest_seed(cfg.random_seed) + tree_id, ctx=ctx)
    del rgb, labels
    setup_s = time.perf_counter() - t0
    with ClockSampler(local) as tclk:
        time.sleep(0.5)
        t_call = time.perf_counter()
        tree, snaps, _ = cf.train_tree_snapshots(ds, samples, C3["classes"], cfg, LEVELS, tree_id=tree_id,
                                                 seed_counter=counter)
    ev, dev_ms, nlev = tree.train_stats()
    # each level's time beside the SM clock and power-cap samples taken while it ran (the level's start
    # is known on the device timeline; the training's first device work follows the call by the
    # samples' upload, a few ms)
    levels_ms = []
    for (n_, s_, ms_), st in zip(tree.level_stats(), tree.level_starts()):
        mhz, capped = tclk.between(t_call + st / 1e3, t_call + (st + ms_) / 1e3)
        levels_ms.append([n_, s_, round(ms_, 1), mhz, None if capped is None else round(capped, 2)])
    out["tree"] = {"tree_id": tree_id, "nodes": tree.num_nodes, "depth": tree.depth, "levels": nlev,
                   "samples": len(samples), "device_ms": dev_ms, "feature_evals": ev,
                   "feature_evals_per_s": ev / (dev_ms / 1e3),
                   "note": "the whole tree trained once (level-batched) while the snapshots were taken; "
                           "setup (frames, upload, integral images, device sampling) %.1f s" % setup_s,
                   "levels_ms": levels_ms,
                   "levels_ms_columns": ["open nodes", "samples", "split search ms", "median SM MHz while it ran",
                                         "fraction of clock samples with sw_power_cap active"]}
    tree.close()
    assert [s.level for s in snaps] == list(LEVELS), "the tree did not reach every benchmarked level"

    for i in range(args.warmup):
        snaps[i % len(snaps)].run()
    torch.cuda.synchronize()
    barrier()
    ctx.reset_timing()
    ctx.set_timing(True)
    launches0 = ctx.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per_level = {s.level: [] for s in snaps}
    total_evals = 0
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        barrier()
        start.record(stream)
        for i in range(args.steps):
            s = snaps[i % len(snaps)]
            if i == args.profile_step:   # an Nsight Compute range (ncu --profile-from-start off)
                torch.cuda.synchronize()
                torch.cuda.profiler.start()
            r = s.run()
            if i == args.profile_step:
                torch.cuda.synchronize()
                torch.cuda.profiler.stop()
            total_evals += r["evals"]
            per_level[s.level].append(r["ms"])
        end.record(stream)
        torch.cuda.synchronize()
        barrier()
    ctx.set_timing(False)
    launches = ctx.launch_count() - launches0
    ms = start.elapsed_time(end)
    ms_max = max_over_ranks(ms)
    out["value"] = sum_over_ranks(total_evals) / (ms_max / 1e3)
    out["ms_per_step"] = ms_max / args.steps
    out["evals_per_step"] = total_evals / args.steps
    out["gpu_launches"] = int(launches)
    out["clocks"] = clocks.summary()
    # the split search is level_eval (fused, or pass 2 reading staged bins) plus stage_bins (pass 1 of
    # the staged levels); the roofline is that of the two together, with each kernel's share beside it
    eval_ms, eval_launches = ctx.kernel_time("level_eval")
    stage_ms, stage_launches = ctx.kernel_time("stage_bins")
    out["kernel_ms"] = {k: ctx.kernel_time(k)[0] for k in ("level_eval", "stage_bins", "stage_rows", "node_consts",
                                                            "gen_features", "sort_features", "route_flags",
                                                            "route_scatter", "scan", "reduce_candidates")}
    bytes_per_eval = (BYTES_DEPTH_EVAL + BYTES_COLOR_EVAL) / 2.0
    search_ms = eval_ms + stage_ms
    achieved = total_evals * bytes_per_eval / (search_ms / 1e3) / 1e9 if search_ms > 0 else None
    peak, peak_kind = load_peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "split_search_traffic.txt")
    if os.path.exists(tp):
        for ln in open(tp):
            if ln.startswith("dram_bytes_per_feature_eval:"):
                traffic = float(ln.split(":")[1]) * total_evals / max(1, args.steps)
    out["roofline"] = {"bound": "hbm", "kernel": "split search (level_eval + stage_bins)", "achieved": achieved,
                       "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                       "traffic": traffic, "traffic_per": "step (one level)", "peak_source": peak_kind,
                       "bytes_per_eval": bytes_per_eval, "ms_per_step": search_ms / max(1, args.steps),
                       "kernels": {"level_eval": {"ms": eval_ms, "launches": eval_launches,
                                                  "share": eval_ms / search_ms if search_ms else None},
                                   "stage_bins": {"ms": stage_ms, "launches": stage_launches,
                                                  "share": stage_ms / search_ms if search_ms else None}}}
    out["levels"] = [{"level": s.level, "nodes": s.num_nodes, "samples": s.num_samples,
                      "ms": statistics.median(per_level[s.level]) if per_level[s.level] else None,
                      "feature_evals_per_s": s.num_samples * C3["features"] / (statistics.median(per_level[s.level]) / 1e3)
                      if per_level[s.level] else None} for s in snaps]

    # the plain per-node form on the same levels: identical splits required
    if not args.no_per_node:
        rows, lb_total, pn_total, same_all = [], 0.0, 0.0, True
        for s in snaps:
            lb = s.run(cf.LEVEL_BATCHED, splits=True)
            pn = s.run(cf.PER_NODE, splits=True)
            same = splits_equal(lb["splits"], pn["splits"]) and (lb["next_nodes"], lb["next_samples"]) == \
                (pn["next_nodes"], pn["next_samples"])
            same_all &= same
            lb_total += lb["ms"]
            pn_total += pn["ms"]
            rows.append({"level": s.level, "nodes": s.num_nodes, "level_batched_ms": lb["ms"], "per_node_ms": pn["ms"],
                         "speedup": pn["ms"] / lb["ms"], "splits_identical": same})
        ev = sum(s.num_samples for s in snaps) * C3["features"]
        out["per_node"] = {"value": ev / (pn_total / 1e3), "unit": "feature-evals/s",
                           "level_batched_value": ev / (lb_total / 1e3), "speedup": pn_total / lb_total,
                           "splits_identical": bool(same_all), "levels": rows,
                           "note": "one run of each level in each form; splits, next-level nodes and samples "
                                   "compared"}

    # end to end through the host-buffer entry points: candidate generation and evaluateBestSplits
    # from pinned host samples, the candidate table and splits back to the host
    if args.e2e_steps > 0:
        tot_ev, tot_s, h2d, d2h, same_all = 0, 0.0, 0, 0, True
        for s in snaps:
            offsets, hs, seed = s.export()
            ref = s.run(cf.LEVEL_BATCHED, splits=True)["splits"]
            pinned, keep = pinned_copy(hs)
            for _ in range(args.e2e_steps):
                barrier()
                t0 = time.perf_counter()
                feats, thr = cf.generate_features(ds, pinned, seed, C3["features"], C3["thresholds"],
                                                  C3["box_radius"], C3["region_size"])
                best = cf.evaluate_best_splits(ds, offsets, pinned, C3["classes"], feats, thr)
                tot_s += time.perf_counter() - t0
                tot_ev += s.num_samples * C3["features"]
                h2d += 2 * hs.nbytes + feats.nbytes + thr.nbytes + offsets.nbytes
                d2h += feats.nbytes + thr.nbytes + best.nbytes
                same_all &= splits_equal(best, ref)
            del pinned, keep
        steps = args.e2e_steps * len(snaps)
        tot_s = max_over_ranks(tot_s)
        out["e2e"] = {"value": sum_over_ranks(tot_ev) / tot_s, "unit": "feature-evals/s",
                      "h2d_bytes_per_step": int(h2d / steps), "d2h_bytes_per_step": int(d2h / steps),
                      "splits_identical": bool(same_all),
                      "note": "per level: cf_generate_features + cf_evaluate_best_splits (ImageFeatureEvaluation::"
                              "evaluateBestSplits) from pinned host samples, splits to the host; host wall clock; "
                              "%d call(s) per level" % args.e2e_steps}
    for s in snaps:
        s.close()
    ds.close()
    return out


# ----------------------------------------------------------------------------------------- config 2
def config2(ctx, stream, args):
    """The plain-method full-size configuration: 3 trees per step on the resident dataset (device time),
    the plain per-node form on tree 0, cf_forest_train from host frames end to end. Returns the
    section, the dataset and its frames (the prediction forest trains on them)."""
    import torch
    import curfil_b200 as cf
    out = {"workload": "plain method full size: 200 RGB-D frames 640x480, 40 classes, 4000 samples/image, 3 trees "
                       "depth 20, 2000 features x 20 thresholds, minSampleCount 50; a step trains the 3 trees"}
    rgb, depth, labels = frames(C2)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    cfg = train_config(C2)
    seed = cf.forest_seed(cfg.random_seed)
    per_tree = []
    for t in range(C2["trees"]):
        s, prior, counter = cf.sample_tree_pixels(labels, depth, C2["classes"], cfg, C2["trees"], seed + t)
        per_tree.append((t, s, prior, counter))
    if not args.no_autotune:
        t0_, s0_, _, c0_ = per_tree[0]
        tuned = cf.autotune_split_search(ds, s0_, C2["classes"], cfg, tree_id=t0_, seed_counter=c0_)
        tuned.pop("key", None)
        out["autotune"] = tuned

    def step():
        trees, evals = [], 0
        for t, s, prior, counter in per_tree:
            tree, _ = cf.train_tree(ds, s, C2["classes"], cfg, tree_id=t, seed_counter=counter)
            evals += tree.train_stats()[0]
            trees.append(tree)
        return trees, evals

    trees, _ = step()
    for t in trees:
        t.close()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    evals = 0
    steps = 3
    for _ in range(steps):
        trees, ev = step()
        evals += ev
        levels0 = trees[0].level_stats()
        for t in trees:
            t.close()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out.update({"value": evals / (ms / 1e3), "unit": "feature-evals/s", "steps": steps, "ms_per_step": ms / steps,
                "split_search_tuning": ctx.get_tuning().as_dict(),
                "levels_tree0": [[n, s, round(m, 3)] for n, s, m in levels0]})
    if not args.no_per_node:
        t, s, prior, counter = per_tree[0]
        res = {}
        for name, mode in (("level_batched", cf.LEVEL_BATCHED), ("per_node", cf.PER_NODE)):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            tree, _ = cf.train_tree(ds, s, C2["classes"], cfg, tree_id=t, seed_counter=counter, mode=mode)
            b.record(stream)
            torch.cuda.synchronize()
            res[name] = (tree.arrays(), a.elapsed_time(b), tree.train_stats()[0])
            tree.close()
        (A, lb_ms, lb_ev), (B, pn_ms, pn_ev) = res["level_batched"], res["per_node"]
        out["per_node"] = {"value": pn_ev / (pn_ms / 1e3), "ms_per_tree": pn_ms, "level_batched_ms_per_tree": lb_ms,
                           "speedup": pn_ms / lb_ms, "trees_identical": bool(lb_ev == pn_ev and trees_equal(A, B))}
    if args.e2e_steps > 0:
        c = train_config(C2, sampler=1)
        for t in cf.train_forest(ctx, rgb, depth, labels, C2["classes"], c, C2["trees"]):
            t.close()
        t0 = time.perf_counter()
        ev = 0
        for _ in range(args.e2e_steps):
            for t in cf.train_forest(ctx, rgb, depth, labels, C2["classes"], c, C2["trees"]):
                ev += t.train_stats()[0]
                t.close()
        dt = time.perf_counter() - t0
        out["e2e"] = {"value": ev / dt, "unit": "feature-evals/s", "calls": args.e2e_steps,
                      "h2d_bytes_per_step": int(rgb.nbytes + 2 * depth.nbytes + labels.nbytes),
                      "note": "cf_forest_train (RandomForestImage::train): host frames uploaded, integral images, "
                              "device class-uniform sampling, level-batched training, trees to the host"}
    return out, ds, (rgb, depth, labels)


# ----------------------------------------------------------------------------------------- config 1
def config1(ctx, stream):
    """The plain-method small configuration: one tree on 16 frames 320x240 (8 classes, void class 0
    ignored, 500 samples per class and image, reference sampler), trained level-batched, per node and
    by the CPU oracle (the reference's CPU path) with all host cores; trees compared; 4 held-out
    frames predicted on the GPU and by the oracle."""
    import torch
    import curfil_b200 as cf
    from oracle import pyoracle as orc
    n, C = C1["images"], C1["classes"]
    rgb, depth, labels = frames(C1, seed=SEED + 1, n=n + C1["predict_images"])
    ignore = np.zeros(C, np.uint8)
    ignore[0] = 1
    cfg = train_config(C1)
    seed = cf.forest_seed(cfg.random_seed)
    s, prior, counter = cf.sample_tree_pixels(labels[:n], depth[:n], C, cfg, 1, seed, ignored=ignore)
    ds = cf.Dataset.from_raw(ctx, rgb[:n], depth[:n])
    out = {"workload": "plain method small: 16 RGB-D frames 320x240, 8 classes (void ignored), 500 samples per class "
                       "and image (%d samples), 1 tree depth 12, 500 features x 20 thresholds" % len(s)}
    gpu = {}
    for name, mode in (("level_batched", cf.LEVEL_BATCHED), ("per_node", cf.PER_NODE)):
        cf.train_tree(ds, s, C, cfg, seed_counter=counter, mode=mode)[0].close()   # warm
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        tree, _ = cf.train_tree(ds, s, C, cfg, seed_counter=counter, mode=mode)
        b.record(stream)
        torch.cuda.synchronize()
        ev = tree.train_stats()[0]
        gpu[name] = (tree, a.elapsed_time(b), ev)
    tree, lb_ms, ev = gpu["level_batched"]
    threads = host_threads()
    ods = orc.integral(rgb[:n], depth[:n])
    t0 = time.perf_counter()
    rc, ot, _ = orc.train_tree(ods, s.view(orc.SAMPLE_DTYPE), C, C1["features"], C1["thresholds"], C1["max_depth"],
                               C1["min_samples"], C1["box_radius"], C1["region_size"], counter, threads=threads)
    cpu_s = time.perf_counter() - t0
    A = tree.arrays()
    O = {k: getattr(ot, k) for k in ("level", "left", "feature", "threshold", "histogram", "num_samples")}
    same_oracle = rc == 0 and trees_equal({k: A[k] for k in O}, O)
    out.update({"nodes": tree.num_nodes, "feature_evals": ev,
                "level_batched": {"ms": lb_ms, "feature_evals_per_s": ev / (lb_ms / 1e3)},
                "per_node": {"ms": gpu["per_node"][1], "feature_evals_per_s": ev / (gpu["per_node"][1] / 1e3)},
                "cpu": {"seconds": cpu_s, "feature_evals_per_s": ev / cpu_s, "cores": threads, "cpu": cpu_model(),
                        "kind": "port"},
                "trees_identical_gpu_forms": trees_equal(A, gpu["per_node"][0].arrays()),
                "tree_identical_to_cpu": bool(same_oracle)})
    # prediction of the held-out frames: GPU from host frames vs the oracle (the reference's CPU predict)
    forest = cf.Forest(ctx, [tree], prior=prior)
    hr, hd = rgb[n:], depth[n:]
    forest.predict(hr, hd)
    t0 = time.perf_counter()
    probs, lab = forest.predict(hr, hd)
    gpu_s = time.perf_counter() - t0
    normalized = np.stack([orc.normalize_histogram(h, prior, 0.0, True) for h in A["histogram"]])
    otv = orc.Tree(len(A["left"]), C)
    otv.left, otv.feature, otv.threshold = A["left"], A["feature"], A["threshold"]
    hods = orc.integral(hr, hd)
    t0 = time.perf_counter()
    agree, pdiff = [], 0.0
    for i in range(len(hr)):
        op, ol = orc.predict(hods, i, [otv], [normalized], C, threads=threads)
        agree.append((ol == lab[i]).mean())
        pdiff = max(pdiff, float(np.abs(op - probs[i]).max()))
    cpu_p = time.perf_counter() - t0
    px = hr.shape[0] * hr.shape[1] * hr.shape[2]
    out["predict"] = {"frames": len(hr), "gpu_mpx_per_s": px / gpu_s / 1e6, "cpu_mpx_per_s": px / cpu_p / 1e6,
                      "cpu_cores": threads, "label_agreement": float(np.mean(agree)), "max_probability_diff": pdiff,
                      "heldout_pixel_accuracy": float((lab == labels[n:]).mean()),
                      "note": "GPU from host frames (upload, integral images, classify, results back)"}
    forest.close()
    for t, _, _ in gpu.values():
        t.close()
    ds.close()
    return out


# ----------------------------------------------------------------------------------------- prediction
def forest_trees(ds, rgb, depth, labels, n_trees):
    """n_trees trees trained as in config 2 (the forest's sampling split over n_trees)."""
    import curfil_b200 as cf
    cfg = train_config(C2)
    seed = cf.forest_seed(cfg.random_seed)
    trees = []
    for t in range(n_trees):
        s, prior, counter = cf.sample_tree_pixels(labels, depth, C2["classes"], cfg, n_trees, seed + t)
        tree, _ = cf.train_tree(ds, s, C2["classes"], cfg, tree_id=t, seed_counter=counter)
        tree.set_prior(prior)
        trees.append(tree)
    return trees


def timed_events(stream, fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def timed_wall(fn, reps):
    fn()
    t0 = time.perf_counter()
    for _ in range(reps):
        r = fn()
    return (time.perf_counter() - t0) / reps, r


def predict_section(ctx, stream, ds, trees, local, serve_seconds):
    """Config 4: a 10-tree depth-20 forest on 64 frames 640x480. Resident frames: the batched kernel
    (one launch for all frames and trees) against the plain per-image launch form. From host frames,
    with equal outputs on both sides: one CUDA-graph replay against the plain per-image form as
    RandomForestImage::predict runs it, labels only and with probabilities. The reference's CPU
    prediction (oracle, all host cores) on two of the frames. Poisson serving and the refiner."""
    import torch
    import curfil_b200 as cf
    from oracle import pyoracle as orc
    n, C, H, Wd = C4["images"], C2["classes"], C2["height"], C2["width"]
    px = n * H * Wd
    forest = cf.Forest(ctx, trees)
    out = {"images": n, "frame": "%dx%d" % (Wd, H), "trees": len(trees), "forest_nodes": forest.num_nodes}
    pa = torch.empty((n, C, H, Wd), dtype=torch.float32, device=local)
    la = torch.empty((n, H, Wd), dtype=torch.uint8, device=local)
    ctx.reset_timing()
    ctx.set_timing(True)
    ms = timed_events(stream, lambda: forest.predict_dataset(ds, 0, n, pa.data_ptr(), la.data_ptr()), 5)
    ctx.set_timing(False)
    k_ms, k_n = ctx.kernel_time("classify")
    peak, peak_kind = load_peaks()
    bpp = 20 + 4 * C + 1   # integral images (colour 12 B + depth 8 B) read, probabilities and label written
    achieved = px * bpp / (k_ms / k_n / 1e3) / 1e9
    out["batched"] = {"mpx_per_s": px / (ms / 1e3) / 1e6, "ms_per_batch": ms, "ms_per_frame": ms / n,
                      "roofline": {"bound": "hbm", "kernel": "classify", "achieved": achieved, "peak": peak,
                                   "unit": "GB/s", "frac": achieved / peak, "bytes_per_px": bpp,
                                   "avg_launch_ms": k_ms / k_n, "peak_source": peak_kind}}
    pb = torch.empty_like(pa)
    lb = torch.empty_like(la)
    pms = timed_events(stream, lambda: forest.predict_dataset_plain(ds, 0, n, pb.data_ptr(), lb.data_ptr()), 1)
    out["plain_per_image"] = {"mpx_per_s": px / (pms / 1e3) / 1e6, "ms_per_frame": pms / n,
                              "note": "one launch + synchronisation per tree per image, then normalise and argmax"}
    out["speedup_vs_plain"] = pms / ms
    out["labels_identical"] = bool(torch.equal(la, lb))
    out["probabilities_identical"] = bool(torch.equal(pa.view(torch.int32), pb.view(torch.int32)))
    del pa, pb

    # from host frames, equal outputs on both sides
    rgb, depth, _ = frames(C2, seed=SEED + 7, n=n)
    sub = 16
    spx = sub * H * Wd
    host = {}
    for probs in (False, True):
        g = cf.PredictGraph(forest, n, Wd, H, probabilities=probs)
        g.rgb[...] = rgb
        g.depth[...] = depth
        gs, _ = timed_wall(g.run, 3)
        glabels = g.labels[:sub].copy()
        g.close()
        if probs:
            ps, (_, pl) = timed_wall(lambda: forest.predict_plain(rgb[:sub], depth[:sub], probabilities=True), 1)
        else:
            # the plain per-image launches from host frames with only the labels copied back
            pds = cf.Dataset(ctx, sub, Wd, H)
            lab_dev = torch.empty((sub, H, Wd), dtype=torch.uint8, device=local)

            def plain_labels():
                pds.upload_raw(rgb[:sub], depth[:sub])
                forest.predict_dataset_plain(pds, 0, sub, 0, lab_dev.data_ptr())
                return lab_dev.cpu().numpy()
            ps, pl = timed_wall(plain_labels, 1)
            pds.close()
        key = "with_probabilities" if probs else "labels_only"
        host[key] = {"graph_mpx_per_s": px / gs / 1e6, "graph_ms_per_batch": gs * 1e3,
                     "plain_mpx_per_s": spx / ps / 1e6, "plain_frames": sub, "speedup": (px / gs) / (spx / ps),
                     "labels_identical": bool(np.array_equal(pl, glabels)),
                     "h2d_bytes_per_frame": H * Wd * 5, "d2h_bytes_per_frame": H * Wd * (1 + (4 * C if probs else 0))}
    host["note"] = ("graph: pinned host RGB-D -> H2D -> integral images -> classify -> results D2H, one replay of all "
                    "64 frames; plain: per image upload, integral images, one launch + sync per tree, normalise, "
                    "argmax, results back (cf_predict_host_plain with probabilities; with labels only, the same "
                    "launches with only the labels copied back)")
    out["host_frames"] = host

    # the reference's CPU prediction (random_forest_image.cpp:307-345, oracle restatement, all host cores)
    threads = host_threads()
    arrays = [t.arrays() for t in trees]
    views, normalized = [], []
    for t, A in zip(trees, arrays):
        pr = t.prior()
        normalized.append(np.stack([orc.normalize_histogram(h, pr, 0.0, True) for h in A["histogram"]]))
        v = orc.Tree(len(A["left"]), C)
        v.left, v.feature, v.threshold = A["left"], A["feature"], A["threshold"]
        views.append(v)
    k = 2
    ods = orc.integral(rgb[:k], depth[:k])
    probs_g, labels_g = forest.predict(rgb[:k], depth[:k])
    t0 = time.perf_counter()
    agree, pdiff = [], 0.0
    for i in range(k):
        op, ol = orc.predict(ods, i, views, normalized, C, threads=threads)
        agree.append((ol == labels_g[i]).mean())
        pdiff = max(pdiff, float(np.abs(op - probs_g[i]).max()))
    cpu_s = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": k * H * Wd / cpu_s / 1e6, "unit": "Mpx/s", "cores": threads, "kind": "port",
                           "cpu": cpu_model(), "sample": "%d frames 640x480 through the 10-tree forest (oracle "
                                                         "restatement of the CPU branch of RandomForestImage::predict, "
                                                         "rows in parallel)" % k,
                           "label_agreement_with_gpu": float(np.mean(agree)), "max_probability_diff": pdiff}
    if serve_seconds > 0:
        out["serving"] = serve(forest, serve_seconds)
    out["refiner"] = refiner_section(ctx, stream, ds, forest, local)
    forest.close()
    return out


def refiner_section(ctx, stream, ds, forest, local):
    """The learned part: the refinement network trained on 32 dataset frames' labels, pixel accuracy
    of forest and forest + network on 8 held-out frames of the same generator."""
    import torch
    import curfil_b200 as cf
    n_train, n_test = min(32, ds.n), 8
    _, _, labels = frames(C2, n=n_train)
    # held out: the frames after the dataset's in the same seeded sequence (same class appearance)
    rgb_t, depth_t, labels_t = frames(C2, n=n_test, first=ds.n)
    test = cf.Dataset.from_raw(ctx, rgb_t, depth_t)
    r = cf.Refiner(ctx, C2["classes"], hidden=64, epochs=8, batch=4096, pixels_per_image=20000, seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = r.train(forest, ds, 0, n_train, labels)
    train_s = time.perf_counter() - t0
    lab = torch.empty((n_test, C2["height"], C2["width"]), dtype=torch.uint8, device=local)
    forest.predict_dataset(test, 0, n_test, 0, lab.data_ptr())
    torch.cuda.synchronize()
    base = float((lab.cpu().numpy() == labels_t).mean())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r.predict(forest, test, 0, n_test, 0, lab.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    refined = float((lab.cpu().numpy() == labels_t).mean())
    px = n_test * C2["width"] * C2["height"]
    r.close()
    test.close()
    return {"train_frames": n_train, "train_pixels": n_train * 20000, "epochs": 8, "train_s": train_s,
            "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
            "heldout_frames": n_test, "forest_pixel_accuracy": base, "refined_pixel_accuracy": refined,
            "refined_predict_mpx_per_s": px / (e0.elapsed_time(e1) / 1e3) / 1e6}


# ----------------------------------------------------------------------------------------- serving
def serve(forest, seconds):
    """Config 5: Poisson arrivals (seeded) at each offered rate, frame sizes 160x120 : 320x240 :
    640x480 : 1280x960 = 1:2:4:1; latency = completion - submission on the server's clock. The top
    rate is run twice: without a queueing limit, and with load shedding (max_queue_ms), where
    requests that waited too long are refused and the latency of the admitted ones is reported."""
    import curfil_b200 as cf
    pool = {}
    for w, h, _ in SERVE_SIZES:
        rgb, depth, _ = cf.synthetic_frames(SEED + w, 4, w, h, C2["cells"], C2["classes"])
        pool[(w, h)] = (rgb, depth)
    weights = np.array([k for _, _, k in SERVE_SIZES], np.float64)
    results = []
    runs = [(r, 0.0) for r in SERVE_RATES] + [(SERVE_RATES[-1], SHED_MS)]
    for rate, shed in runs:
        rng = np.random.default_rng(rate)
        count = max(8, int(rate * seconds))
        gaps = rng.exponential(1.0 / rate, count)
        kinds = rng.choice(len(SERVE_SIZES), count, p=weights / weights.sum())
        which = rng.integers(0, 4, count)
        srv = cf.Server(forest, hbm_budget_bytes=8 << 30, max_pending=1 << 16, max_queue_ms=shed, **SERVE_CONFIG)
        for w, h, _ in SERVE_SIZES:   # warm the server with one frame of each size
            rgb, depth = pool[(w, h)]
            srv.wait(srv.submit(rgb[0], depth[0]), (h, w))
        ids, done, refused = [], {}, []

        def drain():
            for rid, shape in iter(q.get, None):
                try:
                    _, _, st = srv.wait(rid, shape, timeout_s=60.0)
                    done[rid] = (st.submit_ms, st.admitted_ms, st.done_ms, shape)
                except cf.CurfilError as e:
                    if e.status != 7:
                        raise
                    refused.append(shape)

        q = queue.Queue()
        waiter = threading.Thread(target=drain)
        waiter.start()
        t = time.perf_counter()
        for i in range(count):
            t += gaps[i]
            while time.perf_counter() < t:
                pass
            w, h, _ = SERVE_SIZES[kinds[i]]
            rgb, depth = pool[(w, h)]
            rid = srv.submit(rgb[which[i]], depth[which[i]])
            ids.append(rid)
            q.put((rid, (h, w)))
        q.put(None)
        waiter.join()
        ok = [r for r in ids if r in done]
        lat = np.array([done[r][2] - done[r][0] for r in ok])
        qwait = np.array([done[r][1] - done[r][0] for r in ok])
        shapes = np.array([done[r][3] for r in ok])
        big = (shapes[:, 0] == 480) & (shapes[:, 1] == 640)
        by_size = {f"{w}x{h}": float(np.percentile(lat[(shapes[:, 0] == h) & (shapes[:, 1] == w)], 99))
                   for w, h, _ in SERVE_SIZES if ((shapes[:, 0] == h) & (shapes[:, 1] == w)).any()}
        span = (max(done[r][2] for r in ok) - min(done[r][0] for r in ok)) / 1e3
        pxs = sum(done[r][3][0] * done[r][3][1] for r in ok)
        offered_px = sum(SERVE_SIZES[k][0] * SERVE_SIZES[k][1] for k in kinds)
        c = srv.counters()
        srv.close()
        results.append({"offered_fps": rate, "frames": count, "max_queue_ms": shed or None,
                        "offered_mpx_per_s": rate * offered_px / count / 1e6,
                        "served": len(ok), "rejected": len(refused), "rejected_fraction": len(refused) / count,
                        "mpx_per_s": pxs / span / 1e6, "p50_ms": float(np.percentile(lat, 50)),
                        "p99_ms": float(np.percentile(lat, 99)),
                        "p99_ms_640x480": float(np.percentile(lat[big], 99)) if big.any() else None,
                        "p99_ms_by_size": by_size, "p99_admission_wait_ms": float(np.percentile(qwait, 99)),
                        "batches": c["batches"] - len(SERVE_SIZES)})
    return {"sizes": "160x120:320x240:640x480:1280x960 = 1:2:4:1", "trees": forest.num_trees,
            "server": dict(SERVE_CONFIG), "rates": results,
            "note": "latency percentiles over the served frames; with max_queue_ms, refused frames are counted in "
                    "rejected and excluded from the percentiles"}


# ----------------------------------------------------------------------------------------- our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--images", type=int, default=C3["images"], help="frames of the headline workload")
    ap.add_argument("--e2e-steps", type=int, default=1, help="host-buffer calls per level for the e2e figure")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-node", action="store_true", help="skip the plain per-node comparisons")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default split-search launch shape")
    ap.add_argument("--headline-only", action="store_true", help="skip configs 1, 2, 4 and 5")
    ap.add_argument("--sections", default="headline,config1,config2,predict",
                    help="comma-separated parts to run (profiling runs pick one); predict needs config2's forest data")
    ap.add_argument("--serve-seconds", type=float, default=1.5, help="Poisson load per offered rate (0: skip)")
    ap.add_argument("--tuning", default="", help="split-search launch shape overrides, e.g. ctas_per_sm=4,"
                    "bins_budget_words=10240 (cf_eval_tuning field names)")
    ap.add_argument("--profile-step", type=int, default=-1,
                    help="bracket this timed headline step (0-based; steps cycle the levels) with a profiler range")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import curfil_b200 as cf

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def reduce(x, op):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max_over_ranks(x):
        return reduce(x, dist.ReduceOp.MAX if dist else None)

    def sum_over_ranks(x):
        return reduce(x, dist.ReduceOp.SUM if dist else None)

    ctx = cf.Context(local)
    if args.tuning:
        overrides = {}
        for kv in args.tuning.split(","):
            k, v = kv.split("=")
            overrides[k.strip()] = float(v) if k.strip() == "items_per_slot" else int(v)
        ctx.set_tuning(**overrides)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)

    C3["images"] = args.images
    sections = set(args.sections.split(","))
    if "headline" not in sections:
        # a profiling run of other parts only
        if "config1" in sections:
            config1(ctx, stream)
        if "config2" in sections or "predict" in sections:
            c2, ds2, (rgb2, depth2, labels2) = config2(ctx, stream, args)
            if "predict" in sections:
                ptrees = forest_trees(ds2, rgb2, depth2, labels2, C4["trees"])
                predict_section(ctx, stream, ds2, ptrees, local, args.serve_seconds)
        ctx.close()
        return
    head = headline(ctx, stream, local, rank, world, args, barrier, max_over_ranks, sum_over_ranks)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_train()
    extra = {}
    if rank == 0 and world == 1 and not args.headline_only:
        if "config1" in sections:
            extra["config1"] = config1(ctx, stream)
        if "config2" in sections or "predict" in sections:
            c2, ds2, (rgb2, depth2, labels2) = config2(ctx, stream, args)
            extra["config2"] = c2
            if "predict" in sections:
                ptrees = forest_trees(ds2, rgb2, depth2, labels2, C4["trees"])
                extra["predict"] = predict_section(ctx, stream, ds2, ptrees, local, args.serve_seconds)
                for t in ptrees:
                    t.close()
            ds2.close()
    if rank == 0:
        line = {"metric": METRIC, "value": head["value"], "unit": "feature-evals/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded RGB-D generator; no dataset offline)",
                "config": dict(workload_config(), parallelism="one tree per GPU (tree id = rank), %d GPU(s)" % world,
                               split_search_tuning=ctx.get_tuning().as_dict() if args.tuning else "default"),
                "roofline": head["roofline"], "cpu_baseline": cpu, "e2e": head.get("e2e"),
                "gpu_launches": head["gpu_launches"], "clocks": head["clocks"],
                "per_node": head.get("per_node"), "levels": head["levels"], "tree": head["tree"],
                "kernel_ms": head["kernel_ms"], "feature_evals_per_step": head["evals_per_step"],
                # split evaluations: every feature evaluation is binned against all T thresholds
                "split_evals_per_s": head["value"] * C3["thresholds"]}
        line.update(extra)
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
