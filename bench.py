#!/usr/bin/env python
"""Benchmark of CURFIL's random-forest training hot path on B200.

Workload (the plain-method full-size configuration): 200 seeded synthetic RGB-D frames 640x480
(40 Voronoi cells, 40 classes, uint8 colour, uint16 depth with 10% holes), 4000 samples per image
(class-uniform, divided over the trees as RandomForestImage::train does), 3 trees to depth 20,
2000 candidate features x 20 thresholds per level, minSampleCount 50, offsets <= 60, boxes <= 15.

A step trains the forest's trees level-batched from their sample lists on the resident dataset
(integral images 1.2 GB, larger than L2). Metric: feature evaluations per second (one evaluation =
one (sample, candidate feature) response compared against all thresholds and binned). The split
search's launch shape is chosen by the autotuner before timing.
Reported beside it: `e2e` (cf_forest_train from host frames: upload, integral images, device
sampling, training, tree download; also with the reference's host sampler), the plain per-node form
on the same tree (identity checked), the CPU oracle, and prediction with a 10-tree forest on 64
frames (batched, plain per-image form, CUDA-graph replay from host frames, Poisson serving).
Under torchrun every rank trains its own trees (trees are independent; no collective on the data path).
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

W = dict(images=200, width=640, height=480, cells=40, classes=40, samples_per_image=4000, trees=3, max_depth=20,
         features=2000, thresholds=20, min_samples=50, box_radius=60, region_size=15, predict_images=64,
         predict_trees=10, seed=2026)
# serving: Poisson arrivals of mixed frame sizes (weights 1:2:4:1) at these offered rates
SERVE_RATES = (200, 1000, 4000)
# cf_server_config of the serving runs: one 640x480 frame already fills the GPU, so one frame per batch
# costs no throughput and keeps a frame from waiting for a long batch; smallest frames first (with a
# 20 ms age limit) lets small frames pass queued large ones, and device priorities let their thread
# blocks pass a large frame already running. At 1000 frames/s this moves the p99 of 640x480 frames from
# 8.8 to 6.0 ms and of 160x120 frames from 6.4 to 1.6 ms; 1280x960 frames wait longer (17 -> 18 ms).
SERVE_CONFIG = dict(max_batch_frames=1, pipeline_depth=6, policy=1, max_wait_ms=20.0, device_priority=1)
SERVE_SIZES = ((160, 120, 1), (320, 240, 2), (640, 480, 4), (1280, 960, 1))
BYTES_DEPTH_EVAL = 64   # 2 boxes x 4 corners x (int32 depth sum + int32 valid count)
BYTES_COLOR_EVAL = 32   # 2 boxes x 4 corners x float32
METRIC = "train feature-evals/s"


def workload_config():
    return {"workload": "plain method full size: %d RGB-D frames %dx%d, %d classes, %d samples/image, %d trees "
                        "depth %d, %d features x %d thresholds, minSampleCount %d" % (
                            W["images"], W["width"], W["height"], W["classes"], W["samples_per_image"], W["trees"],
                            W["max_depth"], W["features"], W["thresholds"], W["min_samples"]),
            "images": W["images"], "frame": "%dx%d" % (W["width"], W["height"]), "classes": W["classes"],
            "trees_per_gpu": W["trees"], "max_depth": W["max_depth"], "features": W["features"],
            "thresholds": W["thresholds"], "samples_per_image": W["samples_per_image"],
            "l2": "inputs larger than L2 (integral images 1.23 GB)"}


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


def make_data():
    import curfil_b200 as cf
    return cf.synthetic_frames(W["seed"], W["images"], W["width"], W["height"], W["cells"], W["classes"])


def train_config():
    import curfil_b200 as cf
    return cf.TrainConfig(random_seed=4711, samples_per_image=W["samples_per_image"], feature_count=W["features"],
                          min_sample_count=W["min_samples"], max_depth=W["max_depth"], box_radius=W["box_radius"],
                          region_size=W["region_size"], thresholds=W["thresholds"])


def tree_samples(labels, depth, cfg, tree_ids):
    import curfil_b200 as cf
    seed = cf.forest_seed(cfg.random_seed)
    out = []
    for t in tree_ids:
        s, prior, counter = cf.sample_tree_pixels(labels, depth, W["classes"], cfg, W["trees"], seed + t)
        out.append((t, s, prior, counter))
    return out


# ----------------------------------------------------------------------------------------- CPU baseline
def cpu_root_split_search(rgb, depth, labels, seconds=15.0, threads=None):
    """The reference's CPU split search (FeatureEvaluationCPU + calculateScores + argmax) on the oracle,
    for the root node of tree 0 with as many candidate features as fit in ~`seconds`."""
    import curfil_b200 as cf
    from oracle import pyoracle as orc
    threads = threads or os.cpu_count()
    cfg = train_config()
    (_, samples, _, counter), = tree_samples(labels, depth, cfg, [0])
    ods = orc.integral(rgb, depth)
    s = samples.view(orc.SAMPLE_DTYPE)
    feats, thr = orc.generate_features(ods, s, 12345, W["features"], W["thresholds"], W["box_radius"],
                                       W["region_size"])
    hist = np.bincount(s["label"], minlength=W["classes"]).astype(np.uint32)

    def run(F):
        idx = np.linspace(0, W["features"] - 1, F).astype(int)   # keep the depth/colour mix
        f, t = np.ascontiguousarray(feats[:, idx]), np.ascontiguousarray(thr[:, idx])
        t0 = time.perf_counter()
        counters = orc.histograms(ods, s, f, t, W["classes"], threads=threads)
        sc = orc.scores(counters, hist)
        orc.best_split(sc)
        return time.perf_counter() - t0

    probe_f = 8
    dt = run(probe_f)
    F = int(max(probe_f, min(W["features"], probe_f * seconds / max(dt, 1e-6))))
    F = max(2, F - F % 2)
    dt = run(F)
    evals = len(s) * F
    return {"value": evals / dt, "unit": "feature-evals/s", "cores": threads, "kind": "port",
            "sample": "root-node split search of tree 0: %d samples x %d of %d candidate features x %d thresholds "
                      "(oracle restatement of FeatureEvaluationCPU + calculateScores, OpenMP)" % (
                          len(s), F, W["features"], W["thresholds"]),
            "seconds": dt}, ods


# ----------------------------------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import curfil_b200 as cf  # noqa: F401  (synthetic frames only)
    rgb, depth, labels = make_data()
    budget = max(5.0, 60.0 / max(1, args.steps + args.warmup))
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        base, _ = cpu_root_split_search(rgb, depth, labels, seconds=budget)
        if i >= args.warmup:
            vals.append(base["value"])
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": "feature-evals/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": base["seconds"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(),
            "cpu_baseline": {"value": value, "unit": "feature-evals/s", "cores": base["cores"], "kind": "port",
                             "sample": base["sample"]},
            "e2e": {"value": value, "unit": "feature-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference cannot be built here (Boost, TBB, Vigra, cuv::ndarray absent; texture references "
                    "removed in CUDA 12); its CPU path is timed through the oracle restatement"}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------- prediction
def forest_trees(ds, labels, depth, cfg, n_trees):
    """n_trees trees trained with the full-size settings, the forest sampling split over n_trees."""
    import curfil_b200 as cf
    seed = cf.forest_seed(cfg.random_seed)
    trees = []
    for t in range(n_trees):
        s, prior, counter = cf.sample_tree_pixels(labels, depth, W["classes"], cfg, n_trees, seed + t)
        tree, _ = cf.train_tree(ds, s, W["classes"], cfg, tree_id=t, seed_counter=counter)
        tree.set_prior(prior)
        trees.append(tree)
    return trees


def predict_section(ctx, stream, ds, trees, local, serve_seconds):
    """Batch prediction of resident frames (one launch), the plain per-image launch form on the same
    frames (identical results required), a CUDA-graph replay from pinned host frames, and Poisson
    serving of mixed frame sizes."""
    import torch
    import curfil_b200 as cf
    n, C, H, Wd = W["predict_images"], W["classes"], W["height"], W["width"]
    px = n * H * Wd
    forest = cf.Forest(ctx, trees)
    out = {"images": n, "frame": "%dx%d" % (Wd, H), "trees": len(trees), "forest_nodes": forest.num_nodes}
    pa = torch.empty((n, C, H, Wd), dtype=torch.float32, device=local)
    la = torch.empty((n, H, Wd), dtype=torch.uint8, device=local)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ctx.reset_timing()
    ctx.set_timing(True)
    ms = timed(lambda: forest.predict_dataset(ds, 0, n, pa.data_ptr(), la.data_ptr()), 5)
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
    pms = timed(lambda: forest.predict_dataset_plain(ds, 0, n, pb.data_ptr(), lb.data_ptr()), 1)
    out["plain_per_image"] = {"mpx_per_s": px / (pms / 1e3) / 1e6, "ms_per_frame": pms / n,
                              "note": "one launch + synchronisation per tree per image, then normalise and argmax"}
    out["speedup_vs_plain"] = pms / ms
    out["labels_identical"] = bool(torch.equal(la, lb))
    out["probabilities_identical"] = bool(torch.equal(pa.view(torch.int32), pb.view(torch.int32)))
    del pa, la, pb, lb

    # the same 64 frames from pinned host buffers through one CUDA graph replay (labels back to the host)
    rgb, depth, _ = cf.synthetic_frames(W["seed"] + 7, n, Wd, H, W["cells"], C)
    g = cf.PredictGraph(forest, n, Wd, H, probabilities=False)
    g.rgb[...] = rgb
    g.depth[...] = depth
    g.run()
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        g.run()
    gs = (time.perf_counter() - t0) / reps
    out["graph_e2e"] = {"mpx_per_s": px / gs / 1e6, "ms_per_batch": gs * 1e3,
                        "h2d_bytes_per_batch": int(rgb.nbytes + depth.nbytes), "d2h_bytes_per_batch": int(px),
                        "note": "pinned host RGB-D -> H2D -> integral images -> classify -> labels D2H, one graph"}
    # the plain per-image form from the same host frames, as RandomForestImage::predict runs on the
    # GPU: upload, one launch + sync per tree, normalise, argmax, probabilities and labels copied back
    sub = min(n, 16)
    forest.predict_plain(rgb[:1], depth[:1], probabilities=False)
    t0 = time.perf_counter()
    _, lp = forest.predict_plain(rgb[:sub], depth[:sub], probabilities=False)
    ps = time.perf_counter() - t0
    spx = sub * H * Wd
    out["plain_per_image_host"] = {"mpx_per_s": spx / ps / 1e6, "frames": sub, "ms_per_frame": ps * 1e3 / sub,
                                   "d2h_bytes_per_frame": H * Wd * (4 * C + 1)}
    out["e2e_speedup_vs_plain"] = (px / gs) / (spx / ps)
    out["e2e_labels_identical"] = bool(np.array_equal(lp, g.labels[:sub]))
    g.close()
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
    _, _, labels = cf.synthetic_frames(W["seed"], n_train, W["width"], W["height"], W["cells"], W["classes"])
    # held out: the frames after the dataset's in the same seeded sequence (same class appearance)
    rgb_t, depth_t, labels_t = cf.synthetic_frames(W["seed"], n_test, W["width"], W["height"], W["cells"],
                                                   W["classes"], first=ds.n)
    test = cf.Dataset.from_raw(ctx, rgb_t, depth_t)
    r = cf.Refiner(ctx, W["classes"], hidden=64, epochs=8, batch=4096, pixels_per_image=20000, seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = r.train(forest, ds, 0, n_train, labels)
    train_s = time.perf_counter() - t0
    lab = torch.empty((n_test, W["height"], W["width"]), dtype=torch.uint8, device=local)
    forest.predict_dataset(test, 0, n_test, 0, lab.data_ptr())
    torch.cuda.synchronize()
    base = float((lab.cpu().numpy() == labels_t).mean())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r.predict(forest, test, 0, n_test, 0, lab.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    refined = float((lab.cpu().numpy() == labels_t).mean())
    px = n_test * W["width"] * W["height"]
    r.close()
    test.close()
    return {"train_frames": n_train, "train_pixels": n_train * 20000, "epochs": 8, "train_s": train_s,
            "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
            "heldout_frames": n_test, "forest_pixel_accuracy": base, "refined_pixel_accuracy": refined,
            "refined_predict_mpx_per_s": px / (e0.elapsed_time(e1) / 1e3) / 1e6}


def serve(forest, seconds):
    """Poisson arrivals (seeded) at each offered rate, frame sizes 160x120 : 320x240 : 640x480 :
    1280x960 = 1:2:4:1; latency = completion - submission on the server's clock."""
    import curfil_b200 as cf
    pool = {}
    for w, h, _ in SERVE_SIZES:
        rgb, depth, _ = cf.synthetic_frames(W["seed"] + w, 4, w, h, W["cells"], W["classes"])
        pool[(w, h)] = (rgb, depth)
    weights = np.array([k for _, _, k in SERVE_SIZES], np.float64)
    results = []
    for rate in SERVE_RATES:
        rng = np.random.default_rng(rate)
        count = max(8, int(rate * seconds))
        gaps = rng.exponential(1.0 / rate, count)
        kinds = rng.choice(len(SERVE_SIZES), count, p=weights / weights.sum())
        which = rng.integers(0, 4, count)
        srv = cf.Server(forest, hbm_budget_bytes=8 << 30, max_pending=1 << 16, **SERVE_CONFIG)
        # warm the server with one frame of each size
        for w, h, _ in SERVE_SIZES:
            rgb, depth = pool[(w, h)]
            srv.wait(srv.submit(rgb[0], depth[0]), (h, w))
        ids = []
        done = {}

        def drain():
            for rid, shape in iter(q.get, None):
                _, _, st = srv.wait(rid, shape, timeout_s=60.0)
                done[rid] = (st.submit_ms, st.admitted_ms, st.done_ms, shape)

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
        lat = np.array([done[r][2] - done[r][0] for r in ids])
        qwait = np.array([done[r][1] - done[r][0] for r in ids])
        big = np.array([done[r][3] == (480, 640) for r in ids])
        shapes = np.array([done[r][3] for r in ids])
        by_size = {f"{w}x{h}": float(np.percentile(lat[(shapes[:, 0] == h) & (shapes[:, 1] == w)], 99))
                   for w, h, _ in SERVE_SIZES if ((shapes[:, 0] == h) & (shapes[:, 1] == w)).any()}
        span = (max(done[r][2] for r in ids) - min(done[r][0] for r in ids)) / 1e3
        pxs = sum(done[r][3][0] * done[r][3][1] for r in ids)
        c = srv.counters()
        srv.close()
        results.append({"offered_fps": rate, "frames": count, "offered_mpx_per_s": rate * pxs / count / 1e6,
                        "mpx_per_s": pxs / span / 1e6, "p50_ms": float(np.percentile(lat, 50)),
                        "p99_ms": float(np.percentile(lat, 99)),
                        "p99_ms_640x480": float(np.percentile(lat[big], 99)) if big.any() else None,
                        "p99_ms_by_size": by_size,
                        "p99_admission_wait_ms": float(np.percentile(qwait, 99)),
                        "batches": c["batches"] - len(SERVE_SIZES), "rejected": c["rejected"]})
    return {"sizes": "160x120:320x240:640x480:1280x960 = 1:2:4:1", "trees": forest.num_trees,
            "server": dict(SERVE_CONFIG), "rates": results}


# ----------------------------------------------------------------------------------------- our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3,
                    help="timed cf_forest_train calls (after one untimed call) for the end-to-end figure")
    ap.add_argument("--no-per-node", action="store_true", help="skip the plain per-node comparison tree")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default split-search launch shape")
    # workload size (defaults: the full-size configuration); smaller cases are for profiler captures
    ap.add_argument("--images", type=int, default=W["images"])
    ap.add_argument("--trees", type=int, default=W["trees"])
    ap.add_argument("--max-depth", type=int, default=W["max_depth"])
    ap.add_argument("--predict-images", type=int, default=W["predict_images"])
    ap.add_argument("--predict-trees", type=int, default=W["predict_trees"])
    ap.add_argument("--serve-seconds", type=float, default=1.5, help="Poisson load per offered rate (0: skip)")
    ap.add_argument("--tuning", default="", help="split-search launch shape overrides, e.g. ctas_per_sm=4,"
                    "bins_budget_words=10240 (cf_eval_tuning field names)")
    ap.add_argument("--serve-config", default="", help="serving overrides, e.g. max_batch_frames=4,pipeline_depth=2")
    args = ap.parse_args()
    for kv in filter(None, args.serve_config.split(",")):
        k, v = kv.split("=")
        SERVE_CONFIG[k.strip()] = float(v) if k.strip() == "max_wait_ms" else int(v)
    W.update(images=args.images, trees=args.trees, max_depth=args.max_depth,
             predict_images=min(args.predict_images, args.images), predict_trees=args.predict_trees)
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

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    rgb, depth, labels = make_data()
    cfg = train_config()
    ctx = cf.Context(local)
    if args.tuning:
        overrides = {}
        for kv in args.tuning.split(","):
            k, v = kv.split("=")
            overrides[k.strip()] = float(v) if k.strip() == "items_per_slot" else int(v)
        ctx.set_tuning(**overrides)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    from curfil_b200 import distributed as cfdist
    # every rank trains W["trees"] trees of a world * W["trees"] forest (treeId % world == rank)
    tree_ids = cfdist.tree_ids_for_rank(rank, world, world * W["trees"])
    per_tree = tree_samples(labels, depth, cfg, tree_ids)
    # the split search's launch shape, chosen by the autotuner on this rank's first tree (untimed)
    autotune = None
    if not args.tuning and not args.no_autotune:
        t0_, s0_, _, c0_ = per_tree[0]
        autotune = cf.autotune_split_search(ds, s0_, W["classes"], cfg, tree_id=t0_, seed_counter=c0_)
        autotune.pop("key", None)

    def step():
        trees, evals = [], 0
        for t, s, prior, counter in per_tree:
            tree, _ = cf.train_tree(ds, s, W["classes"], cfg, tree_id=t, seed_counter=counter)
            tree.set_prior(prior)
            evals += tree.train_stats()[0]
            trees.append(tree)
        return trees, evals

    for _ in range(args.warmup):
        trees, evals_per_step = step()
    torch.cuda.synchronize()
    barrier()
    ctx.reset_timing()
    ctx.set_timing(True)
    launches0 = ctx.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        barrier()
        start.record(stream)
        total_evals = 0
        for _ in range(args.steps):
            trees, ev = step()
            total_evals += ev
        end.record(stream)
        torch.cuda.synchronize()
        barrier()
    ctx.set_timing(False)
    launches = ctx.launch_count() - launches0
    ms = start.elapsed_time(end)
    ms_max = max_over_ranks(ms)
    all_evals = sum_over_ranks(total_evals)
    value = all_evals / (ms_max / 1e3)
    eval_ms, eval_launches = ctx.kernel_time("level_eval")
    kernel_ms = {k: ctx.kernel_time(k)[0] for k in ("level_eval", "gen_features", "route_flags", "route_scatter",
                                                     "scan", "reduce_candidates", "sort_features")}
    # the forest of all ranks assembled on every rank (the only exchange; untimed)
    n_forest_trees = len(cfdist.gather_forest(trees)) if dist is not None else len(trees)

    # algorithmic bytes of the level-batched evaluation: half the candidates are depth features
    bytes_per_eval = (BYTES_DEPTH_EVAL + BYTES_COLOR_EVAL) / 2.0
    achieved = total_evals * bytes_per_eval / (eval_ms / 1e3) / 1e9 if eval_ms > 0 else None
    peak, peak_kind = load_peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "level_eval_traffic.txt")
    if os.path.exists(tp):
        for ln in open(tp):
            if ln.startswith("dram_bytes_per_feature_eval:"):
                traffic = float(ln.split(":")[1]) * total_evals / max(1, eval_launches)

    # prediction: a forest of predict_trees trees trained with the same settings, 64 resident frames
    predict = None
    if W["predict_images"] > 0:
        ptrees = forest_trees(ds, labels, depth, cfg, W["predict_trees"])
        predict = predict_section(ctx, stream, ds, ptrees, local, args.serve_seconds)
        for t in ptrees:
            t.close()

    # end to end through cf_forest_train with host buffers: frames in, trees out
    def forest_e2e(sampler, steps):
        c = train_config()
        c.sampler = sampler
        # one untimed step first: the first cf_forest_train call of a sampler pays one-time costs
        # (its device buffers, the sampler's stream and pinned staging)
        for t in cf.train_forest(ctx, rgb, depth, labels, W["classes"], c, W["trees"]):
            t.close()
        barrier()
        t0 = time.perf_counter()
        e2e_evals = 0
        d2h = 0
        for _ in range(steps):
            ts = cf.train_forest(ctx, rgb, depth, labels, W["classes"], c, W["trees"])
            for t in ts:
                e2e_evals += t.train_stats()[0]
                d2h += t.num_nodes * (4 * 4 + 11 + 4 + 8 + 4 * W["classes"])
                t.close()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        h2d = rgb.nbytes + depth.nbytes + (labels.nbytes + depth.nbytes if sampler == 1 else 0)
        return {"value": sum_over_ranks(e2e_evals) / e2e_s, "unit": "feature-evals/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h / steps)}

    e2e = None
    if args.e2e_steps > 0:
        e2e = forest_e2e(1, args.e2e_steps)
        e2e["note"] = ("cf_forest_train: frames and labels uploaded, GPU integral images, device class-uniform "
                       "sampling, level-batched training, trees downloaded")
        e2e["reference_sampler"] = forest_e2e(0, 1)
        e2e["reference_sampler"]["note"] = ("the same with the reference's class-uniform reservoir on one host "
                                            "thread (its RNG streams)")

    # the plain per-node form (reference-structured kernels: responses to HBM, one block per
    # (threshold, feature), score kernel, host argmax, node by node) on this rank's first tree:
    # same tree required, feature-evals/s compared
    per_node = None
    if not args.no_per_node:
        t, s, prior, counter = per_tree[0]
        res = {}
        for name, mode in (("level_batched", cf.LEVEL_BATCHED), ("per_node", cf.PER_NODE)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            tree, _ = cf.train_tree(ds, s, W["classes"], cfg, tree_id=t, seed_counter=counter, mode=mode)
            e1.record(stream)
            torch.cuda.synchronize()
            res[name] = (tree.arrays(), e0.elapsed_time(e1), tree.train_stats()[0],
                         [round(float(x[2]), 2) for x in tree.level_stats()])
        (A, lb_ms, lb_ev, lb_lv), (B, pn_ms, pn_ev, pn_lv) = res["level_batched"], res["per_node"]
        # leaves carry a NaN threshold, which must compare equal
        identical = lb_ev == pn_ev and all(np.array_equal(A[k], B[k], equal_nan=A[k].dtype.kind == "f") for k in A)
        per_node = {"value": pn_ev / (pn_ms / 1e3), "unit": "feature-evals/s", "ms_per_tree": pn_ms,
                    "level_batched_value": lb_ev / (lb_ms / 1e3), "level_batched_ms_per_tree": lb_ms,
                    "speedup": pn_ms / lb_ms, "trees_identical": bool(identical), "tree": int(t),
                    "split_search_ms_per_level": {"per_node": pn_lv, "level_batched": lb_lv}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, _ = cpu_root_split_search(rgb, depth, labels, seconds=15.0)
        cpu.pop("seconds", None)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "feature-evals/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(workload_config(), parallelism="trees sharded over %d GPU(s)" % world,
                               split_search_tuning=ctx.get_tuning().as_dict(), autotune=autotune),
                "roofline": {"bound": "hbm", "kernel": "level_eval", "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                             "peak_source": peak_kind, "bytes_per_eval": bytes_per_eval,
                             "avg_launch_ms": eval_ms / max(1, eval_launches), "launches": eval_launches},
                "kernel_ms": kernel_ms,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "forest_trees": n_forest_trees,
                "clocks": clocks.summary(),
                "predict": predict,
                "per_node": per_node,
                "levels_tree0": [[n, s, round(ms, 3)] for n, s, ms in trees[0].level_stats()],
                "feature_evals_per_step": total_evals / args.steps,
                # split evaluations: every feature evaluation is binned against all T thresholds
                "split_evals_per_s": value * W["thresholds"],
                "per_node_split_evals_per_s": per_node["value"] * W["thresholds"] if per_node else None}
        print(json.dumps(line), flush=True)
    ds.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
