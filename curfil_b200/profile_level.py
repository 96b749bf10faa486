"""Runs one tree level of the split search inside a profiler range, for Nsight Compute.

    ncu --profile-from-start off ... python -m curfil_b200.profile_level --images 200 --features 1000 --level 12

Synthetic frames (the seeded generator of `synthetic_frames`), device class-uniform sampling of 8000
pixels per frame, one tree trained to the level with the batching configuration's settings
(minSampleCount 1, box radius 60, region 15), the level captured as a snapshot and run twice
unprofiled; the third run is the profiled one. Prints the level's shape and the split-search kernels'
times of that run (CUDA events).
"""
import argparse

import torch

import curfil_b200 as cf


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--images", type=int, default=200)
    ap.add_argument("--features", type=int, default=1000)
    ap.add_argument("--thresholds", type=int, default=32)
    ap.add_argument("--level", type=int, default=12)
    ap.add_argument("--tuning", default="", help="cf_eval_tuning overrides, e.g. stage_bins=0")
    args = ap.parse_args(argv)
    rgb, depth, labels = cf.synthetic_frames(2026, args.images, 640, 480, 40, 40)
    ctx = cf.Context(0)
    if args.tuning:
        kw = {}
        for kv in args.tuning.split(","):
            k, v = kv.split("=")
            kw[k] = float(v) if k == "items_per_slot" else int(v)
        ctx.set_tuning(**kw)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    cfg = cf.TrainConfig(random_seed=4711, samples_per_image=80000, feature_count=args.features, min_sample_count=1,
                         max_depth=args.level + 1, box_radius=60, region_size=15, thresholds=args.thresholds, sampler=1)
    s, _, counter = cf.sample_tree_pixels(labels, depth, 40, cfg, 10, cf.forest_seed(4711), ctx=ctx)
    tree, snaps, _ = cf.train_tree_snapshots(ds, s, 40, cfg, [args.level], seed_counter=counter)
    sn = snaps[0]
    print("level", sn.level, "nodes", sn.num_nodes, "samples", sn.num_samples, flush=True)
    for _ in range(2):
        sn.run()
    ctx.set_timing(True)
    ctx.reset_timing()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    r = sn.run()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print("level ms", round(r["ms"], 3), {k: ctx.kernel_time(k) for k in ("stage_bins", "level_eval")}, flush=True)


if __name__ == "__main__":
    main()
