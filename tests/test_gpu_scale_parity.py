"""Parity with the oracle at the benchmark configurations' own sizes, not only on small scenes:

- plain method, small: one tree on 16 frames 320x240 (8 classes, void ignored, 500 samples per class
  and image, 500 features x 20 thresholds, depth 12), in full;
- plain method, full size: tree 0 of the 3-tree forest on 200 frames 640x480 (40 classes, 2000
  features x 20 thresholds, depth 20, minSampleCount 50), in full, against the oracle's tree with all
  host threads (about half a minute of CPU);
- batched prediction: a 10-tree depth-20 forest trained with the full-size settings, two 640x480
  frames predicted on the GPU and by the oracle (labels >= 99.9 % equal, probabilities within 1e-5).

Trees are compared path by path (helpers.compare_trees): identical histograms and splits, a
different split accepted only where the two scores tie within 1e-6 relative.
"""
import os

import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H

pytestmark = pytest.mark.gpu

THREADS = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


def gpu_and_oracle_tree(ctx, rgb, depth, labels, C, cfg, num_trees, tree, ignored=None, ods=None):
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    seed = cf.forest_seed(cfg.random_seed)
    s, prior, counter = cf.sample_tree_pixels(labels, depth, C, cfg, num_trees, seed + tree, ignored=ignored)
    g, _ = cf.train_tree(ds, s, C, cfg, tree_id=tree, seed_counter=counter)
    ods = ods if ods is not None else orc.integral(rgb, depth)
    rc, o, _ = orc.train_tree(ods, s.view(orc.SAMPLE_DTYPE), C, cfg.feature_count, cfg.thresholds, cfg.max_depth,
                              cfg.min_sample_count, cfg.box_radius, cfg.region_size, counter, threads=THREADS)
    assert rc == 0
    A = g.arrays()
    g.close()
    ds.close()
    return A, H.oracle_tree_dict(o), len(s)


def test_plain_method_small_configuration_tree(ctx):
    C = 8
    rgb, depth, labels = cf.synthetic_frames(2027, 16, 320, 240, 12, C)
    ignore = np.zeros(C, np.uint8)
    ignore[0] = 1
    cfg = cf.TrainConfig(random_seed=4711, samples_per_image=3500, feature_count=500, thresholds=20, max_depth=12,
                         min_sample_count=1, box_radius=60, region_size=15)
    g, o, n = gpu_and_oracle_tree(ctx, rgb, depth, labels, C, cfg, 1, 0, ignored=ignore)
    assert n == 56000
    compared = H.compare_trees(g, o)
    assert compared > 500


def test_plain_method_full_size_tree0(ctx):
    C = 40
    rgb, depth, labels = cf.synthetic_frames(2026, 200, 640, 480, 40, C)
    cfg = cf.TrainConfig(random_seed=4711, samples_per_image=4000, feature_count=2000, thresholds=20, max_depth=20,
                         min_sample_count=50, box_radius=60, region_size=15)
    g, o, n = gpu_and_oracle_tree(ctx, rgb, depth, labels, C, cfg, 3, 0)
    assert n == 266600
    compared = H.compare_trees(g, o)
    assert compared > 2000


def test_batched_prediction_ten_tree_forest(ctx):
    C = 40
    rgb, depth, labels = cf.synthetic_frames(2026, 200, 640, 480, 40, C)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    cfg = cf.TrainConfig(random_seed=4711, samples_per_image=4000, feature_count=2000, thresholds=20, max_depth=20,
                         min_sample_count=50, box_radius=60, region_size=15, sampler=1)
    trees = cf.train_forest(ctx, rgb, depth, labels, C, cfg, 10)
    ds.close()
    forest = cf.Forest(ctx, trees)
    frgb, fdepth, _ = cf.synthetic_frames(2026 + 7, 2, 640, 480, 40, C)
    probs, lab = forest.predict(frgb, fdepth)
    views, normalized = [], []
    for t in trees:
        A = t.arrays()
        pr = t.prior()
        normalized.append(np.stack([orc.normalize_histogram(h, pr, 0.0, True) for h in A["histogram"]]))
        v = orc.Tree(len(A["left"]), C)
        v.left, v.feature, v.threshold = A["left"], A["feature"], A["threshold"]
        views.append(v)
    assert min(v.num_nodes for v in views) > 1000
    ods = orc.integral(frgb, fdepth)
    for i in range(2):
        op, ol = orc.predict(ods, i, views, normalized, C, threads=THREADS)
        assert (ol == lab[i]).mean() >= 0.999
        np.testing.assert_allclose(probs[i], op, atol=1e-5)
    forest.close()
    for t in trees:
        t.close()
