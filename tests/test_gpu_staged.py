"""Staged bins: the split search in two passes (bins of every (sample, feature) computed in frame order
into a byte table, then histogrammed node by node) gives the counts, splits and trees of the fused
search and of the oracle. `stage_bins = 2` forces the two passes on these small frames (by default they
run only where the integral images exceed L2); `stage_max_mb = 1` cuts a level into feature chunks."""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H

pytestmark = pytest.mark.gpu

W, HT, N_IMG, C = 96, 72, 5, 40


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def scene(ctx):
    rgb, depth, labels = H.frames(seed=17, n=N_IMG, w=W, h=HT, cells=12, classes=C)
    return dict(rgb=rgb, depth=depth, labels=labels, ods=orc.integral(rgb, depth),
                ds=cf.Dataset.from_raw(ctx, rgb, depth))


def expected_chunks(rows, F, max_mb):
    """Feature chunks of the staged table: whole 32-feature blocks, at most max_mb MiB, as even as
    possible."""
    tiles = -(-F // 32)
    tiles_max = max(1, (max_mb << 20) // rows // 32)
    n = -(-tiles // tiles_max)
    chunk = -(-tiles // n) * 32
    return -(-F // chunk)


def staged_launches(ctx, fn):
    """Runs fn with kernel timing on; returns (fn's result, stage_bins launches)."""
    ctx.set_timing(True)
    ctx.reset_timing()
    try:
        out = fn()
        _, n = ctx.kernel_time("stage_bins")
    finally:
        ctx.set_timing(False)
    return out, n


@pytest.mark.parametrize("T", [20, 32, 45, 100])
@pytest.mark.parametrize("max_mb", [8192, 1])
def test_staged_counts_equal_fused_and_oracle(ctx, scene, T, max_mb):
    """Pass 1 + pass 2 (in one or several feature chunks) against the fused search and the oracle."""
    rng = np.random.default_rng(T + max_mb)
    # many nodes of ragged sizes, samples spread over all frames, flips 0 / 1 / 2
    sizes = [1, 2, 3, 900, 40, 257, 5, 1200, 64, 1, 333] + [int(x) for x in rng.integers(1, 120, 40)]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, N_IMG, W, HT, C, int(offsets[-1]), depth=scene["depth"], flips=True)
    F = 331   # not a multiple of the 32-feature pass-1 tile
    fe, th = orc.generate_features(scene["ods"], s, 7 + T, F, T, 60, 15)
    th[1, :] = th[0, :]   # duplicate thresholds
    try:
        ctx.set_tuning(stage_bins=0)
        best0, left0 = cf.level_left_counts(scene["ds"], offsets, s, C, fe, th)
        ctx.set_tuning(stage_bins=2, stage_max_mb=max_mb)
        (best2, left2), launches = staged_launches(
            ctx, lambda: cf.level_left_counts(scene["ds"], offsets, s, C, fe, th))
    finally:
        ctx.set_tuning()
    assert launches == expected_chunks(int(offsets[-1]), F, max_mb) and launches >= 1
    np.testing.assert_array_equal(left2, left0)
    # (flags, which depend on how the items split the features, are not compared)
    for k in ("score", "feature", "threshold_index", "threshold"):
        np.testing.assert_array_equal(best2[k], best0[k], err_msg=k)
    for i in (0, 3, 7, 10):
        sl = s[offsets[i]:offsets[i + 1]]
        o = orc.histograms(scene["ods"], sl.view(orc.SAMPLE_DTYPE), fe, th, C, threads=4)
        np.testing.assert_array_equal(left2[i], o[:, :, :, 0].transpose(1, 2, 0), err_msg="node %d" % i)


def test_staged_tree_equals_fused_tree_and_oracle(ctx, scene):
    samples, _ = H.class_uniform_samples(scene["labels"], scene["depth"], C, 60)
    cfg = cf.TrainConfig(feature_count=200, thresholds=16, max_depth=12, min_sample_count=2, box_radius=60,
                         region_size=15)
    trees = {}
    try:
        for stage in (0, 2):
            ctx.set_tuning(stage_bins=stage, stage_max_mb=1)
            (tree, _), n = staged_launches(ctx, lambda: cf.train_tree(scene["ds"], samples, C, cfg, seed_counter=4))
            assert (n > 0) == (stage == 2)
            trees[stage] = tree.arrays()
            tree.close()
    finally:
        ctx.set_tuning()
    for k in trees[0]:
        np.testing.assert_array_equal(trees[2][k], trees[0][k], err_msg=k)
    assert trees[2]["left"].size > 30
    rc, otree, _ = orc.train_tree(scene["ods"], samples.view(orc.SAMPLE_DTYPE), C, 200, 16, 12, 2, 60, 15, 4,
                                  threads=4)
    assert rc == 0
    assert H.compare_trees(trees[2], H.oracle_tree_dict(otree)) > 30


def test_staging_off_above_255_thresholds(ctx, scene):
    """Bins are stored in bytes: with more than 255 thresholds the level runs fused."""
    rng = np.random.default_rng(3)
    offsets = np.array([0, 300, 500], np.int64)
    s = H.random_samples(rng, N_IMG, W, HT, C, 500, depth=scene["depth"])
    fe, th = orc.generate_features(scene["ods"], s, 99, 40, 300, 60, 15)
    try:
        ctx.set_tuning(stage_bins=2)
        (best, left), n = staged_launches(ctx, lambda: cf.level_left_counts(scene["ds"], offsets, s, C, fe, th))
    finally:
        ctx.set_tuning()
    assert n == 0
    o = orc.histograms(scene["ods"], s[:300].view(orc.SAMPLE_DTYPE), fe, th, C, threads=4)
    np.testing.assert_array_equal(left[0], o[:, :, :, 0].transpose(1, 2, 0))


def test_sorted_sample_copy_gives_the_same_counts(ctx, scene):
    """The one-pass search over the copy sorted by (node, frame, Morton code) counts what the level's own
    order counts, sliced nodes included."""
    rng = np.random.default_rng(11)
    sizes = [9000, 1, 17, 2500, 300] + [int(x) for x in rng.integers(1, 200, 30)]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, N_IMG, W, HT, C, int(offsets[-1]), depth=scene["depth"], flips=True)
    fe, th = orc.generate_features(scene["ods"], s, 21, 120, 24, 60, 15)
    out = {}
    try:
        for order in (0, 2):
            ctx.set_tuning(stage_bins=0, sample_order=order)
            ctx.set_timing(True)
            ctx.reset_timing()
            out[order] = cf.level_left_counts(scene["ds"], offsets, s, C, fe, th)
            assert (ctx.kernel_time("gather_sorted_samples")[1] > 0) == (order == 2)
            ctx.set_timing(False)
    finally:
        ctx.set_timing(False)
        ctx.set_tuning()
    np.testing.assert_array_equal(out[2][1], out[0][1])
    for k in ("score", "feature", "threshold_index", "threshold"):
        np.testing.assert_array_equal(out[2][0][k], out[0][0][k], err_msg=k)
