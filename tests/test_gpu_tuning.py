"""Split-search launch shapes (cf_eval_tuning) change speed only: counts, splits and trees are the same
under every valid tuning, and the generic threshold search (T > 31) is as exact as the padded one."""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H

pytestmark = pytest.mark.gpu

TUNINGS = [
    {},
    {"warp_aggregate": 1},
    {"sample_groups": 0},
    {"sample_groups": 0, "warp_aggregate": 1},
    {"ctas_per_sm": 4, "bins_budget_words": 4096},
    {"bins_budget_words": 1024, "features_per_tile": 2, "feature_granule": 1, "items_per_slot": 1000.0,
     "min_item_evals": 256},
    {"items_per_slot": 8192.0, "min_item_evals": 256},
    {"sample_groups": 0, "bins_budget_words": 1024, "features_per_tile": 2, "feature_granule": 1},
    {"ctas_per_sm": 1, "items_per_slot": 0.5, "feature_granule": 64, "features_per_tile": 64},
    {"sample_groups": 0, "ctas_per_sm": 1, "feature_granule": 64, "features_per_tile": 64},
    {"ctas_per_sm": 2, "bins_budget_words": 49152, "items_per_slot": 4.0, "feature_granule": 4},
    {"stage_bins": 2},
    {"stage_bins": 2, "warp_aggregate": 1, "stage_max_mb": 1},
    {"stage_bins": 2, "sample_groups": 0, "bins_budget_words": 1024, "features_per_tile": 2, "feature_granule": 1,
     "stage_max_mb": 1},
    {"stage_bins": 0},
    {"stage_bins": 0, "sample_order": 2},
    {"stage_bins": 0, "sample_order": 2, "sample_groups": 0, "warp_aggregate": 1},
    {"stage_bins": 0, "sample_order": 0},
]


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def scene(ctx):
    rgb, depth, labels = H.frames(seed=5, n=4, w=96, h=72, cells=12, classes=40)
    return dict(rgb=rgb, depth=depth, labels=labels, ods=orc.integral(rgb, depth),
                ds=cf.Dataset.from_raw(ctx, rgb, depth))


def test_default_tuning_and_reset(ctx):
    ctx.set_tuning()
    d = ctx.get_tuning().as_dict()
    assert d["ctas_per_sm"] == 3 and d["warp_aggregate"] == 0 and d["features_per_tile"] == 16
    assert d["sample_groups"] == 1 and d["stage_bins"] == 1 and d["stage_max_mb"] == 8192
    assert d["sample_order"] == 1
    ctx.set_tuning(items_per_slot=2.0)
    assert ctx.get_tuning().items_per_slot == 2.0
    ctx.set_tuning()
    assert ctx.get_tuning().as_dict() == d


@pytest.mark.parametrize("bad", [{"ctas_per_sm": 0}, {"ctas_per_sm": 5}, {"features_per_tile": 1},
                                 {"features_per_tile": 65}, {"bins_budget_words": 100},
                                 {"bins_budget_words": 49153}, {"warp_aggregate": 2}, {"feature_granule": 0},
                                 {"items_per_slot": 0.0}, {"items_per_slot": 9000.0}, {"min_item_evals": 100},
                                 {"stage_bins": 3}, {"stage_max_mb": 0}, {"sample_order": 3}])
def test_invalid_tuning_rejected(ctx, bad):
    ctx.set_tuning()
    before = ctx.get_tuning().as_dict()
    with pytest.raises(cf.CurfilError) as e:
        ctx.set_tuning(**bad)
    assert e.value.status == 1
    assert ctx.get_tuning().as_dict() == before


def test_tuning_changes_speed_not_results(ctx, scene):
    rng = np.random.default_rng(8)
    sizes = [900, 1, 40, 257, 3]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, 4, 96, 72, 40, int(offsets[-1]), depth=scene["depth"], flips=True)
    fe, th = orc.generate_features(scene["ods"], s, 5, 72, 12, 60, 15)
    samples, _ = H.class_uniform_samples(scene["labels"], scene["depth"], 40, 60)
    cfg = cf.TrainConfig(feature_count=96, thresholds=10, max_depth=7, min_sample_count=4, box_radius=40,
                         region_size=10)
    ref = None
    try:
        for t in TUNINGS:
            ctx.set_tuning()
            if t:
                ctx.set_tuning(**t)
            best, left = cf.level_left_counts(scene["ds"], offsets, s, 40, fe, th)
            tree, _ = cf.train_tree(scene["ds"], samples, 40, cfg, seed_counter=9)
            arrays = tree.arrays()
            if ref is None:
                ref = (best, left, arrays)
                continue
            np.testing.assert_array_equal(left, ref[1], err_msg=str(t))
            for k in ("score", "feature", "threshold_index", "threshold"):
                np.testing.assert_array_equal(best[k], ref[0][k], err_msg="%s %s" % (t, k))
            for k in arrays:
                np.testing.assert_array_equal(arrays[k], ref[2][k], err_msg="%s %s" % (t, k))
        assert ref[2]["left"].size > 30
    finally:
        ctx.set_tuning()


def test_autotune_keeps_the_tree_and_caches(ctx, scene, tmp_path):
    samples, _ = H.class_uniform_samples(scene["labels"], scene["depth"], 40, 40)
    cfg = cf.TrainConfig(feature_count=64, thresholds=10, max_depth=6, min_sample_count=4, box_radius=40,
                         region_size=10)
    ctx.set_tuning()
    before, _ = cf.train_tree(scene["ds"], samples, 40, cfg, seed_counter=3)
    cache = str(tmp_path / "tuning.json")
    try:
        r = cf.autotune_split_search(scene["ds"], samples, 40, cfg, seed_counter=3, cache=cache)
        assert not r["from_cache"] and r["trials"] >= 10
        assert r["split_search_ms"] <= r["start_ms"]
        assert ctx.get_tuning().as_dict() == r["tuning"]
        after, _ = cf.train_tree(scene["ds"], samples, 40, cfg, seed_counter=3)
        A, B = before.arrays(), after.arrays()
        for k in A:
            np.testing.assert_array_equal(A[k], B[k], err_msg=k)
        ctx.set_tuning()
        again = cf.autotune_split_search(scene["ds"], samples, 40, cfg, seed_counter=3, cache=cache)
        assert again["from_cache"] and again["tuning"] == r["tuning"]
        assert ctx.get_tuning().as_dict() == r["tuning"]
    finally:
        ctx.set_tuning()


@pytest.mark.parametrize("T", [31, 32, 45])
def test_counts_bit_exact_around_search_padding(ctx, scene, T):
    """T <= 31 takes the branch-free search over 32 padded positions, larger T the generic one."""
    rng = np.random.default_rng(T)
    sizes = [700, 2, 300]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, 4, 96, 72, 40, int(offsets[-1]), depth=scene["depth"], flips=True)
    fe, th = orc.generate_features(scene["ods"], s, 31 + T, 40, T, 60, 15)
    th[1, :] = th[0, :]
    _, left = cf.level_left_counts(scene["ds"], offsets, s, 40, fe, th)
    for i in range(len(sizes)):
        sl = s[offsets[i]:offsets[i + 1]]
        o = orc.histograms(scene["ods"], sl.view(orc.SAMPLE_DTYPE), fe, th, 40, threads=4)
        np.testing.assert_array_equal(left[i], o[:, :, :, 0].transpose(1, 2, 0), err_msg="node %d" % i)
