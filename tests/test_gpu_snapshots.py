"""Level snapshots: one level of a tree's training run again on its own (the loop body of
RandomTreeTrain::train, random_tree.h:1262-1410). A snapshot's run must reproduce the splits the
tree took at that level, in both split-search forms, and the level's next-level sizes; its exported
inputs through the host-buffer entry points (candidate generation + evaluateBestSplits) must give
the same splits."""
import numpy as np
import pytest

import curfil_b200 as cf
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


def tree_level_splits(a, level):
    """(feature id, threshold) of the split nodes of one level, breadth-first (the open nodes)."""
    m = (a["level"] == level) & (a["left"] >= 0)
    return a["feature_id"][m], a["threshold"][m], a["score"][m]


def test_snapshots_reproduce_their_levels(ctx):
    C = 10
    rgb, depth, labels = H.frames(seed=12, n=4, w=96, h=72, cells=12, classes=C)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    samples, _ = H.class_uniform_samples(labels, depth, C, 150)
    cfg = cf.TrainConfig(feature_count=120, thresholds=10, max_depth=9, min_sample_count=4)
    plain, sc0 = cf.train_tree(ds, samples, C, cfg, seed_counter=5)
    tree, snaps, sc1 = cf.train_tree_snapshots(ds, samples, C, cfg, [1, 3, 5, 30], seed_counter=5)
    assert sc0 == sc1
    A, B = plain.arrays(), tree.arrays()
    for k in A:
        np.testing.assert_array_equal(A[k], B[k], err_msg=k)   # capturing changes nothing
    assert [s.level for s in snaps] == [1, 3, 5]                # level 30 is beyond the tree
    stats = tree.level_stats()
    for s in snaps:
        nodes, nsamp, _ = stats[s.level - 1]
        assert (s.num_nodes, s.num_samples) == (nodes, nsamp)
        fid, thr, score = tree_level_splits(B, s.level)
        runs = [s.run(cf.LEVEL_BATCHED, splits=True), s.run(cf.LEVEL_BATCHED, splits=True),
                s.run(cf.PER_NODE, splits=True)]
        for r in runs:
            np.testing.assert_array_equal(r["splits"]["feature"], fid)
            np.testing.assert_array_equal(r["splits"]["threshold"], thr)
            np.testing.assert_allclose(r["splits"]["score"], score, rtol=1e-12)
            assert r["evals"] == s.num_samples * 120
            if s.level < len(stats):
                assert (r["next_nodes"], r["next_samples"]) == stats[s.level][:2]
            assert r["ms"] > 0
        # the exported inputs through the host-buffer entry points give the same splits
        offsets, lsamples, seed = s.export()
        assert offsets[-1] == s.num_samples and len(offsets) == s.num_nodes + 1
        if s.level == 1:
            np.testing.assert_array_equal(lsamples.view(np.uint8), samples.view(np.uint8))
        feats, thresholds = cf.generate_features(ds, lsamples, seed, 120, 10, cfg.box_radius, cfg.region_size)
        best = cf.evaluate_best_splits(ds, offsets, lsamples, C, feats, thresholds)
        np.testing.assert_array_equal(best["feature"], fid)
        np.testing.assert_array_equal(best["threshold"], thr)
    for s in snaps:
        s.close()
    tree.close()
    plain.close()
    ds.close()
