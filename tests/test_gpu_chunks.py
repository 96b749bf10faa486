"""Split search over sample chunks: where a level has fewer work items than four per resident CTA, the
items of nodes with at least 8192 samples are cut into sample chunks whose counts are merged in global
memory (the last chunk to finish scores them). Nodes of 20 000 and 9 000 samples with 96 features give
a few dozen items, so both are chunked (4 and 2 chunks); the counts and trees must equal the oracle's."""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def scene(ctx):
    rgb, depth, labels = H.frames(seed=41, n=12, w=160, h=120, cells=14, classes=12)
    return dict(rgb=rgb, depth=depth, labels=labels, ods=orc.integral(rgb, depth),
                ds=cf.Dataset.from_raw(ctx, rgb, depth))


@pytest.mark.parametrize("flips", [False, True])
def test_chunked_level_counts_bit_exact(ctx, scene, flips):
    rng = np.random.default_rng(71 + flips)
    sizes = [20000, 9000, 300, 1]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, 12, 160, 120, 40, int(offsets[-1]), depth=scene["depth"], flips=flips)
    fe, th = orc.generate_features(scene["ods"], s, 96, 96, 12, 60, 15)
    best, left = cf.level_left_counts(scene["ds"], offsets, s, 40, fe, th)
    for i in range(len(sizes)):
        sl = s[offsets[i]:offsets[i + 1]]
        o = orc.histograms(scene["ods"], sl.view(orc.SAMPLE_DTYPE), fe, th, 40, threads=8)   # [C][F][T][2]
        np.testing.assert_array_equal(left[i], o[:, :, :, 0].transpose(1, 2, 0), err_msg="node %d" % i)


@pytest.mark.parametrize("flip", [False, True])
def test_chunked_train_tree_matches_oracle(ctx, scene, flip):
    samples, _ = H.class_uniform_samples(scene["labels"], scene["depth"], 12, 2000)
    assert len(samples) >= 2 * 8192
    if flip:
        samples["flip"] = 2
    cfg = cf.TrainConfig(feature_count=100, thresholds=12, max_depth=8, min_sample_count=4, box_radius=40,
                         region_size=10)
    tree, counter = cf.train_tree(scene["ds"], samples, 12, cfg, tree_id=0, seed_counter=640)
    rc, otree, ocounter = orc.train_tree(scene["ods"], samples.view(orc.SAMPLE_DTYPE), 12, 100, 12, 8, 4, 40, 10, 640,
                                         threads=8)
    assert rc == 0
    assert counter == ocounter
    g = tree.arrays()
    o = H.oracle_tree_dict(otree)
    n = H.compare_trees(g, o)
    assert n > 20
