"""Edge configurations against the oracle: one feature and one threshold, threshold counts on both
sides of the padded searches (63, 64, 100), many classes in training and in prediction (the 128- and
256-class prediction kernels)."""
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
    rgb, depth, labels = H.frames(seed=31, n=3, w=80, h=64, cells=14, classes=12)
    return dict(rgb=rgb, depth=depth, labels=labels, ods=orc.integral(rgb, depth),
                ds=cf.Dataset.from_raw(ctx, rgb, depth))


@pytest.mark.parametrize("F,T,C,depth", [(1, 1, 2, 5), (7, 64, 12, 6), (33, 63, 12, 6), (20, 100, 12, 5),
                                         (60, 10, 200, 6)])
def test_train_tree_edges_match_oracle(ctx, scene, F, T, C, depth):
    labels = scene["labels"] % C
    absent = (np.bincount(labels.ravel(), minlength=C) == 0).astype(np.uint8)   # not sampled, as ignored
    samples, _ = H.class_uniform_samples(labels, scene["depth"], C, 40, ignore=absent)
    cfg = cf.TrainConfig(feature_count=F, thresholds=T, max_depth=depth, min_sample_count=2, box_radius=30,
                         region_size=8)
    rc, otree, ocounter = orc.train_tree(scene["ods"], samples.view(orc.SAMPLE_DTYPE), C, F, T, depth, 2, 30, 8,
                                         900, threads=4)
    if rc == -1:   # an empty child: the reference throws, so must the GPU path
        with pytest.raises(cf.CurfilError) as e:
            cf.train_tree(scene["ds"], samples, C, cfg, tree_id=1, seed_counter=900)
        assert e.value.status == 4
        return
    assert rc == 0
    tree, counter = cf.train_tree(scene["ds"], samples, C, cfg, tree_id=1, seed_counter=900)
    assert counter == ocounter
    g = tree.arrays()
    o = H.oracle_tree_dict(otree)
    H.compare_trees(g, o)
    assert tree.num_nodes >= 3


@pytest.mark.parametrize("C", [100, 200])
def test_predict_many_classes_matches_oracle(ctx, scene, C):
    labels = scene["labels"] * (C // 12) % C   # spread the present classes over 0..C-1
    prior = np.bincount(labels.ravel(), minlength=C).astype(np.uint32)
    trees, otrees, normalized = [], [], []
    for t in range(2):
        absent = (prior == 0).astype(np.uint8)
        samples, _ = H.class_uniform_samples(labels, scene["depth"], C, 30, seed_counter=70 + 5 * t, ignore=absent)
        cfg = cf.TrainConfig(feature_count=80, thresholds=10, max_depth=8, min_sample_count=2, box_radius=30,
                             region_size=8)
        tree, _ = cf.train_tree(scene["ds"], samples, C, cfg, tree_id=t, seed_counter=3 + t)
        trees.append(tree)
        a = tree.arrays()
        ot = orc.Tree(len(a["left"]), C)
        ot.left, ot.feature, ot.threshold, ot.histogram = a["left"], a["feature"], a["threshold"], a["histogram"]
        otrees.append(ot)
        normalized.append(np.stack([orc.normalize_histogram(h, prior, 0.0, True) for h in a["histogram"]]))
    forest = cf.Forest(ctx, trees, prior=prior)
    probs, lab = forest.predict(scene["rgb"], scene["depth"])
    for i in range(scene["rgb"].shape[0]):
        op, ol = orc.predict(scene["ods"], i, otrees, normalized, C, threads=4)
        assert (lab[i] == ol).mean() >= 0.999
        np.testing.assert_allclose(probs[i], op, atol=1e-5, rtol=0)
    assert lab.max() > 12
    forest.close()
