"""Tree packing and traversal against the reference's packing tests (src/tests/
random_tree_image_gpu_test.cu:990-1304): the two-split recall tree and degenerate trees longer than
the reference's 2048-node layers, imported through cf_tree_import and packed by cf_forest_create,
must send every pixel to the leaf the oracle's traversal reaches and give that leaf's normalised
histogram (random_tree.cpp:54-104) as its probabilities."""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests.golden import reference_kats as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


def frame(seed, H=480, W=640):
    """Random colour with channel 2 zero in the left half, depth in 16x16 blocks of 1 m or 60 m, so
    that the recall tree's depth split (threshold -29.1 m) sends pixels both ways."""
    rng = np.random.default_rng(seed)
    blocks = rng.choice([1000, 60000], (H // 16, W // 16), p=[0.6, 0.4]).astype(np.uint16)
    depth = np.kron(blocks, np.ones((16, 16), np.uint16))[None]
    rgb = rng.integers(0, 256, (1, H, W, 3), dtype=np.uint8)
    rgb[0, :, : W // 2, 2] = 0
    return rgb, depth


def predict_both(ctx, left, feature, threshold, hist, prior, rgb, depth):
    C = hist.shape[1]
    tree = cf.Tree.from_arrays(0, left, feature, threshold, hist)
    forest = cf.Forest(ctx, [tree], prior=prior)
    probs, labels = forest.predict(rgb, depth)
    forest.close()
    tree.close()
    normalized = np.stack([orc.normalize_histogram(h, prior, 0.0, True) for h in hist])
    view = orc.Tree(len(left), C)
    view.left, view.feature, view.threshold = left, feature, threshold
    op, ol = orc.predict(orc.integral(rgb, depth), 0, [view], [normalized], C, threads=8)
    return probs[0], labels[0], op, ol, normalized


def test_recall_tree_leaf_paths_and_normalised_histograms(ctx):
    R = K.RECALL_TREE
    left = np.array([1, 3, -1, -1, -1], np.int32)
    feature = np.zeros((5, 11), np.int8)
    feature[0] = R["split2"]["feature"]   # n0: depth feature
    feature[1] = R["split1"]["feature"]   # n1: colour feature
    threshold = np.array([R["split2"]["threshold"], R["split1"]["threshold"], np.nan, np.nan, np.nan], np.float32)
    h = R["hist"]
    hist = np.array([[a + b for a, b in zip(h[1], h[2])], h[1], h[2], h[3], h[4]], np.uint32)
    prior = np.array(R["prior"], np.uint32)
    rgb, depth = frame(5)
    probs, labels, op, ol, normalized = predict_both(ctx, left, feature, threshold, hist, prior, rgb, depth)
    np.testing.assert_array_equal(labels, ol)
    np.testing.assert_allclose(probs, op, atol=1e-6)
    # every leaf is reached, and a pixel's probabilities are its leaf's normalised histogram
    for leaf in (2, 3, 4):
        v = (normalized[leaf] / normalized[leaf].sum()).astype(np.float32)
        at = np.abs(probs - v[:, None, None]).max(0) < 1e-6
        assert at.sum() > 1000, "leaf %d reached by %d pixels" % (leaf, at.sum())
    # the normalised histograms themselves (equal priors: the counts over their sum)
    for leaf in (1, 2, 3, 4):
        np.testing.assert_allclose(normalized[leaf] * 3.0, hist[leaf] / hist[leaf].sum(), rtol=1e-15)


@pytest.mark.parametrize("num_nodes", [10, 100, 3 * 2048 + 2])
def test_degenerate_trees_beyond_one_node_layer(ctx, num_nodes):
    """The degenerate trees of testRecallLargeForest: each left child splits again, so the tree has
    num_nodes + 1 nodes in a chain of levels (the reference packs at most 2048 nodes per layer)."""
    rng = np.random.default_rng(num_nodes)
    n = num_nodes + 1
    left = np.full(n, -1, np.int32)
    node = 0
    for child in range(1, num_nodes, 2):
        left[node] = child
        node = child
    split = left >= 0
    feature = np.zeros((n, 11), np.int8)
    feature[:, 0] = rng.integers(0, 2, n)
    feature[:, 1:5] = rng.integers(-120, 121, (n, 4))
    feature[:, 5:9] = rng.integers(1, 21, (n, 4))
    feature[:, 9:11] = np.where(feature[:, :1] == 1, rng.integers(0, 3, (n, 2)), 0)
    feature[~split] = 0
    threshold = np.where(split, rng.uniform(-2, 2, n), np.nan).astype(np.float32)
    hist = rng.integers(0, 50, (n, 3)).astype(np.uint32)
    hist[:, 0] += 1
    prior = np.array([100, 100, 100], np.uint32)
    rgb, depth = frame(num_nodes, H=240, W=320)
    depth[depth == 60000] = 3000
    probs, labels, op, ol, _ = predict_both(ctx, left, feature, threshold, hist, prior, rgb, depth)
    assert (labels == ol).mean() >= 0.999
    np.testing.assert_allclose(probs, op, atol=1e-5)
