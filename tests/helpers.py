"""Shared fixtures: seeded synthetic frames, oracle datasets and sample lists."""
import numpy as np

import curfil_b200 as cf
from oracle import pyoracle as orc


def frames(seed=1, n=4, w=96, h=72, cells=10, classes=6):
    """Seeded synthetic RGB-D frames (rgb, depth_mm, labels) from the library's host generator."""
    return cf.synthetic_frames(seed, n, w, h, cells, classes)


def oracle_dataset(rgb, depth):
    return orc.integral(rgb, depth)


def class_uniform_samples(labels, depth, num_classes, per_image, seed_counter=100, ignore=None):
    ign = np.zeros(num_classes, np.uint8) if ignore is None else np.asarray(ignore, np.uint8)
    n, status = None, None
    status, s, counter = orc.sample_class_uniform(labels, depth, num_classes, ign, per_image, seed_counter)
    assert status > 0, "sampling failed (%d)" % status
    out = np.zeros(len(s), cf.SAMPLE_DTYPE)
    for k in ("x", "y", "image", "depth", "label", "flip"):
        out[k] = s[k]
    return out, counter


def random_samples(rng, n_images, w, h, num_classes, count, depth=None, flips=False):
    s = np.zeros(count, cf.SAMPLE_DTYPE)
    s["image"] = rng.integers(0, n_images, count)
    s["x"] = rng.integers(0, w, count)
    s["y"] = rng.integers(0, h, count)
    s["label"] = rng.integers(0, num_classes, count)
    if depth is None:
        s["depth"] = (rng.integers(500, 5001, count).astype(np.float32) / np.float32(1000.0))
    else:
        mm = depth[s["image"], s["y"], s["x"]]
        s["depth"] = np.where(mm > 0, mm.astype(np.float32) / np.float32(1000.0), np.float32(0.0))
    if flips:
        s["flip"] = rng.integers(0, 3, count)
    return s


def random_features(rng, F, box_radius=60, region_size=15, depth_fraction=0.5):
    f = np.zeros((11, F), np.int8)
    f[0] = (rng.random(F) >= depth_fraction).astype(np.int8)
    for r in (1, 2, 3, 4):
        f[r] = rng.integers(-box_radius, box_radius + 1, F)
    for r in (5, 6, 7, 8):
        f[r] = rng.integers(1, region_size + 1, F)
    f[9] = np.where(f[0] == 1, rng.integers(0, 3, F), 0)
    f[10] = np.where(f[0] == 1, rng.integers(0, 3, F), 0)
    same = (f[1] == f[3]) & (f[2] == f[4])
    f[3][same] += 1
    return f


def compare_trees(gpu, ora, rel=1e-6):
    """Path-by-path comparison of two breadth-first trees (dicts of arrays).

    Both trees are walked from the root together. At every pair of nodes reached by the same path the
    histograms must be identical, and so must the split (leaf or not, feature parameters, threshold);
    the score must agree to 1e-12. A differing split is accepted only where the two scores tie within
    `rel` relative; the two subtrees below it then differ and are skipped, while every other subtree
    is still compared. Returns the number of node pairs compared.
    """
    compared, skipped = 0, 0
    stack = [(0, 0)]
    while stack:
        a, b = stack.pop()
        np.testing.assert_array_equal(gpu["histogram"][a], ora["histogram"][b],
                                      err_msg="histogram of node %d (oracle node %d)" % (a, b))
        compared += 1
        leaf_a, leaf_b = gpu["left"][a] < 0, ora["left"][b] < 0
        assert leaf_a == leaf_b, "node %d / oracle node %d: leaf in one tree only" % (a, b)
        if leaf_a:
            continue
        same = np.array_equal(gpu["feature"][a], ora["feature"][b]) and gpu["threshold"][a] == ora["threshold"][b]
        if not same:
            if abs(gpu["score"][a] - ora["score"][b]) <= rel * abs(ora["score"][b]):
                skipped += 1
                continue
            raise AssertionError("node %d differs: gpu feat=%s thr=%r score=%r | oracle node %d feat=%s thr=%r "
                                 "score=%r" % (a, gpu["feature"][a], gpu["threshold"][a], gpu["score"][a], b,
                                               ora["feature"][b], ora["threshold"][b], ora["score"][b]))
        assert gpu["score"][a] == __import__("pytest").approx(ora["score"][b], rel=1e-12, abs=1e-14)
        la, lb = int(gpu["left"][a]), int(ora["left"][b])
        stack.append((la + 1, lb + 1))
        stack.append((la, lb))
    if skipped == 0:
        assert len(gpu["left"]) == len(ora["left"]), "node counts differ: %d vs %d" % (len(gpu["left"]),
                                                                                      len(ora["left"]))
    return compared


def oracle_tree_dict(t):
    return dict(level=t.level, left=t.left, feature=t.feature, threshold=t.threshold, score=t.score,
                feature_id=t.feature_id, histogram=t.histogram, num_samples=t.num_samples)
