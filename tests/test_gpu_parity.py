"""CUDA path vs the CPU oracle on the same seeded inputs and candidate features.

Bars (from the task's parity contract): histogram counts, routing and integral images bit-exact;
feature responses bit-identical to the oracle's double computation; scores within 1e-12 relative
(the two sides differ only by their log2 implementations); chosen splits identical except where
scores tie within 1e-6 relative; pixel labels agree on >= 99.9% of pixels; probabilities within 1e-5.
"""
import math

import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H
from tests.golden import reference_kats as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


def gpu_dataset_from_oracle(ctx, ods):
    """Upload oracle integrals (int64 depth wrapped to int32, as the device layout keeps it)."""
    depth = np.stack([ods.depth_sum.astype(np.int64).astype(np.int32), ods.depth_valid], axis=1)
    return cf.Dataset.from_integral(ctx, ods.color, np.ascontiguousarray(depth))


# ----------------------------------------------------------------------------------- integral images
@pytest.mark.parametrize("shape", [(3, 1, 1), (2, 7, 5), (2, 37, 53), (1, 480, 640)])
def test_integral_bit_exact(ctx, shape):
    n, h, w = shape
    rng = np.random.default_rng(h * w)
    rgb = rng.integers(0, 256, (n, h, w, 3), dtype=np.uint8)
    depth = rng.integers(500, 5001, (n, h, w)).astype(np.uint16)
    depth[rng.random(depth.shape) < 0.1] = 0
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    color, dint = ds.download_integral()
    ods = orc.integral(rgb, depth)
    np.testing.assert_array_equal(color.view(np.uint32), ods.color.view(np.uint32))
    np.testing.assert_array_equal(dint[:, 0], (ods.depth_sum & 0xFFFFFFFF).astype(np.uint32).view(np.int32))
    np.testing.assert_array_equal(dint[:, 1], ods.depth_valid)


def test_integral_1280x960_box_sums_exact_beyond_int32(ctx):
    """The reference's int depth integral overflows here (6.1e9 mm); box sums must stay exact."""
    h, w = 960, 1280
    rgb = np.full((1, h, w, 3), 255, np.uint8)
    depth = np.full((1, h, w), 5000, np.uint16)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    color, dint = ds.download_integral()
    s = dint[0, 0].view(np.uint32).astype(np.int64)
    # the whole-frame sum (6.1e9) wraps; every box a feature can reach (< 2^31 mm) is exact
    assert s[h - 1, w - 1] == (h * w * 5000) % (1 << 32)
    for (x0, y0, x1, y1) in [(100, 200, 160, 260), (1200, 900, 1279, 959), (0, 0, 300, 280)]:
        box = ((s[y1, x1] - s[y0, x1]) + (s[y0, x0] - s[y1, x0])) % (1 << 32)
        assert box == (x1 - x0) * (y1 - y0) * 5000
    assert color[0, 0, h - 1, w - 1] == np.float32(255.0 * h * w)


# ----------------------------------------------------------------------------------- responses / KATs
def kat_dataset_from_planes(ctx, planes, depth_mm):
    from tests.test_oracle_kats import make_dataset
    ods = make_dataset(planes, depth_mm)
    return ods, gpu_dataset_from_oracle(ctx, ods)


def test_depth_feature_kat(ctx):
    kat = K.DEPTH_FEATURE
    w, h = kat["width"], kat["height"]
    d = np.zeros((1, h, w), np.uint16)
    for (x, y), mm in kat["pixels_mm"].items():
        d[0, y, x] = mm
    ods, ds = kat_dataset_from_planes(ctx, np.zeros((1, 3, h, w), np.float32), d)
    feats = np.array(kat["feature"], np.int8).reshape(11, 1)
    thr = np.array(kat["thresholds"], np.float32).reshape(-1, 1)
    x, y = kat["sample_xy"]
    s = cf.samples_array(2)
    s["x"], s["y"], s["label"] = x, y, [0, 1]
    s["depth"] = np.float32(1.0)
    r = cf.feature_responses(ds, s, feats)
    assert r[0, 0] == pytest.approx(kat["expected_response"], rel=1e-12)
    assert r[0, 0] == orc.feature_responses(ods, s, feats)[0, 0]
    counters = cf.histograms(ds, s, feats, thr, 2)  # [F][T][C][2]
    for label in range(2):
        for t in range(len(kat["thresholds"])):
            assert counters[0, t, label, 0] == int(t >= kat["first_left_threshold"])
            assert counters[0, t, label, 1] == int(t < kat["first_left_threshold"])


def test_color_feature_complex_kat(ctx):
    from tests.test_oracle_kats import complex_dataset, samples_of
    kat = K.COLOR_FEATURE_COMPLEX
    ods = complex_dataset()
    ds = gpu_dataset_from_oracle(ctx, ods)
    feats = np.array(kat["features"], np.int8).T.copy()
    thr = np.array(kat["thresholds"], np.float32)
    s = samples_of(kat["samples"]).view(cf.SAMPLE_DTYPE)
    r = cf.feature_responses(ds, s, feats)
    for f in range(3):
        for i in range(4):
            exp = kat["responses"][f][i]
            assert (math.isnan(r[f, i]) if exp is None else r[f, i] == exp), (f, i, r[f, i])
    counters = cf.histograms(ds, s, feats, thr, 2)
    for (f, t), per_label in kat["counters"].items():
        for label in range(2):
            assert list(counters[f, t, label]) == per_label[label]


@pytest.fixture(scope="module")
def scene(ctx):
    rgb, depth, labels = H.frames(seed=3, n=4, w=96, h=72, cells=12, classes=40)
    ods = orc.integral(rgb, depth)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    return dict(rgb=rgb, depth=depth, labels=labels, ods=ods, ds=ds)


def test_responses_bit_identical(ctx, scene):
    rng = np.random.default_rng(11)
    s = H.random_samples(rng, 4, 96, 72, 40, 700, depth=scene["depth"], flips=True)
    feats = H.random_features(rng, 64, box_radius=60, region_size=15)
    g = cf.feature_responses(scene["ds"], s, feats)
    o = orc.feature_responses(scene["ods"], s, feats)
    assert np.isnan(o).any() and (~np.isnan(o)).sum() > 1000
    np.testing.assert_array_equal(np.isnan(g), np.isnan(o))
    np.testing.assert_array_equal(g[~np.isnan(g)].view(np.uint64), o[~np.isnan(o)].view(np.uint64))


@pytest.mark.parametrize("C", [2, 33, 40, 200])
def test_histograms_bit_exact(ctx, scene, C):
    """Exact counts for any class count (the reference GPU kernel breaks at >= 32 classes)."""
    rng = np.random.default_rng(C)
    s = H.random_samples(rng, 4, 96, 72, C, 1500, depth=scene["depth"], flips=True)
    feats = H.random_features(rng, 24)
    thr = (rng.standard_normal((9, 24)) * 200).astype(np.float32)
    thr[0, :] = 0.0
    thr[3, :] = thr[2, :]   # duplicated thresholds
    g = cf.histograms(scene["ds"], s, feats, thr, C)
    o = orc.histograms(scene["ods"], s, feats, thr, C, threads=4)
    np.testing.assert_array_equal(g, o.transpose(1, 2, 0, 3))


def test_scores_match_oracle(ctx, scene):
    rng = np.random.default_rng(5)
    s = H.random_samples(rng, 4, 96, 72, 40, 2000, depth=scene["depth"])
    feats = H.random_features(rng, 32)
    thr = (rng.standard_normal((12, 32)) * 300).astype(np.float32)
    counters = orc.histograms(scene["ods"], s, feats, thr, 40)
    hist = np.bincount(s["label"], minlength=40).astype(np.uint32)
    g = cf.scores(ctx, counters.transpose(1, 2, 0, 3).copy(), hist)
    o = orc.scores(counters, hist)
    np.testing.assert_allclose(g, o, rtol=1e-12, atol=1e-15)
    assert (o > 0).sum() > 100


def test_generate_features_bit_exact(ctx, scene):
    rng = np.random.default_rng(9)
    s = H.random_samples(rng, 4, 96, 72, 40, 3000, depth=scene["depth"])
    for use_depth in (True, False):
        gf, gt = cf.generate_features(scene["ds"], s, 123456, 300, 20, 60, 15, use_depth)
        of, ot = orc.generate_features(scene["ods"], s, 123456, 300, 20, 60, 15, use_depth)
        np.testing.assert_array_equal(gf, of)
        np.testing.assert_array_equal(gt.view(np.uint32), ot.view(np.uint32))
    keys = [(int(gf[0, i]) << 30) | (int(gf[9, i]) << 26) | (int(gf[10, i]) << 22) |
            ((int(gf[2, i]) + 127) << 14) | ((int(gf[1, i]) + 127) << 6) for i in range(300)]
    assert keys == sorted(keys)


def _oracle_best(ods, samples, feats, thr, C):
    counters = orc.histograms(ods, samples, feats, thr, C, threads=4)
    hist = np.zeros(C, np.uint32)
    for lab, fl in zip(samples["label"], samples["flip"]):
        hist[lab] += 2 if fl == 2 else 1
    scores = orc.scores(counters, hist)
    f, t, s = orc.best_split(scores)
    return f, t, s, scores


def test_evaluate_best_splits_level(ctx, scene):
    """Level-batched evaluation of skewed nodes (1 .. 3000 samples) against per-node oracle argmax."""
    rng = np.random.default_rng(21)
    sizes = [3000, 1, 2, 17, 250, 999, 5, 64]
    total = sum(sizes)
    s = H.random_samples(rng, 4, 96, 72, 40, total, depth=scene["depth"])
    # cluster labels per node so nodes have different class mixes
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    for i in range(len(sizes)):
        s["label"][offsets[i]:offsets[i + 1]] = rng.integers(0, 2 + 5 * i, sizes[i]) % 40
    fe, th = orc.generate_features(scene["ods"], s, 777, 200, 20, 60, 15)
    best = cf.evaluate_best_splits(scene["ds"], offsets, s, 40, fe, th)
    for i in range(len(sizes)):
        sl = s[offsets[i]:offsets[i + 1]]
        f, t, sc, scores = _oracle_best(scene["ods"], sl, fe, th, 40)
        g = best[i]
        if (g["feature"], g["threshold_index"]) != (f, t):
            # allowed only for a tie within 1e-6 relative in the oracle's own scores
            assert scores[g["threshold_index"], g["feature"]] == pytest.approx(sc, rel=1e-6), (i, g, f, t, sc)
        else:
            assert g["score"] == pytest.approx(sc, rel=1e-12, abs=1e-15)
            assert g["threshold"] == th[t, f]


@pytest.mark.parametrize("flips", [False, True])
def test_level_batched_counts_bit_exact(ctx, scene, flips):
    """The level-batched kernel's accumulated counts equal the oracle's per-node counters exactly
    (this exercises its fast paths: fallback-checked divisions and float depth estimates)."""
    rng = np.random.default_rng(33 + flips)
    sizes = [1500, 1, 7, 300, 64, 2]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, 4, 96, 72, 40, int(offsets[-1]), depth=scene["depth"], flips=flips)
    # a few samples with invalid depth and on the image border
    s["depth"][5] = 0.0
    s["x"][6], s["y"][6] = 0, 0
    s["x"][7], s["y"][7] = 95, 71
    fe, th = orc.generate_features(scene["ods"], s, 99, 96, 12, 60, 15)
    th[3, :] = th[2, :]               # tied thresholds
    th[4, :5] = 0.0
    best, left = cf.level_left_counts(scene["ds"], offsets, s, 40, fe, th)
    for i in range(len(sizes)):
        sl = s[offsets[i]:offsets[i + 1]]
        o = orc.histograms(scene["ods"], sl.view(orc.SAMPLE_DTYPE), fe, th, 40, threads=4)   # [C][F][T][2]
        np.testing.assert_array_equal(left[i], o[:, :, :, 0].transpose(1, 2, 0), err_msg="node %d" % i)


def train_cfg(**kw):
    d = dict(feature_count=120, thresholds=10, max_depth=8, min_sample_count=4, box_radius=40, region_size=10)
    d.update(kw)
    return cf.TrainConfig(**d)


def _oracle_score_ok(ods, samples_by_node):
    return lambda i: True


@pytest.mark.parametrize("flip", [False, True])
def test_train_tree_matches_oracle(ctx, scene, flip):
    samples, _ = H.class_uniform_samples(scene["labels"], scene["depth"], 40, 60)
    if flip:
        samples["flip"] = 2
    cfg = train_cfg()
    tree, counter = cf.train_tree(scene["ds"], samples, 40, cfg, tree_id=0, seed_counter=500)
    rc, otree, ocounter = orc.train_tree(scene["ods"], samples.view(orc.SAMPLE_DTYPE), 40, 120, 10, 8, 4, 40, 10, 500,
                                         threads=4)
    assert rc == 0
    assert counter == ocounter
    g = tree.arrays()
    o = H.oracle_tree_dict(otree)
    n = H.compare_trees(g, o)
    assert n > 20


def test_level_batched_equals_per_node(ctx, scene):
    samples, _ = H.class_uniform_samples(scene["labels"], scene["depth"], 40, 80)
    cfg = train_cfg(feature_count=200, thresholds=16, max_depth=10)
    a, _ = cf.train_tree(scene["ds"], samples, 40, cfg, seed_counter=42, mode=cf.LEVEL_BATCHED)
    b, _ = cf.train_tree(scene["ds"], samples, 40, cfg, seed_counter=42, mode=cf.PER_NODE)
    A, B = a.arrays(), b.arrays()
    for k in A:
        np.testing.assert_array_equal(A[k], B[k], err_msg=k)
    assert a.num_nodes > 50


def test_empty_child_is_an_error(ctx):
    """Two samples of different labels at the same pixel: no split separates them, the reference
    throws 'no samples in left node' (random_tree.h:1388-1393)."""
    rgb = np.zeros((1, 40, 40, 3), np.uint8)
    depth = np.full((1, 40, 40), 1000, np.uint16)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    s = cf.samples_array(2)
    s["x"], s["y"], s["depth"], s["label"] = 20, 20, np.float32(1.0), [0, 1]
    with pytest.raises(cf.CurfilError) as e:
        cf.train_tree(ds, s, 2, train_cfg(feature_count=8, thresholds=3, max_depth=3, min_sample_count=1))
    assert e.value.status == 4


def test_invalid_inputs_rejected(ctx, scene):
    s = cf.samples_array(3)
    s["label"] = [0, 1, 50]
    feats = H.random_features(np.random.default_rng(0), 4)
    with pytest.raises(cf.CurfilError) as e:
        cf.histograms(scene["ds"], s, feats, np.zeros((2, 4), np.float32), 40)
    assert e.value.status == 1
    s["label"] = 0
    with pytest.raises(cf.CurfilError):
        cf.histograms(scene["ds"], s, feats, np.full((2, 4), np.nan, np.float32), 40)
    s["x"] = 5000
    with pytest.raises(cf.CurfilError):
        cf.feature_responses(scene["ds"], s, feats)


# ----------------------------------------------------------------------------------- prediction
@pytest.fixture(scope="module")
def forest_and_oracle(ctx, scene):
    trees, otrees, normalized = [], [], []
    prior = np.bincount(scene["labels"].ravel(), minlength=40).astype(np.uint32)
    for t in range(3):
        samples, _ = H.class_uniform_samples(scene["labels"], scene["depth"], 40, 50, seed_counter=900 + 10 * t)
        tree, _ = cf.train_tree(scene["ds"], samples, 40, train_cfg(max_depth=10), tree_id=t, seed_counter=77 + t)
        trees.append(tree)
        a = tree.arrays()
        ot = orc.Tree(len(a["left"]), 40)
        ot.left, ot.feature, ot.threshold = a["left"], a["feature"], a["threshold"]
        ot.histogram = a["histogram"]
        otrees.append(ot)
        normalized.append(np.stack([orc.normalize_histogram(h, prior, 0.0, True) for h in a["histogram"]]))
    forest = cf.Forest(ctx, trees, prior=prior)
    return forest, otrees, normalized


def test_predict_matches_oracle(ctx, scene, forest_and_oracle):
    forest, otrees, normalized = forest_and_oracle
    rgb, depth, _ = H.frames(seed=99, n=2, w=96, h=72, cells=12, classes=40)
    ods = orc.integral(rgb, depth)
    probs, labels = forest.predict(rgb, depth)
    for i in range(2):
        op, ol = orc.predict(ods, i, otrees, normalized, 40, threads=4)
        agree = (labels[i] == ol).mean()
        assert agree >= 0.999, agree
        np.testing.assert_allclose(probs[i], op, atol=1e-5, rtol=0)
    assert labels.max() > 0


def test_predict_dataset_equals_host_path(ctx, scene, forest_and_oracle):
    import torch
    forest, _, _ = forest_and_oracle
    probs_h, labels_h = forest.predict(scene["rgb"], scene["depth"])
    n, h, w = scene["depth"].shape
    probs_d = torch.empty((n, 40, h, w), dtype=torch.float32, device="cuda:0")
    labels_d = torch.empty((n, h, w), dtype=torch.uint8, device="cuda:0")
    ctx.synchronize()
    forest.predict_dataset(scene["ds"], 0, n, probs_d.data_ptr(), labels_d.data_ptr())
    ctx.synchronize()
    np.testing.assert_array_equal(probs_d.cpu().numpy(), probs_h)
    np.testing.assert_array_equal(labels_d.cpu().numpy(), labels_h)


def test_predict_batched_equals_plain_per_image(ctx, scene, forest_and_oracle):
    """The batched kernel (fast-path responses with exact fallback, reciprocal-corrected division) and
    the reference-structured plain form (exact double responses, one launch per tree and image, plain
    division) agree bit for bit. Thresholds are responses of training pixels, so the training frames
    hit responses equal to thresholds and exercise the fallback."""
    import torch
    forest, _, _ = forest_and_oracle
    n, h, w = scene["depth"].shape
    pa = torch.empty((n, 40, h, w), dtype=torch.float32, device="cuda:0")
    la = torch.empty((n, h, w), dtype=torch.uint8, device="cuda:0")
    pb = torch.empty_like(pa)
    lb = torch.empty_like(la)
    ctx.synchronize()
    forest.predict_dataset(scene["ds"], 0, n, pa.data_ptr(), la.data_ptr())
    forest.predict_dataset_plain(scene["ds"], 0, n, pb.data_ptr(), lb.data_ptr())
    ctx.synchronize()
    np.testing.assert_array_equal(pa.cpu().numpy().view(np.uint32), pb.cpu().numpy().view(np.uint32))
    np.testing.assert_array_equal(la.cpu().numpy(), lb.cpu().numpy())


def test_predict_host_plain_equals_batched(ctx, forest_and_oracle):
    forest, _, _ = forest_and_oracle
    rgb, depth, _ = H.frames(seed=321, n=2, w=96, h=72, cells=12, classes=40)
    p1, l1 = forest.predict(rgb, depth)
    p2, l2 = forest.predict_plain(rgb, depth)
    np.testing.assert_array_equal(p1.view(np.uint32), p2.view(np.uint32))
    np.testing.assert_array_equal(l1, l2)
    _, l3 = forest.predict_plain(rgb, depth, probabilities=False)
    np.testing.assert_array_equal(l1, l3)


def test_predict_graph_equals_host_path(ctx, forest_and_oracle):
    forest, _, _ = forest_and_oracle
    g = cf.PredictGraph(forest, 3, 96, 72, probabilities=True)
    try:
        for seed in (123, 124):
            rgb, depth, _ = H.frames(seed=seed, n=3, w=96, h=72, cells=12, classes=40)
            g.rgb[...] = rgb
            g.depth[...] = depth
            g.run()
            probs, labels = forest.predict(rgb, depth)
            np.testing.assert_array_equal(g.labels, labels)
            np.testing.assert_array_equal(g.probabilities, probs)
    finally:
        g.close()


def test_device_sampler_matches_oracle(ctx):
    rgb, depth, labels = H.frames(seed=8, n=3, w=80, h=60, cells=10, classes=6)
    ign = np.zeros(6, np.uint8)
    ign[0] = 1
    cfg = train_cfg(samples_per_image=300, sampler=1)
    s, prior, counter = cf.sample_tree_pixels(labels, depth, 6, cfg, 2, 77, ignored=ign, ctx=ctx)
    rc, o, ocounter = orc.sample_class_uniform_keys(labels, depth, 6, ign, 300 // 2, 77)
    assert rc == len(s) == 5 * int(np.ceil(3 * 150 / 5))
    assert counter == ocounter
    for k in ("x", "y", "image", "label", "flip"):
        np.testing.assert_array_equal(s[k], o[k], err_msg=k)
    np.testing.assert_array_equal(s["depth"].view(np.uint32), o["depth"].view(np.uint32))
    np.testing.assert_array_equal(prior, np.bincount(labels.ravel(), minlength=6))
    assert (s["label"] != 0).all()
    # a class with too few eligible pixels is an error, as in the reference
    with pytest.raises(cf.CurfilError):
        cf.sample_tree_pixels(labels, depth, 6, train_cfg(samples_per_image=60000, sampler=1), 1, 77, ctx=ctx)


def test_device_sampler_at_scale_matches_oracle(ctx):
    """The device sampler's selection and ordering (radix sorts on the GPU) at 40 classes, 20 frames
    640x480 and 8000 samples per frame, against the oracle's restatement."""
    rgb, depth, labels = cf.synthetic_frames(2026, 20, 640, 480, 40, 40)
    cfg = train_cfg(samples_per_image=80000, sampler=1)
    s, prior, counter = cf.sample_tree_pixels(labels, depth, 40, cfg, 10, 4242, ctx=ctx)
    rc, o, ocounter = orc.sample_class_uniform_keys(labels, depth, 40, np.zeros(40, np.uint8), 8000, 4242)
    assert rc == len(s) == 40 * 4000 and counter == ocounter
    for k in ("x", "y", "image", "label", "flip"):
        np.testing.assert_array_equal(s[k], o[k], err_msg=k)
    np.testing.assert_array_equal(s["depth"].view(np.uint32), o["depth"].view(np.uint32))
    np.testing.assert_array_equal(prior, np.bincount(labels.ravel(), minlength=40))


@pytest.mark.parametrize("shape", [(3, 64, 48, 8, 300), (4, 640, 480, 40, 8000)])
def test_device_pixel_uniform_sampler_matches_oracle(ctx, shape):
    """pixelUniform on the device (the reference's random streams, one thread per sample) against the
    oracle's restatement of random_tree_image.cpp:840-883 with the block sort, void class ignored."""
    n, w, h, C, per_image = shape
    rgb, depth, labels = cf.synthetic_frames(4, n, w, h, 10, C)
    ign = np.zeros(C, np.uint8)
    ign[0] = 1
    cfg = train_cfg(samples_per_image=2 * per_image, subsampling_type=1, sampler=1)
    seed = cf.forest_seed(4711)
    s, prior, counter = cf.sample_tree_pixels(labels, depth, C, cfg, 2, seed + 1, ignored=ign, ctx=ctx)
    rc, o, ocounter = orc.sample_pixel_uniform(labels, depth, ign, per_image, seed + 1)
    assert rc == len(s) == n * per_image and counter == ocounter
    for k in ("x", "y", "image", "label", "flip"):
        np.testing.assert_array_equal(s[k], o[k], err_msg=k)
    np.testing.assert_array_equal(s["depth"].view(np.uint32), o["depth"].view(np.uint32))
    np.testing.assert_array_equal(prior, np.bincount(labels.ravel(), minlength=C))
    assert (s["label"] != 0).all()
    # the host form of the same definition gives the same samples
    hs, _, hcounter = cf.sample_tree_pixels(labels, depth, C, cfg, 2, seed + 1, ignored=ign)
    assert hcounter == counter
    np.testing.assert_array_equal(hs.view(np.uint8), s.view(np.uint8))


def test_forest_train_device_sampler_matches_oracle(ctx):
    rgb, depth, labels = H.frames(seed=6, n=3, w=80, h=60, cells=10, classes=6)
    cfg = train_cfg(random_seed=4711, samples_per_image=120, max_depth=7, sampler=1)
    trees = cf.train_forest(ctx, rgb, depth, labels, 6, cfg, num_trees=2)
    ods = orc.integral(rgb, depth)
    SEED = int(orc.sampler_draws(4711, 0, 0xFFFE, 1)[0])
    for t, tree in enumerate(trees):
        rc, s, counter = orc.sample_class_uniform_keys(labels, depth, 6, np.zeros(6, np.uint8), 120 // 2, SEED + t)
        assert rc > 0
        rc, ot, _ = orc.train_tree(ods, s, 6, 120, 10, 7, 4, 40, 10, counter, threads=4)
        assert rc == 0
        g = tree.arrays()
        o = H.oracle_tree_dict(ot)
        H.compare_trees(g, o)


def test_forest_train_end_to_end_matches_oracle(ctx):
    """RandomForestImage::train on raw frames (sampling on the host) vs oracle sampling + training."""
    rgb, depth, labels = H.frames(seed=5, n=3, w=80, h=60, cells=10, classes=6)
    cfg = train_cfg(random_seed=4711, samples_per_image=120, max_depth=7)
    trees = cf.train_forest(ctx, rgb, depth, labels, 6, cfg, num_trees=2)
    ods = orc.integral(rgb, depth)
    # forest seed (random_forest_image.cpp:150-151): SEED = first draw of Sampler(4711, 0, 0xFFFE)
    SEED = int(orc.sampler_draws(4711, 0, 0xFFFE, 1)[0])
    for t, tree in enumerate(trees):
        counter = SEED + t
        rc, s, counter = orc.sample_class_uniform(labels, depth, 6, np.zeros(6, np.uint8), 120 // 2, counter)
        assert rc > 0
        rc, ot, _ = orc.train_tree(ods, s, 6, 120, 10, 7, 4, 40, 10, counter, threads=4)
        assert rc == 0
        g = tree.arrays()
        o = H.oracle_tree_dict(ot)
        H.compare_trees(g, o)
        np.testing.assert_array_equal(tree.prior(), np.bincount(labels.ravel(), minlength=6))


def test_host_entry_point_large_level_matches_oracle(ctx, scene):
    """cf_evaluate_best_splits on 600 000 host samples: the entry point checks the samples and counts
    the node histograms on several host threads (ranges that split nodes between threads), and the
    splits are the oracle's; an invalid sample is reported by its index, the first one when several are
    invalid."""
    rng = np.random.default_rng(600)
    sizes = [290001, 1, 7, 210000, 99991]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, 4, 96, 72, 40, int(offsets[-1]), depth=scene["depth"], flips=True)
    for i in range(len(sizes)):
        s["label"][offsets[i]:offsets[i + 1]] = rng.integers(0, 3 + 9 * i, sizes[i]) % 40
    fe, th = orc.generate_features(scene["ods"], s[:20000], 61, 8, 5, 60, 15)
    got = cf.evaluate_best_splits(scene["ds"], offsets, s, 40, fe, th)
    for i in range(len(sizes)):
        sl = s[offsets[i]:offsets[i + 1]]
        node_hist = np.zeros(40, np.uint32)
        np.add.at(node_hist, sl["label"], np.where(sl["flip"] == 2, 2, 1).astype(np.uint32))
        sc = orc.scores(orc.histograms(scene["ods"], sl.view(orc.SAMPLE_DTYPE), fe, th, 40, threads=8), node_hist)
        bf, bt, bs = orc.best_split(sc)
        mine = sc[got["threshold_index"][i], got["feature"][i]]
        if (got["feature"][i], got["threshold_index"][i]) != (bf, bt):
            assert abs(mine - bs) <= 1e-6 * abs(bs), i
        assert got["score"][i] == pytest.approx(mine, rel=1e-12, abs=1e-15), i
    bad = s.copy()
    bad["label"][450000] = 40
    bad["x"][123456] = 96
    with pytest.raises(cf.CurfilError) as e:
        cf.evaluate_best_splits(scene["ds"], offsets, bad, 40, fe, th)
    assert "sample 123456: pixel outside" in str(e.value), str(e.value)
