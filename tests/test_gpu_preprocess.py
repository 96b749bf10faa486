"""Preprocessing (depth filling, CIE L*a*b*) and evaluation helpers on the device vs the oracle.

Bars: depth filling bit-exact (integer work); L*a*b* within one float ulp (the device's double cbrt
and the host's may differ in the last double bit before the rounding to float); the L*a*b* integral
within one float ulp plus the double summation-order error; pixel accuracy and the confusion matrix
exact (integer counts), the class average to 1e-15.
"""
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


def holey_depth(rng, n, h, w, frac):
    d = rng.integers(500, 5001, (n, h, w)).astype(np.uint16)
    d[rng.random(d.shape) < frac] = 0
    return d


# ------------------------------------------------------------------------------------ depth filling
def test_fill_depth_kat(ctx):
    """The reference's own fillDepth test image (image_test.cpp:425-456)."""
    k = K.DEPTH_FILL
    d = np.zeros((k["height"], k["width"]), np.uint16)
    for (x, y), mm in k["seeds"].items():
        d[y, x] = mm
    f = cf.fill_depth(ctx, d)[0]
    assert (f[:k["split_row"]] == k["above"]).all()
    assert (f[k["split_row"]:] == k["below"]).all()


@pytest.mark.parametrize("shape,frac", [((1, 1, 1), 1.0), ((2, 1, 17), 0.6), ((2, 13, 1), 0.6), ((3, 37, 53), 0.3),
                                        ((2, 37, 53), 0.97), ((1, 480, 640), 0.1)])
def test_fill_depth_matches_oracle(ctx, shape, frac):
    rng = np.random.default_rng(sum(shape) + int(frac * 100))
    d = holey_depth(rng, *shape, frac)
    d[0, :, :] = 0 if shape[1] * shape[2] < 4 else d[0]
    got = cf.fill_depth(ctx, d)
    np.testing.assert_array_equal(got, orc.fill_depth(d))
    # valid pixels keep their depth
    np.testing.assert_array_equal(got[d > 0], d[d > 0])


def test_fill_depth_all_missing_stays_missing(ctx):
    d = np.zeros((2, 9, 11), np.uint16)
    np.testing.assert_array_equal(cf.fill_depth(ctx, d), d)


# ------------------------------------------------------------------------------------------ L*a*b*
def _assert_within_ulps(got, want, ulps=1):
    """One float ulp, plus 1e-12 absolute for a* and b* near zero, where 500 (fx - fy) cancels terms of
    size ~100 whose last double bits differ between the device (fused multiply-adds) and the host."""
    diff = np.abs(got.astype(np.float64) - want.astype(np.float64))
    bound = ulps * np.spacing(np.abs(want).astype(np.float32)).astype(np.float64) + 1e-12
    bad = diff > bound
    assert not bad.any(), (got[bad][:5], want[bad][:5])


def test_lab_matches_oracle_all_grey_levels_and_random(ctx):
    rng = np.random.default_rng(3)
    grey = np.repeat(np.arange(256, dtype=np.uint8)[:, None], 3, axis=1).reshape(1, 16, 16, 3)
    rnd = rng.integers(0, 256, (2, 16, 16, 3), dtype=np.uint8)
    rgb = np.concatenate([grey, rnd])
    got = cf.rgb_to_cielab(ctx, rgb)
    want = orc.rgb_to_lab(rgb)
    _assert_within_ulps(got, want)
    # white and black
    assert abs(got[0, 0, 15, 15] - 100.0) < 1e-3 and abs(got[0, 0, 0, 0]) < 1e-6


def test_lab_integral_matches_oracle(ctx):
    rng = np.random.default_rng(11)
    n, h, w = 2, 61, 83
    rgb = rng.integers(0, 256, (n, h, w, 3), dtype=np.uint8)
    depth = holey_depth(rng, n, h, w, 0.2)
    ds = cf.Dataset.from_raw(ctx, rgb, depth, cie_lab=True)
    color, dint = ds.download_integral()
    lab = orc.rgb_to_lab(rgb)
    for i in range(n):
        want = orc.integral_float_color(lab[i])
        absum = np.cumsum(np.cumsum(np.abs(lab[i].astype(np.float64)), axis=1), axis=2)
        diff = np.abs(color[i].astype(np.float64) - want.astype(np.float64))
        bound = np.spacing(np.abs(want)).astype(np.float64) + 1e-12 * absum
        assert (diff <= bound).all()
    # depth channels untouched by the colour conversion
    ods = orc.integral(rgb, depth)
    np.testing.assert_array_equal(dint[:, 1], ods.depth_valid)


def test_upload_with_fill_depth_equals_filled_upload(ctx):
    rng = np.random.default_rng(5)
    n, h, w = 3, 40, 52
    rgb = rng.integers(0, 256, (n, h, w, 3), dtype=np.uint8)
    depth = holey_depth(rng, n, h, w, 0.4)
    a = cf.Dataset.from_raw(ctx, rgb, depth, fill_depth=True)
    filled = orc.fill_depth(depth)
    b = cf.Dataset.from_raw(ctx, rgb, filled)
    ca, da = a.download_integral()
    cb, db = b.download_integral()
    np.testing.assert_array_equal(ca.view(np.uint32), cb.view(np.uint32))
    np.testing.assert_array_equal(da, db)
    ods = orc.integral(rgb, filled)
    np.testing.assert_array_equal(da[:, 1], ods.depth_valid)


def test_predict_host_applies_forest_preprocessing(ctx):
    """A forest marked as trained on filled depth and L*a*b* predicts raw frames like the dataset path
    over frames uploaded with the same preprocessing."""
    import torch
    rgb, depth, labels = H.frames(seed=21, n=3, w=64, h=48, classes=4)
    depth = depth.copy()
    depth[np.random.default_rng(1).random(depth.shape) < 0.2] = 0
    ds = cf.Dataset.from_raw(ctx, rgb, depth, fill_depth=True, cie_lab=True)
    samples, _ = H.class_uniform_samples(labels, orc.fill_depth(depth), 4, 300)
    cfg = cf.TrainConfig(feature_count=64, thresholds=10, max_depth=6, min_sample_count=4, box_radius=20,
                         region_size=6, use_cie_lab=1, use_depth_filling=1)
    trees = [cf.train_tree(ds, samples, 4, cfg, tree_id=t, seed_counter=5 + t)[0] for t in range(2)]
    forest = cf.Forest(ctx, trees, prior=np.bincount(labels.ravel(), minlength=4).astype(np.uint32))
    forest.set_preprocessing(fill_depth=True, cie_lab=True)
    probs_host, labels_host = forest.predict(rgb, depth)
    n, h, w = depth.shape
    probs_dev = torch.empty((n, 4, h, w), dtype=torch.float32, device="cuda")
    labels_dev = torch.empty((n, h, w), dtype=torch.uint8, device="cuda")
    forest.predict_dataset(ds, 0, n, probs_dev.data_ptr(), labels_dev.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(labels_host, labels_dev.cpu().numpy())
    np.testing.assert_array_equal(probs_host, probs_dev.cpu().numpy())


# -------------------------------------------------------------------------------------- evaluation
def _accuracy_restated(pred, truth, C, ignored, include_void):
    """calculatePixelAccuracy (predict.cpp:148-207) over the given frames."""
    conf = np.zeros((C, C), np.uint64)
    keep = np.ones(truth.shape, bool) if include_void or ignored is None else ~np.asarray(ignored, bool)[truth]
    np.add.at(conf, (truth[keep], pred[keep]), 1)
    correct = int((pred[keep] == truth[keep]).sum())
    pixels = truth.size if include_void else int(keep.sum())
    return correct / pixels, conf


@pytest.mark.parametrize("C", [3, 40, 90])
@pytest.mark.parametrize("include_void", [True, False])
def test_pixel_accuracy_and_confusion(ctx, C, include_void):
    import torch
    rng = np.random.default_rng(C)
    truth = rng.integers(0, C, (3, 37, 45), dtype=np.uint8)
    pred = np.where(rng.random(truth.shape) < 0.7, truth, rng.integers(0, C, truth.shape)).astype(np.uint8)
    ignored = np.zeros(C, np.uint8)
    ignored[0] = 1
    want_acc, want_conf = _accuracy_restated(pred, truth, C, ignored, include_void)
    conf = np.zeros((C, C), np.uint64)
    conf[0, 0] = 5   # accumulated, not overwritten
    t_pred = torch.from_numpy(pred).cuda()
    t_truth = torch.from_numpy(truth).cuda()
    acc = cf.pixel_accuracy(ctx, t_pred.data_ptr(), t_truth.data_ptr(), 3, 45, 37, C, ignored, include_void, conf)
    assert acc == pytest.approx(want_acc, rel=0, abs=1e-15)
    want_conf[0, 0] += 5
    np.testing.assert_array_equal(conf, want_conf)
    avg, norm = cf.average_class_accuracy(conf, ignored, include_void)
    sums = want_conf.astype(np.float64).sum(axis=1, keepdims=True)
    want_norm = np.where(sums == 0, want_conf.astype(np.float64), want_conf / np.where(sums == 0, 1, sums))
    np.testing.assert_allclose(norm, want_norm, rtol=1e-15, atol=0)
    classes = [c for c in range(C) if include_void or not ignored[c]]
    assert avg == pytest.approx(np.mean([want_norm[c, c] for c in classes]), rel=1e-15)


def test_pixel_accuracy_rejects_out_of_range_labels(ctx):
    import torch
    truth = torch.full((1, 4, 4), 7, dtype=torch.uint8, device="cuda")
    pred = torch.zeros((1, 4, 4), dtype=torch.uint8, device="cuda")
    with pytest.raises(cf.CurfilError):
        cf.pixel_accuracy(ctx, pred.data_ptr(), truth.data_ptr(), 1, 4, 4, 5)


# --------------------------------------------------------------------------------------------- padding
def padded_scene(ctx, seed=41, n=3, w=70, h=50, pad_w=96, pad_h=72, classes=40):
    rgb, depth, labels = H.frames(seed=seed, n=n, w=w, h=h, cells=10, classes=classes)
    ds = cf.Dataset(ctx, n, pad_w, pad_h)
    ds.upload_raw_padded(rgb, depth)
    ods = orc.pad_integral(orc.integral(rgb, depth), pad_w, pad_h)
    pdepth = np.zeros((n, pad_h, pad_w), np.uint16)
    pdepth[:, :h, :w] = depth
    return ds, ods, pdepth, cf.pad_labels(labels, pad_w, pad_h, 0)


def test_padded_upload_matches_oracle(ctx):
    ds, ods, _, labels = padded_scene(ctx)
    color, dint = ds.download_integral()
    np.testing.assert_array_equal(np.isnan(color), np.isnan(ods.color))
    np.testing.assert_array_equal(color.view(np.uint32)[~np.isnan(color)], ods.color.view(np.uint32)[~np.isnan(color)])
    np.testing.assert_array_equal(dint[:, 0], ods.depth_sum.astype(np.int32))
    np.testing.assert_array_equal(dint[:, 1], ods.depth_valid)
    assert (labels[:, 50:, :] == 0).all() and (labels[:, :, 70:] == 0).all()
    ds.close()


def test_padded_upload_with_preprocessing(ctx):
    rng = np.random.default_rng(2)
    rgb = rng.integers(0, 256, (2, 30, 40, 3), dtype=np.uint8)
    depth = holey_depth(rng, 2, 30, 40, 0.3)
    ds = cf.Dataset(ctx, 2, 64, 48)
    ds.upload_raw_padded(rgb, depth, fill_depth=True)
    _, dint = ds.download_integral()
    ods = orc.pad_integral(orc.integral(rgb, orc.fill_depth(depth)), 64, 48)
    np.testing.assert_array_equal(dint[:, 1], ods.depth_valid)
    np.testing.assert_array_equal(dint[:, 0], ods.depth_sum.astype(np.int32))
    with pytest.raises(cf.CurfilError):
        ds.upload_raw_padded(np.zeros((1, 50, 40, 3), np.uint8), np.zeros((1, 50, 40), np.uint16))
    ds.close()


@pytest.mark.parametrize("flips", [False, True])
def test_level_counts_on_padded_frames_bit_exact(ctx, flips):
    """Boxes that reach the padding see NaN colour and negative depth counts (the reference divides
    by them); the level-batched kernel's fast paths must count exactly as the oracle does."""
    ds, ods, pdepth, _ = padded_scene(ctx)
    rng = np.random.default_rng(7 + flips)
    sizes = [900, 3, 250, 40]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, 3, 96, 72, 40, int(offsets[-1]), depth=pdepth, flips=flips)
    # half of the samples near the edges of the real frame, where boxes straddle the padding
    k = len(s) // 2
    s["x"][:k] = rng.integers(50, 70, k)
    s["y"][:k] = rng.integers(30, 50, k)
    mm = pdepth[s["image"][:k], s["y"][:k], s["x"][:k]]
    s["depth"][:k] = np.where(mm > 0, mm.astype(np.float32) / np.float32(1000.0), np.float32(0.0))
    fe, th = orc.generate_features(ods, s, 123, 96, 12, 60, 15)
    best, left = cf.level_left_counts(ds, offsets, s, 40, fe, th)
    for i in range(len(sizes)):
        sl = s[offsets[i]:offsets[i + 1]]
        o = orc.histograms(ods, sl.view(orc.SAMPLE_DTYPE), fe, th, 40, threads=4)
        np.testing.assert_array_equal(left[i], o[:, :, :, 0].transpose(1, 2, 0), err_msg="node %d" % i)
    ds.close()


def test_predict_on_padded_frames_matches_oracle(ctx):
    import torch
    C = 6
    ds, ods, pdepth, labels = padded_scene(ctx, classes=C)
    ignore = np.zeros(C, np.uint8)
    ignore[0] = 1   # the padding label is ignored, as getPaddingLabel's colour is
    samples, _ = H.class_uniform_samples(labels, pdepth, C, 200, ignore=ignore)
    cfg = cf.TrainConfig(feature_count=128, thresholds=10, max_depth=8, min_sample_count=4, box_radius=40,
                         region_size=10)
    tree, _ = cf.train_tree(ds, samples, C, cfg, tree_id=0, seed_counter=9)
    prior = np.bincount(labels.ravel(), minlength=C).astype(np.uint32)
    forest = cf.Forest(ctx, [tree], prior=prior)
    a = tree.arrays()
    ot = orc.Tree(len(a["left"]), C)
    ot.left, ot.feature, ot.threshold, ot.histogram = a["left"], a["feature"], a["threshold"], a["histogram"]
    normalized = np.stack([orc.normalize_histogram(hh, prior, 0.0, True) for hh in a["histogram"]])
    probs = torch.empty((3, C, 72, 96), dtype=torch.float32, device="cuda")
    lab = torch.empty((3, 72, 96), dtype=torch.uint8, device="cuda")
    forest.predict_dataset(ds, 0, 3, probs.data_ptr(), lab.data_ptr())
    torch.cuda.synchronize()
    probs, lab = probs.cpu().numpy(), lab.cpu().numpy()
    for i in range(3):
        op, ol = orc.predict(ods, i, [ot], [normalized], C, threads=4)
        assert (lab[i] == ol).mean() >= 0.999
        np.testing.assert_allclose(probs[i], op, atol=1e-5, rtol=0)
    forest.close()
    ds.close()


# ------------------------------------------------------------------------------ reference-layout integral
def test_integrate_planes_matches_oracle(ctx):
    """cf_integrate_planes (RGBDImage::calculateIntegral on setColor/setDepth layouts): integer-valued
    colours bit-exact, arbitrary floats within one float ulp of the reference's Kahan scan, depth exact."""
    rng = np.random.default_rng(17)
    n, h, w = 2, 45, 67
    rgb = rng.integers(0, 256, (n, h, w, 3), dtype=np.uint8)
    depth = holey_depth(rng, n, h, w, 0.2)
    planes = np.ascontiguousarray(rgb.transpose(0, 3, 1, 2).astype(np.float32))
    dplanes = np.stack([depth.astype(np.int32), (depth > 0).astype(np.int32)], axis=1)
    color, dint = cf.integrate_planes(ctx, planes, dplanes)
    ods = orc.integral(rgb, depth)
    np.testing.assert_array_equal(color.view(np.uint32), ods.color.view(np.uint32))
    np.testing.assert_array_equal(dint[:, 0], ods.depth_sum.astype(np.int32))
    np.testing.assert_array_equal(dint[:, 1], ods.depth_valid)
    floats = (rng.standard_normal((n, 3, h, w)) * 37.3).astype(np.float32)
    color, _ = cf.integrate_planes(ctx, floats, dplanes)
    for i in range(n):
        want = orc.integral_float_color(floats[i])
        absum = np.cumsum(np.cumsum(np.abs(floats[i].astype(np.float64)), axis=1), axis=2)
        diff = np.abs(color[i].astype(np.float64) - want.astype(np.float64))
        assert (diff <= np.spacing(np.abs(want)).astype(np.float64) + 1e-12 * absum).all()


def test_predict_dataset_host_equals_device_outputs(ctx):
    import torch
    rgb, depth, labels = H.frames(seed=8, n=2, w=64, h=48, classes=5)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    samples, _ = H.class_uniform_samples(labels, depth, 5, 200)
    cfg = cf.TrainConfig(feature_count=64, thresholds=10, max_depth=6, min_sample_count=4, box_radius=20,
                         region_size=6)
    tree, _ = cf.train_tree(ds, samples, 5, cfg)
    forest = cf.Forest(ctx, [tree], prior=np.bincount(labels.ravel(), minlength=5).astype(np.uint32))
    probs_dev = torch.empty((2, 5, 48, 64), dtype=torch.float32, device="cuda")
    labels_dev = torch.empty((2, 48, 64), dtype=torch.uint8, device="cuda")
    forest.predict_dataset(ds, 0, 2, probs_dev.data_ptr(), labels_dev.data_ptr())
    torch.cuda.synchronize()
    probs, lab = forest.predict_dataset_host(ds, 0, 2)
    np.testing.assert_array_equal(probs, probs_dev.cpu().numpy())
    np.testing.assert_array_equal(lab, labels_dev.cpu().numpy())
    _, lab1 = forest.predict_dataset_host(ds, 1, 1, probabilities=False)
    np.testing.assert_array_equal(lab1[0], lab[1])
