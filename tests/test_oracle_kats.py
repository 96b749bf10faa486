"""CPU oracle pinned against the known-answer values of the reference's unit tests.

These run without a GPU. Every expected value comes from tests/golden/reference_kats.py,
which cites the reference test it was transcribed from.
"""
import math

import numpy as np
import pytest

from oracle import pyoracle as orc
from tests.golden import reference_kats as K


def make_dataset(color_planes, depth_mm):
    """color_planes float [n][3][H][W] (raw), depth_mm int [n][H][W] -> oracle Dataset."""
    color_planes = np.asarray(color_planes, np.float32)
    depth_mm = np.asarray(depth_mm, np.uint16)
    n, _, h, w = color_planes.shape
    rgb0 = np.zeros((n, h, w, 3), np.uint8)
    depth_ds = orc.integral(rgb0, depth_mm)
    color = np.stack([orc.integral_float_color(color_planes[i]) for i in range(n)])
    return orc.Dataset(color, depth_ds.depth_sum, depth_ds.depth_valid)


def samples_of(rows):
    """rows of (image, label, depth_mm, x, y[, flip])"""
    s = np.zeros(len(rows), orc.SAMPLE_DTYPE)
    for i, r in enumerate(rows):
        img, label, dmm, x, y = r[:5]
        s[i]["image"], s[i]["label"], s[i]["x"], s[i]["y"] = img, label, x, y
        s[i]["depth"] = np.float32(dmm) / np.float32(1000.0)
        s[i]["flip"] = r[5] if len(r) > 5 else 0
    return s


# --------------------------------------------------------------------------- scores
@pytest.mark.parametrize("left,right,all_,expected,rel,ig", K.SCORE_KATS)
def test_score_kats(left, right, all_, expected, rel, ig):
    s = orc.score(left, right, all_)
    assert s == pytest.approx(expected, rel=rel)
    if ig is not None:
        assert orc.score(left, right, all_, information_gain_only=True) == pytest.approx(ig, rel=1e-5)


def test_score_extremes():
    for num in K.SCORE_RANGE:
        assert orc.score([num, num], [num, num], [2 * num, 2 * num]) == 0.0
        assert orc.score([0, 2 * num], [2 * num, 0], [2 * num, 2 * num]) == 1.0


# --------------------------------------------------------------------------- integral images
def test_color_integral_3x3():
    p = np.array(K.COLOR_INTEGRAL_3X3["pixels"], np.float32)
    planes = np.stack([p, p, p])
    out = orc.integral_float_color(planes)
    for c in range(3):
        np.testing.assert_array_equal(out[c], np.array(K.COLOR_INTEGRAL_3X3["integral"], np.float32))


def test_color_integral_large_box():
    kat = K.COLOR_INTEGRAL_LARGE
    w, h = kat["width"], kat["height"]
    rgb = np.full((1, h, w, 3), kat["value"], np.uint8)
    ds = orc.integral(rgb, np.zeros((1, h, w), np.uint16))
    bw, bh = kat["box"]
    x, y = w - bw - 1, h - bh - 1
    for c in range(3):
        I = ds.color[0, c].astype(np.float64)
        s = I[y + bh, x + bw] - I[y - bh, x + bw] - I[y + bh, x - bw] + I[y - bh, x - bw]
        assert s == 2 * bw * 2 * bh * 255.0


def test_depth_integral_3x2():
    kat = K.DEPTH_INTEGRAL_3X2
    d = np.zeros((1, 2, 3), np.uint16)
    for (x, y), mm in kat["writes"]:
        d[0, y, x] = mm
    ds = orc.integral(np.zeros((1, 2, 3, 3), np.uint8), d)
    np.testing.assert_array_equal(ds.depth_sum[0], np.array(kat["integral_mm"]))
    np.testing.assert_array_equal(ds.depth_valid[0], np.array(kat["valid"]))
    # pixel depth recovery (random_tree_image.h:140-165)
    for y in range(2):
        for x in range(3):
            got = orc.pixel_depth(ds, 0, x, y)
            if d[0, y, x] == 0:
                assert math.isnan(got)
            else:
                assert got == np.float32(d[0, y, x]) / np.float32(1000.0)


def test_integral_matches_exact_integer_scan():
    rng = np.random.default_rng(5)
    rgb = rng.integers(0, 256, (2, 37, 53, 3), dtype=np.uint8)
    depth = rng.integers(0, 5001, (2, 37, 53)).astype(np.uint16)
    depth[rng.random(depth.shape) < 0.1] = 0
    ds = orc.integral(rgb, depth)
    exact = np.cumsum(np.cumsum(rgb.astype(np.int64), axis=1), axis=2).transpose(0, 3, 1, 2)
    np.testing.assert_array_equal(ds.color, exact.astype(np.float32))
    np.testing.assert_array_equal(ds.depth_sum, np.cumsum(np.cumsum(depth.astype(np.int64), 1), 2))
    np.testing.assert_array_equal(ds.depth_valid, np.cumsum(np.cumsum((depth > 0).astype(np.int32), 1), 2))


# --------------------------------------------------------------------------- feature responses
def _depth_feature_dataset(pixels_mm, w, h, constant=None):
    d = np.zeros((1, h, w), np.uint16)
    if constant is not None:
        d[:] = constant
    for (x, y), mm in pixels_mm.items():
        d[0, y, x] = mm
    return make_dataset(np.zeros((1, 3, h, w), np.float32), d)


def _check_counts(counters, thresholds, first_left, num_labels):
    # counters [C][F][T][2]
    for label in range(num_labels):
        for t in range(len(thresholds)):
            assert counters[label, 0, t, 0] + counters[label, 0, t, 1] == 1
            assert counters[label, 0, t, 0] == int(t >= first_left)


def test_depth_feature_kat():
    kat = K.DEPTH_FEATURE
    w, h = kat["width"], kat["height"]
    feats = np.array(kat["feature"], np.int8).reshape(11, 1)
    thr = np.array(kat["thresholds"], np.float32).reshape(-1, 1)
    x, y = kat["sample_xy"]
    samples = samples_of([(0, lab, kat["sample_depth_mm"], x, y) for lab in kat["labels"]])
    # all-zero depth image: no valid pixel in the boxes -> NaN (goes right everywhere)
    ds0 = _depth_feature_dataset({}, w, h)
    assert math.isnan(orc.feature_responses(ds0, samples, feats)[0, 0])
    ds = _depth_feature_dataset(kat["pixels_mm"], w, h)
    r = orc.feature_responses(ds, samples, feats)
    assert r[0, 0] == pytest.approx(kat["expected_response"], rel=1e-8)
    counters = orc.histograms(ds, samples, feats, thr, 2)
    _check_counts(counters, kat["thresholds"], kat["first_left_threshold"], 2)
    dsc = _depth_feature_dataset({}, w, h, constant=kat["constant_depth_mm"])
    assert orc.feature_responses(dsc, samples, feats)[0, 0] == 0.0
    counters = orc.histograms(dsc, samples, feats, thr, 2)
    _check_counts(counters, kat["thresholds"], kat["constant_first_left_threshold"], 2)


def test_color_feature_simple_kat():
    kat = K.COLOR_FEATURE_SIMPLE
    w, h = kat["width"], kat["height"]
    feats = np.array(kat["feature"], np.int8).reshape(11, 1)
    thr = np.array(kat["thresholds"], np.float32).reshape(-1, 1)
    x, y = kat["sample_xy"]
    samples = samples_of([(0, lab, kat["sample_depth_mm"], x, y) for lab in kat["labels"]])
    for name, expected, left_flags in kat["cases"]:
        planes = np.zeros((1, 3, h, w), np.float32)
        if name == "pixel_7_2_half":
            planes[0, 0, 2, 7] = 0.5
        elif name == "ones":
            planes[0, 0] = 1.0
        ds = make_dataset(planes, np.zeros((1, h, w), np.uint16))
        assert orc.feature_responses(ds, samples, feats)[0, 0] == expected
        counters = orc.histograms(ds, samples, feats, thr, 2)
        for label in range(2):
            for t, lf in enumerate(left_flags):
                assert counters[label, 0, t, 0] == lf
                assert counters[label, 0, t, 1] == 1 - lf


def complex_dataset():
    kat = K.COLOR_FEATURE_COMPLEX
    w, h = kat["width"], kat["height"]
    planes = np.zeros((2, 3, h, w), np.float32)
    for c in range(3):
        for yy in range(h):
            for xx in range(w):
                v = np.float32(100 * c + yy * w + xx)
                planes[0, c, yy, xx] = v
                planes[1, c, yy, xx] = v / np.float32(2.0)
    return make_dataset(planes, np.zeros((2, h, w), np.uint16))


def test_color_feature_complex_kat():
    kat = K.COLOR_FEATURE_COMPLEX
    ds = complex_dataset()
    h, w = kat["height"], kat["width"]
    for c in range(3):
        assert ds.color[0, c, h - 1, w - 1] == kat["integral_bottom_right"][c]
        assert ds.color[1, c, h - 1, w - 1] == kat["integral_bottom_right"][c] / 2.0
    feats = np.array(kat["features"], np.int8).T.copy()
    thr = np.array(kat["thresholds"], np.float32)
    samples = samples_of(kat["samples"])
    r = orc.feature_responses(ds, samples, feats)
    for f in range(3):
        for s in range(4):
            exp = kat["responses"][f][s]
            if exp is None:
                assert math.isnan(r[f, s])
            else:
                assert r[f, s] == exp
    counters = orc.histograms(ds, samples, feats, thr, 2)
    for (f, t), per_label in kat["counters"].items():
        for label in range(2):
            assert list(counters[label, f, t]) == per_label[label]


def test_histogram_threads_agree():
    ds = complex_dataset()
    kat = K.COLOR_FEATURE_COMPLEX
    feats = np.array(kat["features"], np.int8).T.copy()
    thr = np.array(kat["thresholds"], np.float32)
    rng = np.random.default_rng(1)
    rows = [(int(rng.integers(2)), int(rng.integers(3)), int(rng.integers(500, 4000)), int(rng.integers(12)),
             int(rng.integers(15)), int(rng.integers(3))) for _ in range(700)]
    samples = samples_of(rows)
    a = orc.histograms(ds, samples, feats, thr, 3, threads=1)
    b = orc.histograms(ds, samples, feats, thr, 3, threads=4)
    np.testing.assert_array_equal(a, b)
    # flip Both counts twice per sample
    both = (samples["flip"] == 2).sum()
    assert a[:, 0, 0, :].sum() == len(samples) + both


# --------------------------------------------------------------------------- normalisation
@pytest.mark.parametrize("hist,prior,bias,expected", K.NORMALIZE_KATS)
def test_normalize_histogram_kats(hist, prior, bias, expected):
    out = orc.normalize_histogram(hist, prior, bias, True)
    for a, b in zip(out, expected):
        assert a == pytest.approx(b, rel=1e-15, abs=1e-300)


# --------------------------------------------------------------------------- argmax tie rule
def test_best_split_tie_rule():
    s = np.zeros((3, 4))
    s[1, 2] = 0.5
    s[0, 3] = 0.5 + 0.5e-13   # within 1e-13 of a later, larger score: first in thresh-major order wins
    f, t, v = orc.best_split(s)
    assert (f, t) == (3, 0)
    s[2, 0] = 0.5 + 2e-13     # clearly larger -> replaces
    f, t, v = orc.best_split(s)
    assert (f, t) == (0, 2)


# --------------------------------------------------------------------------- random numbers
@pytest.mark.parametrize("inp,out", K.PHILOX_KATS)
def test_philox_kat(inp, out):
    got = orc.philox(*inp)
    assert [int(v) for v in got] == list(out)


def test_sampler_range_and_determinism():
    a = orc.sampler_draws(4711, -120, 120, 1000)
    b = orc.sampler_draws(4711, -120, 120, 1000)
    np.testing.assert_array_equal(a, b)
    assert a.min() >= -120 and a.max() <= 120
    # std::mt19937 default-seed first output is 3499211612 (C++ standard, [rand.predef]);
    # a full-range sampler passes engine words through unchanged
    assert int(orc.sampler_draws(5489, 0, -1, 1)[0]) & 0xFFFFFFFF == 3499211612


def test_fill_depth_kat():
    k = K.DEPTH_FILL
    d = np.zeros((k["height"], k["width"]), np.uint16)
    for (x, y), mm in k["seeds"].items():
        d[y, x] = mm
    f = orc.fill_depth(d)[0]
    assert (f[:k["split_row"]] == k["above"]).all()
    assert (f[k["split_row"]:] == k["below"]).all()


def test_fill_depth_leaves_valid_pixels_and_empty_images():
    rng = np.random.default_rng(4)
    d = rng.integers(500, 5000, (2, 13, 17)).astype(np.uint16)
    d[rng.random(d.shape) < 0.4] = 0
    d[1] = 0                                      # an image without any depth stays empty
    f = orc.fill_depth(d)
    assert (f[0][d[0] > 0] == d[0][d[0] > 0]).all()
    assert (f[0] > 0).all()
    assert (f[1] == 0).all()


def test_lab_reference_white_and_black():
    rgb = np.array([[[[255, 255, 255], [0, 0, 0], [255, 0, 0]]]], np.uint8)
    lab = orc.rgb_to_lab(rgb)[0]
    assert lab[0, 0, 0] == pytest.approx(100.0, abs=1e-4) and abs(lab[1, 0, 0]) < 1e-3 and abs(lab[2, 0, 0]) < 1e-3
    assert lab[:, 0, 1].tolist() == [0.0, 0.0, 0.0]
    # pure red (linear RGB): L* = 116 cbrt(0.212671) - 16 = 53.24, a* and b* strongly positive
    assert lab[0, 0, 2] == pytest.approx(53.2408, abs=1e-3)
    assert lab[1, 0, 2] > 70 and lab[2, 0, 2] > 60
