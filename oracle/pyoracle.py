"""ctypes bindings for the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU legs of
bench.py to check or time the reference algorithm; the curfil_b200 product never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

SAMPLE_DTYPE = np.dtype([("x", "<u2"), ("y", "<u2"), ("image", "<u4"), ("depth", "<f4"),
                         ("label", "u1"), ("flip", "u1"), ("reserved", "<u2")])
assert SAMPLE_DTYPE.itemsize == 16


class _Dataset(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("color", ctypes.c_void_p), ("depth_sum", ctypes.c_void_p),
                ("depth_valid", ctypes.c_void_p)]


class _TrainConfig(ctypes.Structure):
    _fields_ = [("num_features", ctypes.c_int), ("num_thresholds", ctypes.c_int),
                ("max_depth", ctypes.c_int), ("min_sample_count", ctypes.c_int),
                ("box_radius", ctypes.c_int), ("region_size", ctypes.c_int),
                ("use_depth_images", ctypes.c_int), ("num_threads", ctypes.c_int)]


class _TreeOut(ctypes.Structure):
    _fields_ = [("max_nodes", ctypes.c_int), ("num_nodes", ctypes.c_int),
                ("level", ctypes.c_void_p), ("left", ctypes.c_void_p),
                ("feature", ctypes.c_void_p), ("threshold", ctypes.c_void_p),
                ("score", ctypes.c_void_p), ("feature_id", ctypes.c_void_p),
                ("histogram", ctypes.c_void_p), ("num_samples", ctypes.c_void_p)]


class _TreeView(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int), ("left", ctypes.c_void_p),
                ("feature", ctypes.c_void_p), ("threshold", ctypes.c_void_p),
                ("normalized", ctypes.c_void_p)]


_lib = None


def build():
    """Compile the oracle with its Makefile (g++ + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_pixel_depth.restype = ctypes.c_float
        _lib.orc_feature_response.restype = ctypes.c_double
        _lib.orc_score.restype = ctypes.c_double
        _lib.orc_information_gain.restype = ctypes.c_double
        _lib.orc_train_tree.restype = ctypes.c_int
        _lib.orc_sample_class_uniform.restype = ctypes.c_int
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


class Dataset:
    """Integral images of n equal-size frames in the reference layout (int64 depth sums)."""

    def __init__(self, color, depth_sum, depth_valid):
        self.color = np.ascontiguousarray(color, dtype=np.float32)
        self.depth_sum = np.ascontiguousarray(depth_sum, dtype=np.int64)
        self.depth_valid = np.ascontiguousarray(depth_valid, dtype=np.int32)
        n, _, h, w = self.color.shape
        self._c = _Dataset(n, w, h, self.color.ctypes.data, self.depth_sum.ctypes.data,
                           self.depth_valid.ctypes.data)

    @property
    def n(self):
        return self._c.n

    @property
    def width(self):
        return self._c.width

    @property
    def height(self):
        return self._c.height

    def ref(self):
        return ctypes.byref(self._c)


def integral(rgb, depth_mm):
    """rgb uint8 [n][H][W][3], depth_mm uint16 [n][H][W] -> Dataset."""
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    depth_mm = np.ascontiguousarray(depth_mm, dtype=np.uint16)
    n, h, w = depth_mm.shape
    color = np.empty((n, 3, h, w), np.float32)
    dsum = np.empty((n, h, w), np.int64)
    dvalid = np.empty((n, h, w), np.int32)
    for i in range(n):
        lib().orc_integral(w, h, _p(rgb[i]), _p(depth_mm[i]), _p(color[i]), _p(dsum[i]), _p(dvalid[i]))
    return Dataset(color, dsum, dvalid)


def integral_float_color(color_planes):
    """color_planes float32 [3][H][W] -> integrated float32 [3][H][W] (reference Kahan scan)."""
    color_planes = np.ascontiguousarray(color_planes, dtype=np.float32)
    _, h, w = color_planes.shape
    out = np.empty_like(color_planes)
    lib().orc_integral_float_color(w, h, _p(color_planes), _p(out))
    return out


def pad_integral(ds, width, height):
    """RGBDImage::resizeImage (image.cpp:450-475) on integrated frames: the frames go to the top-left
    corner of width x height frames; colour NaN and depth sum / valid count 0 elsewhere."""
    n, _, h, w = ds.color.shape
    color = np.full((n, 3, height, width), np.nan, np.float32)
    color[:, :, :h, :w] = ds.color
    dsum = np.zeros((n, height, width), np.int64)
    dsum[:, :h, :w] = ds.depth_sum
    dvalid = np.zeros((n, height, width), np.int32)
    dvalid[:, :h, :w] = ds.depth_valid
    return Dataset(color, dsum, dvalid)


def pixel_depth(ds, image, x, y):
    return lib().orc_pixel_depth(ds.ref(), image, x, y)


def feature_responses(ds, samples, features):
    samples = np.ascontiguousarray(samples, dtype=SAMPLE_DTYPE)
    features = np.ascontiguousarray(features, dtype=np.int8)
    F = features.shape[1]
    out = np.empty((F, len(samples)), np.float64)
    lib().orc_feature_responses(ds.ref(), len(samples), _p(samples), F, _p(features), _p(out))
    return out


def histograms(ds, samples, features, thresholds, num_classes, threads=1):
    """counters uint32[C][F][T][2] (FeatureEvaluationCPU layout)."""
    samples = np.ascontiguousarray(samples, dtype=SAMPLE_DTYPE)
    features = np.ascontiguousarray(features, dtype=np.int8)
    thresholds = np.ascontiguousarray(thresholds, dtype=np.float32)
    T, F = thresholds.shape
    out = np.empty((num_classes, F, T, 2), np.uint32)
    lib().orc_histograms(ds.ref(), len(samples), _p(samples), F, T, _p(features), _p(thresholds),
                         num_classes, _p(out), threads)
    return out


def score(left, right, all_classes, information_gain_only=False):
    left = np.ascontiguousarray(left, dtype=np.uint32)
    right = np.ascontiguousarray(right, dtype=np.uint32)
    all_classes = np.ascontiguousarray(all_classes, dtype=np.uint32)
    fn = lib().orc_information_gain if information_gain_only else lib().orc_score
    return fn(len(left), _p(left), _p(right), 1, _p(all_classes), ctypes.c_double(float(left.sum())),
              ctypes.c_double(float(right.sum())))


def scores(counters, node_histogram):
    counters = np.ascontiguousarray(counters, dtype=np.uint32)
    node_histogram = np.ascontiguousarray(node_histogram, dtype=np.uint32)
    C, F, T, _ = counters.shape
    out = np.empty((T, F), np.float64)
    lib().orc_scores(C, F, T, _p(counters), _p(node_histogram), _p(out))
    return out


def best_split(scores_tf):
    scores_tf = np.ascontiguousarray(scores_tf, dtype=np.float64)
    T, F = scores_tf.shape
    bf, bt, bs = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    lib().orc_best_split(F, T, _p(scores_tf), ctypes.byref(bf), ctypes.byref(bt), ctypes.byref(bs))
    return bf.value, bt.value, bs.value


def sampler_draws(seed, lo, hi, count):
    out = np.empty(count, np.int32)
    lib().orc_sampler_draws(seed, lo, hi, count, _p(out))
    return out


def philox(key0, key1, c0, c1, c2, c3):
    out = np.empty(4, np.uint32)
    lib().orc_philox4x32(ctypes.c_uint32(key0), ctypes.c_uint32(key1), ctypes.c_uint32(c0),
                         ctypes.c_uint32(c1), ctypes.c_uint32(c2), ctypes.c_uint32(c3), _p(out))
    return out


def generate_features(ds, samples, seed, num_features, num_thresholds, box_radius, region_size,
                      use_depth_images=True):
    samples = np.ascontiguousarray(samples, dtype=SAMPLE_DTYPE)
    feats = np.empty((11, num_features), np.int8)
    thr = np.empty((num_thresholds, num_features), np.float32)
    lib().orc_generate_features(ds.ref(), len(samples), _p(samples), ctypes.c_uint32(seed), num_features,
                                num_thresholds, box_radius, region_size, int(use_depth_images), _p(feats),
                                _p(thr))
    return feats, thr


class Tree:
    """Breadth-first node arrays of a trained tree (index = nodeId - treeId)."""

    def __init__(self, max_nodes, num_classes):
        self.C = num_classes
        self.level = np.zeros(max_nodes, np.int32)
        self.left = np.zeros(max_nodes, np.int32)
        self.feature = np.zeros((max_nodes, 11), np.int8)
        self.threshold = np.zeros(max_nodes, np.float32)
        self.score = np.zeros(max_nodes, np.float64)
        self.feature_id = np.zeros(max_nodes, np.int32)
        self.histogram = np.zeros((max_nodes, num_classes), np.uint32)
        self.num_samples = np.zeros(max_nodes, np.uint32)
        self._c = _TreeOut(max_nodes, 0, self.level.ctypes.data, self.left.ctypes.data,
                           self.feature.ctypes.data, self.threshold.ctypes.data, self.score.ctypes.data,
                           self.feature_id.ctypes.data, self.histogram.ctypes.data,
                           self.num_samples.ctypes.data)

    def trim(self):
        n = self._c.num_nodes
        for name in ("level", "left", "feature", "threshold", "score", "feature_id", "histogram",
                     "num_samples"):
            setattr(self, name, getattr(self, name)[:n].copy())
        return self

    @property
    def num_nodes(self):
        return len(self.level)


def train_tree(ds, samples, num_classes, num_features, num_thresholds, max_depth, min_sample_count,
               box_radius, region_size, seed_counter, use_depth_images=True, threads=1, max_nodes=None):
    """Returns (status, Tree, new_seed_counter)."""
    samples = np.ascontiguousarray(samples, dtype=SAMPLE_DTYPE)
    if max_nodes is None:
        max_nodes = 2 * len(samples) + 1
    tree = Tree(max_nodes, num_classes)
    cfg = _TrainConfig(num_features, num_thresholds, max_depth, min_sample_count, box_radius, region_size,
                       int(use_depth_images), threads)
    sc = ctypes.c_int(seed_counter)
    rc = lib().orc_train_tree(ds.ref(), len(samples), _p(samples), num_classes, ctypes.byref(cfg),
                              ctypes.byref(sc), ctypes.byref(tree._c))
    return rc, tree.trim(), sc.value


def normalize_histogram(histogram, prior, bias, use_labels_prior=True):
    histogram = np.ascontiguousarray(histogram, dtype=np.uint32)
    prior = np.ascontiguousarray(prior, dtype=np.uint32)
    out = np.empty(len(histogram), np.float64)
    lib().orc_normalize_histogram(len(histogram), _p(histogram), _p(prior), ctypes.c_double(bias),
                                  int(use_labels_prior), _p(out))
    return out


def predict(ds, image, trees, normalized, num_classes, threads=1):
    """trees: list of Tree; normalized: list of float64 [nodes][C]."""
    views = (_TreeView * len(trees))()
    keep = []
    for i, (t, nh) in enumerate(zip(trees, normalized)):
        nh = np.ascontiguousarray(nh, dtype=np.float64)
        keep.append(nh)
        views[i] = _TreeView(t.num_nodes, t.left.ctypes.data, t.feature.ctypes.data, t.threshold.ctypes.data,
                             nh.ctypes.data)
    probs = np.empty((num_classes, ds.height, ds.width), np.float32)
    labels = np.empty((ds.height, ds.width), np.uint8)
    lib().orc_predict(ds.ref(), image, len(trees), views, num_classes, _p(probs), _p(labels), threads)
    return probs, labels


def fill_depth(depth_mm):
    """RGBDImage::fillDepth of uint16 [n][H][W] (a filled copy)."""
    d = np.array(depth_mm, dtype=np.uint16, copy=True, order="C")
    if d.ndim == 2:
        d = d[None]
    n, h, w = d.shape
    lib().orc_fill_depth(n, w, h, _p(d))
    return d


def rgb_to_lab(rgb):
    """L*a*b* float32 [n][3][H][W] of uint8 [n][H][W][3]."""
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    n, h, w, _ = rgb.shape
    out = np.empty((n, 3, h, w), np.float32)
    lib().orc_rgb_to_lab(n, w, h, _p(rgb), _p(out))
    return out


def mlp_loss_grad(params, X, Y, hidden, num_classes):
    """(mean loss, gradient float64 [P]) of the refinement network in double."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.uint8)
    n, D = X.shape
    grad = np.empty(params.size, np.float64)
    loss = ctypes.c_double()
    lib().orc_mlp_loss_grad(n, D, hidden, num_classes, _p(params), _p(X), _p(Y), _p(grad), ctypes.byref(loss))
    return loss.value, grad


def sample_class_uniform_keys(labels, depth_mm, num_classes, ignore, subsample_count, seed_counter):
    """The device sampler's definition (keys per pixel); same calling convention as below."""
    labels = np.ascontiguousarray(labels, dtype=np.uint8)
    depth_mm = np.ascontiguousarray(depth_mm, dtype=np.uint16)
    ignore = np.ascontiguousarray(ignore, dtype=np.uint8)
    n, h, w = labels.shape
    cap = n * h * w
    out = np.empty(cap, SAMPLE_DTYPE)
    sc = ctypes.c_int(seed_counter)
    rc = lib().orc_sample_class_uniform_keys(n, w, h, _p(labels), _p(depth_mm), num_classes, _p(ignore),
                                             subsample_count, ctypes.byref(sc), cap, _p(out))
    if rc < 0:
        return rc, None, sc.value
    return rc, out[:rc].copy(), sc.value


def sample_class_uniform(labels, depth_mm, num_classes, ignore, subsample_count, seed_counter):
    labels = np.ascontiguousarray(labels, dtype=np.uint8)
    depth_mm = np.ascontiguousarray(depth_mm, dtype=np.uint16)
    ignore = np.ascontiguousarray(ignore, dtype=np.uint8)
    n, h, w = labels.shape
    cap = n * h * w
    out = np.empty(cap, SAMPLE_DTYPE)
    sc = ctypes.c_int(seed_counter)
    rc = lib().orc_sample_class_uniform(n, w, h, _p(labels), _p(depth_mm), num_classes, _p(ignore),
                                        subsample_count, ctypes.byref(sc), cap, _p(out))
    if rc < 0:
        return rc, None, sc.value
    return rc, out[:rc].copy(), sc.value


def synthetic_frames(seed, num_images, width, height, num_cells, num_classes, first=0):
    """(rgb uint8 [n][H][W][3], depth uint16 [n][H][W], labels uint8 [n][H][W]) of the workloads'
    seeded synthetic generator (restated here; frames first .. first + n - 1)."""
    rgb = np.empty((num_images, height, width, 3), np.uint8)
    depth = np.empty((num_images, height, width), np.uint16)
    labels = np.empty((num_images, height, width), np.uint8)
    lib().orc_synthetic_frames(ctypes.c_uint64(seed), first, num_images, width, height, num_cells, num_classes,
                               _p(rgb), _p(depth), _p(labels))
    return rgb, depth, labels


def sample_pixel_uniform(labels, depth_mm, ignore, subsample_count, seed_counter):
    """Pixel-uniform sampling with the block sort; returns (count, samples, new seed counter)."""
    labels = np.ascontiguousarray(labels, dtype=np.uint8)
    depth_mm = np.ascontiguousarray(depth_mm, dtype=np.uint16)
    ignore = np.ascontiguousarray(ignore, dtype=np.uint8)
    n, h, w = labels.shape
    cap = n * subsample_count
    out = np.empty(cap, SAMPLE_DTYPE)
    sc = ctypes.c_int(seed_counter)
    rc = lib().orc_sample_pixel_uniform(n, w, h, _p(labels), _p(depth_mm), _p(ignore), subsample_count,
                                        ctypes.byref(sc), cap, _p(out))
    if rc < 0:
        return rc, None, sc.value
    return rc, out[:rc].copy(), sc.value
