"""curfil_b200: CURFIL's random-forest training split search and dense prediction on B200.

Python bindings over the C-ABI of libcurfil_b200.so (include/curfil_b200.h). Host arrays are
numpy arrays; device arrays may be passed as raw pointers (e.g. ``torch.Tensor.data_ptr()``).
The CUDA library is required: importing succeeds without it, but every call raises
``RuntimeError`` until ``curfil_b200._build.build()`` has produced libcurfil_b200.so.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcurfil_b200.so")

SAMPLE_DTYPE = np.dtype([("x", "<u2"), ("y", "<u2"), ("image", "<u4"), ("depth", "<f4"),
                         ("label", "u1"), ("flip", "u1"), ("reserved", "<u2")])
SPLIT_DTYPE = np.dtype([("score", "<f8"), ("feature", "<i4"), ("threshold_index", "<i4"),
                        ("threshold", "<f4"), ("flags", "<i4")])
assert SAMPLE_DTYPE.itemsize == 16 and SPLIT_DTYPE.itemsize == 24

LEVEL_BATCHED = 0
PER_NODE = 1

STATUS = {0: "CF_OK", 1: "CF_ERR_INVALID", 2: "CF_ERR_CUDA", 3: "CF_ERR_OOM", 4: "CF_ERR_EMPTY_CHILD",
          5: "CF_ERR_CAPACITY", 6: "CF_ERR_TIMEOUT", 7: "CF_ERR_REJECTED", 8: "CF_ERR_IO", 9: "CF_ERR_STATE"}


class CurfilError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS.get(status, status), message))
        self.status = status


class TrainConfig(ctypes.Structure):
    """TrainingConfiguration (random_tree.h:187-493)."""
    _fields_ = [("random_seed", ctypes.c_int32), ("samples_per_image", ctypes.c_uint32),
                ("feature_count", ctypes.c_uint32), ("min_sample_count", ctypes.c_uint32),
                ("max_depth", ctypes.c_int32), ("box_radius", ctypes.c_uint16),
                ("region_size", ctypes.c_uint16), ("thresholds", ctypes.c_uint16),
                ("sampler", ctypes.c_uint16), ("num_threads", ctypes.c_int32),
                ("max_images", ctypes.c_int32), ("image_cache_size", ctypes.c_int32),
                ("max_samples_per_batch", ctypes.c_uint32), ("acceleration_mode", ctypes.c_int32),
                ("use_cie_lab", ctypes.c_int32), ("use_depth_filling", ctypes.c_int32),
                ("use_depth_images", ctypes.c_int32), ("horizontal_flipping", ctypes.c_int32),
                ("subsampling_type", ctypes.c_int32)]

    def __init__(self, **kw):
        defaults = dict(random_seed=4711, samples_per_image=500, feature_count=500, min_sample_count=32,
                        max_depth=12, box_radius=60, region_size=15, thresholds=20, num_threads=1,
                        max_images=0, image_cache_size=1 << 30, max_samples_per_batch=50000,
                        acceleration_mode=1, use_cie_lab=0, use_depth_filling=0, use_depth_images=1,
                        horizontal_flipping=0, subsampling_type=0)
        defaults.update(kw)
        super().__init__(**defaults)


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_int64), ("max_batch_frames", ctypes.c_int32),
                ("max_pending", ctypes.c_int32), ("pipeline_depth", ctypes.c_int32),
                ("return_probabilities", ctypes.c_int32), ("policy", ctypes.c_int32), ("max_wait_ms", ctypes.c_float),
                ("device_priority", ctypes.c_int32), ("max_queue_ms", ctypes.c_float)]


class EvalTuning(ctypes.Structure):
    """cf_eval_tuning: launch shape of the level-batched split search (speed only, never results)."""
    _fields_ = [("features_per_tile", ctypes.c_int32), ("bins_budget_words", ctypes.c_int32),
                ("warp_aggregate", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("feature_granule", ctypes.c_int32), ("items_per_slot", ctypes.c_float),
                ("sample_groups", ctypes.c_int32), ("min_item_evals", ctypes.c_int32),
                ("stage_bins", ctypes.c_int32), ("stage_max_mb", ctypes.c_int32),
                ("sample_order", ctypes.c_int32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class RequestStats(ctypes.Structure):
    _fields_ = [("submit_ms", ctypes.c_double), ("admitted_ms", ctypes.c_double), ("done_ms", ctypes.c_double),
                ("batch_id", ctypes.c_int32), ("batch_frames", ctypes.c_int32)]


_lib = None
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64


def lib():
    """The loaded libcurfil_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libcurfil_b200.so is missing: run curfil_b200._build.build() (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        L.cf_version.restype = ctypes.c_char_p
        L.cf_last_error.restype = ctypes.c_size_t
        L.cf_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.cf_context_launch_count.restype = ctypes.c_int64
        L.cf_context_launch_count.argtypes = [_vp]
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        buf = ctypes.create_string_buffer(4096)
        lib().cf_last_error(buf, 4096)
        raise CurfilError(status, buf.value.decode(errors="replace"))


def _p(a):
    if a is None:
        return _vp(0)
    if isinstance(a, int):
        return _vp(a)
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays passed to curfil_b200 must be C-contiguous")
    return _vp(a.ctypes.data)


def version():
    return lib().cf_version().decode()


class Context:
    """cf_context: one CUDA device, one stream, optional per-kernel event timing."""

    def __init__(self, device=0):
        h = _vp()
        _check(lib().cf_context_create(int(device), ctypes.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            _check(lib().cf_context_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        _check(lib().cf_context_set_stream(self.handle, _vp(int(stream_handle) if stream_handle else 0)))

    def synchronize(self):
        _check(lib().cf_context_synchronize(self.handle))

    def set_timing(self, enable=True):
        _check(lib().cf_context_set_timing(self.handle, int(enable)))

    def reset_timing(self):
        _check(lib().cf_context_reset_timing(self.handle))

    def kernel_time(self, name="*"):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _check(lib().cf_context_kernel_time(self.handle, name.encode(), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def launch_count(self):
        return lib().cf_context_launch_count(self.handle)

    def device(self):
        """{'name', 'sms', 'cc'} of the context's device."""
        name = ctypes.create_string_buffer(256)
        sms, major, minor = _i32(), _i32(), _i32()
        _check(lib().cf_context_device(self.handle, name, 256, ctypes.byref(sms), ctypes.byref(major),
                                       ctypes.byref(minor)))
        return {"name": name.value.decode(), "sms": sms.value, "cc": "%d.%d" % (major.value, minor.value)}

    def get_tuning(self):
        t = EvalTuning()
        _check(lib().cf_context_get_tuning(self.handle, ctypes.byref(t)))
        return t

    def set_tuning(self, tuning=None, **fields):
        """Set the split-search launch shape: an EvalTuning, and/or field=value overrides of the
        current one; no arguments restore the defaults."""
        if tuning is None and not fields:
            _check(lib().cf_context_set_tuning(self.handle, _vp(0)))
            return
        t = self.get_tuning() if tuning is None else EvalTuning(*[getattr(tuning, n) for n, _ in EvalTuning._fields_])
        for k, v in fields.items():
            if k not in dict(EvalTuning._fields_):
                raise ValueError("unknown tuning field %r" % k)
            setattr(t, k, v)
        _check(lib().cf_context_set_tuning(self.handle, ctypes.byref(t)))


class Dataset:
    """cf_dataset: integral images of equal-size frames resident in device memory."""

    def __init__(self, ctx, num_images, width, height):
        h = _vp()
        _check(lib().cf_dataset_create(ctx.handle, int(num_images), int(width), int(height), ctypes.byref(h)))
        self.handle, self.ctx = h, ctx
        self.n, self.width, self.height = int(num_images), int(width), int(height)

    @classmethod
    def from_raw(cls, ctx, rgb, depth_mm, fill_depth=False, cie_lab=False):
        rgb = np.ascontiguousarray(rgb, np.uint8)
        depth_mm = np.ascontiguousarray(depth_mm, np.uint16)
        n, h, w = depth_mm.shape
        ds = cls(ctx, n, w, h)
        ds.upload_raw(rgb, depth_mm, fill_depth=fill_depth, cie_lab=cie_lab)
        return ds

    @classmethod
    def from_integral(cls, ctx, color, depth):
        color = np.ascontiguousarray(color, np.float32)
        depth = np.ascontiguousarray(depth, np.int32)
        n, _, h, w = color.shape
        ds = cls(ctx, n, w, h)
        _check(lib().cf_dataset_upload_integral(ds.handle, 0, n, _p(color), _p(depth)))
        return ds

    def upload_raw(self, rgb, depth_mm, first=0, fill_depth=False, cie_lab=False):
        """Raw frames to integral images; fill_depth / cie_lab as useDepthFilling / useCIELab."""
        if isinstance(rgb, int):
            _check(lib().cf_dataset_upload_raw_ex(self.handle, first, int(depth_mm[1]), _vp(rgb), _vp(depth_mm[0]), 1,
                                                  int(fill_depth), int(cie_lab)))
            return
        n = depth_mm.shape[0]
        _check(lib().cf_dataset_upload_raw_ex(self.handle, int(first), int(n), _p(rgb), _p(depth_mm), 0,
                                              int(fill_depth), int(cie_lab)))

    def upload_raw_padded(self, rgb, depth_mm, first=0, fill_depth=False, cie_lab=False):
        """Frames smaller than the dataset's, padded as loadImages pads them (RGBDImage::resizeImage)."""
        rgb = np.ascontiguousarray(rgb, np.uint8)
        depth_mm = np.ascontiguousarray(depth_mm, np.uint16)
        if depth_mm.ndim == 2:
            rgb, depth_mm = rgb[None], depth_mm[None]
        n, h, w = depth_mm.shape
        _check(lib().cf_dataset_upload_raw_padded(self.handle, int(first), int(n), int(w), int(h), _p(rgb),
                                                  _p(depth_mm), 0, int(fill_depth), int(cie_lab)))

    def upload_raw_device(self, rgb_ptr, depth_ptr, count, first=0):
        _check(lib().cf_dataset_upload_raw(self.handle, int(first), int(count), _vp(rgb_ptr), _vp(depth_ptr), 1))

    def download_integral(self, first=0, count=None):
        count = self.n - first if count is None else count
        color = np.empty((count, 3, self.height, self.width), np.float32)
        depth = np.empty((count, 2, self.height, self.width), np.int32)
        _check(lib().cf_dataset_download_integral(self.handle, first, count, _p(color), _p(depth)))
        return color, depth

    def close(self):
        if self.handle:
            _check(lib().cf_dataset_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def samples_array(n):
    return np.zeros(n, SAMPLE_DTYPE)


def feature_responses(ds, samples, features):
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    features = np.ascontiguousarray(features, np.int8)
    F = features.shape[1]
    out = np.empty((F, len(samples)), np.float64)
    _check(lib().cf_feature_responses(ds.handle, len(samples), _p(samples), F, _p(features), _p(out)))
    return out


def histograms(ds, samples, features, thresholds, num_classes):
    """counters uint32 [F][T][C][2] (reference GPU layout)."""
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    features = np.ascontiguousarray(features, np.int8)
    thresholds = np.ascontiguousarray(thresholds, np.float32)
    T, F = thresholds.shape
    out = np.empty((F, T, num_classes, 2), np.uint32)
    _check(lib().cf_histograms(ds.handle, len(samples), _p(samples), F, T, _p(features), _p(thresholds),
                               int(num_classes), _p(out)))
    return out


def scores(ctx, counters, node_histogram):
    """scores double [T][F] from counters [F][T][C][2]."""
    counters = np.ascontiguousarray(counters, np.uint32)
    node_histogram = np.ascontiguousarray(node_histogram, np.uint32)
    F, T, C, _ = counters.shape
    out = np.empty((T, F), np.float64)
    _check(lib().cf_scores(ctx.handle, C, F, T, _p(counters), _p(node_histogram), _p(out)))
    return out


def score_bounds(ctx, counters, node_histogram):
    """(lower, upper) float32 [T][F] enclosing scores(ctx, counters, node_histogram)."""
    counters = np.ascontiguousarray(counters, np.uint32)
    node_histogram = np.ascontiguousarray(node_histogram, np.uint32)
    F, T, C, _ = counters.shape
    lo = np.empty((T, F), np.float32)
    up = np.empty((T, F), np.float32)
    _check(lib().cf_score_bounds(ctx.handle, C, F, T, _p(counters), _p(node_histogram), _p(lo), _p(up)))
    return lo, up


def generate_features(ds, samples, seed, num_features, num_thresholds, box_radius, region_size, use_depth_images=True):
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    feats = np.empty((11, num_features), np.int8)
    thr = np.empty((num_thresholds, num_features), np.float32)
    _check(lib().cf_generate_features(ds.handle, len(samples), _p(samples), ctypes.c_uint32(seed), num_features,
                                      num_thresholds, box_radius, region_size, int(use_depth_images), _p(feats),
                                      _p(thr)))
    return feats, thr


def evaluate_best_splits(ds, node_offsets, samples, num_classes, features, thresholds):
    node_offsets = np.ascontiguousarray(node_offsets, np.int64)
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    features = np.ascontiguousarray(features, np.int8)
    thresholds = np.ascontiguousarray(thresholds, np.float32)
    T, F = thresholds.shape
    M = len(node_offsets) - 1
    out = np.empty(M, SPLIT_DTYPE)
    _check(lib().cf_evaluate_best_splits(ds.handle, M, _p(node_offsets), _p(samples), int(num_classes), F, T,
                                         _p(features), _p(thresholds), _p(out)))
    return out


def level_left_counts(ds, node_offsets, samples, num_classes, features, thresholds):
    """(best splits, left counts uint32 [M][F][T][C]) as accumulated by the level-batched kernel."""
    node_offsets = np.ascontiguousarray(node_offsets, np.int64)
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    features = np.ascontiguousarray(features, np.int8)
    thresholds = np.ascontiguousarray(thresholds, np.float32)
    T, F = thresholds.shape
    M = len(node_offsets) - 1
    best = np.empty(M, SPLIT_DTYPE)
    left = np.empty((M, F, T, num_classes), np.uint32)
    _check(lib().cf_level_left_counts(ds.handle, M, _p(node_offsets), _p(samples), int(num_classes), F, T,
                                      _p(features), _p(thresholds), _p(best), _p(left)))
    return best, left


def evaluate_best_splits_noalloc(ctx, color_ptr, depth_ptr, num_images, width, height, node_offsets, samples_ptr,
                                 node_hist_ptr, num_classes, num_features, num_thresholds, features_ptr,
                                 thresholds_ptr, best_ptr):
    """cf_evaluate_best_splits without device allocation: every array argument except the host
    `node_offsets` is a device pointer owned by the caller (see include/curfil_b200.h)."""
    node_offsets = np.ascontiguousarray(node_offsets, np.int64)
    _check(lib().cf_evaluate_best_splits_noalloc(
        ctx.handle, _vp(color_ptr), _vp(depth_ptr), int(num_images), int(width), int(height),
        len(node_offsets) - 1, _p(node_offsets), _vp(samples_ptr), _vp(node_hist_ptr), int(num_classes),
        int(num_features), int(num_thresholds), _vp(features_ptr), _vp(thresholds_ptr), _vp(best_ptr)))


class Tree:
    """cf_tree: a trained tree in breadth-first node arrays (index = nodeId - treeId)."""

    def __init__(self, handle):
        self.handle = handle
        n, c, d, tid = _i32(), _i32(), _i32(), _i32()
        _check(lib().cf_tree_info(handle, ctypes.byref(n), ctypes.byref(c), ctypes.byref(d), ctypes.byref(tid)))
        self.num_nodes, self.num_classes, self.depth, self.tree_id = n.value, c.value, d.value, tid.value

    def arrays(self):
        n, C = self.num_nodes, self.num_classes
        a = dict(level=np.empty(n, np.int32), left=np.empty(n, np.int32), feature=np.empty((n, 11), np.int8),
                 threshold=np.empty(n, np.float32), score=np.empty(n, np.float64),
                 feature_id=np.empty(n, np.int32), histogram=np.empty((n, C), np.uint32),
                 num_samples=np.empty(n, np.uint32))
        _check(lib().cf_tree_export(self.handle, _p(a["level"]), _p(a["left"]), _p(a["feature"]), _p(a["threshold"]),
                                    _p(a["score"]), _p(a["feature_id"]), _p(a["histogram"]), _p(a["num_samples"])))
        return a

    def prior(self):
        cnt = _i32()
        _check(lib().cf_tree_prior(self.handle, _vp(0), 0, ctypes.byref(cnt)))
        out = np.empty(cnt.value, np.uint32)
        if cnt.value:
            _check(lib().cf_tree_prior(self.handle, _p(out), cnt.value, ctypes.byref(cnt)))
        return out

    def set_prior(self, prior):
        prior = np.ascontiguousarray(prior, np.uint32)
        _check(lib().cf_tree_set_prior(self.handle, _p(prior), len(prior)))

    def level_stats(self):
        """[(open nodes, samples, split-search ms)] per level of the last training."""
        n = _i32()
        _check(lib().cf_tree_level_stats(self.handle, 0, ctypes.byref(n), _vp(0), _vp(0), _vp(0)))
        nodes = np.zeros(n.value, np.int32)
        samples = np.zeros(n.value, np.int64)
        ms = np.zeros(n.value, np.float32)
        _check(lib().cf_tree_level_stats(self.handle, n.value, ctypes.byref(n), _p(nodes), _p(samples), _p(ms)))
        return list(zip(nodes.tolist(), samples.tolist(), ms.tolist()))

    def level_starts(self):
        """Start of each level's split search, ms after the training's first device work."""
        n = len(self.level_stats())
        out = np.zeros(n, np.float32)
        _check(lib().cf_tree_level_starts(self.handle, n, _p(out)))
        return out.tolist()

    def train_stats(self):
        ev, ms, lv = ctypes.c_int64(), ctypes.c_double(), _i32()
        _check(lib().cf_tree_train_stats(self.handle, ctypes.byref(ev), ctypes.byref(ms), ctypes.byref(lv)))
        return ev.value, ms.value, lv.value

    @classmethod
    def from_arrays(cls, tree_id, left, feature, threshold, histogram, level=None, score=None, feature_id=None):
        left = np.ascontiguousarray(left, np.int32)
        feature = np.ascontiguousarray(feature, np.int8)
        threshold = np.ascontiguousarray(threshold, np.float32)
        histogram = np.ascontiguousarray(histogram, np.uint32)
        n, C = histogram.shape
        lv = None if level is None else np.ascontiguousarray(level, np.int32)
        sc = None if score is None else np.ascontiguousarray(score, np.float64)
        fi = None if feature_id is None else np.ascontiguousarray(feature_id, np.int32)
        h = _vp()
        _check(lib().cf_tree_import(int(tree_id), int(n), int(C), _p(lv), _p(left), _p(feature), _p(threshold),
                                    _p(sc), _p(fi), _p(histogram), ctypes.byref(h)))
        return cls(h)

    def write_json(self, path, config=None, prior=None, verbose=False):
        cfg = config if config is not None else TrainConfig()
        prior = self.prior() if prior is None else np.ascontiguousarray(prior, np.uint32)
        _check(lib().cf_tree_write_json(self.handle, ctypes.byref(cfg), _p(prior) if len(prior) else _vp(0),
                                        str(path).encode(), int(verbose)))

    @classmethod
    def read_json(cls, path, max_classes=256):
        cfg = TrainConfig()
        prior = np.zeros(max_classes, np.uint32)
        h = _vp()
        _check(lib().cf_tree_read_json(str(path).encode(), ctypes.byref(cfg), _p(prior), max_classes, ctypes.byref(h)))
        t = cls(h)
        return t, cfg, prior[:t.num_classes].copy()

    def close(self):
        if self.handle:
            _check(lib().cf_tree_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def train_tree(ds, samples, num_classes, config, tree_id=0, seed_counter=0, mode=LEVEL_BATCHED):
    """RandomTreeImage::train from a sample list. Returns (Tree, advanced seed counter)."""
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    sc = _i32(seed_counter)
    h = _vp()
    _check(lib().cf_train_tree(ds.handle, len(samples), _p(samples), int(num_classes), ctypes.byref(config),
                               int(tree_id), ctypes.byref(sc), int(mode), ctypes.byref(h)))
    return Tree(h), sc.value


class LevelSnapshot:
    """cf_level_snapshot: the input state of one level of a tree's training, which can be trained
    again on its own (candidate generation, split search, routing)."""

    def __init__(self, handle):
        self.handle = handle
        lv, m, n = _i32(), _i32(), _i64()
        _check(lib().cf_level_snapshot_info(handle, ctypes.byref(lv), ctypes.byref(m), ctypes.byref(n)))
        self.level, self.num_nodes, self.num_samples = lv.value, m.value, n.value

    def export(self):
        """(node_offsets int64 [M+1], samples [n], level seed)."""
        offsets = np.empty(self.num_nodes + 1, np.int64)
        samples = np.empty(self.num_samples, SAMPLE_DTYPE)
        seed = ctypes.c_uint32()
        _check(lib().cf_level_snapshot_export(self.handle, _p(offsets), _p(samples), ctypes.byref(seed)))
        return offsets, samples, seed.value

    def run(self, mode=LEVEL_BATCHED, splits=False):
        """Trains the level again; returns dict(ms, evals, next_nodes, next_samples[, splits])."""
        ms, ev, nn, ns = ctypes.c_double(), _i64(), _i32(), _i64()
        best = np.empty(self.num_nodes, SPLIT_DTYPE) if splits else None
        _check(lib().cf_level_snapshot_run(self.handle, int(mode), _p(best), ctypes.byref(ms), ctypes.byref(ev),
                                           ctypes.byref(nn), ctypes.byref(ns)))
        out = dict(ms=ms.value, evals=ev.value, next_nodes=nn.value, next_samples=ns.value)
        if splits:
            out["splits"] = best
        return out

    def close(self):
        if self.handle:
            lib().cf_level_snapshot_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def train_tree_snapshots(ds, samples, num_classes, config, levels, tree_id=0, seed_counter=0):
    """cf_train_tree_snapshots: (Tree, [LevelSnapshot of each listed level the tree reaches],
    advanced seed counter)."""
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    lv = np.ascontiguousarray(levels, np.int32)
    handles = (_vp * max(1, len(lv)))()
    got = _i32()
    sc = _i32(seed_counter)
    h = _vp()
    _check(lib().cf_train_tree_snapshots(ds.handle, len(samples), _p(samples), int(num_classes),
                                         ctypes.byref(config), int(tree_id), ctypes.byref(sc), len(lv), _p(lv),
                                         handles, ctypes.byref(got), ctypes.byref(h)))
    return Tree(h), [LevelSnapshot(_vp(handles[i])) for i in range(got.value)], sc.value


_ALLGATHER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p)


def train_tree_sharded(ds, samples, num_classes, config, rank, world, allgather, tree_id=0, seed_counter=0):
    """One tree trained by `world` processes together (cf_train_tree_sharded). `allgather(payload: bytes)`
    must return the concatenation of every rank's payload in rank order (see
    curfil_b200.distributed.allgather_bytes). Returns (Tree, advanced seed counter)."""
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    errors = []

    def trampoline(send, nbytes, recv, user):
        try:
            out = allgather(ctypes.string_at(send, nbytes))
            if len(out) != nbytes * world:
                raise ValueError("all-gather returned %d bytes, expected %d" % (len(out), nbytes * world))
            ctypes.memmove(recv, out, len(out))
            return 0
        except Exception as e:  # reported through the status below
            errors.append(e)
            return 1

    fn = _ALLGATHER_FN(trampoline)
    sc = _i32(seed_counter)
    h = _vp()
    status = lib().cf_train_tree_sharded(ds.handle, len(samples), _p(samples), int(num_classes), ctypes.byref(config),
                                         int(tree_id), ctypes.byref(sc), int(rank), int(world), fn, None,
                                         ctypes.byref(h))
    if status != 0 and errors:
        raise errors[0]
    _check(status)
    return Tree(h), sc.value


def autotune_split_search(ds, samples, num_classes, config, tree_id=0, seed_counter=0, repeats=1, cache=None):
    """Choose the split search's launch shape for this workload (cf_autotune_split_search) and set it on
    the dataset's context. With `cache` (a JSON file path) a previous choice for the same device and
    workload signature is reused without measuring. Returns a dict with the shape and timings."""
    import json
    samples = np.ascontiguousarray(samples, SAMPLE_DTYPE)
    ctx = ds.ctx
    dev = ctx.device()
    key = "%s/%dSM|C=%d F=%d T=%d depth=%d N=%d frames=%dx%dx%d" % (
        dev["name"], dev["sms"], num_classes, config.feature_count, config.thresholds, config.max_depth,
        len(samples), ds.n, ds.width, ds.height)
    table = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            table = json.load(f)
        if key in table:
            ctx.set_tuning(**table[key]["tuning"])
            return dict(table[key], key=key, from_cache=True)
    best = EvalTuning()
    best_ms, start_ms, trials = ctypes.c_double(), ctypes.c_double(), _i32()
    _check(lib().cf_autotune_split_search(ds.handle, len(samples), _p(samples), int(num_classes),
                                          ctypes.byref(config), int(tree_id), _i32(seed_counter), int(repeats),
                                          ctypes.byref(best), ctypes.byref(best_ms), ctypes.byref(start_ms),
                                          ctypes.byref(trials)))
    entry = {"tuning": best.as_dict(), "split_search_ms": best_ms.value, "start_ms": start_ms.value,
             "trials": trials.value}
    if cache:
        table[key] = entry
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, cache)
    return dict(entry, key=key, from_cache=False)


def forest_seed(random_seed):
    """SEED of RandomForestImage::train; tree t starts its random source at SEED + t."""
    s = _i32()
    _check(lib().cf_forest_seed(int(random_seed), ctypes.byref(s)))
    return s.value


def sample_tree_pixels(labels, depth_mm, num_classes, config, num_trees, seed_counter, ignored=None, ctx=None):
    """Training pixels of one tree (sampling + block sort). Returns (samples, prior, new seed counter).
    With `ctx`, classUniform sampling runs on that context's device (cf_sample_tree_pixels_device)."""
    labels = np.ascontiguousarray(labels, np.uint8)
    depth_mm = np.ascontiguousarray(depth_mm, np.uint16)
    n, h, w = labels.shape
    ign = None if ignored is None else np.ascontiguousarray(ignored, np.uint8)
    sc = _i32(seed_counter)
    cnt = ctypes.c_int64()
    # class-uniform draws ceil(n * sub / classes) per class, pixel-uniform n * sub: bounded by n * sub + classes
    cap = n * (config.samples_per_image // max(1, num_trees)) + num_classes
    out = np.empty(cap, SAMPLE_DTYPE)
    prior = np.empty(num_classes, np.uint32)
    if ctx is not None:
        _check(lib().cf_sample_tree_pixels_device(ctx.handle, n, w, h, _p(labels), _p(depth_mm), int(num_classes),
                                                  _p(ign), ctypes.byref(config), int(num_trees), ctypes.byref(sc),
                                                  _p(out), ctypes.c_int64(len(out)), ctypes.byref(cnt), _p(prior)))
    else:
        _check(lib().cf_sample_tree_pixels(n, w, h, _p(labels), _p(depth_mm), int(num_classes), _p(ign),
                                           ctypes.byref(config), int(num_trees), ctypes.byref(sc), _p(out),
                                           ctypes.c_int64(len(out)), ctypes.byref(cnt), _p(prior)))
    return out[:cnt.value].copy(), prior, sc.value


def train_forest(ctx, rgb, depth_mm, labels, num_classes, config, num_trees, ignored=None, mode=LEVEL_BATCHED):
    """RandomForestImage::train on raw host frames; returns the list of Trees."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    depth_mm = np.ascontiguousarray(depth_mm, np.uint16)
    labels = np.ascontiguousarray(labels, np.uint8)
    n, h, w = depth_mm.shape
    ign = None if ignored is None else np.ascontiguousarray(ignored, np.uint8)
    handles = (_vp * num_trees)()
    _check(lib().cf_forest_train(ctx.handle, n, w, h, _p(rgb), _p(depth_mm), _p(labels), int(num_classes), _p(ign),
                                 ctypes.byref(config), int(num_trees), int(mode), handles))
    return [Tree(_vp(handles[i])) for i in range(num_trees)]


class Forest:
    """cf_forest: normalised, packed trees resident on the device (RandomForestImage + convertTree)."""

    def __init__(self, ctx, trees, prior=None, histogram_bias=0.0, use_labels_prior=True):
        arr = (_vp * len(trees))(*[t.handle.value if isinstance(t.handle, _vp) else t.handle for t in trees])
        pr = None if prior is None else np.ascontiguousarray(prior, np.uint32)
        h = _vp()
        _check(lib().cf_forest_create(ctx.handle, len(trees), arr, _p(pr), ctypes.c_double(histogram_bias),
                                      int(use_labels_prior), ctypes.byref(h)))
        self.handle, self.ctx = h, ctx
        nt, nc, nn = _i32(), _i32(), ctypes.c_int64()
        _check(lib().cf_forest_info(h, ctypes.byref(nt), ctypes.byref(nc), ctypes.byref(nn)))
        self.num_trees, self.num_classes, self.num_nodes = nt.value, nc.value, nn.value

    def predict_dataset(self, ds, first, count, probs_ptr, labels_ptr):
        """Device pointers (ints) for the outputs; either may be 0."""
        _check(lib().cf_predict_dataset(self.handle, ds.handle, int(first), int(count), _vp(probs_ptr),
                                        _vp(labels_ptr)))

    def predict_dataset_host(self, ds, first, count, probabilities=True):
        """cf_predict_dataset with host results: (probs float32 [n][C][H][W] or None, labels uint8 [n][H][W])."""
        h, w = ds.height, ds.width
        probs = np.empty((count, self.num_classes, h, w), np.float32) if probabilities else None
        labels = np.empty((count, h, w), np.uint8)
        _check(lib().cf_predict_dataset_host(self.handle, ds.handle, int(first), int(count), _p(probs), _p(labels)))
        return probs, labels

    def set_preprocessing(self, fill_depth=False, cie_lab=False):
        """Preprocessing of raw frames before prediction, as the forest was trained."""
        _check(lib().cf_forest_set_preprocessing(self.handle, int(fill_depth), int(cie_lab)))

    def predict_dataset_plain(self, ds, first, count, probs_ptr, labels_ptr):
        """The plain per-image launch form (one launch per tree per image, synchronised)."""
        _check(lib().cf_predict_dataset_plain(self.handle, ds.handle, int(first), int(count), _vp(probs_ptr),
                                              _vp(labels_ptr)))

    def predict_plain(self, rgb, depth_mm, probabilities=True):
        """RandomForestImage::predict's GPU flow image by image (the plain per-image launch form)."""
        rgb = np.ascontiguousarray(rgb, np.uint8)
        depth_mm = np.ascontiguousarray(depth_mm, np.uint16)
        if depth_mm.ndim == 2:
            rgb, depth_mm = rgb[None], depth_mm[None]
        n, h, w = depth_mm.shape
        probs = np.empty((n, self.num_classes, h, w), np.float32) if probabilities else None
        labels = np.empty((n, h, w), np.uint8)
        _check(lib().cf_predict_host_plain(self.handle, n, w, h, _p(rgb), _p(depth_mm), _p(probs), _p(labels)))
        return probs, labels

    def predict(self, rgb, depth_mm, probabilities=True):
        rgb = np.ascontiguousarray(rgb, np.uint8)
        depth_mm = np.ascontiguousarray(depth_mm, np.uint16)
        if depth_mm.ndim == 2:
            rgb, depth_mm = rgb[None], depth_mm[None]
        n, h, w = depth_mm.shape
        probs = np.empty((n, self.num_classes, h, w), np.float32) if probabilities else None
        labels = np.empty((n, h, w), np.uint8)
        _check(lib().cf_predict_host(self.handle, n, w, h, _p(rgb), _p(depth_mm), _p(probs), _p(labels)))
        return probs, labels

    def close(self):
        if self.handle:
            _check(lib().cf_forest_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PredictGraph:
    """cf_predict_graph: a fixed batch of raw frames predicted by one CUDA graph replay. `rgb`,
    `depth`, `labels` (and `probabilities`) are numpy views of the graph's pinned staging buffers."""

    def __init__(self, forest, count, width, height, probabilities=False):
        h = _vp()
        _check(lib().cf_predict_graph_create(forest.handle, int(count), int(width), int(height), int(probabilities),
                                             ctypes.byref(h)))
        self.handle, self.forest = h, forest
        rgb, dep, pr, lab = _vp(), _vp(), _vp(), _vp()
        _check(lib().cf_predict_graph_buffers(h, ctypes.byref(rgb), ctypes.byref(dep), ctypes.byref(pr),
                                              ctypes.byref(lab)))
        n, C = int(count), forest.num_classes

        def view(ptr, ctype, shape):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctype)), shape=shape)
        self.rgb = view(rgb, ctypes.c_uint8, (n, height, width, 3))
        self.depth = view(dep, ctypes.c_uint16, (n, height, width))
        self.labels = view(lab, ctypes.c_uint8, (n, height, width))
        self.probabilities = view(pr, ctypes.c_float, (n, C, height, width)) if probabilities else None

    def run(self):
        _check(lib().cf_predict_graph_run(self.handle))

    def close(self):
        if self.handle:
            _check(lib().cf_predict_graph_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefinerConfig(ctypes.Structure):
    _fields_ = [("hidden", ctypes.c_int32), ("radius1", ctypes.c_int32), ("radius2", ctypes.c_int32),
                ("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("pixels_per_image", ctypes.c_int32),
                ("learning_rate", ctypes.c_float), ("seed", ctypes.c_uint32)]

    def __init__(self, **kw):
        d = dict(hidden=64, radius1=4, radius2=16, epochs=8, batch=4096, pixels_per_image=20000,
                 learning_rate=3e-3, seed=1)
        d.update(kw)
        super().__init__(**d)


class Refiner:
    """cf_refiner: the per-pixel refinement network trained on the forest's output (the learned part)."""

    def __init__(self, ctx, num_classes, **config):
        self.config = RefinerConfig(**config)
        h = _vp()
        _check(lib().cf_refiner_create(ctx.handle, int(num_classes), ctypes.byref(self.config), ctypes.byref(h)))
        self.handle, self.ctx, self.num_classes = h, ctx, int(num_classes)
        self.num_features = 3 * self.num_classes + 2

    def train(self, forest, ds, first, count, labels, ignored=None):
        """Returns the mean training loss of every epoch."""
        labels = np.ascontiguousarray(labels, np.uint8)
        ign = None if ignored is None else np.ascontiguousarray(ignored, np.uint8)
        losses = np.zeros(max(1, self.config.epochs), np.float32)
        _check(lib().cf_refiner_train(self.handle, forest.handle, ds.handle, int(first), int(count), _p(labels),
                                      _p(ign), _p(losses)))
        return losses[:self.config.epochs]

    def predict(self, forest, ds, first, count, probs_ptr, labels_ptr):
        """Device pointers (ints) for the outputs; either may be 0."""
        _check(lib().cf_refiner_predict(self.handle, forest.handle, ds.handle, int(first), int(count), _vp(probs_ptr),
                                        _vp(labels_ptr)))

    def params(self, new=None):
        n = _i32()
        _check(lib().cf_refiner_params(self.handle, _vp(0), _vp(0), ctypes.byref(n)))
        if new is not None:
            new = np.ascontiguousarray(new, np.float32)
            if new.size != n.value:
                raise ValueError("expected %d parameters" % n.value)
            _check(lib().cf_refiner_params(self.handle, _vp(0), _p(new), ctypes.byref(n)))
        out = np.empty(n.value, np.float32)
        _check(lib().cf_refiner_params(self.handle, _p(out), _vp(0), ctypes.byref(n)))
        return out

    def loss_grad(self, features, labels):
        features = np.ascontiguousarray(features, np.float32)
        labels = np.ascontiguousarray(labels, np.uint8)
        n = _i32()
        _check(lib().cf_refiner_params(self.handle, _vp(0), _vp(0), ctypes.byref(n)))
        grad = np.empty(n.value, np.float32)
        loss = ctypes.c_double()
        _check(lib().cf_refiner_loss_grad(self.handle, len(labels), _p(features), _p(labels), _p(grad),
                                          ctypes.byref(loss)))
        return loss.value, grad

    def features(self, forest, ds, frame, xy):
        xy = np.ascontiguousarray(xy, np.int32)
        out = np.empty((len(xy), self.num_features), np.float32)
        _check(lib().cf_refiner_features(self.handle, forest.handle, ds.handle, int(frame), len(xy), _p(xy), _p(out)))
        return out

    def close(self):
        if self.handle:
            _check(lib().cf_refiner_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """cf_server: continuous-batching dense prediction on a resident forest."""

    def __init__(self, forest, hbm_budget_bytes=8 << 30, max_batch_frames=16, max_pending=4096, pipeline_depth=2,
                 return_probabilities=False, policy=0, max_wait_ms=0.0, device_priority=0, max_queue_ms=0.0):
        cfg = ServerConfig(int(hbm_budget_bytes), int(max_batch_frames), int(max_pending), int(pipeline_depth),
                           int(return_probabilities), int(policy), float(max_wait_ms), int(device_priority),
                           float(max_queue_ms))
        h = _vp()
        _check(lib().cf_server_create(forest.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self.handle, self.forest = h, forest
        self.return_probabilities = bool(return_probabilities)

    def submit(self, rgb, depth_mm):
        rgb = np.ascontiguousarray(rgb, np.uint8)
        depth_mm = np.ascontiguousarray(depth_mm, np.uint16)
        h, w = depth_mm.shape
        rid = ctypes.c_int64()
        _check(lib().cf_server_submit(self.handle, w, h, _p(rgb), _p(depth_mm), ctypes.byref(rid)))
        return rid.value

    def wait(self, request_id, shape, timeout_s=30.0, probabilities=False):
        h, w = shape
        labels = np.empty((h, w), np.uint8)
        probs = np.empty((self.forest.num_classes, h, w), np.float32) if probabilities else None
        st = RequestStats()
        _check(lib().cf_server_wait(self.handle, ctypes.c_int64(request_id), ctypes.c_double(timeout_s), _p(labels),
                                    _p(probs), ctypes.byref(st)))
        return labels, probs, st

    def counters(self):
        vals = [ctypes.c_int64() for _ in range(4)]
        _check(lib().cf_server_counters(self.handle, *[ctypes.byref(v) for v in vals]))
        return dict(zip(("submitted", "completed", "rejected", "batches"), [v.value for v in vals]))

    def close(self):
        if self.handle:
            _check(lib().cf_server_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def integrate_planes(ctx, color, depth):
    """RGBDImage::calculateIntegral of images in the reference layout: colour float32 [n][3][H][W] and
    depth int32 [n][2][H][W] (mm with 0 invalid, valid flag). Returns the integrated copies."""
    color = np.array(color, np.float32, copy=True, order="C")
    depth = np.array(depth, np.int32, copy=True, order="C")
    n, _, h, w = color.shape
    if depth.shape != (n, 2, h, w):
        raise ValueError("depth must be int32 [n][2][H][W]")
    _check(lib().cf_integrate_planes(ctx.handle, n, w, h, _p(color), _p(depth), _p(color), _p(depth), 0))
    return color, depth


def normalize_histogram(histogram, prior, bias=0.0, use_labels_prior=True):
    """detail::normalizeHistogram of one histogram with the class prior (host)."""
    h = np.ascontiguousarray(histogram, np.uint32)
    p = np.ascontiguousarray(prior, np.uint32)
    out = np.empty(len(h), np.float64)
    _check(lib().cf_normalize_histogram(len(h), _p(h), _p(p), ctypes.c_double(bias), int(use_labels_prior), _p(out)))
    return out


def pad_labels(labels, width, height, padding_label):
    """LabelImage::resizeImage (image.cpp:763-777): label frames [n][h][w] placed top-left in [n][height][width]
    frames filled with `padding_label` (getPaddingLabel: the first ignored colour's label, else black's)."""
    labels = np.asarray(labels, np.uint8)
    if labels.ndim == 2:
        labels = labels[None]
    n, h, w = labels.shape
    if w > width or h > height:
        raise ValueError("label frames larger than the padded size")
    out = np.full((n, height, width), padding_label, np.uint8)
    out[:, :h, :w] = labels
    return out


def fill_depth(ctx, depth_mm):
    """RGBDImage::fillDepth on the device; returns a filled copy of uint16 [n][H][W]."""
    d = np.array(depth_mm, dtype=np.uint16, copy=True, order="C")
    if d.ndim == 2:
        d = d[None]
    n, h, w = d.shape
    _check(lib().cf_fill_depth(ctx.handle, n, w, h, _p(d), 0))
    return d


def rgb_to_cielab(ctx, rgb):
    """L*a*b* float32 [n][3][H][W] of uint8 [n][H][W][3], on the device."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    n, h, w, _ = rgb.shape
    out = np.empty((n, 3, h, w), np.float32)
    _check(lib().cf_rgb_to_cielab(ctx.handle, n, w, h, _p(rgb), _p(out), 0))
    return out


def pixel_accuracy(ctx, prediction_ptr, truth_ptr, count, width, height, num_classes, ignored=None, include_void=True,
                   confusion=None):
    """calculatePixelAccuracy over `count` label frames (DEVICE pointers); confusion (uint64 [C][C]) is
    accumulated when given. Returns the accuracy."""
    ign = None if ignored is None else np.ascontiguousarray(ignored, np.uint8)
    if confusion is not None and (confusion.dtype != np.uint64 or confusion.shape != (num_classes, num_classes)):
        raise ValueError("confusion must be uint64 [C][C]")
    acc = ctypes.c_double()
    _check(lib().cf_pixel_accuracy(ctx.handle, int(count), int(width), int(height), _vp(prediction_ptr),
                                   _vp(truth_ptr), int(num_classes), _p(ign), int(include_void), _p(confusion),
                                   ctypes.byref(acc), 1))
    return acc.value


def average_class_accuracy(confusion, ignored=None, include_void=True):
    """(ConfusionMatrix::averageClassAccuracy, normalised matrix) of a uint64 [C][C] confusion matrix."""
    confusion = np.ascontiguousarray(confusion, np.uint64)
    C = confusion.shape[0]
    ign = None if ignored is None else np.ascontiguousarray(ignored, np.uint8)
    norm = np.empty((C, C), np.float64)
    avg = ctypes.c_double()
    _check(lib().cf_confusion_average_class_accuracy(C, _p(confusion), _p(ign), int(include_void), _p(norm),
                                                     ctypes.byref(avg)))
    return avg.value, norm


def synthetic_frames(seed, num_images, width, height, num_cells, num_classes, void_class=-1, first=0):
    """Seeded Voronoi RGB-D scenes: (rgb uint8 [n][H][W][3], depth uint16 [n][H][W], labels uint8 [n][H][W]),
    frames first .. first + n - 1 of the seed's sequence."""
    rgb = np.empty((num_images, height, width, 3), np.uint8)
    depth = np.empty((num_images, height, width), np.uint16)
    labels = np.empty((num_images, height, width), np.uint8)
    _check(lib().cf_synthetic_frames_from(ctypes.c_uint64(seed), int(first), num_images, width, height, num_cells,
                                          num_classes, void_class, _p(rgb), _p(depth), _p(labels)))
    return rgb, depth, labels
