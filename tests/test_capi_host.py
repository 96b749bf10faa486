"""CPU-only checks of the C-ABI library: it loads, exports every declared entry point, reports
errors as status codes, and its host-only parts (tree import/export, JSON files, synthetic frames)
work without a GPU."""
import os
import re

import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from curfil_b200 import _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def built_library():
    _build.build()
    yield


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(cf_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = cf.lib()
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, "not exported: %s" % missing


def test_version_string():
    assert "sm_100a" in cf.version()


def test_errors_are_status_codes_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-device path")
    with pytest.raises(cf.CurfilError) as e:
        cf.Context(0)
    assert e.value.status in (1, 2)


def test_synthetic_frames_deterministic():
    a = cf.synthetic_frames(7, 3, 64, 48, 12, 8)
    b = cf.synthetic_frames(7, 3, 64, 48, 12, 8)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    rgb, depth, labels = a
    assert rgb.shape == (3, 48, 64, 3) and depth.shape == (3, 48, 64)
    assert labels.max() < 8
    holes = (depth == 0).mean()
    assert 0.05 < holes < 0.15
    assert depth[depth > 0].min() >= 500 and depth.max() <= 5000
    # frames are independent given (seed, index): a later slice of the sequence equals the tail
    tail = cf.synthetic_frames(7, 2, 64, 48, 12, 8, first=1)
    for x, y in zip(a, tail):
        np.testing.assert_array_equal(x[1:], y)


@pytest.mark.parametrize("args", [(7, 3, 64, 48, 12, 8, 0), (2026, 1, 640, 480, 40, 40, 0), (5, 2, 80, 60, 10, 6, 3)])
def test_oracle_generator_equals_library_generator(args):
    """The CPU baseline makes its frames with the oracle's restatement of the generator; they must be
    the library's frames byte for byte."""
    seed, n, w, h, cells, classes, first = args
    a = cf.synthetic_frames(seed, n, w, h, cells, classes, first=first)
    b = orc.synthetic_frames(seed, n, w, h, cells, classes, first=first)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def small_tree(C=3):
    # n0 -> (n1, n2); n1 -> (n3, n4)   (random_tree_image_gpu_test.cu:990-1130)
    left = np.array([1, 3, -1, -1, -1], np.int32)
    feature = np.zeros((5, 11), np.int8)
    feature[0] = [0, -18, 25, 9, 28, 4, 19, 1, 16, 0, 0]
    feature[1] = [1, -10, 5, 27, -19, 7, 3, 65, 73, 1, 2]
    threshold = np.array([-29.1245, 28.391, np.nan, np.nan, np.nan], np.float32)
    hist = np.array([[70, 60, 30], [10, 10, 10], [60, 60, 20], [10, 0, 20], [0, 50, 20]], np.uint32)
    score = np.array([0.9371, 0.392, np.nan, np.nan, np.nan])
    fid = np.array([2, 1, -1, -1, -1], np.int32)
    return cf.Tree.from_arrays(0, left, feature, threshold, hist, score=score, feature_id=fid)


def test_tree_import_export_roundtrip():
    t = small_tree()
    a = t.arrays()
    assert t.num_nodes == 5 and t.depth == 3
    np.testing.assert_array_equal(a["level"], [1, 2, 2, 3, 3])
    np.testing.assert_array_equal(a["left"], [1, 3, -1, -1, -1])
    assert a["threshold"][0] == np.float32(-29.1245)


def test_tree_json_roundtrip(tmp_path):
    t = small_tree()
    t.set_prior([100, 100, 100])
    cfg = cf.TrainConfig(feature_count=1000, thresholds=50, max_depth=15, box_radius=127, region_size=50)
    path = tmp_path / "tree0.json.gz"
    t.write_json(path, cfg)
    t2, cfg2, prior2 = cf.Tree.read_json(path)
    a, b = t.arrays(), t2.arrays()
    for k in ("level", "left", "feature", "feature_id", "histogram"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    np.testing.assert_array_equal(a["threshold"][a["left"] >= 0], b["threshold"][b["left"] >= 0])
    np.testing.assert_array_equal(a["score"][a["left"] >= 0], b["score"][b["left"] >= 0])
    np.testing.assert_array_equal(prior2, [100, 100, 100])
    assert (cfg2.feature_count, cfg2.thresholds, cfg2.max_depth, cfg2.box_radius, cfg2.region_size) == \
        (1000, 50, 15, 127, 50)
    # file is gzip JSON with string values, as boost::property_tree writes it
    import gzip
    import json
    doc = json.loads(gzip.open(path).read().decode())
    assert doc["tree"]["split"]["featureId"] == "2"
    assert doc["tree"]["left"]["split"]["feature"]["type"] == "color"
    assert doc["tree"]["split"]["feature"]["offset1"] == ["-18", "25"]
    assert "deviceId" in doc and doc["classLabelPriorDistribution"]["1"] == "100"


def test_tree_json_rejects_corrupt_files(tmp_path):
    p = tmp_path / "bad.json.gz"
    import gzip
    with gzip.open(p, "wb") as f:
        f.write(b'{"tree": {"id": "0"')
    with pytest.raises(cf.CurfilError) as e:
        cf.Tree.read_json(p)
    assert e.value.status == 8
    with pytest.raises(cf.CurfilError):
        cf.Tree.read_json(tmp_path / "missing.json.gz")


def test_tree_import_rejects_bad_child_index():
    left = np.array([5, -1, -1], np.int32)
    with pytest.raises(cf.CurfilError) as e:
        cf.Tree.from_arrays(0, left, np.zeros((3, 11), np.int8), np.zeros(3, np.float32),
                            np.ones((3, 2), np.uint32))
    assert e.value.status == 1


def test_tree_sampling_matches_oracle():
    """cf_sample_tree_pixels (product) vs the oracle restatement of class-uniform sampling."""
    from oracle import pyoracle as orc
    rgb, depth, labels = cf.synthetic_frames(4, 3, 64, 48, 10, 8)
    cfg = cf.TrainConfig(samples_per_image=300)
    seed = cf.forest_seed(4711)
    assert seed == int(orc.sampler_draws(4711, 0, 0xFFFE, 1)[0])
    ignore = np.zeros(8, np.uint8)
    ignore[0] = 1
    for t in range(2):
        s, prior, counter = cf.sample_tree_pixels(labels, depth, 8, cfg, 2, seed + t, ignored=ignore)
        rc, o, ocounter = orc.sample_class_uniform(labels, depth, 8, ignore, 150, seed + t)
        assert rc == len(s) and counter == ocounter
        for k in ("x", "y", "image", "label", "flip"):
            np.testing.assert_array_equal(s[k], o[k], err_msg=k)
        np.testing.assert_array_equal(s["depth"].view(np.uint32), o["depth"].view(np.uint32))
        np.testing.assert_array_equal(prior, np.bincount(labels.ravel(), minlength=8))
        assert (s["label"] != 0).all()


@pytest.mark.parametrize("kat", range(5))
def test_normalize_histogram_entry_point_kats(kat):
    """cf_normalize_histogram (host) against random_tree_test.cpp:46-154 and the oracle."""
    from oracle import pyoracle as orc
    from tests.golden import reference_kats as K
    hist, prior, bias, expected = K.NORMALIZE_KATS[kat]
    for use_prior in (True, False):
        got = cf.normalize_histogram(hist, prior, bias, use_prior)
        np.testing.assert_array_equal(got, orc.normalize_histogram(hist, prior, bias, use_prior))
    np.testing.assert_allclose(cf.normalize_histogram(hist, prior, bias, True), expected, rtol=1e-15, atol=1e-300)


def test_normalize_histogram_rejects_empty_prior():
    with pytest.raises(cf.CurfilError):
        cf.normalize_histogram([1, 2], [0, 0])


def test_reads_a_tree_file_laid_out_as_the_reference_writes_it(tmp_path):
    """A gzip JSON file with the reference's header keys (numCores, numPhysicalCPUs, processorModels,
    deviceId, ...) and node layout (export.cpp:180-290) holding the recall tree of
    random_tree_image_gpu_test.cu:990-1130 is read back exactly."""
    from tests.golden import reference_kats as K
    from tests.golden import reference_tree_file as R
    path = tmp_path / "tree0.json.gz"
    R.write(path)
    t, cfg, prior = cf.Tree.read_json(path)
    a = t.arrays()
    np.testing.assert_array_equal(a["left"], [1, 3, -1, -1, -1])
    np.testing.assert_array_equal(a["level"], [0, 1, 1, 2, 2])
    np.testing.assert_array_equal(a["feature"][0], K.RECALL_TREE["split2"]["feature"])
    np.testing.assert_array_equal(a["feature"][1], K.RECALL_TREE["split1"]["feature"])
    assert a["threshold"][0] == np.float32(K.RECALL_TREE["split2"]["threshold"])
    assert a["threshold"][1] == np.float32(K.RECALL_TREE["split1"]["threshold"])
    assert a["score"][0] == K.RECALL_TREE["split2"]["score"] and a["score"][1] == K.RECALL_TREE["split1"]["score"]
    np.testing.assert_array_equal(a["feature_id"][:2], [2, 1])
    for i in (1, 2, 3, 4):
        np.testing.assert_array_equal(a["histogram"][i], K.RECALL_TREE["hist"][i])
    np.testing.assert_array_equal(a["num_samples"], [170, 30, 140, 30, 70])
    np.testing.assert_array_equal(prior, K.RECALL_TREE["prior"])
    assert (cfg.random_seed, cfg.samples_per_image, cfg.feature_count, cfg.thresholds, cfg.max_depth) == \
        (4711, 100, 1000, 50, 15)
    assert (cfg.box_radius, cfg.region_size, cfg.min_sample_count, cfg.max_samples_per_batch) == (127, 50, 32, 100000)
    assert (cfg.num_threads, cfg.max_images, cfg.image_cache_size, cfg.acceleration_mode) == (1, 5, 5, 2)
    assert (cfg.use_cie_lab, cfg.use_depth_filling, cfg.use_depth_images, cfg.subsampling_type) == (1, 0, 1, 0)
    # written back by the library: the reference's header keys in the reference's order
    import gzip
    import json
    out = tmp_path / "again.json.gz"
    t.write_json(out, cfg, prior=prior)
    doc = json.loads(gzip.open(out).read().decode())
    assert list(doc.keys()) == R.HEADER_KEYS
    assert int(doc["numCores"]) >= 1 and int(doc["numPhysicalCPUs"]) >= 0
    assert isinstance(doc["processorModels"], list) and doc["deviceId"] == ["0"]
    t2, _, _ = cf.Tree.read_json(out)
    b = t2.arrays()
    for k in ("level", "left", "feature", "threshold", "feature_id", "histogram", "num_samples"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_pixel_uniform_sampling_matches_oracle():
    """cf_sample_tree_pixels with pixelUniform (host form) vs the oracle's restatement of
    random_tree_image.cpp:840-883 and the block sort."""
    rgb, depth, labels = cf.synthetic_frames(4, 3, 64, 48, 10, 8)
    cfg = cf.TrainConfig(samples_per_image=300, subsampling_type=1)
    seed = cf.forest_seed(4711)
    ignore = np.zeros(8, np.uint8)
    ignore[0] = 1
    s, prior, counter = cf.sample_tree_pixels(labels, depth, 8, cfg, 2, seed, ignored=ignore)
    rc, o, ocounter = orc.sample_pixel_uniform(labels, depth, ignore, 150, seed)
    assert rc == len(s) == 450 and counter == ocounter
    np.testing.assert_array_equal(s.view(np.uint8), o.view(np.uint8))
    assert (s["label"] != 0).all()
