"""A tree file laid out key for key as the reference writes one.

RandomTreeExport::writeTree (src/curfil/export.cpp:180-290) puts the header keys below, in this
order, into a boost::property_tree and writes it with write_json (export.cpp:292-313), which makes
every value a string, every XY pair a two-element array, and keys containing dots nested objects
(classLabelPriorDistribution.N, histogram entries "R,G,B (label)", split.*). The node fields follow
writeTree(pt, RandomTree) (export.cpp:233-290); children are "left" and "right". The device list is
written as "deviceId" (export.cpp:202), although the reader looks for "deviceIds" (import.cpp:244).

The tree is the two-split recall tree of src/tests/random_tree_image_gpu_test.cu:990-1130 with the
training configuration of that test (1000 features, 50 thresholds, depth 15, box radius 127,
region size 50, GPU_AND_CPU_COMPARE) and a prior of 100 per class.
"""
import gzip
import json

from tests.golden import reference_kats as K

COLORS = ["0,0,0", "128,0,0", "0,128,0"]


def _hist(h):
    return {"%s (%d)" % (COLORS[i], i): str(v) for i, v in enumerate(h)}


def _xy(x, y):
    return [str(x), str(y)]


def _feature(row):
    """writeFeatureDetails (export.cpp:68-86) of an int8 [11] feature row."""
    t, o1x, o1y, o2x, o2y, r1x, r1y, r2x, r2y, c1, c2 = row
    d = {"type": "color" if t == 1 else "depth"}
    if t == 1:
        d["channel1"] = str(c1)
        d["channel2"] = str(c2)
    d["offset1"] = _xy(o1x, o1y)
    d["region1"] = _xy(r1x, r1y)
    d["offset2"] = _xy(o2x, o2y)
    d["region2"] = _xy(r2x, r2y)
    return d


def _node(node_id, level, hist, split=None, left=None, right=None):
    d = {"id": str(node_id), "level": str(level), "samples": str(sum(hist)), "leaf": "false" if split else "true",
         "histogram": _hist(hist)}
    if split:
        d["split"] = {"threshold": repr(split["threshold"]), "score": repr(split["score"]),
                      "featureId": str(split["feature_id"]), "feature": _feature(split["feature"])}
        d["left"] = left
        d["right"] = right
    return d


def recall_tree_document():
    h = K.RECALL_TREE["hist"]
    root_hist = [a + b for a, b in zip(h[1], h[2])]
    n1 = _node(1, 1, h[1], K.RECALL_TREE["split1"], _node(3, 2, h[3]), _node(4, 2, h[4]))
    tree = _node(0, 0, root_hist, K.RECALL_TREE["split2"], n1, _node(2, 1, h[2]))
    doc = {
        "hostname": "trainer01",
        "buildType": "RELEASE",
        "version": "0.0.1",
        "date": "2013-Apr-20 13:44:08",
        "randomSeed": "4711",
        "folderTraining": "/data/training",
        "numCores": "16",
        "numPhysicalCPUs": "2",
        "processorModels": ["Intel(R) Xeon(R) CPU E5-2650 0 @ 2.00GHz"],
        "accelerationMode": "compare",
        "deviceId": ["0"],
        "samplesPerImage": "100",
        "featureCount": "1000",
        "thresholds": "50",
        "boxRadius": "127",
        "regionSize": "50",
        "maxDepth": "15",
        "numThreads": "1",
        "minSampleCount": "32",
        "maxSamplesPerBatch": "100000",
        "maxImages": "5",
        "imageCacheSize": "5",
        "subsamplingType": "classUniform",
        "useCIELab": "true",
        "useDepthFilling": "false",
        "useDepthImages": "true",
        "ignoredColors": ["0,0,0"],
        "classLabelPriorDistribution": {str(i): str(v) for i, v in enumerate(K.RECALL_TREE["prior"])},
        "tree": tree,
    }
    return doc


HEADER_KEYS = ["hostname", "buildType", "version", "date", "randomSeed", "folderTraining", "numCores",
               "numPhysicalCPUs", "processorModels", "accelerationMode", "deviceId", "samplesPerImage",
               "featureCount", "thresholds", "boxRadius", "regionSize", "maxDepth", "numThreads", "minSampleCount",
               "maxSamplesPerBatch", "maxImages", "imageCacheSize", "subsamplingType", "useCIELab", "useDepthFilling",
               "useDepthImages", "ignoredColors", "classLabelPriorDistribution", "tree"]


def write(path):
    with gzip.open(path, "wb") as f:
        f.write(json.dumps(recall_tree_document(), indent=4).encode())
