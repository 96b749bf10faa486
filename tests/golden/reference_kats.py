"""Known-answer values transcribed from the reference's own unit tests.

Each constant cites the test file and line range of deeplearningais/curfil it comes from
(paths relative to the reference project root). They are values, not code: the tests in
this repository recompute them with the CPU oracle and with the CUDA path.
"""

# ---- split scores: src/tests/random_tree_image_gpu_test.cu:106-240 --------------------
# (left, right, all, expected NormalizedInformationGain, relative tolerance, expected IG)
SCORE_KATS = [
    ([5, 8], [3, 1], [8, 9], 0.080185, 1e-6, None),                                   # :160-175
    ([2, 8], [6, 1], [8, 9], 0.33339, 1e-5, None),                                    # :177-192
    ([56, 241, 290, 3, 18], [30, 0, 1, 0, 249], [86, 241, 291, 3, 267], 0.491311, 1e-5,
     0.690912),                                                                       # :194-217
    ([50, 100, 0, 0, 0], [0, 0, 50, 0, 100], [50, 100, 50, 0, 100], 0.68533, 1e-5, 1.0),  # :219-238
]
# :114-158: for num in 1..9, [num,num]/[num,num] scores exactly 0 and [0,2num]/[2num,0] exactly 1.
SCORE_RANGE = range(1, 10)

# ---- depth feature: src/tests/random_tree_image_gpu_test.cu:318-488 --------------------
DEPTH_FEATURE = dict(
    width=16, height=20,
    # type, o1x, o1y, o2x, o2y, r1x, r1y, r2x, r2y, ch1, ch2
    feature=[0, 1, 1, -3, -1, 2, 2, 1, 1, 0, 0],
    thresholds=[(i - 50) / 10.0 for i in range(100)],
    sample_xy=(6, 3), sample_depth_mm=1000, labels=[0, 1],
    # RGBDImage::setDepth(x, y, Depth(metres as float)) -> millimetres
    pixels_mm={(7, 3): 1500, (7, 4): 1700, (8, 4): 4500, (3, 2): 3900},
    expected_response=(1.5 + 1.7 + 4.5) / 3 - 3.9,
    first_left_threshold=37,        # counters(feat, thresh, label, 0) == (thresh >= 37)
    constant_depth_mm=1000,          # all pixels 1.0 m -> response 0
    constant_first_left_threshold=50,
)

# ---- colour feature, simple: src/tests/random_tree_image_gpu_test.cu:490-651 -----------
COLOR_FEATURE_SIMPLE = dict(
    width=16, height=20,
    feature=[1, 3, -2, -3, -2, 4, 2, 1, 2, 0, 0],
    thresholds=[-1.0, 0.0, 1.0],
    sample_xy=(6, 4), sample_depth_mm=1000, labels=[0, 1],
    # (image setup, expected response, expected left flags per threshold)
    cases=[
        ("zero", 0.0, [0, 1, 1]),
        ("pixel_7_2_half", 0.5, [0, 0, 1]),
        ("ones", 8 * 4 - 4 * 2.0, [0, 0, 0]),
    ],
)

# ---- colour feature, complex: src/tests/random_tree_image_gpu_test.cu:653-866 ----------
COLOR_FEATURE_COMPLEX = dict(
    width=12, height=15,
    # image 0: v = 100*c + y*W + x ; image 1: v / 2
    integral_bottom_right=[16110, 34110, 52110],
    features=[
        [1, 2, -1, -3, 4, 2, 1, 1, 2, 0, 2],
        [1, 2, -1, -3, 4, 2, 2, 1, 1, 1, 2],
        [1, -2, 1, 3, -4, 3, 1, 3, 3, 1, 0],
    ],
    thresholds=[[0.0, -300.0, 0.0], [-500.0, 0.0, 500.0]],   # [thresh][feat]
    # (image, label, depth mm, x, y)
    samples=[(0, 0, 1000, 6, 4), (1, 0, 2000, 6, 4), (0, 1, 1500, 5, 5), (1, 1, 3100, 3, 4)],
    # featureResponses(feat, sample); None = NaN
    responses=[[-2040, -444, -884, -424], [1186, -244, -484, -224], [None, 244, 572, 224]],
    # counters(feat, thresh, label, side)
    counters={
        (0, 0): [[2, 0], [2, 0]], (0, 1): [[1, 1], [1, 1]],
        (1, 0): [[0, 2], [1, 1]], (1, 1): [[1, 1], [2, 0]],
        (2, 0): [[0, 2], [0, 2]], (2, 1): [[1, 1], [1, 1]],
    },
)

# ---- integral images: src/tests/image_test.cpp:87-279 ----------------------------------
COLOR_INTEGRAL_3X3 = dict(
    pixels=[[5, 2, 3], [1, 5, 4], [2, 2, 1]],
    integral=[[5, 7, 10], [6, 13, 20], [8, 17, 25]],
)
COLOR_INTEGRAL_LARGE = dict(width=640, height=480, value=255, box=(10, 8))   # :135-162
DEPTH_INTEGRAL_3X2 = dict(
    # setDepth(x, y, Depth(metres)) in call order; the second write to (0,1) wins
    writes=[((0, 0), 5000), ((0, 1), 15000), ((0, 1), 10000), ((1, 0), 35000), ((2, 1), 10000)],
    integral_mm=[[5000, 40000, 40000], [15000, 50000, 60000]],
    valid=[[1, 2, 2], [2, 3, 4]],
)

# ---- histogram normalisation: src/tests/random_tree_test.cpp:46-154 --------------------
# (histogram, prior, bias, expected)
NORMALIZE_KATS = [
    ([850, 50, 100], [100, 100, 100], 0.0, [0.850 / 3.0, 0.050 / 3.0, 0.100 / 3.0]),
    ([50, 50, 50], [80, 10, 10], 0.0, [(1 / 3.0) * 0.8, (1 / 3.0) * 0.1, (1 / 3.0) * 0.1]),
    ([50, 50, 50], [80, 10, 10], 0.5, [0.0, 0.0, 0.0]),
    ([60, 20, 20], [50, 25, 25], 0.5, [0.5, 0.0, 0.0]),
    ([20, 40, 40], [20, 10, 10], 0.2, [0.0, 0.5 * 0.25, 0.5 * 0.25]),
]

# ---- tree packing: src/tests/random_tree_image_gpu_test.cu:990-1130 --------------------
# n0 splits with feature2 into (n1, n2); n1 splits with feature1 into (n3, n4).
RECALL_TREE = dict(
    num_classes=3,
    hist={1: [10, 10, 10], 2: [60, 60, 20], 3: [10, 0, 20], 4: [0, 50, 20]},
    split1=dict(feature_id=1, threshold=28.391, score=0.392,
                feature=[1, -10, 5, 27, -19, 7, 3, 65, 73, 1, 2]),
    split2=dict(feature_id=2, threshold=-29.1245, score=0.9371,
                feature=[0, -18, 25, 9, 28, 4, 19, 1, 16, 0, 0]),
    prior=[100, 100, 100],
)

# ---- Philox4x32-10 known answers (Random123 kat_vectors, Salmon et al. SC'11) -----------
# (key0, key1, c0, c1, c2, c3) -> out
PHILOX_KATS = [
    ((0, 0, 0, 0, 0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF),
     (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0xA4093822, 0x299F31D0, 0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]

# ---- depth filling (image_test.cpp:425-456, testDepthFilling) ------------------------------
# 200x100 image, every depth invalid except (x=20, y=30) = 1.5 m and (x=30, y=20) = 2.5 m; after
# RGBDImage::fillDepth every pixel is valid, 2.5 m for y < 30 and 1.5 m from y = 30 on.
DEPTH_FILL = dict(width=200, height=100, seeds={(20, 30): 1500, (30, 20): 2500}, split_row=30, above=2500,
                  below=1500)
