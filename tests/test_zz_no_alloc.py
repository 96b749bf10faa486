"""The allocation-free split search against the allocating one and the oracle.

cf_evaluate_best_splits_noalloc is for callers that cannot let the library allocate device memory
(a host owning all GPU memory through its own pool, or a loop where cudaMalloc/cudaFree would stall
other streams). Here the caller's buffers are torch tensors; the call must reproduce
cf_evaluate_best_splits on two calls in a row (its scratch array is reused between calls), and
refuse inputs it cannot index safely. This file is collected last so a failure here leaves every
other test already run.
"""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H

pytestmark = pytest.mark.gpu

W, HT, N_IMG, C = 96, 72, 3, 40


class Level:
    """One level's inputs as device tensors the caller owns, plus host copies."""

    def __init__(self, ctx, ods, depth_pairs, offsets, s, feats, thr):
        import torch
        dev = torch.device("cuda", 0)
        M = len(offsets) - 1
        self.offsets, self.s, self.feats, self.thr = offsets, s, feats, thr
        self.hist = np.zeros((M, C), np.uint32)
        for i in range(M):
            self.hist[i] = np.bincount(s["label"][offsets[i]:offsets[i + 1]], minlength=C)
        self.t_color = torch.from_numpy(ods.color).to(dev)
        self.t_depth = torch.from_numpy(depth_pairs).to(dev)
        self.t_samples = torch.from_numpy(s.view(np.uint8)).to(dev)
        self.t_hist = torch.from_numpy(self.hist.view(np.int32)).to(dev)
        self.t_feats = torch.from_numpy(feats).to(dev)
        self.t_thr = torch.from_numpy(thr).to(dev)
        self.t_best = torch.zeros(M * cf.SPLIT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize()

    def call(self, ctx, num_features=None, hist=None, samples=None, thr=None):
        T, F = self.thr.shape
        cf.evaluate_best_splits_noalloc(
            ctx, self.t_color.data_ptr(), self.t_depth.data_ptr(), N_IMG, W, HT, self.offsets,
            (samples if samples is not None else self.t_samples).data_ptr(),
            (hist if hist is not None else self.t_hist).data_ptr(), C, num_features or F, T,
            self.t_feats.data_ptr(), (thr if thr is not None else self.t_thr).data_ptr(), self.t_best.data_ptr())
        return self.t_best.cpu().numpy().view(cf.SPLIT_DTYPE).copy()


@pytest.fixture(scope="module")
def setup():
    from curfil_b200 import _build
    _build.build()
    ctx = cf.Context(0)
    rgb, depth, _ = H.frames(seed=31, n=N_IMG, w=W, h=HT, cells=12, classes=C)
    ods = orc.integral(rgb, depth)
    depth_pairs = np.ascontiguousarray(np.stack([ods.depth_sum.astype(np.int64).astype(np.int32),
                                                 ods.depth_valid], axis=-1))          # [n][H][W][2]
    depth_planes = np.ascontiguousarray(np.moveaxis(depth_pairs, -1, 1))               # [n][2][H][W]
    ds = cf.Dataset.from_integral(ctx, ods.color, depth_planes)
    yield ctx, ods, depth, depth_pairs, ds
    ds.close()
    ctx.close()


def make_level(rng, depth, sizes, label_spread=True):
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, N_IMG, W, HT, C, int(offsets[-1]), depth=depth)
    if label_spread:
        for i in range(len(sizes)):
            s["label"][offsets[i]:offsets[i + 1]] = rng.integers(0, 3 + 6 * i, sizes[i]) % C
    return offsets, s


def assert_same(got, expected, what):
    np.testing.assert_array_equal(got["feature"], expected["feature"], err_msg=what)
    np.testing.assert_array_equal(got["threshold_index"], expected["threshold_index"], err_msg=what)
    np.testing.assert_allclose(got["score"], expected["score"], rtol=1e-12, atol=1e-15, err_msg=what)
    np.testing.assert_array_equal(got["threshold"], expected["threshold"], err_msg=what)


def test_noalloc_split_search_matches_allocating_entry_point_and_oracle(setup):
    ctx, ods, depth, depth_pairs, ds = setup
    rng = np.random.default_rng(8)
    # one node of 20 000 samples: the allocating entry point cuts its items into sample chunks, the
    # allocation-free one never does
    sizes = [20000, 2500, 1, 3, 40, 700, 9]
    offsets, s = make_level(rng, depth, sizes)
    feats, thr = orc.generate_features(ods, s, 4242, 256, 16, 60, 15)
    expected = cf.evaluate_best_splits(ds, offsets, s, C, feats, thr)
    lv = Level(ctx, ods, depth_pairs, offsets, s, feats, thr)
    for call in range(2):
        assert_same(lv.call(ctx), expected, "call %d" % call)
    assert (expected["score"] > 0).sum() >= 5
    # the oracle's split search (FeatureEvaluationCPU + calculateScores + argmax) on every node
    got = lv.call(ctx)
    for i in range(len(sizes)):
        sl = s[offsets[i]:offsets[i + 1]].view(orc.SAMPLE_DTYPE)
        sc = orc.scores(orc.histograms(ods, sl, feats, thr, C, threads=8), lv.hist[i])
        bf, bt, bs = orc.best_split(sc)
        mine = sc[got["threshold_index"][i], got["feature"][i]]
        if (got["feature"][i], got["threshold_index"][i]) != (bf, bt):
            # a different choice is accepted only where the two scores tie within 1e-6 relative
            assert abs(mine - bs) <= 1e-6 * abs(bs), i
        assert got["score"][i] == pytest.approx(mine, rel=1e-12, abs=1e-15)


def test_noalloc_many_work_items_halves_items_per_slot(setup):
    """A level that would need more than the scratch's 65 536 work items at the context's tuning is
    planned with fewer, larger items; the splits are those of the allocating entry point."""
    ctx, ods, depth, depth_pairs, ds = setup
    rng = np.random.default_rng(9)
    sizes = [30 + (i % 7) for i in range(40)]
    offsets, s = make_level(rng, depth, sizes)
    feats, thr = orc.generate_features(ods, s, 777, 16384, 2, 60, 15)
    old = ctx.get_tuning()
    try:
        # 40 nodes x ~2100 items of 4 features (84 000 items), more than the scratch's 65 536
        ctx.set_tuning(items_per_slot=1024.0, min_item_evals=256)
        expected = cf.evaluate_best_splits(ds, offsets, s, C, feats, thr)
        lv = Level(ctx, ods, depth_pairs, offsets, s, feats, thr)
        for call in range(2):
            assert_same(lv.call(ctx), expected, "call %d" % call)
    finally:
        ctx.set_tuning(old)


def test_noalloc_refuses_what_it_cannot_index(setup):
    import torch
    ctx, ods, depth, depth_pairs, ds = setup
    rng = np.random.default_rng(10)
    offsets, s = make_level(rng, depth, [300, 200, 50])
    feats, thr = orc.generate_features(ods, s, 99, 64, 8, 60, 15)
    lv = Level(ctx, ods, depth_pairs, offsets, s, feats, thr)
    good = lv.call(ctx)
    dev = torch.device("cuda", 0)

    def refused(match, **kw):
        with pytest.raises(cf.CurfilError) as e:
            lv.call(ctx, **kw)
        assert e.value.status == 1 and match in str(e.value), str(e.value)

    # sizes beyond the fixed scratch
    refused("fixed scratch", num_features=20000)
    # a histogram that does not count a label present in its node (no histogram row for that class)
    h = lv.hist.copy()
    lab = int(s["label"][offsets[1]])
    h[1, lab] = 0
    refused("not counted in its node's histogram", hist=torch.from_numpy(h.view(np.int32)).to(dev))
    # a node histogram of the wrong node: node 2's labels span fewer classes than node 0's
    h = lv.hist.copy()
    h[0] = 0
    h[0, 0] = 1
    refused("not counted in its node's histogram", hist=torch.from_numpy(h.view(np.int32)).to(dev))
    # image index and pixel out of range, unknown flip setting
    for field, value, match in (("image", N_IMG, "image index"), ("x", W, "pixel outside"),
                                ("y", HT + 3, "pixel outside"), ("flip", 3, "flip setting"),
                                ("label", C, "label >= num_classes")):
        bad = s.copy()
        bad[field][offsets[2] + 7] = value
        refused(match, samples=torch.from_numpy(bad.view(np.uint8)).to(dev))
    t = thr.copy()
    t[3, 5] = np.nan
    refused("NaN threshold", thr=torch.from_numpy(t).to(dev))
    # a refused call leaves the entry point usable: the next good call gives the same splits
    assert_same(lv.call(ctx), good, "after refusals")
