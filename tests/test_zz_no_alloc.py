"""The allocation-free split search against the allocating one.

cf_evaluate_best_splits_noalloc is for callers that cannot let the library allocate device memory
(a host owning all GPU memory through its own pool, or a loop where cudaMalloc/cudaFree would stall
other streams). Here the caller's buffers are torch tensors; the call must reproduce
cf_evaluate_best_splits on two calls in a row (its scratch array is reused between calls).
This file is collected last so a failure here leaves every other test already run.
"""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H

pytestmark = pytest.mark.gpu


def test_noalloc_split_search_matches_allocating_entry_point():
    import torch
    from curfil_b200 import _build
    _build.build()
    ctx = cf.Context(0)
    rgb, depth, _ = H.frames(seed=31, n=3, w=96, h=72, cells=12, classes=40)
    ods = orc.integral(rgb, depth)
    depth_pairs = np.ascontiguousarray(np.stack([ods.depth_sum.astype(np.int64).astype(np.int32),
                                                 ods.depth_valid], axis=-1))          # [n][H][W][2]
    depth_planes = np.ascontiguousarray(np.moveaxis(depth_pairs, -1, 1))               # [n][2][H][W]
    ds = cf.Dataset.from_integral(ctx, ods.color, depth_planes)

    rng = np.random.default_rng(8)
    sizes = [2500, 1, 3, 40, 700, 9]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    s = H.random_samples(rng, 3, 96, 72, 40, int(offsets[-1]), depth=depth)
    for i in range(len(sizes)):
        s["label"][offsets[i]:offsets[i + 1]] = rng.integers(0, 3 + 6 * i, sizes[i]) % 40
    feats, thr = orc.generate_features(ods, s, 4242, 256, 16, 60, 15)
    hist = np.zeros((len(sizes), 40), np.uint32)
    for i in range(len(sizes)):
        hist[i] = np.bincount(s["label"][offsets[i]:offsets[i + 1]], minlength=40)

    expected = cf.evaluate_best_splits(ds, offsets, s, 40, feats, thr)

    dev = torch.device("cuda", 0)
    t_color = torch.from_numpy(ods.color).to(dev)
    t_depth = torch.from_numpy(depth_pairs).to(dev)
    t_samples = torch.from_numpy(s.view(np.uint8)).to(dev)
    t_hist = torch.from_numpy(hist.view(np.int32)).to(dev)
    t_feats = torch.from_numpy(feats).to(dev)
    t_thr = torch.from_numpy(thr).to(dev)
    t_best = torch.zeros(len(sizes) * cf.SPLIT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    for call in range(2):
        t_best.zero_()
        torch.cuda.synchronize()
        cf.evaluate_best_splits_noalloc(ctx, t_color.data_ptr(), t_depth.data_ptr(), 3, 96, 72, offsets,
                                        t_samples.data_ptr(), t_hist.data_ptr(), 40, 256, 16, t_feats.data_ptr(),
                                        t_thr.data_ptr(), t_best.data_ptr())
        got = t_best.cpu().numpy().view(cf.SPLIT_DTYPE)
        np.testing.assert_array_equal(got["feature"], expected["feature"], err_msg="call %d" % call)
        np.testing.assert_array_equal(got["threshold_index"], expected["threshold_index"], err_msg="call %d" % call)
        np.testing.assert_allclose(got["score"], expected["score"], rtol=1e-12, atol=1e-15)
        np.testing.assert_array_equal(got["threshold"], expected["threshold"])
    assert (expected["score"] > 0).sum() >= 4

    # sizes beyond the fixed scratch are refused with a clear error
    with pytest.raises(cf.CurfilError) as e:
        cf.evaluate_best_splits_noalloc(ctx, t_color.data_ptr(), t_depth.data_ptr(), 3, 96, 72, offsets,
                                        t_samples.data_ptr(), t_hist.data_ptr(), 40, 20000, 16, t_feats.data_ptr(),
                                        t_thr.data_ptr(), t_best.data_ptr())
    assert e.value.status == 1 and "fixed scratch" in str(e.value)
    ds.close()
    ctx.close()
