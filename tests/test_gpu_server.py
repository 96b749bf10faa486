"""Serving: continuous batching of mixed-size frames; every result is the same alone and in the mix."""
import numpy as np
import pytest

import curfil_b200 as cf
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def forest():
    from curfil_b200 import _build
    _build.build()
    ctx = cf.Context(0)
    rgb, depth, labels = H.frames(seed=12, n=3, w=96, h=72, cells=12, classes=10)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    trees = []
    for t in range(3):
        samples, _ = H.class_uniform_samples(labels, depth, 10, 40, seed_counter=300 + 7 * t)
        cfg = cf.TrainConfig(feature_count=100, thresholds=10, max_depth=9, min_sample_count=4, box_radius=40,
                             region_size=10)
        tree, _ = cf.train_tree(ds, samples, 10, cfg, tree_id=t, seed_counter=11 * t + 1)
        tree.set_prior(np.bincount(labels.ravel(), minlength=10))
        trees.append(tree)
    f = cf.Forest(ctx, trees)
    yield f
    f.close()
    ctx.close()


SIZES = [(160, 120), (320, 240), (640, 480), (1280, 960)]


def test_alone_and_in_mix_identical(forest):
    server = cf.Server(forest, hbm_budget_bytes=2 << 30, max_batch_frames=8, pipeline_depth=2,
                       return_probabilities=True)
    frames = {}
    for k, (w, h) in enumerate(SIZES):
        rgb, depth, _ = cf.synthetic_frames(500 + k, 1, w, h, 12, 10)
        frames[(w, h)] = (rgb[0], depth[0])
    # alone
    alone = {}
    for key, (rgb, depth) in frames.items():
        rid = server.submit(rgb, depth)
        alone[key] = server.wait(rid, depth.shape, probabilities=True)
    # mixed burst: 1:2:4:1 of the four sizes, submitted back to back
    order = [SIZES[0]] + [SIZES[1]] * 2 + [SIZES[2]] * 4 + [SIZES[3]]
    rng = np.random.default_rng(3)
    rng.shuffle(order)
    ids = [(key, server.submit(*frames[key])) for key in order for _ in range(2)]
    mixed_batches = set()
    for key, rid in ids:
        labels, probs, st = server.wait(rid, frames[key][1].shape, probabilities=True)
        np.testing.assert_array_equal(labels, alone[key][0])
        np.testing.assert_array_equal(probs, alone[key][1])
        if st.batch_frames > 1:
            mixed_batches.add(st.batch_id)
        assert st.done_ms >= st.admitted_ms >= st.submit_ms
    c = server.counters()
    assert c["completed"] == c["submitted"] == len(ids) + len(SIZES)
    assert mixed_batches, "no batch held more than one frame"
    assert c["batches"] < c["submitted"]
    # and the same as the direct prediction path
    for key, (rgb, depth) in frames.items():
        probs, labels = forest.predict(rgb, depth)
        np.testing.assert_array_equal(labels[0], alone[key][0])
        np.testing.assert_array_equal(probs[0], alone[key][1])
    server.close()


def test_admission_rejects_oversized_and_unknown(forest):
    server = cf.Server(forest, hbm_budget_bytes=8 << 20, max_batch_frames=4, pipeline_depth=2)
    rgb, depth, _ = cf.synthetic_frames(1, 1, 1280, 960, 12, 10)
    with pytest.raises(cf.CurfilError) as e:
        server.submit(rgb[0], depth[0])
    assert e.value.status == 7
    small_rgb, small_depth, _ = cf.synthetic_frames(2, 1, 160, 120, 12, 10)
    rid = server.submit(small_rgb[0], small_depth[0])
    labels, _, _ = server.wait(rid, (120, 160))
    assert labels.shape == (120, 160)
    with pytest.raises(cf.CurfilError):
        server.wait(123456789, (1, 1), timeout_s=0.01)
    assert server.counters()["rejected"] == 1
    server.close()


def _burst(forest, policy, max_wait_ms):
    server = cf.Server(forest, hbm_budget_bytes=2 << 30, max_batch_frames=1, pipeline_depth=1, policy=policy,
                       max_wait_ms=max_wait_ms)
    frames = {}
    for k, (w, h) in enumerate(SIZES):
        rgb, depth, _ = cf.synthetic_frames(700 + k, 1, w, h, 12, 10)
        frames[(w, h)] = (rgb[0], depth[0])
    order = [SIZES[3], SIZES[2], SIZES[1], SIZES[0]] * 4
    ids = [(key, server.submit(*frames[key])) for key in order]
    got = []
    for key, rid in ids:
        labels, _, st = server.wait(rid, frames[key][1].shape)
        _, alone = forest.predict(*frames[key], probabilities=False)
        np.testing.assert_array_equal(labels, alone[0])
        got.append((st.batch_id, key[0] * key[1], rid))
    server.close()
    return sorted(got)


def _mean_rank(got, px):
    return np.mean([i for i, (_, p, _) in enumerate(got) if p == px])


def test_smallest_first_policy_orders_queued_frames_by_size(forest):
    # submitted largest first in every group of four: in arrival order the 1280x960 frames run earlier
    # on average than the 160x120 ones; smallest first reverses that (requests that arrive while
    # earlier ones run make the exact order depend on timing, the averages do not)
    fifo = _burst(forest, 0, 0.0)
    assert _mean_rank(fifo, 1280 * 960) < _mean_rank(fifo, 160 * 120)
    assert [rid for _, _, rid in fifo] == sorted(rid for _, _, rid in fifo)
    sjf = _burst(forest, 1, 1e6)
    assert _mean_rank(sjf, 160 * 120) < _mean_rank(sjf, 1280 * 960)
    # every request overdue at once: arrival order again
    aged = _burst(forest, 1, 1e-3)
    assert [rid for _, _, rid in aged] == sorted(rid for _, _, rid in aged)
    with pytest.raises(cf.CurfilError):
        cf.Server(forest, policy=1, max_wait_ms=0.0)
    with pytest.raises(cf.CurfilError):
        cf.Server(forest, policy=2, max_wait_ms=1.0)


def test_device_priority_streams_same_results(forest):
    # four slots, batches of one or two frames on streams of different CUDA priority, results published
    # per slot as each completes: every request still gets exactly its frame's direct prediction
    server = cf.Server(forest, hbm_budget_bytes=2 << 30, max_batch_frames=2, pipeline_depth=4,
                       return_probabilities=True, policy=1, max_wait_ms=50.0, device_priority=1)
    frames = {}
    for k, (w, h) in enumerate(SIZES):
        rgb, depth, _ = cf.synthetic_frames(900 + k, 1, w, h, 12, 10)
        frames[(w, h)] = (rgb[0], depth[0])
    direct = {key: forest.predict(*f) for key, f in frames.items()}
    order = [SIZES[3], SIZES[0], SIZES[2], SIZES[1], SIZES[0], SIZES[2], SIZES[3], SIZES[1]] * 3
    ids = [(key, server.submit(*frames[key])) for key in order]
    for key, rid in ids:
        labels, probs, st = server.wait(rid, frames[key][1].shape, probabilities=True)
        np.testing.assert_array_equal(labels, direct[key][1][0])
        np.testing.assert_array_equal(probs, direct[key][0][0])
        assert st.submit_ms <= st.admitted_ms <= st.done_ms
    c = server.counters()
    assert c["completed"] == c["submitted"] == len(order)
    server.close()
    with pytest.raises(cf.CurfilError):
        cf.Server(forest, device_priority=2)


def test_overload_sheds_requests_that_wait_too_long(forest):
    """With max_queue_ms a request still queued that long after its submission is refused
    (CF_ERR_REJECTED) instead of served late; every served frame is still the frame served alone,
    and no served frame waited in the queue longer than the limit."""
    rgb, depth, _ = cf.synthetic_frames(600, 1, 1280, 960, 12, 10)
    alone = cf.Server(forest, hbm_budget_bytes=1 << 30, max_batch_frames=1, pipeline_depth=1)
    ref = alone.wait(alone.submit(rgb[0], depth[0]), depth[0].shape)[0]
    alone.close()
    server = cf.Server(forest, hbm_budget_bytes=1 << 30, max_batch_frames=1, pipeline_depth=1, max_queue_ms=1.0)
    ids = [server.submit(rgb[0], depth[0]) for _ in range(40)]   # a burst far beyond one slot's pace
    served, refused = 0, 0
    for rid in ids:
        try:
            labels, _, st = server.wait(rid, depth[0].shape)
        except cf.CurfilError as e:
            assert e.status == 7 and "max_queue_ms" in str(e)
            refused += 1
            continue
        served += 1
        np.testing.assert_array_equal(labels, ref)
        assert st.admitted_ms - st.submit_ms <= 1.0 + 0.5   # the limit, plus the launcher's own latency
    c = server.counters()
    assert served >= 1 and refused >= 1 and served + refused == 40
    assert c["rejected"] == refused and c["completed"] == served
    server.close()
    with pytest.raises(cf.CurfilError):
        cf.Server(forest, max_queue_ms=-1.0)
