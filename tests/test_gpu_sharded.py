"""One tree trained by several processes together (cf_train_tree_sharded) equals the tree one process
trains. Ranks are emulated on one GPU by threads, each with its own context and dataset copy, and
exchange through an in-process all-gather. Their kernels never wait on one another: only the host
threads meet, once per level, at the exchange."""
import threading

import numpy as np
import pytest

import curfil_b200 as cf
from tests import helpers as H

pytestmark = pytest.mark.gpu


class LocalGroup:
    """An all-gather among `world` threads of this process (host barrier with a timeout)."""

    def __init__(self, world):
        self.world = world
        self.slots = [None] * world
        self.barrier = threading.Barrier(world, timeout=120)
        self.calls = [0] * world

    def fn(self, rank):
        def allgather(payload):
            self.calls[rank] += 1
            self.slots[rank] = payload
            self.barrier.wait()
            out = b"".join(self.slots)
            self.barrier.wait()
            return out
        return allgather


@pytest.fixture(scope="module")
def scene():
    from curfil_b200 import _build
    _build.build()
    rgb, depth, labels = H.frames(seed=12, n=4, w=96, h=72, cells=12, classes=20)
    samples, _ = H.class_uniform_samples(labels, depth, 20, 120, seed_counter=50)
    return rgb, depth, samples


def _config():
    return cf.TrainConfig(feature_count=200, thresholds=12, max_depth=9, min_sample_count=4, box_radius=40,
                          region_size=10)


def _train_group(rgb, depth, samples, world):
    group = LocalGroup(world)
    results = [None] * world
    errors = []

    def run(rank):
        try:
            ctx = cf.Context(0)
            ds = cf.Dataset.from_raw(ctx, rgb, depth)
            tree, counter = cf.train_tree_sharded(ds, samples, 20, _config(), rank, world, group.fn(rank),
                                                  tree_id=3, seed_counter=77)
            results[rank] = (tree.arrays(), counter, tree.train_stats()[0])
            tree.close()
            ds.close()
            ctx.close()
        except Exception as e:  # surfaced below
            errors.append(e)
            group.barrier.abort()

    threads = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    return results, group


@pytest.mark.parametrize("world", [1, 2, 3])
def test_sharded_tree_equals_single_process_tree(scene, world):
    rgb, depth, samples = scene
    ctx = cf.Context(0)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    ref, ref_counter = cf.train_tree(ds, samples, 20, _config(), tree_id=3, seed_counter=77)
    ref_arrays, ref_evals = ref.arrays(), ref.train_stats()[0]
    results, group = _train_group(rgb, depth, samples, world)
    for rank, (arrays, counter, evals) in enumerate(results):
        assert counter == ref_counter
        for k in ref_arrays:
            np.testing.assert_array_equal(arrays[k], ref_arrays[k], err_msg="rank %d %s" % (rank, k))
    # each rank evaluated its share; together the whole level
    assert sum(r[2] for r in results) == ref_evals
    if world > 1:
        assert len(ref_arrays["left"]) > 15
        assert group.calls[0] == ref.train_stats()[2] and len(set(group.calls)) == 1
    ref.close()
    ds.close()
    ctx.close()


def test_sharded_training_reports_a_failed_exchange(scene):
    rgb, depth, samples = scene
    ctx = cf.Context(0)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)

    def broken(payload):
        raise RuntimeError("peer lost")

    with pytest.raises(RuntimeError, match="peer lost"):
        cf.train_tree_sharded(ds, samples, 20, _config(), 0, 2, broken)
    with pytest.raises(cf.CurfilError):
        cf.train_tree_sharded(ds, samples, 20, _config(), 2, 2, broken)
    # the dataset's trainer is usable afterwards, unsharded
    tree, _ = cf.train_tree(ds, samples, 20, _config(), tree_id=3, seed_counter=77)
    assert tree.num_nodes > 1
    ds.close()
    ctx.close()
