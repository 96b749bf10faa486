"""The multi-process path on CPU: two gloo ranks train disjoint trees (stand-ins built on the host) and
assemble the forest; it equals the single-process forest, tree by tree."""
import os
import socket

import numpy as np
import pytest

import curfil_b200 as cf
from curfil_b200 import distributed as D


def fake_tree(tree_id, C=4):
    """A deterministic small tree per id (the host-side stand-in for a trained tree)."""
    rng = np.random.default_rng(1000 + tree_id)
    left = np.array([1, 3, -1, -1, -1], np.int32)
    feature = rng.integers(-20, 20, (5, 11)).astype(np.int8)
    threshold = rng.standard_normal(5).astype(np.float32)
    threshold[2:] = np.nan
    hist = rng.integers(0, 50, (5, C)).astype(np.uint32)
    score = rng.random(5)
    fid = rng.integers(0, 100, 5).astype(np.int32)
    t = cf.Tree.from_arrays(tree_id, left, feature, threshold, hist, score=score, feature_id=fid)
    t.set_prior(rng.integers(1, 1000, C).astype(np.uint32))
    return t


def _same(a, b):
    assert a.tree_id == b.tree_id
    A, B = a.arrays(), b.arrays()
    for k in A:
        np.testing.assert_array_equal(A[k], B[k], err_msg=k)
    np.testing.assert_array_equal(a.prior(), b.prior())


def _worker(rank, world, port, num_trees, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ids = D.tree_ids_for_rank(rank, world, num_trees)
        forest = D.gather_forest([fake_tree(t) for t in ids])
        with open(os.path.join(out_dir, "rank%d.bin" % rank), "wb") as f:
            for t in forest:
                b = D.tree_to_bytes(t)
                f.write(len(b).to_bytes(8, "little") + b)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _read(path):
    trees = []
    with open(path, "rb") as f:
        while True:
            n = f.read(8)
            if not n:
                return trees
            trees.append(D.tree_from_bytes(f.read(int.from_bytes(n, "little"))))


def test_tree_ids_shard_like_the_reference():
    assert D.tree_ids_for_rank(0, 2, 5) == [0, 2, 4]
    assert D.tree_ids_for_rank(1, 2, 5) == [1, 3]
    all_ids = sorted(i for r in range(3) for i in D.tree_ids_for_rank(r, 3, 10))
    assert all_ids == list(range(10))
    with pytest.raises(ValueError):
        D.tree_ids_for_rank(2, 2, 4)


def test_tree_bytes_roundtrip():
    t = fake_tree(7)
    _same(t, D.tree_from_bytes(D.tree_to_bytes(t)))


def test_two_gloo_ranks_assemble_the_single_process_forest(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    num_trees = 5
    mp.start_processes(_worker, args=(2, port, num_trees, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    single = [fake_tree(t) for t in range(num_trees)]
    for rank in range(2):
        got = _read(os.path.join(str(tmp_path), "rank%d.bin" % rank))
        assert [t.tree_id for t in got] == list(range(num_trees))
        for a, b in zip(got, single):
            _same(a, b)


def _allgather_worker(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        fn = D.allgather_bytes()
        # two rounds, as two levels of a sharded training exchange their candidate lists
        outs = [fn(bytes([rank + 1 + 10 * k]) * (88 * 3)) for k in range(2)]
        with open(os.path.join(out_dir, "ag%d.bin" % rank), "wb") as f:
            f.write(b"".join(outs))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_allgather_bytes_over_two_gloo_ranks(tmp_path):
    """The all-gather train_tree_sharded calls once per level: every rank receives every rank's
    payload, in rank order."""
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_allgather_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    want = b"".join(bytes([r + 1 + 10 * k]) * (88 * 3) for k in range(2) for r in range(2))
    for rank in range(2):
        with open(os.path.join(str(tmp_path), "ag%d.bin" % rank), "rb") as f:
            assert f.read() == want
