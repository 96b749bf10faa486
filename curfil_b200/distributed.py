"""Forest training over several processes (one per GPU).

Trees are independent: the reference spreads them over devices by `treeId % devices`
(random_tree_image_gpu.cu:1727), every tree drawing its samples and features from its own random
source (seed SEED + treeId, random_forest_image.cpp:150-173). So ranks train disjoint trees with no
collective on the data path, and a forest trained on N ranks is the forest trained on one. The only
exchange is assembling the forest afterwards: every rank serialises its trees (a few hundred KB each)
and `gather_forest` all-gathers them, ordered by tree id.

When one tree must span several GPUs, `train_tree_sharded` (with `allgather_bytes`) splits each
level's work items over the ranks and exchanges their candidate lists once per level; the tree is the
one a single process trains.
"""
import io

import numpy as np

from . import Tree


def tree_ids_for_rank(rank, world_size, num_trees):
    """Tree ids trained by `rank`: treeId % world_size == rank, as the reference assigns devices."""
    if not 0 <= rank < world_size:
        raise ValueError("rank %d outside world of %d" % (rank, world_size))
    return list(range(rank, num_trees, world_size))


def tree_to_bytes(tree):
    """A tree's node arrays, prior and id as bytes (numpy .npz)."""
    a = tree.arrays()
    buf = io.BytesIO()
    np.savez(buf, tree_id=np.int32(tree.tree_id), prior=tree.prior(), **a)
    return buf.getvalue()


def tree_from_bytes(data):
    z = np.load(io.BytesIO(data))
    t = Tree.from_arrays(int(z["tree_id"]), z["left"], z["feature"], z["threshold"], z["histogram"],
                         level=z["level"], score=z["score"], feature_id=z["feature_id"])
    if z["prior"].size:
        t.set_prior(z["prior"])
    return t


def gather_forest(local_trees, group=None):
    """All trees of all ranks on every rank, ordered by tree id (torch.distributed must be initialised;
    any backend: gloo on CPU, NCCL on GPUs)."""
    import torch.distributed as dist
    payload = [tree_to_bytes(t) for t in local_trees]
    gathered = [None] * dist.get_world_size(group)
    dist.all_gather_object(gathered, payload, group=group)
    trees = [tree_from_bytes(b) for part in gathered for b in part]
    ids = [t.tree_id for t in trees]
    if len(set(ids)) != len(ids):
        raise RuntimeError("gather_forest: two ranks trained the same tree id")
    return sorted(trees, key=lambda t: t.tree_id)


def allgather_bytes(group=None):
    """An all-gather of equal-size byte strings over torch.distributed, for train_tree_sharded: returns
    a function payload -> the concatenation of every rank's payload in rank order. NCCL exchanges
    through the current CUDA device, gloo through host memory."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else \
        torch.device("cpu")

    def fn(payload):
        t = torch.frombuffer(bytearray(payload), dtype=torch.uint8).to(device)
        out = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(out, t, group=group)
        return b"".join(o.cpu().numpy().tobytes() for o in out)
    return fn
