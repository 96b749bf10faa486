"""CPU checks of the tree comparison the parity tests use: a tolerated tie skips only the subtree
below it, and a difference anywhere else still fails."""
import numpy as np
import pytest

from tests import helpers as H


def tree(lefts, feats, thrs, scores, hists):
    n = len(lefts)
    f = np.zeros((n, 11), np.int8)
    for i, v in enumerate(feats):
        f[i, 1] = v
    return dict(left=np.array(lefts, np.int32), feature=f, threshold=np.array(thrs, np.float32),
                score=np.array(scores, np.float64), histogram=np.array(hists, np.uint32).reshape(n, 1))


# root splits into 1, 2; node 1 splits into 3, 4; node 2 splits into 5, 6
BASE = dict(lefts=[1, 3, 5, -1, -1, -1, -1], feats=[1, 2, 3, 0, 0, 0, 0], thrs=[0.5, 1.5, 2.5, np.nan, np.nan, np.nan,
                                                                             np.nan],
            scores=[0.5, 0.4, 0.3, np.nan, np.nan, np.nan, np.nan], hists=[10, 6, 4, 3, 3, 2, 2])


def test_identical_trees_compare_every_node():
    assert H.compare_trees(tree(**BASE), tree(**BASE)) == 7


def test_tie_skips_only_its_subtree():
    other = {k: list(v) for k, v in BASE.items()}
    other["feats"][1] = 9                       # node 1 splits on another feature with a tied score
    other["scores"][1] = 0.4 * (1 + 1e-9)
    other["hists"][3], other["hists"][4] = 5, 1  # its children differ
    assert H.compare_trees(tree(**BASE), tree(**other)) == 5   # root, 1, 2, 5, 6


def test_difference_outside_the_tied_subtree_fails():
    other = {k: list(v) for k, v in BASE.items()}
    other["feats"][1] = 9
    other["scores"][1] = 0.4 * (1 + 1e-9)
    other["hists"][6] = 7                       # node 6 lies below node 2, not below the tie
    with pytest.raises(AssertionError):
        H.compare_trees(tree(**BASE), tree(**other))


def test_split_difference_without_tie_fails():
    other = {k: list(v) for k, v in BASE.items()}
    other["feats"][2] = 8
    other["scores"][2] = 0.2
    with pytest.raises(AssertionError):
        H.compare_trees(tree(**BASE), tree(**other))
