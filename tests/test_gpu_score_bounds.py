"""The float score bounds that screen (feature, threshold) pairs before exact scoring must enclose the
exact double score of every pair, including the ill-conditioned cases (near-pure nodes, one-sample
sides, gains near zero, counts near 2^31)."""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


def _counters(hist, lefts):
    """counters [F][T][C][2] for left-count vectors lefts [F][T][C] of a node with histogram hist."""
    lefts = np.asarray(lefts, np.uint64)
    right = hist.astype(np.uint64)[None, None, :] - lefts
    return np.stack([lefts, right], axis=-1).astype(np.uint32)


def _cases(rng):
    out = []
    for C, total in [(2, 10), (5, 1000), (40, 266600), (40, 600), (200, 50000), (3, 2 ** 31 - 10)]:
        p = rng.dirichlet(np.ones(C) * 0.5)
        hist = np.maximum(1, np.round(p * total)).astype(np.uint64)
        frac = rng.random((16, 20, C))
        out.append((hist, np.floor(frac * hist).astype(np.uint64)))
    # near-pure node: one dominant class, single samples of the others
    hist = np.array([10 ** 6, 1, 1, 2], np.uint64)
    lefts = rng.integers(0, 2, (8, 20, 4)).astype(np.uint64) * hist
    lefts[:, :, 0] = rng.integers(0, 10 ** 6 + 1, (8, 20))
    out.append((hist, lefts))
    # one-sample sides and proportional splits (gain ~ 0)
    hist = np.array([400, 300, 200, 100], np.uint64)
    lefts = np.zeros((4, 20, 4), np.uint64)
    lefts[0, :, 0] = 1
    lefts[1, :, :] = hist - 1
    lefts[1, :, 1:] = hist[1:]
    for t in range(20):
        lefts[2, t] = (hist * (t + 1)) // 21
    lefts[3, :, :2] = hist[:2]        # perfect split of two class groups
    out.append((hist, lefts))
    # two classes, every left count 0..h
    hist = np.array([37, 41], np.uint64)
    lefts = np.array([[[a, b] for b in range(42)] for a in range(38)], np.uint64)
    out.append((hist, lefts))
    return out


def test_score_bounds_enclose_exact_scores(ctx):
    rng = np.random.default_rng(2026)
    widths = []
    for hist, lefts in _cases(rng):
        counters = _counters(hist, lefts)
        h32 = hist.astype(np.uint32)
        exact = cf.scores(ctx, counters, h32)                  # [T][F]
        lo, up = cf.score_bounds(ctx, counters, h32)
        ora = orc.scores(counters.transpose(2, 0, 1, 3).copy(), h32)   # oracle [T][F]
        # CUDA's and the host's log2 differ by an ulp; the near-pure node amplifies that to ~1e-12
        # relative on its tiny scores
        np.testing.assert_allclose(exact, ora, rtol=1e-10, atol=1e-13)
        assert (lo.astype(np.float64) <= exact).all(), np.argwhere(lo > exact)[:5]
        assert (exact <= up.astype(np.float64)).all(), np.argwhere(exact > up)[:5]
        widths.append(np.median(up - lo))
    # the screening is only useful if typical bounds are tight
    assert np.median(widths) < 2e-5, widths


def test_score_bounds_reject_inconsistent_counters(ctx):
    hist = np.array([5, 5], np.uint32)
    counters = _counters(hist.astype(np.uint64), [[[2, 3]]])
    counters[0, 0, 0, 1] += 1
    with pytest.raises(cf.CurfilError) as e:
        cf.score_bounds(ctx, counters, hist)
    assert e.value.status == 1
