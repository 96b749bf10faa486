"""The learned part: the refinement network's training kernels against the CPU oracle, its inputs against a
numpy restatement, determinism, and what it gains over the forest alone on held-out frames."""
import numpy as np
import pytest

import curfil_b200 as cf
from oracle import pyoracle as orc
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from curfil_b200 import _build
    _build.build()
    c = cf.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("n", [1, 64, 200])
def test_gradients_match_oracle(ctx, n):
    C, hidden = 6, 16
    r = cf.Refiner(ctx, C, hidden=hidden, seed=5)
    rng = np.random.default_rng(n)
    D = 3 * C + 2
    params = (rng.standard_normal(r.params().size) * 0.4).astype(np.float32)
    r.params(params)
    X = rng.random((n, D)).astype(np.float32)
    Y = rng.integers(0, C, n).astype(np.uint8)
    loss, g = r.loss_grad(X, Y)
    oloss, og = orc.mlp_loss_grad(params, X, Y, hidden, C)
    assert loss == pytest.approx(oloss, rel=1e-5)
    np.testing.assert_allclose(g, og, rtol=1e-4, atol=1e-6 * np.abs(og).max())
    r.close()


def _box_mean(p, r):
    """Mean over the (2r+1)^2 box clipped at the border, for planes [C][H][W]."""
    C, Hh, Ww = p.shape
    cs = np.zeros((C, Hh + 1, Ww + 1))
    cs[:, 1:, 1:] = p.astype(np.float64).cumsum(1).cumsum(2)
    out = np.empty_like(p, dtype=np.float64)
    for y in range(Hh):
        y0, y1 = max(0, y - r), min(Hh - 1, y + r)
        for x in range(Ww):
            x0, x1 = max(0, x - r), min(Ww - 1, x + r)
            s = cs[:, y1 + 1, x1 + 1] - cs[:, y0, x1 + 1] - cs[:, y1 + 1, x0] + cs[:, y0, x0]
            out[:, y, x] = s / ((y1 - y0 + 1) * (x1 - x0 + 1))
    return out


@pytest.fixture(scope="module")
def scene(ctx):
    rgb, depth, labels = H.frames(seed=13, n=12, w=96, h=72, cells=8, classes=6)
    ds = cf.Dataset.from_raw(ctx, rgb, depth)
    cfg = cf.TrainConfig(feature_count=64, thresholds=10, max_depth=6, min_sample_count=20, box_radius=30,
                         region_size=8, samples_per_image=600, sampler=1)
    trees = []
    seed = cf.forest_seed(cfg.random_seed)
    for t in range(2):
        s, prior, counter = cf.sample_tree_pixels(labels[:8], depth[:8], 6, cfg, 2, seed + t, ctx=ctx)
        tree, _ = cf.train_tree(ds, s, 6, cfg, tree_id=t, seed_counter=counter)
        tree.set_prior(prior)
        trees.append(tree)
    forest = cf.Forest(ctx, trees)
    return dict(rgb=rgb, depth=depth, labels=labels, ds=ds, forest=forest)


def test_features_match_numpy(ctx, scene):
    import torch
    forest, ds = scene["forest"], scene["ds"]
    r = cf.Refiner(ctx, 6, radius1=2, radius2=5)
    probs = torch.empty((1, 6, 72, 96), dtype=torch.float32, device="cuda:0")
    ctx.synchronize()
    forest.predict_dataset(ds, 3, 1, probs.data_ptr(), 0)
    ctx.synchronize()
    p = probs.cpu().numpy()[0]
    m1, m2 = _box_mean(p, 2), _box_mean(p, 5)
    xy = np.array([[0, 0], [95, 71], [40, 30], [3, 70], [94, 1], [50, 50]], np.int32)
    f = r.features(forest, ds, 3, xy)
    dm = scene["depth"][3].astype(np.float64)
    for i, (x, y) in enumerate(xy):
        np.testing.assert_array_equal(f[i, :6], p[:, y, x])
        np.testing.assert_allclose(f[i, 6:12], m1[:, y, x], rtol=0, atol=2e-6)
        np.testing.assert_allclose(f[i, 12:18], m2[:, y, x], rtol=0, atol=2e-6)
        d = dm[y, x] / 1000.0
        assert f[i, 18] == pytest.approx(d * 0.2, abs=1e-6)
        assert f[i, 19] == (1.0 if dm[y, x] > 0 else 0.0)
    r.close()


def _accuracy(ctx, fn, ds, first, count, labels):
    import torch
    lab = torch.empty((count, ds.height, ds.width), dtype=torch.uint8, device="cuda:0")
    ctx.synchronize()
    fn(first, count, lab.data_ptr())
    ctx.synchronize()
    return float((lab.cpu().numpy() == labels).mean())


def test_training_is_deterministic(ctx, scene):
    cfgs = dict(hidden=32, epochs=2, batch=1024, pixels_per_image=2000, seed=9)
    a, b = cf.Refiner(ctx, 6, **cfgs), cf.Refiner(ctx, 6, **cfgs)
    la = a.train(scene["forest"], scene["ds"], 0, 4, scene["labels"][:4])
    lb = b.train(scene["forest"], scene["ds"], 0, 4, scene["labels"][:4])
    np.testing.assert_array_equal(la, lb)
    np.testing.assert_array_equal(a.params(), b.params())
    a.close()
    b.close()


def test_refinement_gains_over_the_forest(ctx, scene):
    """Trained on the forest's 8 training frames, evaluated on 4 held-out frames."""
    forest, ds, labels = scene["forest"], scene["ds"], scene["labels"]
    r = cf.Refiner(ctx, 6, hidden=64, epochs=10, batch=2048, pixels_per_image=6000, learning_rate=3e-3, seed=3)
    losses = r.train(forest, ds, 0, 8, labels[:8])
    assert losses[-1] < losses[0]
    base = _accuracy(ctx, lambda f, c, p: forest.predict_dataset(ds, f, c, 0, p), ds, 8, 4, labels[8:])
    refined = _accuracy(ctx, lambda f, c, p: r.predict(forest, ds, f, c, 0, p), ds, 8, 4, labels[8:])
    print("held-out pixel accuracy: forest %.4f, refined %.4f" % (base, refined))
    assert refined >= base + 0.02, (base, refined)
    r.close()
