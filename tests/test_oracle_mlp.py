"""The CPU oracle of the refinement network: its gradient equals central finite differences of its loss."""
import numpy as np

from oracle import pyoracle as orc


def test_oracle_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    C, H = 5, 7
    D = 3 * C + 2
    n = 11
    P = H * D + H + C * H + C
    params = (rng.standard_normal(P) * 0.3).astype(np.float32)
    X = rng.random((n, D)).astype(np.float32)
    Y = rng.integers(0, C, n).astype(np.uint8)
    loss, g = orc.mlp_loss_grad(params, X, Y, H, C)
    assert np.isfinite(loss) and loss > 0
    for i in rng.choice(P, 60, replace=False):
        a, b = params.copy(), params.copy()
        a[i] += np.float32(1e-3)
        b[i] -= np.float32(1e-3)
        la, _ = orc.mlp_loss_grad(a, X, Y, H, C)
        lb, _ = orc.mlp_loss_grad(b, X, Y, H, C)
        fd = (la - lb) / (float(a[i]) - float(b[i]))
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_oracle_mlp_uniform_logits_loss_is_log_c():
    C, H = 6, 4
    D = 3 * C + 2
    params = np.zeros(H * D + H + C * H + C, np.float32)
    X = np.ones((3, D), np.float32)
    loss, g = orc.mlp_loss_grad(params, X, np.array([0, 1, 5], np.uint8), H, C)
    assert abs(loss - np.log(C)) < 1e-12
    assert np.abs(g[:H * D + H]).max() == 0.0   # zero weights: no gradient reaches the first layer
