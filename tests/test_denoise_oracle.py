"""The denoiser's CPU oracle (oracle/denoise_ref.py) checked by central finite differences: its
analytic gradients of the mean L1 loss agree with the numerical ones on a 1 x 8 x 8 input."""
import numpy as np

from oracle import denoise_ref as R


def _params(rng):
    p = {}
    for name, cin, cout in R.LAYERS:
        kp = (9 * cin + 63) // 64 * 64
        w = np.zeros((cout, kp))
        w[:, :9 * cin] = rng.normal(0, (2.0 / (9 * cin)) ** 0.5, (cout, 9 * cin))
        p[name] = (w, rng.normal(0, 0.05, cout))
    return p


def test_oracle_gradients_by_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    x0 = rng.normal(0, 1, (1, 8, 8, 8))
    base = rng.uniform(0, 1, (1, 8, 8, 3))
    target = rng.uniform(0, 1, (1, 8, 8, 3))
    loss, g = R.loss_and_grads(p, x0, base, target)
    assert loss > 0
    eps = 1e-6
    checked = 0
    for name in ["c1a", "c2b", "c3a", "c4a", "c5a", "c6"]:
        w, b = p[name]
        cin = dict((n, c) for n, c, _ in R.LAYERS)[name]
        for _ in range(3):
            co, k = rng.integers(0, w.shape[0]), rng.integers(0, 9 * cin)
            w[co, k] += eps
            lp = R.loss_and_grads(p, x0, base, target)[0]
            w[co, k] -= 2 * eps
            lm = R.loss_and_grads(p, x0, base, target)[0]
            w[co, k] += eps
            num = (lp - lm) / (2 * eps)
            ana = g[name][0][co, k]
            assert abs(num - ana) <= 1e-6 + 1e-3 * abs(ana), (name, co, k, num, ana)
            checked += 1
        co = rng.integers(0, w.shape[0])
        b[co] += eps
        lp = R.loss_and_grads(p, x0, base, target)[0]
        b[co] -= 2 * eps
        lm = R.loss_and_grads(p, x0, base, target)[0]
        b[co] += eps
        assert abs((lp - lm) / (2 * eps) - g[name][1][co]) <= 1e-6 + 1e-3 * abs(g[name][1][co])
    assert checked == 18
