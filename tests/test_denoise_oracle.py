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


class _FakeNet:
    """Stands in for the denoiser: its 'weights' are one number, its optimiser state a flag."""

    def __init__(self):
        self.w, self.moments, self.loads = 0, True, 0

    def state_dict(self):
        return {"w": self.w}

    def load_state_dict(self, sd):
        self.w = sd["w"]
        self.loads += 1

    def reset_optimizer(self):
        self.moments = False


def test_collapse_guard_restores_best_weights():
    from conftest import load_package
    load_package()
    from gps_pbvr_web_b200.denoise_train import CollapseGuard
    g, net = CollapseGuard(factor=3.0, warmup=3), _FakeNet()
    losses = [0.10, 0.05, 0.03, 0.025, 0.022, 0.024, 0.093, 0.030, 0.021]
    scales = []
    for step, loss in enumerate(losses):
        net.w = step  # the weights change every step
        scales.append(g.check(step * 100, loss, net))
    # the jump to 0.093 (> 3 x 0.022) restores the weights of step 4 and halves the rate
    assert g.restores == [(600, 0.093, 0.022)] and net.loads == 1 and not net.moments
    assert scales[:6] == [1.0] * 6 and scales[6:] == [0.5, 0.5, 0.5]
    assert g.best == 0.021 and g.snap == {"w": 8}
    # no restore during the warm-up logs, whatever the loss does
    g2, net2 = CollapseGuard(factor=3.0, warmup=3), _FakeNet()
    for step, loss in enumerate([0.01, 0.5, 0.6]):
        g2.check(step, loss, net2)
    assert g2.restores == [] and net2.loads == 0
