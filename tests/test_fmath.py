"""The shared deterministic f32 maths (gps-pbvr-web_b200/csrc/fmath.h) against libm in double
precision: errors stay within a few ulp over the ranges the renderer uses."""
import numpy as np

import oracle as O


def _ulp_err(got, ref):
    ref32 = ref.astype(np.float32)
    spacing = np.spacing(np.abs(ref32).astype(np.float32)).astype(np.float64)
    spacing = np.maximum(spacing, np.finfo(np.float32).tiny)
    return np.abs(got.astype(np.float64) - ref) / spacing


def test_exp_accuracy():
    x = np.linspace(-87.0, 88.0, 400001).astype(np.float32)
    e = _ulp_err(O.o2_fmath(0, x), np.exp(x.astype(np.float64)))
    assert e.max() <= 2.0, e.max()


def test_log_accuracy():
    x = np.concatenate([np.geomspace(1e-37, 1e37, 400001), np.linspace(0.5, 2.0, 200001)]).astype(np.float32)
    ref = np.log(x.astype(np.float64))
    got = O.o2_fmath(1, x)
    err = np.abs(got - ref)
    rel = err / np.maximum(np.abs(ref), 1e-30)
    # a few ulp relative, or absolute 2e-7 next to log(x) = 0
    assert np.all((rel <= 4 * 2.0 ** -24) | (err <= 2e-7)), (rel.max(), err.max())


def test_sin_cos_accuracy():
    x = np.linspace(-7.0, 7.0, 400001).astype(np.float32)
    xd = x.astype(np.float64)
    for which, f in [(2, np.sin), (3, np.cos)]:
        err = np.abs(O.o2_fmath(which, x) - f(xd))
        assert err.max() <= 2.5e-7, (which, err.max())


def test_special_values():
    x = np.array([0.0, 1.0, np.inf, -np.inf, 1e-45, -1.0], np.float32)
    lg = O.o2_fmath(1, x)
    assert lg[0] == -np.inf and lg[1] == 0.0 and lg[2] == np.inf and np.isnan(lg[5])
    assert abs(lg[4] - np.log(float(x[4]))) < 1e-4
    ex = O.o2_fmath(0, np.array([0.0, -200.0, 200.0], np.float32))
    assert ex[0] == 1.0 and ex[1] == 0.0 and ex[2] == np.inf


def test_pow_for_srgb():
    x = np.linspace(0.0031308, 1.0, 100001).astype(np.float32)
    err = np.abs(O.o2_fmath(4, x) - x.astype(np.float64) ** (1 / 2.4))
    assert err.max() <= 3e-7


def test_log_for_positive_normal_arguments_is_log():
    """log_t_pos (log without the special-value test, used where the argument is known positive and
    normal) gives log's bits: every Box-Muller uniform max(k 2^-24, 5.96e-8) and a million floats
    spread over [1e-38, 1] and (1, 1e30]."""
    k = np.arange(1 << 24, dtype=np.float64)
    u = np.maximum((k * 2.0 ** -24).astype(np.float32), np.float32(5.96e-8))
    rng = np.random.default_rng(5)
    wide = np.exp(rng.uniform(np.log(1.2e-38), np.log(1e30), 1_000_000)).astype(np.float32)
    for x in (u, wide):
        a, b = O.o2_fmath(1, x), O.o2_fmath(5, x)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
