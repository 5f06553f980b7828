"""Test oracle (CPU, numpy float64) of the denoiser U-Net of gps-pbvr-web_b200/denoise.py: forward
pass, L1 loss and every parameter gradient, written from the network's definition (3x3
convolutions with zero padding, ReLU, 2x2 average pooling, nearest upsampling, skip concatenation,
residual on the mean colour). Used only by the tests to check the GPU kernels' gradients; it is
not part of the product. Weights use the GPU's (cout, kp) row layout, k = (ky*3 + kx)*cin + ci.
"""
import numpy as np

LAYERS = [("c1a", 8, 32), ("c1b", 32, 32), ("c2a", 32, 64), ("c2b", 64, 64), ("c3a", 64, 128), ("c3b", 128, 128),
          ("c4a", 192, 64), ("c4b", 64, 64), ("c5a", 96, 32), ("c5b", 32, 32), ("c6", 32, 3)]


def _cols(x):
    """im2col of NHWC x with zero padding: (B, H, W, 9 * C), tap-major like the GPU's K axis."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    return np.concatenate([xp[:, ky:ky + H, kx:kx + W] for ky in range(3) for kx in range(3)], axis=-1)


def conv(x, w, b):
    cin = x.shape[-1]
    return _cols(x) @ w[:, :9 * cin].T + b


def conv_grads(x, w, dy):
    """(dw rows (cout, 9 cin), db, dx) of y = conv(x, w, b) given dy."""
    B, H, W, cin = x.shape
    cols = _cols(x).reshape(-1, 9 * cin)
    d2 = dy.reshape(-1, dy.shape[-1])
    dw = d2.T @ cols
    db = d2.sum(axis=0)
    dcols = (d2 @ w[:, :9 * cin]).reshape(B, H, W, 9, cin)
    dx = np.zeros((B, H + 2, W + 2, cin))
    for t in range(9):
        ky, kx = divmod(t, 3)
        dx[:, ky:ky + H, kx:kx + W] += dcols[..., t, :]
    return dw, db, dx[:, 1:-1, 1:-1]


def pool(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def forward(params, x0, base):
    """params[name] = (w (cout, kp), b (cout,)); returns (pred, cache)."""
    relu = lambda v: np.maximum(v, 0.0)
    c = {}
    c["a1"] = relu(conv(x0, *params["c1a"]))
    c["s1"] = relu(conv(c["a1"], *params["c1b"]))
    c["p1"] = pool(c["s1"])
    c["a2"] = relu(conv(c["p1"], *params["c2a"]))
    c["s2"] = relu(conv(c["a2"], *params["c2b"]))
    c["p2"] = pool(c["s2"])
    c["a3"] = relu(conv(c["p2"], *params["c3a"]))
    c["b3"] = relu(conv(c["a3"], *params["c3b"]))
    c["cat2"] = np.concatenate([up(c["b3"]), c["s2"]], axis=-1)
    c["d2a"] = relu(conv(c["cat2"], *params["c4a"]))
    c["d2"] = relu(conv(c["d2a"], *params["c4b"]))
    c["cat1"] = np.concatenate([up(c["d2"]), c["s1"]], axis=-1)
    c["d1a"] = relu(conv(c["cat1"], *params["c5a"]))
    c["d1"] = relu(conv(c["d1a"], *params["c5b"]))
    c["r"] = conv(c["d1"], *params["c6"])
    return base + c["r"], c


def loss_and_grads(params, x0, base, target):
    """Mean L1 loss and {name: (dw (cout, 9 cin), db)} of the whole network."""
    pred, c = forward(params, x0, base)
    n = pred.size
    loss = np.abs(pred - target).sum() / n
    g = {}
    dr = np.sign(pred - target) / n
    dw, db, dd1 = conv_grads(c["d1"], params["c6"][0], dr)
    g["c6"] = (dw, db)

    def layer(name, x, y, dy):
        dz = dy * (y > 0)
        dw, db, dx = conv_grads(x, params[name][0], dz)
        g[name] = (dw, db)
        return dx
    dd1a = layer("c5b", c["d1a"], c["d1"], dd1)
    dcat1 = layer("c5a", c["cat1"], c["d1a"], dd1a)
    dd2 = dcat1[..., :64].reshape(dcat1.shape[0], dcat1.shape[1] // 2, 2, dcat1.shape[2] // 2, 2, 64).sum(axis=(2, 4))
    ds1 = dcat1[..., 64:].copy()
    dd2a = layer("c4b", c["d2a"], c["d2"], dd2)
    dcat2 = layer("c4a", c["cat2"], c["d2a"], dd2a)
    db3 = dcat2[..., :128].reshape(dcat2.shape[0], dcat2.shape[1] // 2, 2, dcat2.shape[2] // 2, 2, 128).sum(axis=(2, 4))
    ds2 = dcat2[..., 128:].copy()
    da3 = layer("c3b", c["a3"], c["b3"], db3)
    dp2 = layer("c3a", c["p2"], c["a3"], da3)
    ds2 += up(dp2) * 0.25
    da2 = layer("c2b", c["a2"], c["s2"], ds2)
    dp1 = layer("c2a", c["p1"], c["a2"], da2)
    ds1 += up(dp1) * 0.25
    da1 = layer("c1b", c["a1"], c["s1"], ds1)
    layer("c1a", x0, c["a1"], da1)
    return loss, g
