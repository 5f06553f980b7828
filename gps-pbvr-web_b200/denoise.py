"""Learned denoiser of few-ensemble accumulations: a 3-level U-Net of 3x3 convolutions whose
forward and backward passes run on the library's tcgen05 kernels (csrc/conv3x3.cu for the
convolutions and data gradients, csrc/denoise.cu for the weight gradients and element-wise steps),
with BF16 weights and activations and FP32 accumulation. bf16 activations are chunk-planar
(B, C/8, H, W, 8) tensors, fp32 buffers pixel-major (B, H, W, C); the 8-channel input features
are the same in both layouts. PyTorch tensors only hold device memory here.
"""
import ctypes as C
import os

from . import abi


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ck(code, what):
    if code != 0:
        raise RuntimeError(f"{what}: CUDA error {code}")


def kp_of(cin):
    """Row length of a weight matrix: 9 * cin rounded up to a multiple of 64."""
    return (9 * cin + 63) // 64 * 64


def conv_fwd(x, cin, w, cout, bias, out, *, xoff=0, ooff=0, relu=False, err):
    """3x3 convolution of the NHWC bf16 tensor x (B, H, W, ldx) channels [xoff, xoff + cin) with
    w (cout, kp) bf16 into out (B, H, W, ldo) channels [ooff, ooff + cout), bf16 or fp32."""
    import torch
    B, H, W, ldx = x.shape
    ldo = out.shape[-1]
    _ck(abi.lib().gpsb_dn_conv_fwd(_p(x), ldx, xoff, cin, B, H, W, _p(w), cout, w.shape[1], _p(bias), _p(out), ldo,
                                   ooff, int(out.dtype == torch.float32), int(relu), _stream(), _p(err)), "conv_fwd")


def conv3_weights(w, cout, cin, wt=None):
    """Weights w (cout, kp) bf16 arranged for conv3 into wt (a uint8 CUDA tensor, allocated when None)."""
    import torch
    L = abi.lib()
    n = int(L.gpsb_dn_conv3_weight_bytes(cout, cin))
    if wt is None or wt.numel() != n:
        wt = torch.zeros(n, dtype=torch.uint8, device=w.device)
    _ck(L.gpsb_dn_conv3_weights(_p(w), cout, cin, w.shape[1], _p(wt), _stream()), "conv3_weights")
    return wt


def dims(t):
    """(B, H, W, channels) of an activation tensor: chunk-planar bf16 (B, C/8, H, W, 8), or
    pixel-major (B, H, W, C) (fp32 buffers, and 8-channel tensors, which are the same in both)."""
    if t.dim() == 5:
        B, C8, H, W, e = t.shape
        assert e == 8
        return B, H, W, 8 * C8
    return tuple(t.shape)


def to_planar(x):
    """(B, H, W, C) pixel-major -> (B, C/8, H, W, 8) chunk-planar (contiguous copy)."""
    B, H, W, C = x.shape
    return x.reshape(B, H, W, C // 8, 8).permute(0, 3, 1, 2, 4).contiguous()


def from_planar(x):
    """(B, C/8, H, W, 8) chunk-planar -> (B, H, W, C) pixel-major."""
    B, C8, H, W, _ = x.shape
    return x.permute(0, 2, 3, 1, 4).reshape(B, H, W, 8 * C8)


def conv3(x, cin, wt, cout, bias, out, *, xoff=0, ooff=0, relu=False, err):
    """The 3x3 convolution on the TMA-staged engine (weights arranged by conv3_weights): x a
    chunk-planar bf16 tensor, out chunk-planar bf16 or pixel-major fp32 (see dims)."""
    import torch
    B, H, W, ldx = dims(x)
    ldo = dims(out)[3]
    _ck(abi.lib().gpsb_dn_conv3(_p(x), ldx, xoff, cin, B, H, W, _p(wt), cout, _p(bias), _p(out), ldo, ooff,
                                int(out.dtype == torch.float32), int(relu), _stream(), _p(err)), "conv3")


def conv_dw(dy, x, cin, cout, dw, *, xoff=0, err):
    """dw (cout, kp) fp32 += weight gradient of the convolution of x channels [xoff, xoff + cin)
    given the bf16 output gradient dy; dy and x chunk-planar (see dims)."""
    B, H, W, ldx = dims(x)
    _ck(abi.lib().gpsb_dn_conv_dw(_p(dy), dims(dy)[3], _p(x), ldx, xoff, cin, B, H, W, cout, dw.shape[1], _p(dw),
                                  _stream(), _p(err)), "conv_dw")


def flip(w, cout, cin, wf, coutp):
    """wf (cin, kp2) = the data-gradient weights of w (cout, kp): W'[ci][8 - t][co] = W[co][t][ci]."""
    _ck(abi.lib().gpsb_dn_flip(_p(w), cout, cin, w.shape[1], _p(wf), coutp, wf.shape[1], _stream()), "flip")


def _L():
    return abi.lib()


# (name, padded input channels, real input channels, output channels); ReLU after all but the last
LAYERS = [("c1a", 8, 6, 32), ("c1b", 32, 32, 32), ("c2a", 32, 32, 64), ("c2b", 64, 64, 64), ("c3a", 64, 64, 128),
          ("c3b", 128, 128, 128), ("c4a", 192, 192, 64), ("c4b", 64, 64, 64), ("c5a", 96, 96, 32),
          ("c5b", 32, 32, 32), ("c6", 32, 32, 3)]


def _pad8(c):
    return (c + 7) // 8 * 8


class Denoiser:
    """3-level U-Net (3x3 convolutions 32/64/128, ReLU, 2x2 average pooling, nearest upsampling,
    skip concatenation) mapping the 8-channel frame features of `pack` to a residual that is added
    to the few-ensemble mean colour. Master weights fp32 (Adam state beside them), compute copies
    bf16; every arithmetic step runs in the library's kernels."""

    def __init__(self, seed=0, device="cuda"):
        import torch
        self.engine = "tma"
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        self.p = {}
        for name, cin, cin_real, cout in LAYERS:
            kp = kp_of(cin)
            w = torch.zeros(cout, kp)
            std = (2.0 / (9 * cin_real)) ** 0.5 if name != "c6" else 1e-3
            wr = torch.randn(cout, 9, cin, generator=g) * std
            if cin_real < cin:
                wr[:, :, cin_real:] = 0.0
            w[:, :9 * cin] = wr.reshape(cout, 9 * cin)
            d = self.device
            self.p[name] = {
                "cin": cin, "cout": cout, "kp": kp, "coutp": _pad8(cout),
                "w": w.to(d), "b": torch.zeros(cout, device=d),
                "wb": torch.zeros(cout, kp, dtype=torch.bfloat16, device=d),
                "wf": torch.zeros(cin, kp_of(_pad8(cout)), dtype=torch.bfloat16, device=d),
                "gw": torch.zeros(cout, kp, device=d), "gb": torch.zeros(cout, device=d),
                "mw": torch.zeros(cout, kp, device=d), "vw": torch.zeros(cout, kp, device=d),
                "mb": torch.zeros(cout, device=d), "vb": torch.zeros(cout, device=d),
            }
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.loss = torch.zeros(1, device=self.device)
        self.t = 0
        self._bufs = {}
        self.sync_weights()

    # ------------------------------------------------------------------ parameters
    def sync_weights(self):
        """bf16 compute copies and flipped data-gradient weights from the fp32 masters."""
        st = _stream()
        for q in self.p.values():
            _ck(_L().gpsb_dn_to_bf16(_p(q["w"]), q["kp"], q["cout"], q["kp"], _p(q["wb"]), q["kp"], st), "to_bf16")
            flip(q["wb"], q["cout"], q["cin"], q["wf"], q["coutp"])
            q["wt"] = conv3_weights(q["wb"], q["cout"], q["cin"], q.get("wt"))
            q["wft"] = conv3_weights(q["wf"], q["cin"], q["coutp"], q.get("wft"))

    def state_dict(self):
        return {n: {"w": q["w"].cpu(), "b": q["b"].cpu()} for n, q in self.p.items()}

    def load_state_dict(self, sd):
        for n, q in self.p.items():
            q["w"].copy_(sd[n]["w"])
            q["b"].copy_(sd[n]["b"])
        self.sync_weights()

    def reset_optimizer(self):
        """Zeroes Adam's moments and step count (after restoring earlier weights)."""
        for q in self.p.values():
            for k in ("mw", "vw", "mb", "vb"):
                q[k].zero_()
        self.t = 0

    def param_count(self):
        return sum(q["cout"] * 9 * c_real + q["cout"] for (n, _, c_real, _), q in zip(LAYERS, self.p.values()))

    # ------------------------------------------------------------------ buffers
    def _buffers(self, B, H, W):
        import torch
        key = (B, H, W)
        if key in self._bufs:
            return self._bufs[key]
        if H % 4 or W % 4:
            raise ValueError("the U-Net needs H and W divisible by 4")
        d, bf, f32 = self.device, torch.bfloat16, torch.float32
        h2, w2, h4, w4 = H // 2, W // 2, H // 4, W // 4

        def t(h, w, c, dt):  # bf16 activations chunk-planar, fp32 buffers pixel-major
            if dt == bf:
                return torch.zeros(B, c // 8, h, w, 8, dtype=dt, device=d)
            return torch.zeros(B, h, w, c, dtype=dt, device=d)
        b = {
            "a1": t(H, W, 32, bf), "cat1": t(H, W, 96, bf), "p1": t(h2, w2, 32, bf), "a2": t(h2, w2, 64, bf),
            "cat2": t(h2, w2, 192, bf), "p2": t(h4, w4, 64, bf), "a3": t(h4, w4, 128, bf), "b3": t(h4, w4, 128, bf),
            "d2a": t(h2, w2, 64, bf), "d2": t(h2, w2, 64, bf), "d1a": t(H, W, 32, bf), "d1": t(H, W, 32, bf),
            "r": t(H, W, 3, f32), "pred": t(H, W, 3, f32),
        }
        self._bufs[key] = b
        return b

    def _grad_buffers(self, B, H, W):
        import torch
        key = ("g", B, H, W)
        if key in self._bufs:
            return self._bufs[key]
        d, bf, f32 = self.device, torch.bfloat16, torch.float32
        h2, w2, h4, w4 = H // 2, W // 2, H // 4, W // 4

        def t(h, w, c, dt):  # bf16 gradients chunk-planar, fp32 ones pixel-major
            if dt == bf:
                return torch.zeros(B, c // 8, h, w, 8, dtype=dt, device=d)
            return torch.zeros(B, h, w, c, dtype=dt, device=d)
        g = {
            "dr": t(H, W, 8, bf), "dz1": t(H, W, 32, bf), "dz2": t(h2, w2, 64, bf), "dz4": t(h4, w4, 128, bf),
            "g1": t(H, W, 32, f32), "dcat1": t(H, W, 96, f32), "g2": t(h2, w2, 64, f32), "dcat2": t(h2, w2, 192, f32),
            "g4": t(h4, w4, 128, f32), "dp2": t(h4, w4, 64, f32), "dp1": t(h2, w2, 32, f32),
        }
        self._bufs[key] = g
        return g

    # ------------------------------------------------------------------ forward
    def _conv(self, name, x, out, *, xoff=0, ooff=0, relu=True):
        q = self.p[name]
        conv3(x, q["cin"], q["wt"], q["cout"], q["b"], out, xoff=xoff, ooff=ooff, relu=relu, err=self.err)

    def forward(self, x0, base):
        """x0 (B, H, W, 8) bf16 features, base (B, H, W, 3) fp32 mean colour -> prediction (B, H, W, 3)."""
        B, H, W, _ = x0.shape
        b = self._buffers(B, H, W)
        L, st = _L(), _stream()
        h2, w2, h4, w4 = H // 2, W // 2, H // 4, W // 4
        self._conv("c1a", x0, b["a1"])
        self._conv("c1b", b["a1"], b["cat1"], ooff=64)
        _ck(L.gpsb_dn_pool2(_p(b["cat1"]), 96, 64, B, h2, w2, 32, _p(b["p1"]), st), "pool2")
        self._conv("c2a", b["p1"], b["a2"])
        self._conv("c2b", b["a2"], b["cat2"], ooff=128)
        _ck(L.gpsb_dn_pool2(_p(b["cat2"]), 192, 128, B, h4, w4, 64, _p(b["p2"]), st), "pool2")
        self._conv("c3a", b["p2"], b["a3"])
        self._conv("c3b", b["a3"], b["b3"])
        _ck(L.gpsb_dn_up2(_p(b["b3"]), 128, B, h4, w4, 128, _p(b["cat2"]), 192, 0, st), "up2")
        self._conv("c4a", b["cat2"], b["d2a"])
        self._conv("c4b", b["d2a"], b["d2"])
        _ck(L.gpsb_dn_up2(_p(b["d2"]), 64, B, h2, w2, 64, _p(b["cat1"]), 96, 0, st), "up2")
        self._conv("c5a", b["cat1"], b["d1a"])
        self._conv("c5b", b["d1a"], b["d1"])
        self._conv("c6", b["d1"], b["r"], relu=False)
        _ck(L.gpsb_dn_residual(_p(base), _p(b["r"]), B * H * W * 3, _p(b["pred"]), st), "residual")
        return b["pred"]

    # ------------------------------------------------------------------ backward
    def _back(self, name, dz, x, gx, *, xoff=0, data_grad=True):
        """weight, bias and (optionally) input gradients of layer `name` from its bf16 output gradient dz"""
        q = self.p[name]
        B, H, W, ld = dims(dz)
        conv_dw(dz, x, q["cin"], q["cout"], q["gw"], xoff=xoff, err=self.err)
        _ck(_L().gpsb_dn_bias_grad(_p(dz), ld, B, H * W, q["cout"], _p(q["gb"]), _stream()), "bias_grad")
        if data_grad:
            conv3(dz, q["coutp"], q["wft"], q["cin"], None, gx, err=self.err)

    def _relu_bwd(self, g, ldg, goff, y, ldy, yoff, C, out):
        B, H, W, ldo = dims(out)
        _ck(_L().gpsb_dn_relu_bwd(_p(g), ldg, goff, _p(y), ldy, yoff, B, H * W, C, _p(out), ldo, _stream()),
            "relu_bwd")

    def backward(self, x0, base, target):
        """L1 loss of the last forward against target; accumulates the parameter gradients (which
        zero_grad clears) and returns the loss tensor (sum of |error|, not yet averaged)."""
        B, H, W, _ = x0.shape
        b, g = self._buffers(B, H, W), self._grad_buffers(B, H, W)
        L, st = _L(), _stream()
        M = B * H * W
        h2, w2, h4, w4 = H // 2, W // 2, H // 4, W // 4
        self.loss.zero_()
        _ck(L.gpsb_dn_l1(_p(base), _p(b["r"]), _p(target), M, _p(self.loss), _p(g["dr"]), 1.0 / (3 * M), st), "l1")
        self._back("c6", g["dr"], b["d1"], g["g1"])
        self._relu_bwd(g["g1"], 32, 0, b["d1"], 32, 0, 32, g["dz1"])
        self._back("c5b", g["dz1"], b["d1a"], g["g1"])
        self._relu_bwd(g["g1"], 32, 0, b["d1a"], 32, 0, 32, g["dz1"])
        self._back("c5a", g["dz1"], b["cat1"], g["dcat1"])
        _ck(L.gpsb_dn_up2_bwd(_p(g["dcat1"]), 96, 0, B, h2, w2, 64, _p(g["g2"]), st), "up2_bwd")
        self._relu_bwd(g["g2"], 64, 0, b["d2"], 64, 0, 64, g["dz2"])
        self._back("c4b", g["dz2"], b["d2a"], g["g2"])
        self._relu_bwd(g["g2"], 64, 0, b["d2a"], 64, 0, 64, g["dz2"])
        self._back("c4a", g["dz2"], b["cat2"], g["dcat2"])
        _ck(L.gpsb_dn_up2_bwd(_p(g["dcat2"]), 192, 0, B, h4, w4, 128, _p(g["g4"]), st), "up2_bwd")
        self._relu_bwd(g["g4"], 128, 0, b["b3"], 128, 0, 128, g["dz4"])
        self._back("c3b", g["dz4"], b["a3"], g["g4"])
        self._relu_bwd(g["g4"], 128, 0, b["a3"], 128, 0, 128, g["dz4"])
        self._back("c3a", g["dz4"], b["p2"], g["dp2"])
        _ck(L.gpsb_dn_pool2_bwd_add(_p(g["dp2"]), B, h4, w4, 64, _p(g["dcat2"]), 192, 128, st), "pool2_bwd")
        dz2s = g["dz2"]
        self._relu_bwd(g["dcat2"], 192, 128, b["cat2"], 192, 128, 64, dz2s)
        self._back("c2b", dz2s, b["a2"], g["g2"])
        self._relu_bwd(g["g2"], 64, 0, b["a2"], 64, 0, 64, g["dz2"])
        self._back("c2a", g["dz2"], b["p1"], g["dp1"])
        _ck(L.gpsb_dn_pool2_bwd_add(_p(g["dp1"]), B, h2, w2, 32, _p(g["dcat1"]), 96, 64, st), "pool2_bwd")
        self._relu_bwd(g["dcat1"], 96, 64, b["cat1"], 96, 64, 32, g["dz1"])
        self._back("c1b", g["dz1"], b["a1"], g["g1"])
        self._relu_bwd(g["g1"], 32, 0, b["a1"], 32, 0, 32, g["dz1"])
        self._back("c1a", g["dz1"], x0, None, data_grad=False)
        return self.loss

    def zero_grad(self):
        for q in self.p.values():
            q["gw"].zero_()
            q["gb"].zero_()

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        L, st = _L(), _stream()
        for q in self.p.values():
            _ck(L.gpsb_dn_adam(_p(q["w"]), _p(q["gw"]), _p(q["mw"]), _p(q["vw"]), q["w"].numel(), lr, b1, b2, eps,
                               self.t, None, st), "adam")
            _ck(L.gpsb_dn_adam(_p(q["b"]), _p(q["gb"]), _p(q["mb"]), _p(q["vb"]), q["b"].numel(), lr, b1, b2, eps,
                               self.t, None, st), "adam")
        self.sync_weights()

    def train_step(self, x0, base, target, lr=1e-3):
        """One Adam step on the mean L1 loss of a batch; returns the loss tensor (mean |error|)."""
        self.zero_grad()
        self.forward(x0, base)
        loss = self.backward(x0, base, target)
        self.adam_step(lr)
        B, H, W, _ = x0.shape
        return loss / (3 * B * H * W)

    def error_word(self):
        return int(self.err.item())


def pack(accum, feat, x, base):
    """Denoiser input of a rendered frame: accum (P, 4) fp32 (rgb sum, count) and feat (P, 8) fp32
    feature sums (or None) -> x (P, 8) bf16 features and base (P, 3) fp32 mean colour."""
    P = accum.shape[0]
    _ck(_L().gpsb_dn_pack(_p(accum), _p(feat), P, _p(x), _p(base), _stream()), "pack")


def crop(x, base, target, crops, ch, cw, xb, baseb, targetb, err=None):
    """Training batch: crops (B, 3) int32 CUDA tensor of (image, y0, x0) windows of ch x cw taken
    from the stacked frames x (N, H, W, 8), base and target (N, H, W, 3) into xb, baseb, targetb."""
    N, H, W, _ = x.shape
    if crops.dim() != 2 or crops.shape[1] != 3 or xb.shape[0] != crops.shape[0]:
        raise ValueError("crops must be (B, 3) with B the batch of xb")
    _ck(_L().gpsb_dn_crop(_p(x), _p(base), _p(target), N, H, W, _p(crops), crops.shape[0], ch, cw, _p(xb), _p(baseb),
                          _p(targetb), _stream(), _p(err)), "crop")


WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "denoiser_pbvr_c3r.npz")


def load_weights(net, path=WEIGHTS):
    """Loads weights saved by denoise_train.save_weights; returns the variance-gate limit."""
    import numpy as np
    import torch
    z = np.load(path)
    sd = {}
    for n, q in net.p.items():
        w = torch.zeros(q["cout"], q["kp"])
        wr = torch.from_numpy(z[f"{n}.w"])
        w[:, :wr.shape[1]] = wr
        sd[n] = {"w": w, "b": torch.from_numpy(z[f"{n}.b"])}
    net.load_state_dict(sd)
    return float(z["gate_limit"])


def render_denoised(renderer, net, cam, params, first_seed, *, ensembles=4, gate_limit, fallback_ensembles=64):
    """A frame of `renderer` (a GpsRenderer) from few ensembles through the denoiser, or, when the
    per-frame variance check fails (mean per-pixel ensemble standard deviation above gate_limit,
    i.e. outside what the network was trained on), the plain accumulation of fallback_ensembles.
    Returns (rgb (H*W, 3) CUDA tensor, used_denoiser, check value)."""
    import torch
    w, h = renderer.size()
    P = w * h
    if h % 4 or w % 4:
        raise ValueError("the denoiser needs width and height divisible by 4")
    feat = torch.zeros(P * 8, device="cuda")
    renderer.reset_accum()
    renderer.set_feature_accum(feat)
    try:
        renderer.render_ensembles(cam, params, first_seed, ensembles)
        renderer.wait_idle()
    finally:
        renderer.set_feature_accum(None)
    acc = torch.from_numpy(renderer.read_accum()).cuda()
    x = torch.zeros(P, 8, dtype=torch.bfloat16, device="cuda")
    base = torch.zeros(P, 3, device="cuda")
    pack(acc, feat, x, base)
    check = float(x[:, 5].float().mean())
    if check <= gate_limit:
        return net.forward(x.view(1, h, w, 8), base.view(1, h, w, 3)).reshape(P, 3).clone(), True, check
    renderer.render_ensembles(cam, params, first_seed + ensembles, fallback_ensembles - ensembles)
    acc = torch.from_numpy(renderer.read_accum()).cuda()
    return acc[:, :3] / acc[:, 3:4].clamp(min=1.0), False, check


class NativeDenoiser:
    """The C-ABI denoiser (gpsb_denoiser_*): the same network sequenced by the library's C++ host
    code, as a Rust or C caller uses it; loaded from the committed weight file."""

    def __init__(self, path=WEIGHTS, device=0):
        import numpy as np
        L = abi.lib()
        h = C.c_void_p()
        _ck(L.gpsb_denoiser_create(device, C.byref(h)), "gpsb_denoiser_create")
        self._h, self._L = h, L
        z = np.load(path)
        for i, (name, cin, _, cout) in enumerate(LAYERS):
            w = np.ascontiguousarray(z[f"{name}.w"], np.float32).reshape(cout, 9 * cin)
            b = np.ascontiguousarray(z[f"{name}.b"], np.float32)
            self._check(L.gpsb_denoiser_set_layer(h, i, w.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p)))
        self.gate_limit = float(z["gate_limit"])
        self._check(L.gpsb_denoiser_set_gate(h, self.gate_limit))

    def _check(self, st):
        if st != 0:
            raise RuntimeError(f"denoiser status {st}: {self._L.gpsb_denoiser_last_error(self._h).decode()}")

    def forward(self, x, base, pred):
        """x (1, H, W, 8) bf16, base (1, H, W, 3) fp32 -> pred (1, H, W, 3) fp32 (CUDA tensors)."""
        H, W = x.shape[1], x.shape[2]
        self._check(self._L.gpsb_denoiser_forward(self._h, _p(x), _p(base), W, H, _p(pred), _stream()))

    def graph_state(self):
        """1: the layers of the current frame size replay a captured CUDA graph; 0: not captured yet;
        -1: a capture failed and the layers launch directly (gpsb_denoiser_graph_state)."""
        return int(self._L.gpsb_denoiser_graph_state(self._h))

    def render(self, renderer, cam, params, first_seed, ensembles=4, gate_limit=0.0, fallback_ensembles=64):
        """gpsb_render_denoised: returns (rgb (H*W, 3) float32 numpy array, used_denoiser, check)."""
        import numpy as np
        w, h = renderer.size()
        rgb = np.zeros((w * h, 3), np.float32)
        used = C.c_int()
        chk = C.c_float()
        cc, pc = cam.to_c(), params.to_c()
        self._check(self._L.gpsb_render_denoised(renderer.handle, self._h, C.byref(cc), C.byref(pc), first_seed,
                                                 ensembles, gate_limit, fallback_ensembles,
                                                 rgb.ctypes.data_as(C.c_void_p), C.byref(used), C.byref(chk)))
        return rgb, bool(used.value), float(chk.value)

    def close(self):
        if self._h:
            self._L.gpsb_denoiser_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
