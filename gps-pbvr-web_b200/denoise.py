"""Learned denoiser of few-ensemble accumulations: a 3-level U-Net of 3x3 convolutions whose
forward and backward passes run on the library's tcgen05 kernels (csrc/denoise.cu), with BF16
weights and activations and FP32 accumulation. PyTorch tensors only hold device memory here.
"""
import ctypes as C

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


def conv_dw(dy, x, cin, cout, dw, *, xoff=0, err):
    """dw (cout, kp) fp32 += weight gradient of the convolution of x channels [xoff, xoff + cin)
    given the bf16 output gradient dy (B, H, W, ldy)."""
    B, H, W, ldx = x.shape
    _ck(abi.lib().gpsb_dn_conv_dw(_p(dy), dy.shape[-1], _p(x), ldx, xoff, cin, B, H, W, cout, dw.shape[1], _p(dw),
                                  _stream(), _p(err)), "conv_dw")


def flip(w, cout, cin, wf, coutp):
    """wf (cin, kp2) = the data-gradient weights of w (cout, kp): W'[ci][8 - t][co] = W[co][t][ci]."""
    _ck(abi.lib().gpsb_dn_flip(_p(w), cout, cin, w.shape[1], _p(wf), coutp, wf.shape[1], _stream()), "flip")
