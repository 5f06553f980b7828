"""Phase 0 of the reference's GPU verification (crates/gps-render/src/lib.rs:99-324) on the CUDA
primitives, plus the radix sort primitive:
  * the two-pass atomicMin winner rule on 3 ensembles x 4096 pixels x 200k synthetic samples with
    many exact-depth ties (p0_sample.wgsl), done here with one packed 64-bit atomicMin, bit-exact
    with the CPU two-pass reference (lib.rs:31-39, 169-183);
  * the exclusive scan at n in {1, 255, 256, 257, 65536, 300000, 1000003} (lib.rs:196-275) and at
    2^28 elements through size-independent properties;
  * the stable radix sort against numpy's stable argsort at 4-, 6- and 8-bit digits.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from conftest import load_package

pytestmark = pytest.mark.gpu
PKG = load_package()


def _pcg(v):
    v = v.astype(np.uint64)
    s = (v * np.uint64(747796405) + np.uint64(2891336453)) & np.uint64(0xFFFFFFFF)
    w = (((s >> ((s >> np.uint64(28)) + np.uint64(4))) ^ s) * np.uint64(277803737)) & np.uint64(0xFFFFFFFF)
    return ((w >> np.uint64(22)) ^ w).astype(np.uint32)


def _renderer():
    return PKG.GpsRenderer(16, 16, 1)


def test_pcg_vectorised_matches_oracle():
    xs = np.array([0, 1, 2, 3, 0xDEADBEEF], np.uint32)
    assert _pcg(xs).tolist() == [O.pcg_hash(int(x)) for x in xs]


def test_atomic_two_pass_winner_rule():
    import torch
    E, PIX, SAMPLES = 3, 4096, 200_000
    r = _renderer()
    dev = torch.device("cuda", 0)
    packed = torch.full((E * PIX,), -1, dtype=torch.int64, device=dev)
    L = PKG.abi.lib()
    for e in range(E):
        assert L.gpsb_p0_sample(r.handle, 1000 + e * 7, e * PIX, PIX, SAMPLES, C.c_void_p(packed.data_ptr())) == 0
    r.wait_idle()
    got = packed.cpu().numpy().view(np.uint64)
    rd = np.full(E * PIX, 0xFFFFFFFF, np.uint64)
    rc = rd.copy()
    ties = 0
    for e in range(E):
        i = np.arange(SAMPLES, dtype=np.uint32)
        h0 = _pcg(i ^ np.uint32(O.pcg_hash(1000 + e * 7)))
        h1 = _pcg(h0)
        h2 = _pcg(h1)
        pix = (e * PIX + (h0 % PIX)).astype(np.int64)
        key = ((np.uint32(0x3F800000) | (h1 & np.uint32(0x007FFFFF))) | np.uint32(0x80000000)) & np.uint32(0xFFFF0000)
        rgb = h2 & np.uint32(0x00FFFFFF)
        np.minimum.at(rd, pix, key.astype(np.uint64))
        win = rd[pix] == key
        ties += int(win.sum())
        np.minimum.at(rc, pix[win], rgb[win].astype(np.uint64))
    assert np.array_equal(got >> np.uint64(32), rd) and np.array_equal(got & np.uint64(0xFFFFFFFF), rc)
    assert ties > E * PIX  # many exact-depth ties were exercised
    r.close()


@pytest.mark.parametrize("n", [1, 255, 256, 257, 65536, 300000, 1000003])
def test_scan_sizes(n):
    import torch
    dev = torch.device("cuda", 0)
    x = (_pcg(np.arange(n, dtype=np.uint32)) % 7).astype(np.uint32)
    t_in = torch.from_numpy(x.view(np.int32)).to(dev)
    t_out = torch.empty_like(t_in)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    r = _renderer()
    L = PKG.abi.lib()
    assert L.gpsb_scan_u32(r.handle, C.c_void_p(t_in.data_ptr()), C.c_void_p(t_out.data_ptr()), n,
                           C.c_void_p(total.data_ptr())) == 0
    r.wait_idle()
    ref = np.concatenate([[0], np.cumsum(x.astype(np.uint64))[:-1]]).astype(np.uint32)
    assert np.array_equal(t_out.cpu().numpy().view(np.uint32), ref)
    assert int(total.item()) == int(x.astype(np.uint64).sum())
    r.close()


@pytest.mark.parametrize("n,offset,full", [(524288, 0, False), (524288 + 8192 * 3 + 5, 0, False),
                                           (4_000_001, 0, False), (600_000, 0, True), (1_000_003, 1, False),
                                           (1_000_003, 2, True)])
def test_scan_large_paths(n, offset, full):
    """Many-tile scans with ragged tails, full-range u32 counts whose total passes 2^32, and
    views that are not 16-byte aligned (scalar loads and stores instead of 128-bit ones)."""
    import torch
    dev = torch.device("cuda", 0)
    h = _pcg(np.arange(n, dtype=np.uint32) + np.uint32(offset * 77))
    x = h if full else (h % 13).astype(np.uint32)
    buf = torch.zeros(n + offset, dtype=torch.int32, device=dev)
    buf[offset:] = torch.from_numpy(x.view(np.int32))
    t_in = buf[offset:]
    obuf = torch.zeros(n + offset, dtype=torch.int32, device=dev)
    t_out = obuf[offset:]
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    r = _renderer()
    L = PKG.abi.lib()
    assert L.gpsb_scan_u32(r.handle, C.c_void_p(t_in.data_ptr()), C.c_void_p(t_out.data_ptr()), n,
                           C.c_void_p(total.data_ptr())) == 0
    r.wait_idle()
    cs = np.cumsum(x.astype(np.uint64))
    ref = np.concatenate([[0], cs[:-1]]).astype(np.uint64) & np.uint64(0xFFFFFFFF)
    assert np.array_equal(t_out.cpu().numpy().view(np.uint32), ref.astype(np.uint32))
    assert int(total.item()) == int(cs[-1])
    assert r.debug_error_word() == 0
    r.close()


def test_scan_full_size_properties():
    import torch
    dev = torch.device("cuda", 0)
    n = 1 << 28
    g = torch.Generator(device=dev).manual_seed(5)
    t_in = torch.randint(0, 16, (n,), dtype=torch.int32, device=dev, generator=g)
    t_out = torch.empty_like(t_in)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    r = _renderer()
    L = PKG.abi.lib()
    assert L.gpsb_scan_u32(r.handle, C.c_void_p(t_in.data_ptr()), C.c_void_p(t_out.data_ptr()), n,
                           C.c_void_p(total.data_ptr())) == 0
    r.wait_idle()
    assert int(total.item()) == int(t_in.sum(dtype=torch.int64).item())
    d = (t_out[1:].to(torch.int64) - t_out[:-1].to(torch.int64)) % (1 << 32)
    assert torch.equal(d, t_in[:-1].to(torch.int64)) and int(t_out[0].item()) == 0
    assert r.debug_error_word() == 0
    r.close()


@pytest.mark.parametrize("bits,key_bits,n", [(4, 24, 300_000), (6, 24, 1_000_000), (8, 24, 5_000_000), (8, 32, 1_000_003)])
def test_radix_sort_stable(bits, key_bits, n):
    import torch
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(bits * 1000 + n)
    keys = rng.integers(0, 1 << key_bits, n, dtype=np.uint64).astype(np.uint32)
    keys[:: 7] = keys[0]  # many equal keys: stability matters
    vals = np.arange(n, dtype=np.uint32)
    r = _renderer()
    r.set_sort_digit_bits(bits)
    ki = torch.from_numpy(keys.view(np.int32).copy()).to(dev)
    vi = torch.from_numpy(vals.view(np.int32).copy()).to(dev)
    ko, vo = torch.empty_like(ki), torch.empty_like(vi)
    L = PKG.abi.lib()
    assert L.gpsb_sort_pairs(r.handle, C.c_void_p(ki.data_ptr()), C.c_void_p(vi.data_ptr()), C.c_void_p(ko.data_ptr()),
                             C.c_void_p(vo.data_ptr()), n, key_bits) == 0
    r.wait_idle()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(vo.cpu().numpy().view(np.uint32), vals[order])
    assert np.array_equal(ko.cpu().numpy().view(np.uint32), keys[order])
    r.close()
