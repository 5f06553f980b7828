"""gpsb_sort_pairs_noalloc: the radix sort for callers that cannot allocate device memory.

Some hosts own the whole GPU memory budget through their own pool, or run a real-time frame loop
in which a cudaMalloc would stall or is not allowed; they sort through this entry point, whose
scratch is a fixed array inside the library. The test sorts, through the C ABI, the same
(depth key, splat id) pairs that the existing sorted-path entry point (gpsb_render_sorted, read
back with gpsb_read_sorted) sorts with its own allocated scratch, and requires identical output
on two calls in a row (different scenes, so the second call must not see the first call's
scratch contents). This file is collected last on purpose.
"""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

PKG = load_package()


def _crowd(n, seed):
    rng = np.random.default_rng(seed)
    g = np.zeros((n, 16), np.float32)
    g[:, 0:2] = rng.uniform(-1.3, 1.3, (n, 2))
    g[:, 2] = rng.uniform(4.0, 9.0, n)
    g[:, 3] = rng.uniform(0.2, 0.9, n)
    s = rng.uniform(0.01, 0.24, n)
    g[:, 4] = np.log(s)
    g[:, 5] = np.log(s * rng.uniform(0.3, 1.3, n))
    g[:, 6] = np.log(s * 0.5)
    q = rng.normal(size=(n, 4))
    g[:, 8:12] = q / np.linalg.norm(q, axis=1, keepdims=True)
    g[:, 12:15] = rng.uniform(0.0, 1.0, (n, 3))
    return g


def _reference_sort(g):
    """Sorted (keys, values) of the existing entry point and the unsorted pairs it sorted."""
    r = PKG.GpsRenderer(128, 96, 1)
    r.set_gaussians(g)
    r.render_sorted(PKG.OracleCamera(focal_x=150.0, focal_y=150.0), PKG.RenderParams(spp_side=1), 1)
    keys, vals = r.read_sorted()
    r.close()
    n = len(g)
    assert sorted(vals.tolist()) == list(range(n))
    key_of = np.empty(n, np.uint32)
    key_of[vals] = keys
    return keys, vals, key_of, np.arange(n, dtype=np.uint32)


def _noalloc_sort(keys_in, vals_in, key_bits, with_err=True):
    import torch
    L = PKG.abi.lib()
    dev = torch.device("cuda", 0)
    ki = torch.from_numpy(keys_in.view(np.int32).copy()).to(dev)
    vi = torch.from_numpy(vals_in.view(np.int32).copy()).to(dev)
    ko = torch.empty_like(ki)
    vo = torch.empty_like(vi)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = L.gpsb_sort_pairs_noalloc(C.c_void_p(ki.data_ptr()), C.c_void_p(vi.data_ptr()), C.c_void_p(ko.data_ptr()),
                                   C.c_void_p(vo.data_ptr()), len(keys_in), key_bits, C.c_void_p(stream.cuda_stream),
                                   C.c_void_p(err.data_ptr()) if with_err else None)
    if not with_err:
        return st, L.gpsb_last_error(None).decode()
    assert st == 0, L.gpsb_last_error(None).decode()
    torch.cuda.synchronize(dev)
    assert int(err.item()) == 0
    return ko.cpu().numpy().view(np.uint32), vo.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_the_sorted_path_twice():
    for n, seed in [(300_000, 5), (3000, 6)]:  # the second call follows a larger one: scratch reuse
        keys, vals, keys_in, vals_in = _reference_sort(_crowd(n, seed))
        ko, vo = _noalloc_sort(keys_in, vals_in, 24)
        assert np.array_equal(ko, keys), f"n={n}: keys differ"
        assert np.array_equal(vo, vals), f"n={n}: values differ (the sort must be stable)"


@pytest.mark.parametrize("key_bits", [16, 32, 7])
def test_noalloc_sort_every_pass_parity(key_bits):
    """Two and four 8-bit passes (an even count starts from a copy of the input in the output
    buffers) and one pass, against numpy's stable argsort, twice in a row."""
    for n, seed in [(200_003, key_bits), (4099, key_bits + 1)]:
        rng = np.random.default_rng(seed)
        keys = rng.integers(0, 1 << key_bits, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 5] = keys[n // 3]  # long runs of equal keys: stability matters
        vals = rng.permutation(n).astype(np.uint32)
        order = np.argsort(keys, kind="stable")
        ko, vo = _noalloc_sort(keys, vals, key_bits)
        assert np.array_equal(ko, keys[order]), f"key_bits={key_bits} n={n}: keys differ"
        assert np.array_equal(vo, vals[order]), f"key_bits={key_bits} n={n}: values differ"


def test_noalloc_sort_requires_an_error_word():
    keys = np.arange(100, dtype=np.uint32)[::-1].copy()
    st, msg = _noalloc_sort(keys, keys.copy(), 8, with_err=False)
    assert st == 1 and "error word" in msg  # GPSB_ERR_INVALID_ARGUMENT


def test_noalloc_sort_rejects_sizes_above_its_scratch():
    L = PKG.abi.lib()
    st = L.gpsb_sort_pairs_noalloc(None, None, None, None, (1 << 21) + 1, 24, None, None)
    assert st == 2  # GPSB_ERR_LIMIT
    assert "exceed" in L.gpsb_last_error(None).decode()
