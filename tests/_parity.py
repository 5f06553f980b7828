"""Shared helpers of the GPU parity tests: run the CUDA renderer through the C ABI and the O2
mirror oracle on the same inputs and compare bit for bit."""
import numpy as np

import oracle as O
from conftest import load_package

PKG = load_package()
LUT = None


def lut():
    global LUT
    if LUT is None:
        LUT = O.radius_lut()
    return LUT


def cuda_render(splats, sh, degree, W, H, side, cam, params, first_seed, count, want_debug=True, renderer=None):
    r = renderer or PKG.GpsRenderer(W, H, side)
    if renderer is None:
        if sh is not None and degree:
            r.set_gaussians_sh(splats, sh, degree)
        else:
            r.set_gaussians(splats)
    r.render_ensembles(cam, params, first_seed, count)
    acc = r.read_accum()
    st = r.read_stats()
    counts = packed = None
    if want_debug:
        particle = params.path == PKG.RenderPath.Particle or params.method != PKG.Method.Gps
        counts = np.stack([r.debug_counts(e) for e in range(count)]) if particle and len(splats) else None
        packed = np.stack([r.debug_subpixels(e) for e in range(count)])
    return r, acc, st, counts, packed


def o2_render(splats, sh, degree, W, H, side, cam, params, first_seed, count):
    return O.o2_render_ensembles(splats, sh, degree, lut(), W, H, side, cam.to_array(), params.to_c(), first_seed,
                                 count, want_counts=True, want_packed=True)


def stats_tuple(st):
    return (st.points, st.truncated_splats, st.dropped_points, st.visible_splats, st.orphan_subpixels, st.candidates,
            st.undercovered_splats, st.skipped_ensembles, st.ensembles, st.probe_demand, st.subpixel_writes,
            st.list_entries)


def assert_bit_exact(splats, sh, degree, W, H, side, cam, params, first_seed=1, count=3):
    r, acc, st, counts, packed = cuda_render(splats, sh, degree, W, H, side, cam, params, first_seed, count)
    oacc, ost, ocounts, opacked = o2_render(splats, sh, degree, W, H, side, cam, params, first_seed, count)
    if counts is not None:
        bad = np.argwhere(counts != ocounts)
        assert bad.size == 0, f"{len(bad)} per-splat counts differ, first {bad[:5].tolist()}"
    diff = np.argwhere(packed != opacked)
    assert diff.size == 0, f"{len(diff)} subpixel winners differ, first {diff[:5].tolist()}: " \
        f"{[hex(int(packed[tuple(d)])) for d in diff[:3]]} vs {[hex(int(opacked[tuple(d)])) for d in diff[:3]]}"
    assert stats_tuple(st) == tuple(int(x) for x in ost), (stats_tuple(st), ost.tolist())
    eq = acc.view(np.uint32) == oacc.view(np.uint32)
    assert eq.all(), f"{(~eq).sum()} accum words differ; max abs {np.abs(acc - oacc).max()}"
    r.close()
    return acc, st
