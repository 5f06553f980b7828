"""Autotuner of the renderer's launch shapes, per (Gaussian count, resolution, method, path).

For the particle path it sweeps items per thread {8, 16, 24} x particle blocks per SM {4, 5, 6}
and times a short trajectory through the captured CUDA graph (gpsb_render_trajectory_graph); for
the depth-sorted path (GPS) it sweeps radix digit width {4, 6, 8} x blend tiles {16x16, 32x8,
32x32} and times render_sorted. Timing: CUDA events on the renderer's stream, median of `reps`
after one warm-up. The best shape per key is cached in a JSON file and applied with
GpsRenderer.set_tuning.
"""
import json
import math
import os
import statistics

PARTICLE_SPACE = [{"particle_items": i, "particle_blocks_per_sm": b} for i in (8, 16, 24) for b in (4, 5, 6)]
SORTED_SPACE = [{"sort_digit_bits": d, "blend_tile_w": w, "blend_tile_h": h}
                for d in (4, 6, 8) for (w, h) in ((16, 16), (32, 8), (32, 32))]


def key(n_splats, width, height, method, sorted_path):
    """Cache key: the Gaussian count rounded to a power of two, the resolution, method and path."""
    nb = 1 << max(0, int(round(math.log2(max(n_splats, 1)))))
    return f"m{int(method)}-{'sorted' if sorted_path else 'particle'}-{width}x{height}-n{nb}"


def _time(stream, fn, reps):
    import torch
    fn()  # warm-up (and graph capture)
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return statistics.median(out)


def tune(renderer, cams, params, *, ensembles=4, sorted_path=False, reps=3, space=None):
    """Times every shape of the space on `cams` (OracleCameras of the renderer's size) and returns
    (best shape, [(shape, ms)]). The renderer must run on a created stream (set_stream)."""
    import torch
    w, h = renderer.size()
    stream = torch.cuda.current_stream()
    renderer.set_stream(stream.cuda_stream)
    space = space or (SORTED_SPACE if sorted_path else PARTICLE_SPACE)
    before = renderer.tuning()
    results = []
    out = torch.zeros(len(cams) * w * h * 4, device="cuda")
    for shape in space:
        renderer.set_tuning(**shape)
        if sorted_path:
            def run():
                for c in cams:
                    renderer.reset_accum()
                    renderer.render_sorted(c, params, ensembles)
        else:
            def run():
                renderer.render_trajectory_graph(cams, params, 1, ensembles, out.data_ptr())
        results.append((shape, _time(stream, run, reps)))
    best = min(results, key=lambda t: t[1])[0]
    renderer.set_tuning(**{k: v for k, v in before.items() if k in best})
    return best, results


def load_cache(path):
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def tuned(renderer, cams, params, n_splats, *, sorted_path=False, cache_path=None, **kw):
    """The cached best shape for this workload (tuning it first when missing), applied to the renderer."""
    w, h = renderer.size()
    k = key(n_splats, w, h, params.method, sorted_path)
    cache = load_cache(cache_path)
    if k not in cache:
        best, results = tune(renderer, cams, params, sorted_path=sorted_path, **kw)
        cache[k] = {"best": best, "ms": {json.dumps(s, sort_keys=True): ms for s, ms in results}}
        if cache_path:
            with open(cache_path, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
    renderer.set_tuning(**cache[k]["best"])
    return cache[k]["best"]
