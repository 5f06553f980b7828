"""Benchmark of the stochastic particle-rendering path on B200.

Workload (the reference's 560k-Gaussian benchmark configuration, synthesised): 560,000 synthetic
Gaussians (64 anisotropic clusters + 10% background, SH degree 3), PBVR Extinction C3+R, spp 1,
per-splat cap 16,384, 1280x720, 64 ensembles at each of three orbit distances (near 2.5, mid 7,
far 20). One step renders the 64 ensembles of all three views (192 ensembles); the metric is
whole-job ensembles per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU (torchrun, one rank per GPU): every rank renders its own ensembles (seeds offset by
rank) of the same views: weak scaling, no collective on the data path; the timed region is
bracketed by a barrier + synchronize and the max over ranks is reported.
`--impl reference` times the reference's CPU implementation of the path (the C++ port of
gps-core's render_particles_3d, oracle/o1_core.cpp) on all host cores, on rank 0 only; it reads
the scene with the oracle's PLY reader and builds the cameras with O1's camera code, so the
renderer library is never loaded on that arm.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, SIDE, ENS, CAP, N_SPLATS = 1280, 720, 1, 64, 16384, 560_000
VIEWS = (("near", 2.5), ("mid", 7.0), ("far", 20.0))


def load_package():
    import importlib.util
    name = "gps_pbvr_web_b200"
    if name in sys.modules:
        return sys.modules[name]
    d = os.path.join(ROOT, "gps-pbvr-web_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload_config():
    return {"workload": "PBVR Extinction C3+R, 560k synthetic Gaussians (64 clusters + 10% background, SH3), "
                        "1280x720 spp1, cap 16384, 64 ensembles x near/mid/far orbit (2.5/7/20)",
            "gaussians": N_SPLATS, "resolution": [W, H], "spp_side": SIDE, "ensembles_per_view": ENS,
            "views": [v for v, _ in VIEWS], "cap": CAP, "method": "PBVR Extinction C3+R", "sh_degree": 3,
            "l2": "inputs larger than L2 (64 subpixel buffers = 472 MB per view, scene 136 MB)"}


def build_scene(pkg):
    from gps_pbvr_web_b200 import scenes
    ply = scenes.cluster_scene(N_SPLATS, seed=0, degree=3)
    return pkg.load_ply(ply)


def params(pkg):
    p = pkg.RenderParams(spp_side=SIDE, max_points_per_splat=CAP, method=pkg.Method.Extinction)
    p.pbvr.calibration = pkg.Calibration.PerSplatFootprint
    p.pbvr.radial_correction = True
    return p


def cameras(pkg, views=None):
    out = []
    for name, d in VIEWS:
        if views and name not in views:
            continue
        cam = pkg.OrbitCamera(target=(0.0, 0.0, 0.0), distance=d, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0), fov_y=0.9)
        out.append((name, cam.to_camera(W, H)))
    return out


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        res = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows)}
        if not self.rows:
            return res
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        res["sm_mhz"] = statistics.median(loaded) if loaded else None
        res["sm_max_mhz"] = max(mx) if mx else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for k, n in enumerate(names):
            if any(r[4 + k].lower() == "active" for r in self.rows):
                res["reasons"].append(n)
        return res


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "of measured"
    except Exception:
        return 6650.0, "of fallback"


def committed_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/traffic.md), or None."""
    import re
    path = os.path.join(ROOT, "profiles", "traffic.md")
    try:
        for line in open(path):
            m = re.match(r"\|\s*(\S+)\s*\|\s*([0-9.eE+]+)\s*\|", line)
            if m and m.group(1) == kernel:
                return float(m.group(2))
    except OSError:
        pass
    return None


def issue_roofline(st, ms, world, clk):
    """The particle kernel is bound by instruction issue, not HBM: generated particles per second
    (live) x warp instructions per particle (ncu, committed) against the SMs' issue peak (148 SMs x
    4 schedulers x one warp instruction per clock at the median SM clock sampled in the timed
    region)."""
    per = committed_traffic("k_particles_warp_inst_per_particle")
    mhz = clk.get("sm_mhz") if clk else None
    if not per or not mhz or not st.particles:
        return None
    achieved = st.particles / (ms / 1000.0) * per  # per GPU: st and ms are this rank's
    peak = 148 * 4 * mhz * 1e6
    return {"kernel": "k_particles", "unit": "warp instructions/s", "achieved": achieved, "peak": peak,
            "frac": achieved / peak, "warp_inst_per_particle": per,
            "note": "particles and time live; instructions per particle from ncu on the near view (estimate)"}


# ------------------------------------------------------------------------------ CPU reference
def scenes_module():
    """gps-pbvr-web_b200/scenes.py loaded on its own (numpy only): the reference arm builds its scene
    without importing the renderer package."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_gpsb_scenes", os.path.join(ROOT, "gps-pbvr-web_b200", "scenes.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_inputs():
    """The workload for the CPU arm, through the oracle alone: the seeded scene read by the oracle's
    PLY reader (a restatement of gps-io) and the orbit cameras built by O1's camera code (a
    restatement of gps-core's camera.rs), both equal to what the renderer receives."""
    import oracle as O
    from oracle import ply
    g, _, _, _ = ply.read_ply(scenes_module().cluster_scene(N_SPLATS, seed=0, degree=3))
    cams = []
    for name, d in VIEWS:
        eye = O.orbit_eye((0.0, 0.0, 0.0), d, 0.6, 0.25, (0.0, -1.0, 0.0))
        cams.append((name, O.look_at(eye, (0.0, 0.0, 0.0), (0.0, -1.0, 0.0), 0.9, W, H)))
    return g, cams


def o1_call(g, cam17, seed):
    """Wall seconds of one O1 render_particles_3d call (the C++ port of gps-core, with the GPU's
    per-splat cap): one ensemble of the splats g on one thread."""
    import oracle as O
    from oracle import ply
    sc = ply.o1_scene(g)
    t = time.perf_counter()
    O.render_particles_3d(sc, cam17, W, H, SIDE, 1, (0.05, 0.05, 0.08), seed, level=3, rule=1, radial_correction=True,
                          per_particle_seed=True, threads=1, max_points_per_splat=CAP)
    return time.perf_counter() - t


def o1_concurrent(parts, cam17, first_seed):
    """Runs o1_call on every splat array of `parts` at once, one host thread each (the calls release
    the interpreter lock); returns their wall times."""
    out = [0.0] * len(parts)

    def run(k):
        out[k] = o1_call(parts[k], cam17, first_seed + k)

    ths = [threading.Thread(target=run, args=(k,)) for k in range(len(parts))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return out


def cpu_reference(g, cams, threads, stride=64, step=0):
    """Full-scene seconds per ensemble of each view, all host threads busy. Thread t renders one
    ensemble of its own uniform 1/stride subset of the splats (subset (step * threads + t) mod
    stride, disjoint across threads; the generator shuffles splats), so the sample averages over
    `threads` subsets; the per-ensemble fixed cost a (framebuffer set-up and resolve, measured the
    same way on one splat) is not multiplied: full = a + stride (mean t - a), and with all threads
    busy the job renders `threads` such ensembles in that time. Returns (ensembles/s, per-view
    ms/ensemble, per-view fixed ms, per-view coefficient of variation of the subsets' per-splat
    times)."""
    per_view, fixed, spread = {}, {}, {}
    total = 0.0
    for name, cam in cams:
        a = statistics.median(o1_concurrent([g[:1]] * threads, cam, 1))
        parts = [g[((step * threads + t) % stride)::stride] for t in range(threads)]
        ts = o1_concurrent(parts, cam, 1 + step * threads)
        var = [max(t - a, 0.0) for t in ts]
        mean = statistics.fmean(var)
        full = a + stride * mean  # one full-scene ensemble on one thread
        s_per_ens = full / threads
        per_view[name] = 1000.0 * s_per_ens
        fixed[name] = 1000.0 * a
        spread[name] = statistics.pstdev(var) / max(mean, 1e-12)
        total += s_per_ens
    return len(cams) / total, per_view, fixed, spread


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    g, cams = reference_inputs()
    threads = os.cpu_count() or 1
    stride = int(round(1.0 / args.cpu_fraction))
    for k in range(args.warmup):
        cpu_reference(g, cams, threads, stride, k)
    rates, views, fixed, spread = [], [], [], []
    t0 = time.perf_counter()
    for k in range(args.steps):
        r, v, a, sp = cpu_reference(g, cams, threads, stride, args.warmup + k)
        rates.append(r)
        views.append(v)
        fixed.append(a)
        spread.append(sp)
    wall = time.perf_counter() - t0
    value = statistics.median(rates)
    sample = (f"per view {threads} host threads, each rendering one ensemble of its own disjoint 1/{stride} splat "
              f"subset; full-scene time = fixed per-ensemble cost (measured on one splat) + {stride} x the mean "
              f"per-splat part; successive steps take the next subsets")
    line = {"impl": "reference", "metric": "ensembles/s (PBVR Ext C3+R, 560k Gaussians SH3, 1280x720, near/mid/far)",
            "value": value, "unit": "ensembles/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * wall / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(),
            "ms_per_ensemble": {k: statistics.median([v[k] for v in views]) for k in views[0]},
            "fixed_ms_per_call": {k: statistics.median([v[k] for v in fixed]) for k in fixed[0]},
            "subset_cv": {k: max(v[k] for v in spread) for k in spread[0]},
            "cpu_baseline": {"value": value, "unit": "ensembles/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "ensembles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------ GPU arm
def algorithmic_bytes_per_launch(stage, writes, entries, E, n_splats, P):
    """Bytes one launch of `stage` must move (the roofline basis, one view of E ensembles):
    writes / entries = on-screen particle writes and compact-list entries of that launch."""
    if stage == "particles":   # one 8-byte atomicMin per written particle, list entry + 96-byte record per entry
        return 8.0 * writes + (8.0 + 96.0) * entries
    if stage == "count_scan":  # 8-byte count descriptor per splat and ensemble, 8-byte list entry written
        return 8.0 * n_splats * E + 8.0 * entries
    if stage == "resolve":     # every subpixel word of every ensemble, accum read + write
        return 8.0 * P * SIDE * SIDE * E + 32.0 * P
    if stage == "clear":       # every subpixel word of every ensemble
        return 8.0 * P * SIDE * SIDE * E
    if stage == "geometry":    # splat + SH3 read, record + descriptor + colour written
        return (64.0 + 180.0 + 96.0 + 8.0 + 16.0) * n_splats
    return 0.0


def micro_scan_sort(pkg, r, stream, peak):
    """HBM throughput of the two data-movement primitives at sizes far above L2:
    exclusive scan of 2^28 u32 counts (8 algorithmic bytes per element: read + write) and the
    stable radix sort of 2^26 (24-bit key, value) pairs with 8-bit digits (4 bytes of histogram read
    + 3 passes x 16 bytes of key/value read and write = 52 bytes per pair)."""
    import ctypes as C
    import torch
    L = pkg.abi.lib()
    out = {}
    n = 1 << 28
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randint(0, 16, (n,), dtype=torch.int32, device="cuda", generator=g)
    y = torch.empty_like(x)
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    def scan():
        assert L.gpsb_scan_u32(r.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), n, C.c_void_p(tot.data_ptr())) == 0
    ms = _time_events(scan, stream, 3, 10)
    out["scan_u32"] = {"n": n, "ms": ms, "alg_bytes": 8 * n, "GBps": 8 * n / (ms / 1e3) / 1e9,
                       "frac": 8 * n / (ms / 1e3) / 1e9 / peak}
    del x, y
    n = 1 << 26
    keys = torch.randint(0, 1 << 24, (n,), dtype=torch.int32, device="cuda", generator=g)
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ka, va, kb, vb = keys.clone(), vals.clone(), torch.empty_like(keys), torch.empty_like(vals)
    for bits in (8, 6, 4):
        r.set_tuning(sort_digit_bits=bits)
        passes = -(-24 // bits)
        def sort():
            ka.copy_(keys)
            va.copy_(vals)
        def run():
            assert L.gpsb_sort_pairs(r.handle, C.c_void_p(ka.data_ptr()), C.c_void_p(va.data_ptr()),
                                     C.c_void_p(kb.data_ptr()), C.c_void_p(vb.data_ptr()), n, 24) == 0
        # inputs are clobbered by the ping-pong passes: restore them outside the timed region
        tms = []
        for k in range(6):
            sort()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run()
            b.record(stream)
            torch.cuda.synchronize()
            if k >= 2:
                tms.append(a.elapsed_time(b))
        ms = statistics.median(tms)
        alg = (4 + 16 * passes + (8 if passes % 2 == 0 else 0)) * n
        out[f"sort_pairs_{bits}bit"] = {"n": n, "ms": ms, "alg_bytes": alg, "GBps": alg / (ms / 1e3) / 1e9,
                                        "frac": alg / (ms / 1e3) / 1e9 / peak}
    r.set_tuning(sort_digit_bits=8)
    # the sort by time: the fastest digit width against the fewest algorithmic bytes (8-bit digits:
    # 4 B histogram read + 3 passes x 16 B = 52 B per pair), so extra passes do not count as bandwidth
    best = min((k for k in out if k.startswith("sort_pairs_")), key=lambda k: out[k]["ms"])
    alg8 = 52 * n
    out["sort_pairs_by_time"] = {"n": n, "fastest": best, "ms": out[best]["ms"], "alg_bytes": alg8,
                                 "GBps": alg8 / (out[best]["ms"] / 1e3) / 1e9,
                                 "frac": alg8 / (out[best]["ms"] / 1e3) / 1e9 / peak}
    return out


def equal_psnr_target(ms_per_ensemble, denoiser_ms, psnr_denoised, plain_ensembles, target=8.0):
    """Whether the denoised frame (4 ensembles + the network) is at least `target` times faster than
    the plain accumulation of equal PSNR, and if not, the measured reason in one sentence."""
    frame = 4 * ms_per_ensemble + denoiser_ms
    if plain_ensembles is None:
        return {"target": target, "met": None,
                "why_not": f"the plain curve does not reach the denoised {psnr_denoised:.1f} dB within its largest "
                           "measured count, so the speed-up is larger than the curve can show"}
    plain = plain_ensembles * ms_per_ensemble
    speedup = plain / frame
    if speedup >= target:
        return {"target": target, "met": True, "why_not": None}
    return {"target": target, "met": False,
            "why_not": f"the plain path matches the denoised {psnr_denoised:.1f} dB after {plain_ensembles:.0f} "
                       f"ensembles = {plain:.2f} ms, while the denoised frame costs {4 * ms_per_ensemble:.2f} ms of "
                       f"rendering (4 ensembles at {ms_per_ensemble:.3f} ms) + {denoiser_ms:.2f} ms of network: "
                       f"{speedup:.1f}x"}


def denoise_measure(pkg, r, stream, cams, p, per_view_ms, ref_ens=256, w=None, h=None,
                    counts=(4, 8, 16, 32, 64, 128, 256, 512), big_ref=4096, big_ref_views=("mid", "far")):
    """The "ms to PSNR vs the 256-ensemble reference: denoised batch vs plain" comparison, per view:
    the 4-ensemble frame through the trained denoiser (committed weights) against the plain
    accumulation. PSNR (peak 1, linear RGB clamped to [0, 1]) against a 256-ensemble reference with
    disjoint seeds; the plain path's PSNR is measured at every count of `counts`, and the ensembles
    it needs to match the denoised PSNR are read off that measured curve (interpolated in log n
    between measured counts; the fitted error model MSE(N) = s2 (1/N + 1/256) is reported beside
    it). For the views in big_ref_views the denoised and plain frames are also compared with a
    `big_ref`-ensemble reference, whose own noise is 1/16 of the 256-ensemble one, and the plain
    curve extends to 1024 ensembles: there the 40 dB question has a measured answer. Each view
    states whether the denoised frame is >= 8x faster than the plain one of equal PSNR, and if not,
    the measured reason. Times are ensembles x the view's ms per ensemble of this run,
    plus the denoiser's GPU time."""
    import torch
    from gps_pbvr_web_b200 import denoise as dn
    from gps_pbvr_web_b200 import denoise_train as T
    nat = dn.NativeDenoiser()
    gate = nat.gate_limit
    out = {"weights": "gps-pbvr-web_b200/weights/denoiser_pbvr_c3r.npz", "engine": "tma+graph (C ABI)",
           "reference_ensembles": ref_ens, "input_ensembles": 4, "big_reference_ensembles": big_ref, "views": {}}
    w, h = w or W, h or H
    P = w * h
    with torch.cuda.stream(stream):
        for name, cam in cams:
            r.reset_accum()
            r.render_ensembles(cam, p, 5_000_000, ref_ens)
            ref = T.mean_rgb(torch.from_numpy(r.read_accum()).cuda())
            feat = torch.zeros(P * 8, device="cuda")
            r.reset_accum()
            r.set_feature_accum(feat)
            r.render_ensembles(cam, p, 6_000_000, 4)
            r.set_feature_accum(None)
            acc = torch.from_numpy(r.read_accum()).cuda()
            x = torch.zeros(P, 8, dtype=torch.bfloat16, device="cuda")
            base = torch.zeros(P, 3, device="cuda")
            dn.pack(acc, feat, x, base)
            ok, check = T.variance_gate(x, gate)
            # the network through the C ABI (gpsb_denoiser_forward: input copies, the U-Net as one
            # replayed CUDA graph, output copy, error-word read): GPU time of each call on `stream`
            pred = torch.empty(1, h, w, 3, device="cuda")
            for _ in range(3):  # first call of a frame size: direct launches, then the capture
                nat.forward(x.view(1, h, w, 8), base.view(1, h, w, 3), pred)
            ts = []
            for _ in range(10):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                nat.forward(x.view(1, h, w, 8), base.view(1, h, w, 3), pred)
                b.record(stream)
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b))
            dn_ms = statistics.median(ts)
            out["graph_state"] = nat.graph_state()  # 1: the timed calls replayed the captured graph
            pred = pred.reshape(P, 3).clone()
            ps_dn, me_dn = T.psnr(pred, ref)
            view_counts = list(counts)
            if name in big_ref_views and big_ref and view_counts[-1] < 1024:
                view_counts.append(1024)  # extends the plain curve against the big reference past 40 dB at mid
            prog = T.progressive(r, cam, p, 6_000_000, view_counts)
            curve = {n: T.psnr(T.mean_rgb(v), ref)[0] for n, v in prog.items()}
            s2 = T.noise_model(curve, ref_ens)
            n_model = T.n_model(s2, ref_ens, ps_dn)
            n_same = T.n_to_reach(curve, ps_dn)
            ms_ens = per_view_ms[name]
            frame_ms = 4 * ms_ens + dn_ms
            row = {
                "psnr_denoised": ps_dn, "maxerr_denoised": me_dn, "psnr_plain": curve,
                "psnr_ceiling_vs_reference": 10.0 * math.log10(ref_ens / s2), "variance_check_passed": ok,
                "denoiser_ms": dn_ms, "denoised_frame_ms": frame_ms,
                "plain_ensembles_for_same_psnr": n_same, "plain_ensembles_for_same_psnr_model": n_model,
                "plain_ms_for_same_psnr": None if n_same is None else n_same * ms_ens,
                "speedup_at_same_psnr": None if n_same is None else n_same * ms_ens / frame_ms,
                "reaches_40db": {"denoised": ps_dn >= 40.0, "plain_max_measured": max(curve.values()) >= 40.0},
                "equal_psnr_8x": equal_psnr_target(ms_ens, dn_ms, ps_dn, n_same)}
            if name in big_ref_views and big_ref:
                r.reset_accum()
                r.render_ensembles(cam, p, 20_000_000, big_ref)
                bref = T.mean_rgb(torch.from_numpy(r.read_accum()).cuda())
                ps_b, me_b = T.psnr(pred, bref)
                curve_b = {n: T.psnr(T.mean_rgb(v), bref)[0] for n, v in prog.items()}
                n_b = T.n_to_reach(curve_b, ps_b)
                n40 = T.n_to_reach(curve_b, 40.0)
                row["vs_big_reference"] = {
                    "psnr_denoised": ps_b, "maxerr_denoised": me_b, "psnr_plain": curve_b,
                    "plain_ensembles_for_same_psnr": n_b,
                    "speedup_at_same_psnr": None if n_b is None else n_b * ms_ens / frame_ms,
                    "plain_ensembles_for_40db": n40,
                    "plain_ms_for_40db": None if n40 is None else n40 * ms_ens,
                    "reaches_40db": {"denoised": ps_b >= 40.0, "plain_max_measured": max(curve_b.values()) >= 40.0},
                    "equal_psnr_8x": equal_psnr_target(ms_ens, dn_ms, ps_b, n_b)}
            out["views"][name] = row
    nat.close()
    return out


def _time_events(fn, stream, warmup, reps):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def run_trajectory(args, rank, world):
    """Configuration 3 (one line, not the default): the cluster generator scaled to 2,000,000
    Gaussians (SH3) at 1920x1080, a 360-degree orbit of 16 cameras x E ensembles (distance 7)
    rendered through one captured CUDA graph, for PBVR Extinction C3+R and ScreenOccupancy, with
    the launch shape chosen by the autotuner (sweep on 2 cameras x 2 ensembles)."""
    import torch
    pkg = load_package()
    from gps_pbvr_web_b200 import autotune, scenes
    n, Wt, Ht, ncam = args.traj_gaussians, 1920, 1080, 16
    splats, sh, deg = pkg.load_ply(scenes.cluster_scene(n, seed=0, degree=3))
    stream = torch.cuda.Stream()
    r = pkg.GpsRenderer(Wt, Ht, 1)
    r.set_stream(stream.cuda_stream)
    r.set_gaussians_sh(splats, sh, deg)
    cams = [pkg.OrbitCamera(target=(0.0, 0.0, 0.0), distance=7.0, yaw=2 * math.pi * k / ncam, pitch=0.25,
                            up=(0.0, -1.0, 0.0), fov_y=0.9).to_camera(Wt, Ht) for k in range(ncam)]
    out = torch.zeros(ncam * Wt * Ht * 4, device="cuda")
    E = args.ensembles
    rows = {}
    clocks = ClockSampler(0)
    clocks.start()
    with torch.cuda.stream(stream):
        for name, method in (("PBVR Extinction C3+R", pkg.Method.Extinction), ("ScreenOccupancy", pkg.Method.ScreenOccupancy)):
            p = pkg.RenderParams(spp_side=1, max_points_per_splat=CAP, method=method)
            if method == pkg.Method.Extinction:
                p.pbvr.calibration = pkg.Calibration.PerSplatFootprint
                p.pbvr.radial_correction = True
            best, sweep = autotune.tune(r, cams[:2], p, ensembles=2, reps=2)
            r.set_tuning(**best)
            for _ in range(max(1, args.warmup)):  # the first call captures the graph
                r.render_trajectory_graph(cams, p, 1, E, out.data_ptr())
            torch.cuda.synchronize()
            l0 = r.profile()["total_launches"]
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                r.render_trajectory_graph(cams, p, 1, E, out.data_ptr())
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / args.steps
            rows[name] = {"ms_per_trajectory": ms, "gpu_launches_per_trajectory": (r.profile()["total_launches"] - l0) / args.steps, "ensembles_per_s": ncam * E / (ms / 1e3),
                          "ms_per_ensemble": ms / (ncam * E), "autotuned": best,
                          "sweep_ms": [[sh_, round(t, 3)] for sh_, t in sweep]}
    clk = clocks.stop()
    line = {"metric": "ensembles/s (trajectory, captured CUDA graph)", "clocks": clk, "value": rows["PBVR Extinction C3+R"]["ensembles_per_s"],
            "unit": "ensembles/s", "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup), "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": f"{n} synthetic Gaussians SH3, 1920x1080 spp1, cap {CAP}, 16-camera 360-degree orbit "
                                   f"(distance 7) x {E} ensembles, one captured CUDA graph per method",
                       "gaussians": n, "resolution": [Wt, Ht], "cameras": ncam, "ensembles_per_camera": E},
            "methods": rows}
    print(json.dumps(line))
    r.close()
    return 0


def run_stress(args, rank, world):
    """Configuration 5 (one line, not the default): the cluster generator scaled to 6,000,000
    Gaussians (SH3), PBVR Extinction C3+R with a per-splat cap of 65,536 at 3840x2160, near / mid /
    far orbit views. Per view: ms per ensemble of the plain path (CUDA events over 4 ensembles),
    the algorithmic GB/s of each stage, and the denoised 4-ensemble frame against the plain 64-
    and 256-ensemble accumulations (PSNR and max abs error against a reference of --stress-ref
    ensembles with disjoint seeds, ms per frame)."""
    import torch
    pkg = load_package()
    from gps_pbvr_web_b200 import scenes
    n = args.stress_gaussians
    sw, sh_ = (int(v) for v in args.stress_res.lower().split("x"))
    splats, sh, deg = pkg.load_ply(scenes.cluster_scene(n, seed=0, degree=3))
    stream = torch.cuda.Stream()
    r = pkg.GpsRenderer(sw, sh_, 1)
    r.set_stream(stream.cuda_stream)
    r.set_gaussians_sh(splats, sh, deg)
    p = pkg.RenderParams(spp_side=1, max_points_per_splat=args.stress_cap, method=pkg.Method.Extinction)
    p.pbvr.calibration = pkg.Calibration.PerSplatFootprint
    p.pbvr.radial_correction = True
    cams = [(name, pkg.OrbitCamera(target=(0.0, 0.0, 0.0), distance=d, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                                   fov_y=0.9).to_camera(sw, sh_)) for name, d in VIEWS]
    per_view, stages = {}, {}
    P = sw * sh_
    clocks = ClockSampler(0)
    clocks.start()
    for name, cam in cams:
        r.reset_accum()
        r.render_ensembles(cam, p, 1, 1)  # warm-up
        r.reset_stats()
        r.profile_enable(True)
        p0 = r.profile()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r.reset_accum()
        a.record(stream)
        r.render_ensembles(cam, p, 1, 4)
        b.record(stream)
        torch.cuda.synchronize()
        per_view[name] = a.elapsed_time(b) / 4
        prof, st = r.profile(), r.read_stats()
        rows = {}
        for sname in ["particles", "count_scan", "resolve", "clear", "geometry"]:
            launches = prof["launches"][sname] - p0["launches"][sname]
            ms = prof["ms"][sname] - p0["ms"][sname]
            if launches and ms > 0:
                byts = algorithmic_bytes_per_launch(sname, st.subpixel_writes / launches, st.list_entries / launches,
                                                    4, n, P)
                rows[sname] = {"ms": ms, "launches": launches, "alg_GBps": byts * launches / (ms / 1e3) / 1e9}
        # an ensemble whose particle total passes 2^32 - 1 is skipped (the reference's u32 rule,
        # gps_splat.wgsl:635-663); candidates is the particle demand before the per-splat cap
        stages[name] = {"stages": rows, "particles": st.particles, "points": st.points,
                        "subpixel_writes": st.subpixel_writes, "skipped_ensembles": st.skipped_ensembles,
                        "ensembles": st.ensembles, "candidates_before_cap": st.candidates}
    clk = clocks.stop()
    # reference ensembles per view (--stress-ref, overridden per view by --stress-ref-views)
    refs = {name: args.stress_ref for name, _ in cams}
    for item in filter(None, args.stress_ref_views.split(",")):
        k, v = item.split(":")
        refs[k] = int(v)
    dnz = {"views": {}, "reference_ensembles": refs, "input_ensembles": 4}
    for name, cam in cams:
        one = denoise_measure(pkg, r, stream, [(name, cam)], p, per_view, ref_ens=refs[name], w=sw, h=sh_,
                              counts=tuple(c for c in (4, 16, 64, 256) if c <= refs[name]), big_ref=0)
        dnz["views"][name] = one["views"][name]
        dnz["engine"] = one["engine"]
    line = {"metric": "stress: denoised 4-ensemble frames vs plain 64 / 256 ensembles", "unit": "dB, ms",
            "n_gpus": 1, "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": f"{n} synthetic Gaussians SH3, {sw}x{sh_} spp1, cap {args.stress_cap}, "
                                   "PBVR Extinction C3+R, near/mid/far orbit (2.5/7/20)",
                       "gaussians": n, "resolution": [sw, sh_], "cap": args.stress_cap,
                       "reference_ensembles": refs},
            "ms_per_ensemble": per_view, "per_view": stages, "clocks": clk, "denoise": dnz}
    print(json.dumps(line))
    r.close()
    return 0


def run_case(args):
    """Small single-kernel-family workloads for ncu captures (each a few launches of a case larger
    than the 126 MB L2 but a few GB at most on the device); prints the device error word:
      scan                 exclusive scan of 2^26 u32 counts, 3 times (k_scan_u32_staged)
      sort                 stable radix sort of 2^24 (24-bit key, value) pairs, 8-bit digits, 3 times
      denoise-train        two training steps of the denoiser on 2 x 256 x 256 crops
      denoise-infer        two 1280 x 720 inferences of the denoiser (conv3 and the element-wise steps)
      particles-near       PBVR Ext C3+R, 560k cluster scene, 1280 x 720, near view, 2 ensembles in one
                           launch of k_particles, fast decisions on
      particles-near-exact the same with the fast decisions off"""
    import ctypes as C
    import torch
    pkg = load_package()
    L = pkg.abi.lib()
    case = args.case
    g = torch.Generator(device="cuda").manual_seed(3)
    err = 0
    if case in ("scan", "sort"):
        r = pkg.GpsRenderer(16, 16, 1)
        if case == "scan":
            n = 1 << 26
            x = torch.randint(0, 16, (n,), dtype=torch.int32, device="cuda", generator=g)
            y = torch.empty_like(x)
            tot = torch.zeros(1, dtype=torch.int64, device="cuda")
            for _ in range(3):
                assert L.gpsb_scan_u32(r.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), n,
                                       C.c_void_p(tot.data_ptr())) == 0
        else:
            m = 1 << 24
            keys = torch.randint(0, 1 << 24, (m,), dtype=torch.int32, device="cuda", generator=g)
            vals = torch.arange(m, dtype=torch.int32, device="cuda")
            kb, vb = torch.empty_like(keys), torch.empty_like(vals)
            for _ in range(3):
                ka, va = keys.clone(), vals.clone()
                assert L.gpsb_sort_pairs(r.handle, C.c_void_p(ka.data_ptr()), C.c_void_p(va.data_ptr()),
                                         C.c_void_p(kb.data_ptr()), C.c_void_p(vb.data_ptr()), m, 24) == 0
                r.wait_idle()
        r.wait_idle()
        err = r.debug_error_word()
        r.close()
    elif case.startswith("denoise"):
        from gps_pbvr_web_b200 import denoise as dn
        net = dn.Denoiser()
        dn.load_weights(net)
        gc = torch.Generator().manual_seed(0)
        if case == "denoise-train":
            x0 = torch.zeros(2, 256, 256, 8)
            x0[..., :6] = torch.rand(2, 256, 256, 6, generator=gc)
            base = torch.rand(2, 256, 256, 3, generator=gc).cuda()
            x0 = x0.to(torch.bfloat16).cuda()
            for _ in range(2):
                net.train_step(x0, base, base, lr=1e-4)
        else:
            x = torch.rand(1, H, W, 8, generator=gc).to(torch.bfloat16).cuda()
            base = torch.zeros(1, H, W, 3, device="cuda")
            for _ in range(2):
                net.forward(x, base)
        torch.cuda.synchronize()
        err = net.error_word()
    else:
        splats, sh, deg = build_scene(pkg)
        cam = cameras(pkg, ["near"])[0][1]
        r = pkg.GpsRenderer(W, H, SIDE)
        r.set_gaussians_sh(splats, sh, deg)
        r.set_fast_decisions(0 if case == "particles-near-exact" else 1)
        r.render_ensembles(cam, params(pkg), 1, 2)
        torch.cuda.synchronize()
        err = r.debug_error_word()
        r.close()
    print(case, "error word", err)
    return 1 if err else 0


def run_b200(args, rank, world):
    import torch
    pkg = load_package()
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    splats, sh, deg = build_scene(pkg)
    cams = cameras(pkg, args.views)
    ENS = args.ensembles
    p = params(pkg)
    stream = torch.cuda.Stream(device=dev)
    r = pkg.GpsRenderer(W, H, SIDE, device=dev)
    r.set_stream(stream.cuda_stream)
    r.set_gaussians_sh(splats, sh, deg)
    from gps_pbvr_web_b200 import multi
    # weak scaling: every rank renders ENS ensembles per view; the ranks' seeds are disjoint
    seed0 = multi.rank_first_seed(1, world * ENS, world, rank)

    def step(seed):
        for _, cam in cams:
            r.reset_accum()
            r.render_ensembles(cam, p, seed, ENS)

    def barrier():
        if dist is not None:
            dist.barrier()

    for k in range(args.warmup):
        step(seed0)
    torch.cuda.synchronize()
    r.reset_stats()
    r.profile_enable(True)
    clocks = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        step(seed0)
    t_end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = t_start.elapsed_time(t_end)
    prof = r.profile()
    st = r.read_stats()
    ms = multi.max_over_ranks(ms, dist, device="cuda")
    ens_total = world * args.steps * len(cams) * ENS
    value = ens_total / (ms / 1000.0)

    # per-view breakdown (outside the timed region)
    per_view = {}
    for name, cam in cams:
        r.reset_accum()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r.render_ensembles(cam, p, seed0, ENS)
        b.record(stream)
        torch.cuda.synchronize()
        per_view[name] = a.elapsed_time(b) / ENS

    # roofline of the dominant kernel: algorithmic bytes per launch / average launch duration
    P = W * H
    views_per_step = len(cams)
    writes_pl = st.subpixel_writes / (args.steps * views_per_step)
    entries_pl = st.list_entries / (args.steps * views_per_step)
    stage = max(prof["ms"], key=lambda k: prof["ms"][k])
    avg_launch_ms = prof["ms"][stage] / max(prof["launches"][stage], 1)
    bytes_per_launch = algorithmic_bytes_per_launch(stage, writes_pl, entries_pl, ENS, len(splats), P)
    achieved = bytes_per_launch / (avg_launch_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peak()
    kernel_name = {"particles": "k_particles", "count_scan": "k_count_scan", "resolve": "k_resolve",
                   "geometry": "k_geometry", "clear": "memset"}.get(stage, stage)
    traffic = committed_traffic(kernel_name)
    stage_gbs = {}
    for sname in ["particles", "count_scan", "resolve", "clear", "geometry"]:
        if prof["launches"][sname]:
            b = algorithmic_bytes_per_launch(sname, writes_pl, entries_pl, ENS, len(splats), P)
            t_ms = prof["ms"][sname] / prof["launches"][sname]
            stage_gbs[sname] = {"ms_per_launch": t_ms, "alg_GBps": b / (t_ms / 1000.0) / 1e9,
                                "share": prof["ms"][sname] / max(sum(prof["ms"].values()), 1e-9)}

    # end to end through the public API: host scene upload, render, host readback, every step
    e2e = None
    if not args.no_e2e:
        pin_g = torch.from_numpy(splats.reshape(-1)).pin_memory()
        pin_s = torch.from_numpy(sh).pin_memory()
        out = torch.empty((P, 4), dtype=torch.float32).pin_memory()
        L = pkg.abi.lib()
        import ctypes as C
        pc = p.to_c()
        cc = [c.to_c() for _, c in cams]

        def ok(status):
            if status != 0:
                raise RuntimeError(L.gpsb_last_error(r.handle).decode())

        def e2e_step():
            ok(L.gpsb_set_gaussians_sh(r.handle, C.c_void_p(pin_g.data_ptr()), len(splats),
                                       C.c_void_p(pin_s.data_ptr()), pin_s.numel(), deg))
            for c in cc:
                ok(L.gpsb_reset_accum(r.handle))
                ok(L.gpsb_render_ensembles(r.handle, C.byref(c), C.byref(pc), seed0, ENS))
                ok(L.gpsb_read_accum(r.handle, C.c_void_p(out.data_ptr())))

        e2e_step()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_steps = max(1, min(args.steps, 5))
        for _ in range(e_steps):
            e2e_step()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        dt = multi.max_over_ranks(dt, dist, device="cuda")
        e2e = {"value": world * e_steps * len(cams) * ENS / dt, "unit": "ensembles/s",
               "h2d_bytes_per_step": int(splats.nbytes + sh.nbytes), "d2h_bytes_per_step": int(len(cams) * P * 16),
               "steps": e_steps, "timing": "host wall clock around synchronised steps"}

    prims = None
    if rank == 0 and not args.no_micro:
        prims = micro_scan_sort(pkg, r, stream, peak)

    dnz = None
    if rank == 0 and not args.no_denoise:
        dnz = denoise_measure(pkg, r, stream, cams, p, per_view)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        stride = int(round(1.0 / args.cpu_fraction))
        rg, rcams = reference_inputs()
        rate, cpu_views, cpu_fixed, cpu_spread = cpu_reference(rg, rcams, threads, stride, 0)
        cpu = {"value": rate, "unit": "ensembles/s", "cores": threads, "kind": "port",
               "sample": f"per view {threads} host threads, each rendering one ensemble of its own disjoint 1/{stride} "
                         f"splat subset; full-scene time = fixed per-ensemble cost (measured on one splat) + {stride} x "
                         f"the mean per-splat part",
               "ms_per_ensemble": cpu_views, "fixed_ms_per_call": cpu_fixed, "subset_cv": cpu_spread}

    if rank == 0:
        line = {"metric": "ensembles/s (PBVR Ext C3+R, 560k Gaussians SH3, 1280x720, near/mid/far)",
                "value": value, "unit": "ensembles/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
                "config": dict(workload_config(), views=[n for n, _ in cams], ensembles_per_view=ENS),
                "ms_per_ensemble": per_view,
                "particles_per_s": world * st.subpixel_writes / (ms / 1000.0) / 1.0,
                "points_per_s": world * st.points / (ms / 1000.0),
                "gaussians_per_s": world * args.steps * len(cams) * ENS * len(splats) / (ms / 1000.0),
                "roofline": {"bound": "hbm", "kernel": kernel_name, "achieved": achieved, "peak": peak,
                             "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic},
                "issue_roofline": issue_roofline(st, ms, world, clk),
                "generated_particles_per_s": world * st.particles / (ms / 1000.0),
                "stages": stage_gbs, "clocks": clk, "gpu_launches": prof["total_launches"],
                "stats_per_step": {"particles": st.particles / args.steps, "points": st.points / args.steps,
                                   "subpixel_writes": st.subpixel_writes / args.steps,
                                   "list_entries": st.list_entries / args.steps,
                                   "truncated_splats": st.truncated_splats / args.steps,
                                   "skipped_ensembles": st.skipped_ensembles},
                "primitives": prims, "denoise": dnz, "e2e": e2e, "cpu_baseline": cpu}
        print(json.dumps(line))
    r.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-micro", action="store_true", help="skip the scan/sort HBM measurements")
    ap.add_argument("--no-denoise", action="store_true", help="skip the denoised-vs-plain PSNR measurement")
    ap.add_argument("--config", default="default", choices=["default", "trajectory", "stress"],
                    help="trajectory: the 2M-Gaussian 1080p 16-camera orbit through one captured graph; "
                         "stress: the 6M-Gaussian 3840x2160 scene with the denoiser in the loop")
    ap.add_argument("--traj-gaussians", type=int, default=2_000_000)
    ap.add_argument("--stress-gaussians", type=int, default=6_000_000)
    ap.add_argument("--stress-res", default="3840x2160")
    ap.add_argument("--stress-cap", type=int, default=65536)
    ap.add_argument("--stress-ref", type=int, default=256, help="ensembles of the stress reference")
    ap.add_argument("--stress-ref-views", default="", help="per-view reference ensembles, e.g. near:64")
    ap.add_argument("--cpu-fraction", type=float, default=1.0 / 64, help="splat fraction each host thread renders")
    ap.add_argument("--views", default="near,mid,far", help="subset of the views (small profiling cases)")
    ap.add_argument("--ensembles", type=int, default=ENS, help="ensembles per view (small profiling cases)")
    ap.add_argument("--case", default=None,
                    choices=["scan", "sort", "denoise-train", "denoise-infer", "particles-near", "particles-near-exact"],
                    help="one small single-kernel-family workload for an ncu capture (no JSON line)")
    args = ap.parse_args()
    args.views = [v for v in args.views.split(",") if v]
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.case:
        return run_case(args)
    if args.config == "trajectory":
        return run_trajectory(args, rank, world)
    if args.config == "stress":
        return run_stress(args, rank, world)
    return run_b200(args, rank, world)


if __name__ == "__main__":
    sys.exit(main())
