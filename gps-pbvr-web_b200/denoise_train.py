"""Training pairs, training and evaluation of the learned denoiser (`denoise.Denoiser`).

Pairs come from the renderer itself: for a seeded synthetic scene (the cluster generator of
`scenes`) and a random orbit camera, the few-ensemble frame (its accumulation and feature sums,
packed by `denoise.pack`) is the input and a many-ensemble accumulation with disjoint seeds is the
target. Evaluation compares, on held-out cameras, the denoised few-ensemble frame and the plain
accumulation of N ensembles with a many-ensemble reference (PSNR with peak 1 on linear RGB
clamped to [0, 1], and the largest absolute error), and finds the ensemble count (and time) the
plain path needs to reach a PSNR.

Run as a program: python gps-pbvr-web_b200/denoise_train.py --out results.json --weights w.npz
"""
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _pkg():
    name = "gps_pbvr_web_b200"
    if name in sys.modules:
        return sys.modules[name]
    import importlib.util
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"), submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def params(pkg, cap=16384):
    """PBVR Extinction C3+R, spp 1 (the configuration the denoiser is trained for)."""
    p = pkg.RenderParams(spp_side=1, max_points_per_splat=cap, method=pkg.Method.Extinction)
    p.pbvr.calibration = pkg.Calibration.PerSplatFootprint
    p.pbvr.radial_correction = True
    return p


def random_cameras(pkg, n, W, H, rng, dmin=2.5, dmax=20.0):
    cams = []
    for _ in range(n):
        d = float(math.exp(rng.uniform(math.log(dmin), math.log(dmax))))
        cams.append((d, pkg.OrbitCamera(target=(0.0, 0.0, 0.0), distance=d, yaw=float(rng.uniform(0, 2 * math.pi)),
                                        pitch=float(rng.uniform(-0.6, 0.6)), up=(0.0, -1.0, 0.0),
                                        fov_y=0.9).to_camera(W, H)))
    return cams


class FrameRenderer:
    """A renderer with a feature buffer, rendering accumulations into CUDA tensors."""

    def __init__(self, pkg, W, H):
        import torch
        self.pkg, self.W, self.H = pkg, W, H
        self.r = pkg.GpsRenderer(W, H, 1)
        self.feat = torch.zeros(W * H * 8, device="cuda")

    def set_scene(self, splats, sh, deg):
        self.r.set_gaussians_sh(splats, sh, deg)

    def accum(self, cam, p, first_seed, count, features=False):
        """(accum (P, 4) CUDA tensor, feature sums or None, GPU ms of the render)."""
        import torch
        self.r.reset_accum()
        if features:
            self.feat.zero_()
        self.r.set_feature_accum(self.feat if features else None)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        self.r.render_ensembles(cam, p, first_seed, count)
        self.r.wait_idle()
        ms = (time.perf_counter() - t0) * 1e3
        a = torch.from_numpy(self.r.read_accum()).cuda()
        self.r.set_feature_accum(None)
        return a, (self.feat.clone() if features else None), ms

    def progressive(self, cam, p, first_seed, counts):
        self.r.set_feature_accum(None)
        return progressive(self.r, cam, p, first_seed, counts)


def progressive(r, cam, p, first_seed, counts):
    """Plain accumulations of renderer r after each of the increasing ensemble counts (one pass)."""
    import torch
    r.reset_accum()
    out, done = {}, 0
    for n in counts:
        r.render_ensembles(cam, p, first_seed + done, n - done)
        done = n
        out[n] = torch.from_numpy(r.read_accum()).cuda()
    return out


def mean_rgb(accum):
    return accum[:, :3] / accum[:, 3:4].clamp(min=1.0)


def psnr(a, b):
    """PSNR (peak 1) of two (P, 3) linear RGB tensors clamped to [0, 1], and their max abs error."""
    a, b = a.clamp(0, 1), b.clamp(0, 1)
    mse = float(((a - b) ** 2).mean())
    return (99.0 if mse == 0 else 10.0 * math.log10(1.0 / mse)), float((a - b).abs().max())


def make_frames(pkg, fr, scene_specs, cams_per_scene, in_ens, tgt_ens, rng, seed_base, time_budget_s=None,
                log=None):
    """Stacked training frames: x (N, H, W, 8) bf16, base and target (N, H, W, 3) fp32, filled in
    place in tensors allocated once (N = scenes x cameras) and trimmed to the frames rendered when
    the optional time budget runs out. Each frame: `in_ens` ensembles with feature sums packed by
    gpsb_dn_pack straight from the renderer's accumulation, and the mean colour of `tgt_ens`
    ensembles with disjoint seeds (gpsb_dn_mean_rgb), both on the device."""
    import torch
    from gps_pbvr_web_b200 import denoise as dn
    from gps_pbvr_web_b200 import scenes
    W, H = fr.W, fr.H
    P = W * H
    p = params(pkg)
    N = len(scene_specs) * cams_per_scene
    xs = torch.zeros(N, H, W, 8, dtype=torch.bfloat16, device="cuda")
    bases = torch.zeros(N, H, W, 3, device="cuda")
    tgts = torch.zeros(N, H, W, 3, device="cuda")
    meta = []
    k = 0
    t0 = time.perf_counter()
    L = pkg.abi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    fr.r.set_stream(stream)
    acc = fr.r.accum_device_ptr()
    import ctypes as C
    for n_splats, sseed in scene_specs:
        splats, sh, deg = pkg.load_ply(scenes.cluster_scene(n_splats, seed=sseed, degree=3))
        fr.set_scene(splats, sh, deg)
        for d, cam in random_cameras(pkg, cams_per_scene, W, H, rng):
            if time_budget_s is not None and time.perf_counter() - t0 > time_budget_s:
                break
            seed = seed_base + 100_000 * k
            fr.r.reset_accum()
            fr.feat.zero_()
            fr.r.set_feature_accum(fr.feat)
            fr.r.render_ensembles(cam, p, seed, in_ens)
            fr.r.set_feature_accum(None)
            dn._ck(L.gpsb_dn_pack(C.c_void_p(acc), dn._p(fr.feat), P, dn._p(xs[k]), dn._p(bases[k]),
                                  C.c_void_p(stream)), "pack")
            fr.r.reset_accum()
            fr.r.render_ensembles(cam, p, seed + 50_000, tgt_ens)
            dn._ck(L.gpsb_dn_mean_rgb(C.c_void_p(acc), P, dn._p(tgts[k]), C.c_void_p(stream)), "mean_rgb")
            meta.append({"scene": [n_splats, sseed], "distance": d})
            k += 1
            if log and k % 100 == 0:
                torch.cuda.synchronize()
                log(f"frames {k}/{N} after {time.perf_counter() - t0:.0f} s")
        else:
            continue
        break
    torch.cuda.synchronize()
    fr.r.set_stream(None)
    return xs[:k], bases[:k], tgts[:k], meta


class CollapseGuard:
    """Watches the logged training loss. Adam at a high rate can throw this network into a state
    it does not leave (a 10,000-step run at lr 1e-3 jumped from 0.022 to 0.09 at step ~2,400 and
    stayed there, its output no better than the input); when a logged loss exceeds `factor` times
    the best one seen after `warmup` logs, the guard restores the weights of that best log,
    clears the optimiser state and halves the rate scale it returns."""

    def __init__(self, factor=3.0, warmup=5):
        self.factor, self.warmup = factor, warmup
        self.best, self.snap, self.logs, self.scale, self.restores = float("inf"), None, 0, 1.0, []

    def check(self, step, loss, net):
        """Called at every logged step; returns the learning-rate scale for the steps that follow."""
        self.logs += 1
        if self.snap is not None and self.logs > self.warmup and loss > self.factor * self.best:
            net.load_state_dict(self.snap)
            net.reset_optimizer()
            self.scale *= 0.5
            self.restores.append((step, loss, self.best))
        elif loss < self.best:
            self.best, self.snap = loss, net.state_dict()
        return self.scale


def train(net, x, base, target, steps, batch, crop, lr, rng, log_every=100, guard=None):
    """Adam on random crop batches (cosine decay, with a CollapseGuard); returns (loss history,
    ms per step). The guard's restores are in guard.restores."""
    import torch
    from gps_pbvr_web_b200 import denoise as dn
    N, H, W, _ = x.shape
    xb = torch.zeros(batch, crop, crop, 8, dtype=torch.bfloat16, device="cuda")
    bb = torch.zeros(batch, crop, crop, 3, device="cuda")
    tb = torch.zeros(batch, crop, crop, 3, device="cuda")
    crops = torch.zeros(batch, 3, dtype=torch.int32, device="cuda")
    hist = []
    guard = guard if guard is not None else CollapseGuard()
    scale = 1.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        c = np.stack([rng.integers(0, N, batch), rng.integers(0, H - crop + 1, batch),
                      rng.integers(0, W - crop + 1, batch)], axis=1).astype(np.int32)
        crops.copy_(torch.from_numpy(c))
        dn.crop(x, base, target, crops, crop, crop, xb, bb, tb, err=net.err)
        step_lr = scale * lr * (0.5 * (1 + math.cos(math.pi * s / steps)))  # cosine decay
        loss = net.train_step(xb, bb, tb, lr=step_lr)
        if s % log_every == 0 or s == steps - 1:
            hist.append((s, float(loss.item())))
            scale = guard.check(s, hist[-1][1], net)
    torch.cuda.synchronize()
    return hist, (time.perf_counter() - t0) * 1e3 / steps


def denoise_frame(net, x, base):
    """Full-frame inference: x (H, W, 8), base (H, W, 3) -> prediction (H*W, 3); GPU ms."""
    import torch
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    pred = net.forward(x.unsqueeze(0), base.unsqueeze(0))
    b.record()
    torch.cuda.synchronize()
    return pred.reshape(-1, 3).clone(), a.elapsed_time(b)


def variance_gate(x, limit):
    """The per-frame variance check: mean per-pixel ensemble standard deviation of the input
    frame (feature 5) within the training range (<= limit); outside it the plain accumulation is
    used instead of the denoiser."""
    v = float(x[..., 5].float().mean())
    return v <= limit, v


def noise_model(curve, ref_ens):
    """Least-squares fit of the plain path's error model MSE(N) = s2 (1/N + 1/ref_ens) (independent
    ensembles against a reference of ref_ens ensembles) to a PSNR curve; returns s2."""
    xs = np.array([1.0 / n + 1.0 / ref_ens for n in curve])
    ys = np.array([10.0 ** (-p / 10.0) for p in curve.values()])
    return float((xs * ys).sum() / (xs * xs).sum())


def n_model(s2, ref_ens, target_db):
    """Ensembles the error model needs for target_db (None: above the reference's own noise)."""
    inv = 10.0 ** (-target_db / 10.0) / s2 - 1.0 / ref_ens
    return None if inv <= 0 else 1.0 / inv


def n_to_reach(curve, target_db):
    """Smallest ensemble count reaching target_db on a plain PSNR curve {n: psnr}, interpolated in
    log n between measured counts; None if the largest count does not reach it."""
    ns = sorted(curve)
    for i, n in enumerate(ns):
        if curve[n] >= target_db:
            if i == 0:
                return float(n)
            n0, p0, p1 = ns[i - 1], curve[ns[i - 1]], curve[n]
            t = (target_db - p0) / max(p1 - p0, 1e-9)
            return float(math.exp(math.log(n0) + t * (math.log(n) - math.log(n0))))
    return None


def evaluate(pkg, net, fr, scene_specs, cams_per_scene, in_ens, ref_ens, counts, rng, seed_base, gate_limit):
    """Per held-out camera: PSNR / max error of the denoised input, of plain N-ensemble frames, the
    plain count reaching the denoised PSNR and 40 dB, and the timings."""
    import torch
    from gps_pbvr_web_b200 import denoise as dn
    from gps_pbvr_web_b200 import scenes
    W, H = fr.W, fr.H
    P = W * H
    p = params(pkg)
    rows = []
    k = 0
    for n_splats, sseed in scene_specs:
        splats, sh, deg = pkg.load_ply(scenes.cluster_scene(n_splats, seed=sseed, degree=3))
        fr.set_scene(splats, sh, deg)
        for d, cam in random_cameras(pkg, cams_per_scene, W, H, rng):
            seed = seed_base + 100_000 * k
            ref, _, ms_ref = fr.accum(cam, p, seed + 50_000, ref_ens)
            refc = mean_rgb(ref)
            a, f, ms_in = fr.accum(cam, p, seed, in_ens, features=True)
            x = torch.zeros(P, 8, dtype=torch.bfloat16, device="cuda")
            base = torch.zeros(P, 3, device="cuda")
            dn.pack(a, f, x, base)
            ok, v = variance_gate(x, gate_limit)
            if k == 0:  # first call: kernel attributes and full-frame buffers
                denoise_frame(net, x.view(H, W, 8), base.view(H, W, 3))
            pred, ms_dn = denoise_frame(net, x.view(H, W, 8), base.view(H, W, 3))
            ps_dn, me_dn = psnr(pred, refc)
            ps_in, me_in = psnr(base, refc)
            prog = fr.progressive(cam, p, seed + 200_000, counts)
            curve = {n: psnr(mean_rgb(acc), refc)[0] for n, acc in prog.items()}
            ms_ens = ms_ref / ref_ens
            n_same = n_to_reach(curve, ps_dn)
            n_40 = n_to_reach(curve, 40.0)
            s2 = noise_model(curve, ref_ens)
            n_same_model = n_model(s2, ref_ens, ps_dn)
            rows.append({"scene": [n_splats, sseed], "distance": d, "ms_per_ensemble": ms_ens,
                         "psnr_denoised": ps_dn, "maxerr_denoised": me_dn, "psnr_input": ps_in, "maxerr_input": me_in,
                         "denoise_ms": ms_dn, "gate_ok": ok, "gate_value": v, "plain_curve": curve,
                         "plain_n_same_psnr": n_same, "plain_n_40db": n_40, "noise_s2": s2,
                         "psnr_ceiling_vs_ref": 10.0 * math.log10(ref_ens / s2),
                         "plain_n_same_psnr_model": n_same_model,
                         "plain_ms_same_psnr_model": None if n_same_model is None else n_same_model * ms_ens,
                         "denoised_frame_ms": in_ens * ms_ens + ms_dn,
                         "plain_ms_same_psnr": None if n_same is None else n_same * ms_ens,
                         "plain_ms_40db": None if n_40 is None else n_40 * ms_ens})
            k += 1
    return rows


def save_weights(net, path, gate_limit):
    """Weights as used (fp32 rows trimmed to 9 * cin) and the variance-gate limit, in an .npz."""
    sd = net.state_dict()
    arrs = {f"{n}.w": v["w"].numpy()[:, :9 * net.p[n]["cin"]].astype(np.float32) for n, v in sd.items()}
    arrs.update({f"{n}.b": v["b"].numpy().astype(np.float32) for n, v in sd.items()})
    np.savez_compressed(path, gate_limit=np.float32(gate_limit), **arrs)


def main(argv=None):
    import argparse
    import torch
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default="denoise_results.json")
    ap.add_argument("--weights", default="denoiser_weights.npz")
    ap.add_argument("--load", default=None, help="evaluate these weights instead of training")
    ap.add_argument("--width", type=int, default=1280)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--train-scenes", default="200000:11,400000:12,600000:13,800000:14")
    ap.add_argument("--eval-scenes", default="560000:21")
    ap.add_argument("--train-cams", type=int, default=12, help="cameras per training scene")
    ap.add_argument("--eval-cams", type=int, default=8, help="held-out cameras per evaluation scene")
    ap.add_argument("--in-ens", type=int, default=4)
    ap.add_argument("--target-ens", type=int, default=128)
    ap.add_argument("--ref-ens", type=int, default=256)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--crop", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--log-every", type=int, default=100)
    ap.add_argument("--data-budget-s", type=float, default=None,
                    help="stop rendering training frames after this many seconds (train on what was rendered)")
    ap.add_argument("--protocol", default=None, choices=[None, "config4"],
                    help="config4: 2,000 random orbit cameras over 8 seeded cluster scenes of 200k-1M Gaussians "
                         "(250 each), 256-ensemble targets, evaluation on 64 held-out cameras of the same scenes "
                         "against the plain 256-ensemble result")
    pre = argparse.ArgumentParser(add_help=False)
    pre.add_argument("--protocol", default=None)
    if pre.parse_known_args(argv)[0].protocol == "config4":  # its values become the defaults
        sc = ",".join(f"{int(round(200_000 + i * 800_000 / 7))}:{11 + i}" for i in range(8))
        ap.set_defaults(train_scenes=sc, eval_scenes=sc, train_cams=250, eval_cams=8, target_ens=256, ref_ens=256,
                        steps=12000, log_every=200)
    args = ap.parse_args(argv)
    pkg = _pkg()
    from gps_pbvr_web_b200 import denoise as dn
    rng = np.random.default_rng(args.seed)
    spec = lambda s: [tuple(int(v) for v in t.split(":")) for t in s.split(",") if t]
    fr = FrameRenderer(pkg, args.width, args.height)
    t0 = time.perf_counter()
    x, base, target, meta = make_frames(pkg, fr, spec(args.train_scenes), args.train_cams, args.in_ens,
                                        args.target_ens, rng, 1, time_budget_s=args.data_budget_s,
                                        log=lambda m: print(m, file=sys.stderr, flush=True))
    t_data = time.perf_counter() - t0
    net = dn.Denoiser(seed=args.seed)
    if args.load:
        gate_limit = dn.load_weights(net, args.load)
        hist, ms_step = [], 0.0
    else:
        guard = CollapseGuard()
        hist, ms_step = train(net, x, base, target, args.steps, args.batch, args.crop, args.lr, rng, guard=guard,
                              log_every=args.log_every)
        gate_limit = 1.5 * float(x[..., 5].float().mean(dim=(1, 2)).max())
    del x, base, target
    torch.cuda.empty_cache()
    if not args.load:  # the weights are kept even if the evaluation does not finish
        save_weights(net, args.weights, gate_limit)
    rows = evaluate(pkg, net, fr, spec(args.eval_scenes), args.eval_cams, args.in_ens, args.ref_ens,
                    [4, 8, 16, 32, 64, 128, 256], rng, 1_500_000_000, gate_limit)
    save_weights(net, args.weights, gate_limit)
    res = {"config": vars(args), "train_frames": len(meta), "data_seconds": t_data, "loss_history": hist,
           "guard_restores": [] if args.load else guard.restores,
           "ms_per_train_step": ms_step, "params": net.param_count(), "gate_limit": gate_limit,
           "error_word": net.error_word(), "eval": rows}
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
    dn_psnr = [r["psnr_denoised"] for r in rows]
    in_psnr = [r["psnr_input"] for r in rows]
    print(json.dumps({"psnr_denoised_mean": float(np.mean(dn_psnr)), "psnr_input_mean": float(np.mean(in_psnr)),
                      "ms_per_train_step": ms_step, "final_loss": hist[-1][1] if hist else None}))


if __name__ == "__main__":
    main()
