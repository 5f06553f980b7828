"""Small, self-contained GPU workloads for profiling one kernel family at a time under ncu (each
runs a few launches of a case larger than the 126 MB L2 but a few GB at most on the device):

  scan           exclusive scan of 2^26 u32 counts, 3 times (k_scan_u32_staged)
  sort           stable radix sort of 2^24 (24-bit key, value) pairs, 8-bit digits, 3 times (k_onesweep)
  denoise-train  two training steps of the denoiser on 2 x 256 x 256 crops (k_conv_fwd, k_conv_dw, ...)
  denoise-infer  two 1280 x 720 inferences of the denoiser
  particles-near       PBVR Extinction C3+R, 560k-Gaussian cluster scene, 1280 x 720, near orbit view
                       (distance 2.5), 2 ensembles in one launch of k_particles, fast decisions on
  particles-near-exact the same with the fast decisions off (every particle on the exact path)

python gps-pbvr-web_b200/profile_cases.py scan|sort|denoise-train|denoise-infer
"""
import ctypes as C
import os
import sys

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


def scan(pkg):
    import torch
    r = pkg.GpsRenderer(16, 16, 1)
    L = pkg.abi.lib()
    n = 1 << 26
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randint(0, 16, (n,), dtype=torch.int32, device="cuda", generator=g)
    y = torch.empty_like(x)
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(3):
        assert L.gpsb_scan_u32(r.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), n,
                               C.c_void_p(tot.data_ptr())) == 0
    r.wait_idle()
    return r.debug_error_word()


def sort(pkg):
    import torch
    r = pkg.GpsRenderer(16, 16, 1)
    L = pkg.abi.lib()
    m = 1 << 24
    g = torch.Generator(device="cuda").manual_seed(3)
    keys = torch.randint(0, 1 << 24, (m,), dtype=torch.int32, device="cuda", generator=g)
    vals = torch.arange(m, dtype=torch.int32, device="cuda")
    kb, vb = torch.empty_like(keys), torch.empty_like(vals)
    for _ in range(3):
        ka, va = keys.clone(), vals.clone()
        assert L.gpsb_sort_pairs(r.handle, C.c_void_p(ka.data_ptr()), C.c_void_p(va.data_ptr()),
                                 C.c_void_p(kb.data_ptr()), C.c_void_p(vb.data_ptr()), m, 24) == 0
        r.wait_idle()
    return r.debug_error_word()


def denoise(pkg, train):
    import torch
    from gps_pbvr_web_b200 import denoise as dn
    net = dn.Denoiser()
    dn.load_weights(net)
    g = torch.Generator().manual_seed(0)
    if train:
        x0 = torch.zeros(2, 256, 256, 8)
        x0[..., :6] = torch.rand(2, 256, 256, 6, generator=g)
        base = torch.rand(2, 256, 256, 3, generator=g).cuda()
        x0 = x0.to(torch.bfloat16).cuda()
        for _ in range(2):
            net.train_step(x0, base, base, lr=1e-4)
    else:
        x = torch.zeros(1, 720, 1280, 8, dtype=torch.bfloat16, device="cuda")
        base = torch.zeros(1, 720, 1280, 3, device="cuda")
        for _ in range(2):
            net.forward(x, base)
    torch.cuda.synchronize()
    return net.error_word()


def particles_near(pkg, fast):
    import torch
    from gps_pbvr_web_b200 import scenes
    splats, sh, deg = pkg.load_ply(scenes.cluster_scene(560_000, seed=0, degree=3))
    w, h = 1280, 720
    cam = pkg.OrbitCamera(target=(0.0, 0.0, 0.0), distance=2.5, yaw=0.6, pitch=0.25, up=(0.0, -1.0, 0.0),
                          fov_y=0.9).to_camera(w, h)
    p = pkg.RenderParams(spp_side=1, max_points_per_splat=16384, method=pkg.Method.Extinction)
    p.pbvr.calibration = pkg.Calibration.PerSplatFootprint
    p.pbvr.radial_correction = True
    r = pkg.GpsRenderer(w, h, 1)
    r.set_gaussians_sh(splats, sh, deg)
    r.set_fast_decisions(1 if fast else 0)
    r.render_ensembles(cam, p, 1, 2)
    torch.cuda.synchronize()
    return r.debug_error_word()


def main(argv=None):
    case = (argv or sys.argv[1:] or ["scan"])[0]
    pkg = _pkg()
    fn = {"scan": scan, "sort": sort, "denoise-train": lambda p: denoise(p, True),
          "denoise-infer": lambda p: denoise(p, False), "particles-near": lambda p: particles_near(p, True),
          "particles-near-exact": lambda p: particles_near(p, False)}[case]
    err = fn(pkg)
    print(case, "error word", err)
    return 1 if err else 0


if __name__ == "__main__":
    sys.exit(main())
