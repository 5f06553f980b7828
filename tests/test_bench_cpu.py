"""Host-side helpers of bench.py (no GPU): the committed ncu figures it reads, the issue roofline it
derives from them, the peak fallback and the workload description."""
import os
import sys
from types import SimpleNamespace

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_committed_figures_parse():
    assert bench.committed_traffic("k_particles") > 1e9
    per = bench.committed_traffic("k_particles_warp_inst_per_particle")
    assert per is not None and 5.0 < per < 40.0
    assert bench.committed_traffic("no_such_kernel") is None


def test_issue_roofline_arithmetic():
    per = bench.committed_traffic("k_particles_warp_inst_per_particle")
    st = SimpleNamespace(particles=7_000_000_000)
    out = bench.issue_roofline(st, 100.0, 1, {"sm_mhz": 2000.0})
    achieved = 7e9 / 0.1 * per
    peak = 148 * 4 * 2000e6
    assert abs(out["achieved"] - achieved) < 1e-6 * achieved and abs(out["peak"] - peak) < 1.0
    assert abs(out["frac"] - achieved / peak) < 1e-12
    # no clock samples or no particles: no estimate
    assert bench.issue_roofline(st, 100.0, 1, {"sm_mhz": None}) is None
    assert bench.issue_roofline(SimpleNamespace(particles=0), 100.0, 1, {"sm_mhz": 2000.0}) is None


def test_peak_and_workload():
    peak, kind = bench.measured_peak()
    assert peak > 1000.0 and kind in ("of measured", "of fallback")
    cfg = bench.workload_config()
    assert cfg["gaussians"] == bench.N_SPLATS and cfg["resolution"] == [bench.W, bench.H]
    assert cfg["views"] == [v for v, _ in bench.VIEWS] and cfg["ensembles_per_view"] == bench.ENS


def test_reference_arm_never_loads_the_renderer():
    """The CPU arm builds its scene and cameras from the oracle alone (oracle PLY reader, O1
    cameras equal to the renderer's) and its timing helper runs O1 in one host thread per subset;
    the renderer library is not mapped into that process."""
    import subprocess
    code = ("import sys; sys.path.insert(0, %r); import bench; g, cams = bench.reference_inputs(); "
            "r = bench.cpu_reference(g[:20000], cams[2:], 2, 64); assert r[0] > 0; "
            "print(any('libgpsb200' in l for l in open('/proc/self/maps')))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().splitlines()[-1] == "False"


def test_reference_cameras_equal_the_renderers():
    import numpy as np
    from conftest import load_package
    pkg = load_package()
    _, cams = bench.reference_inputs()
    for (name, c17), (name2, cam) in zip(cams, bench.cameras(pkg)):
        assert name == name2 and np.array_equal(c17, cam.to_array())


def test_equal_psnr_target_statement():
    met = bench.equal_psnr_target(4.2, 0.45, 33.4, 396.0)
    assert met == {"target": 8.0, "met": True, "why_not": None}
    far = bench.equal_psnr_target(0.283, 0.45, 31.4, 30.9)
    assert far["met"] is False and "31 ensembles" in far["why_not"] and "5.5x" in far["why_not"]
    unknown = bench.equal_psnr_target(4.2, 0.45, 37.0, None)
    assert unknown["met"] is None and "largest" in unknown["why_not"]
