"""gpsb-verify, the restatement of the reference CLI (crates/gps-verify/src/main.rs)."""
import os
import subprocess

import pytest

from conftest import ROOT

CLI = os.path.join(ROOT, "gps-pbvr-web_b200", "gpsb-verify")
PLY = os.path.join(ROOT, "tests", "golden", "synthetic_sh1.ply")


def test_cli_usage_without_gpu():
    p = subprocess.run([CLI], capture_output=True, text=True, timeout=60)
    assert p.returncode == 2 and "bench-ply" in p.stderr


@pytest.mark.gpu
def test_cli_bench_ply():
    p = subprocess.run([CLI, "bench-ply", PLY, "320x180", "1"], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, MAXPTS="4096"))
    assert p.returncode == 0, p.stderr
    rows = [l for l in p.stdout.splitlines() if "ms " in l or l.rstrip().endswith("ms")]
    assert "400 Gaussians, SH degree 1" in p.stdout
    assert sum(1 for l in p.stdout.splitlines() if l.startswith(("near", "mid", "far"))) == 9, p.stdout


@pytest.mark.gpu
def test_cli_bench():
    p = subprocess.run([CLI, "bench"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.count("ms") >= 5
