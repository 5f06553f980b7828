"""The frame-loop session (gps-web Viewer::frame policy, crates/gps-web/src/lib.rs:437-697) on the
CPU against a scripted fake renderer: manual ensembles per tick up to the target, history restarts
on a new camera, adaptive LOD (one ensemble with the moving-camera cap while the camera moves,
growing while still), the point-budget density factor, Auto's sorted/GPS choice from the demand
probe with 0.5 hysteresis, the hand-over to particles when sorting is slow, and PBVR never sorted."""
import importlib

import numpy as np

from conftest import load_package

PKG = load_package()
S = importlib.import_module(PKG.__name__ + ".session")
abi = PKG.abi


class Fake:
    """Records the session's calls; statistics readbacks arrive on the next request."""

    def __init__(self, n_splats=1000, demand=1e6, points_per_ens=1e6, dropped=0):
        self.acc = self.sub = 0
        self.calls = []
        self.n = n_splats
        self.demand = demand
        self.points_per_ens = points_per_ens
        self.dropped = dropped
        self.cur = abi.StatsC()
        self.latest = abi.StatsC()
        self.issued = 0

    def render_ensembles(self, cam, p, seed, n):
        self.calls.append(("ens", seed, n, p.density_scale, p.max_points_per_splat))
        self.acc += n
        self.sub += n
        self.cur.ensembles += n
        self.cur.points += int(self.points_per_ens * n * p.density_scale)
        self.cur.dropped_points += int(self.dropped * n)
        return 0

    def render_sorted(self, cam, p, n):
        self.calls.append(("sorted", n))
        self.acc = n
        self.sub += n
        return 0

    def probe_demand(self, cam, p):
        self.calls.append(("probe",))
        self.cur.probe_demand = int(self.demand)
        return 0

    def request_stats(self):
        self.issued += 1
        self.latest = abi.StatsC.from_buffer_copy(self.cur)
        self.latest.issue = self.issued
        return 0

    def latest_stats(self):
        return self.latest

    def stats_issued(self):
        return self.issued

    def accumulated(self):
        return self.acc

    def submitted(self):
        return self.sub

    def reset_accum(self):
        self.calls.append(("reset",))
        self.acc = self.sub = 0
        return 0

    def reset_stats(self):
        self.cur = abi.StatsC()
        return 0

    def gaussian_count(self):
        return self.n


def _cam(z=5.0):
    c = abi.Camera()
    for i in range(9):
        c.view_rot[i] = 1.0 if i % 4 == 0 else 0.0
    c.view_pos[2] = -z
    c.focal_x = c.focal_y = 100.0
    return c


def _params(method=0, cap=4096):
    p = PKG.RenderParams(spp_side=1, max_points_per_splat=cap)
    p.method = PKG.Method(method)
    return p


def _session(fake, method=0, per_frame=2, target=8, path=0):
    s = S.FrameSession(backend=fake)
    s.configure(_params(method), per_frame, target)
    s.set_render_path(path, 30.0)
    s.set_camera(_cam())
    return s


def test_manual_ensembles_until_target_and_restart_on_camera():
    f = Fake()
    s = _session(f)
    t = 0.0
    presented = []
    for _ in range(6):
        t += 16.7
        presented.append(s.frame(t))
    ens = [c for c in f.calls if c[0] == "ens"]
    assert [c[2] for c in ens] == [2, 2, 2, 2] and f.acc == 8
    assert [c[1] for c in ens] == [1, 3, 5, 7]  # consecutive seeds from the session seed
    assert presented[:4] == [True] * 4 and presented[4:] == [False, False]
    s.set_camera(_cam(6.0))
    s.frame(t + 16.7)
    assert f.calls[-2][0] == "reset" and f.calls[-1][:3] == ("ens", 1, 2)
    assert s.state()["history_epoch"] == 2


def test_adaptive_lod_moving_cap_and_growth():
    f = Fake()
    s = _session(f, per_frame=1, target=10_000)
    s.set_lod(True, 33.3, 512)
    t = 100.0
    s.frame(t)
    s.set_camera(_cam(4.0), user_input=True)
    t += 10.0
    s.frame(t)
    st = s.state()
    assert st["lod_moving"] == 1 and f.calls[-1][0] == "ens" and f.calls[-1][2] == 1 and f.calls[-1][4] == 512
    # still for longer than 250 ms: the history restarts with the full cap, then ensembles grow
    for _ in range(400):
        t += 10.0  # fast frames (ema well below 0.6 * 33.3 ms)
        s.frame(t)
    st = s.state()
    assert st["lod_moving"] == 0 and f.calls[-1][4] == 4096
    assert st["lod_n"] == 4 and f.calls[-1][2] == 4
    # slow frames back off one at a time
    for _ in range(40):
        t += 60.0
        s.frame(t)
    assert s.state()["lod_n"] == 1


def test_point_budget_lowers_density():
    f = Fake(points_per_ens=8e6, dropped=2e6)
    s = _session(f, per_frame=1, target=10_000)
    s.set_point_budget(2.5)  # 2.5 M points per ensemble; demand = 10 M
    t = 0.0
    for _ in range(12):
        t += 16.7
        s.frame(t)
    st = s.state()
    assert abs(st["auto_density"] - 0.25) < 1e-6
    assert any(c[0] == "ens" and abs(c[3] - 0.25) < 1e-6 for c in f.calls)


def test_auto_path_probe_threshold_and_hysteresis():
    f = Fake(demand=50e6)
    s = _session(f, method=0, per_frame=1, target=16, path=2)
    t = 0.0
    for _ in range(3):
        t += 16.7
        s.frame(t)
    assert ("probe",) in f.calls and s.state()["sorted_active"] == 1
    assert any(c[0] == "sorted" for c in f.calls)
    # a new view whose demand is between half the threshold and the threshold keeps the sorted path
    f.demand = 20e6
    s.set_camera(_cam(7.0))
    for _ in range(3):
        t += 16.7
        s.frame(t)
    assert s.state()["sorted_active"] == 1 and s.state()["last_demand"] == 20_000_000
    # below half the threshold: back to GPS particles
    f.demand = 10e6
    s.set_camera(_cam(8.0))
    for _ in range(3):
        t += 16.7
        s.frame(t)
    assert s.state()["sorted_active"] == 0 and f.calls[-1][0] == "ens"


def test_slow_sorting_hands_motion_to_particles():
    f = Fake(demand=50e6)
    s = _session(f, method=0, per_frame=1, target=10_000, path=2)
    t = 0.0
    for _ in range(3):
        t += 16.7
        s.frame(t)
    assert s.state()["sorted_active"] == 1
    for _ in range(60):
        t += 80.0
        s.set_camera(_cam(5.0 + t * 1e-3), user_input=True)
        s.frame(t)
    st = s.state()
    assert st["moving_prefers_gps"] == 1 and st["sorted_active"] == 0


def test_pbvr_never_uses_the_sorted_path():
    f = Fake(demand=90e6)
    s = _session(f, method=2, per_frame=1, target=4, path=2)
    for k in range(6):
        s.frame(16.7 * (k + 1))
    assert not any(c[0] in ("probe", "sorted") for c in f.calls)
    assert f.acc == 4


def test_autotune_key_buckets():
    at = importlib.import_module(PKG.__name__ + ".autotune")
    assert at.key(560_000, 1280, 720, 2, False) == "m2-particle-1280x720-n524288"
    assert at.key(2_000_000, 1920, 1080, 4, False) == "m4-particle-1920x1080-n2097152"
    assert at.key(10_000, 256, 256, 0, True) == "m0-sorted-256x256-n8192"
    assert len(at.PARTICLE_SPACE) == 9 and len(at.SORTED_SPACE) == 9
