"""Python mirror of gps-render's renderer API over the C ABI (crates/gps-render/src/gps.rs).

Names, argument meaning and error behaviour follow the reference: GpsRenderer(...) with
set_gaussians / set_gaussians_sh / resize / reset_accum / reset_stats / render_ensembles /
render_sorted / probe_demand / read_accum / read_stats / request_stats / latest_stats /
stats_issued / read_sorted / accumulated / submitted / composite / wait_idle, and the
RenderParams / PbvrParams / Method / Calibration / RenderPath / GpuStats value types. A failing
call raises GpsError with the library's message (the reference returns Err(String)).
"""
import ctypes as C
import enum
import math
from dataclasses import dataclass, field, replace
from typing import Optional, Sequence, Tuple

import numpy as np

from . import abi


class GpsError(RuntimeError):
    """Err(String) of the reference renderer."""

    def __init__(self, status, message):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Method(enum.IntEnum):  # gps.rs:104-116
    Gps = 0
    Proportional = 1
    Extinction = 2
    ViewConditioned = 3
    ScreenOccupancy = 4

    @staticmethod
    def from_index(i):
        return Method(i) if 0 <= i <= 4 else Method.Gps


class Calibration(enum.IntEnum):  # gps.rs:144-154
    None_ = 0
    ObjectZoom = 1
    PerSplatDepth = 2
    PerSplatFootprint = 3


class RenderPath(enum.IntEnum):  # gps.rs:93-100
    Primitive = 0
    Particle = 1


@dataclass
class PbvrParams:  # gps.rs:169-185
    calibration: Calibration = Calibration.PerSplatFootprint
    radial_correction: bool = False
    centre_depth: bool = False
    low_pass_jitter: bool = True
    base_k: float = 512.0
    reference_pixel_length: float = 0.01


@dataclass
class RenderParams:  # gps.rs:189-229
    spp_side: int = 2
    density_scale: float = 1.0
    max_points_per_splat: int = 1 << 16
    near: float = 0.05
    background: Tuple[float, float, float] = (0.05, 0.05, 0.08)
    exposure: float = 1.0
    srgb_output: bool = True
    exact_radius: bool = False
    sh_degree: int = 3
    path: RenderPath = RenderPath.Particle
    method: Method = Method.Gps
    pbvr: PbvrParams = field(default_factory=PbvrParams)

    def to_c(self) -> abi.ParamsC:
        p = abi.ParamsC()
        p.spp_side = int(self.spp_side)
        p.density_scale = float(self.density_scale)
        p.max_points_per_splat = int(self.max_points_per_splat) & 0xFFFFFFFF
        p.near_z = float(self.near)
        for k in range(3):
            p.background[k] = float(self.background[k])
        p.exposure = float(self.exposure)
        p.srgb_output = int(bool(self.srgb_output))
        p.exact_radius = int(bool(self.exact_radius))
        p.sh_degree = int(self.sh_degree)
        p.path = int(self.path)
        p.method = int(self.method)
        p.pbvr.calibration = int(self.pbvr.calibration)
        p.pbvr.radial_correction = int(bool(self.pbvr.radial_correction))
        p.pbvr.centre_depth = int(bool(self.pbvr.centre_depth))
        p.pbvr.low_pass_jitter = int(bool(self.pbvr.low_pass_jitter))
        p.pbvr.base_k = float(self.pbvr.base_k)
        p.pbvr.reference_pixel_length = float(self.pbvr.reference_pixel_length)
        return p


@dataclass(frozen=True)
class GpuStats:  # gps.rs:231-252
    points: int = 0
    truncated_splats: int = 0
    dropped_points: int = 0
    visible_splats: int = 0
    orphan_subpixels: int = 0
    candidates: int = 0
    undercovered_splats: int = 0
    skipped_ensembles: int = 0
    ensembles: int = 0
    probe_demand: int = 0
    issue: int = 0
    subpixel_writes: int = 0
    list_entries: int = 0
    particles: int = 0

    @staticmethod
    def from_c(s: abi.StatsC) -> "GpuStats":
        return GpuStats(s.points, s.truncated_splats, s.dropped_points, s.visible_splats, s.orphan_subpixels,
                        s.candidates, s.undercovered_splats, s.skipped_ensembles, s.ensembles, s.probe_demand, s.issue,
                        s.subpixel_writes, s.list_entries, s.particles)

    def counters(self):
        """Every counter but the readback issue number (for equality checks between paths)."""
        return (self.points, self.truncated_splats, self.dropped_points, self.visible_splats, self.orphan_subpixels,
                self.candidates, self.undercovered_splats, self.skipped_ensembles, self.ensembles)


@dataclass
class OracleCamera:  # crates/gps-core/src/oracle.rs:33-48
    view_rot: np.ndarray = field(default_factory=lambda: np.eye(3))
    view_pos: np.ndarray = field(default_factory=lambda: np.zeros(3))
    focal_x: float = 200.0
    focal_y: float = 200.0
    cx: float = 0.0
    cy: float = 0.0
    low_pass: float = 0.3

    def to_c(self) -> abi.Camera:
        c = abi.Camera()
        r = np.asarray(self.view_rot, dtype=np.float64).reshape(-1)
        for k in range(9):
            c.view_rot[k] = float(r[k])
        for k in range(3):
            c.view_pos[k] = float(self.view_pos[k])
        c.focal_x, c.focal_y, c.cx, c.cy, c.low_pass = (float(self.focal_x), float(self.focal_y), float(self.cx),
                                                        float(self.cy), float(self.low_pass))
        return c

    def to_array(self) -> np.ndarray:
        """17 doubles in gpsb_camera order (view_rot row-major, view_pos, fx, fy, cx, cy, low_pass)."""
        return np.concatenate([np.asarray(self.view_rot, np.float64).reshape(-1), np.asarray(self.view_pos, np.float64),
                               [self.focal_x, self.focal_y, self.cx, self.cy, self.low_pass]])

    @staticmethod
    def from_c(c: abi.Camera) -> "OracleCamera":
        return OracleCamera(np.array(list(c.view_rot)).reshape(3, 3), np.array(list(c.view_pos)), c.focal_x, c.focal_y,
                            c.cx, c.cy, c.low_pass)

    @staticmethod
    def look_at(eye, target, up, fov_y, w, h) -> "OracleCamera":
        out = abi.Camera()
        _check(None, abi.lib().gpsb_camera_look_at(_d3(eye), _d3(target), _d3(up), float(fov_y), int(w), int(h),
                                                    C.byref(out)))
        return OracleCamera.from_c(out)


@dataclass
class OrbitCamera:  # crates/gps-core/src/camera.rs:9-26
    target: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    distance: float = 5.0
    yaw: float = 0.0
    pitch: float = 0.0
    up: Tuple[float, float, float] = (0.0, 1.0, 0.0)
    fov_y: float = 0.9

    def to_camera(self, w, h) -> OracleCamera:
        out = abi.Camera()
        _check(None, abi.lib().gpsb_orbit_camera(_d3(self.target), float(self.distance), float(self.yaw),
                                                  float(self.pitch), _d3(self.up), float(self.fov_y), int(w), int(h),
                                                  C.byref(out)))
        return OracleCamera.from_c(out)

    def frame_sphere(self, centre, radius):  # camera.rs:87-90
        self.target = tuple(float(x) for x in centre)
        self.distance = (max(radius, 1e-6) / math.sin(0.5 * self.fov_y)) * 1.25

    @staticmethod
    def robust_sphere(splats: np.ndarray):
        g = _splats(splats)
        c = (C.c_double * 3)()
        r = C.c_double()
        _check(None, abi.lib().gpsb_robust_sphere(g.ctypes.data_as(C.c_void_p), g.shape[0], c, C.byref(r)))
        return (c[0], c[1], c[2]), r.value


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def _splats(a) -> np.ndarray:
    g = np.ascontiguousarray(a, dtype=np.float32)
    if g.ndim != 2 or g.shape[1] != 16:
        g = g.reshape(-1, 16)
    return g


def _check(r, status):
    if status != abi.GPSB_OK:
        msg = abi.lib().gpsb_last_error(r).decode(errors="replace")
        raise GpsError(status, msg)


def radius_lut() -> np.ndarray:
    t = np.zeros(65 * 129, np.float32)
    _check(None, abi.lib().gpsb_radius_lut(t.ctypes.data_as(C.c_void_p)))
    return t


def estimate_memory(w, h, spp_side, n):
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    abi.lib().gpsb_estimate_memory(w, h, spp_side, n, C.byref(a), C.byref(b), C.byref(c))
    return {"depth_winner_bytes": a.value, "accum_bytes": b.value, "splat_bytes": c.value}


def load_ply_device(data: bytes):
    """GPU decode of a binary 3DGS PLY (gpsb_load_ply_device): (splats (n, 16) float32 CUDA tensor,
    SH rest float32 CUDA tensor, degree), ready for GpsRenderer.set_gaussians_sh_device."""
    import torch
    L = abi.lib()
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    n = C.c_size_t()
    d = C.c_uint32()
    st = L.gpsb_load_ply_device(buf, len(data), C.byref(n), C.byref(d), None, None, None)
    if st != abi.GPSB_OK:
        raise GpsError(st, L.gpsb_ply_last_error().decode(errors="replace"))
    per = (d.value + 1) ** 2 - 1 if d.value else 0
    g = torch.zeros((n.value, 16), dtype=torch.float32, device="cuda")
    sh = torch.zeros(max(n.value * 3 * per, 1), dtype=torch.float32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = L.gpsb_load_ply_device(buf, len(data), C.byref(n), C.byref(d), C.c_void_p(g.data_ptr()),
                                C.c_void_p(sh.data_ptr()), stream)
    if st != abi.GPSB_OK:
        raise GpsError(st, L.gpsb_ply_last_error().decode(errors="replace"))
    return g, sh[: n.value * 3 * per], d.value


def debug_fmath(which: int, x_dev, out_dev):
    """The shared exp (0) / log (1) / sin (2) / cos (3) / positive-normal log (4) evaluated on the
    device as the kernels evaluate them (which | 8: global tables); x_dev/out_dev are float32 CUDA
    tensors of the same size."""
    _check(None, abi.lib().gpsb_debug_fmath(which, C.c_void_p(x_dev.data_ptr()), C.c_void_p(out_dev.data_ptr()),
                                            x_dev.numel()))


def load_ply(data: bytes):
    """gps-io load_ply + activation + GpuGaussian::from_activated: (splats (n,16) f32, sh_rest f32, degree)."""
    L = abi.lib()
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    n = C.c_size_t()
    d = C.c_uint32()
    st = L.gpsb_load_ply(buf, len(data), C.byref(n), C.byref(d), None, None)
    if st != abi.GPSB_OK:
        raise GpsError(st, L.gpsb_ply_last_error().decode(errors="replace"))
    per = (d.value + 1) ** 2 - 1 if d.value else 0
    g = np.zeros((n.value, 16), np.float32)
    sh = np.zeros(n.value * 3 * per, np.float32)
    st = L.gpsb_load_ply(buf, len(data), C.byref(n), C.byref(d), g.ctypes.data_as(C.c_void_p),
                         sh.ctypes.data_as(C.c_void_p) if sh.size else None)
    if st != abi.GPSB_OK:
        raise GpsError(st, L.gpsb_ply_last_error().decode(errors="replace"))
    return g, sh, d.value


class GpsRenderer:
    """GpsRenderer (gps.rs:302-1065) on a CUDA device."""

    def __init__(self, width: int, height: int, spp_side: int, device: int = 0):
        self._r = C.c_void_p()
        L = abi.lib()
        st = L.gpsb_create(device, width, height, spp_side, C.byref(self._r))
        if st != abi.GPSB_OK:
            raise GpsError(st, L.gpsb_last_error(None).decode(errors="replace"))
        self._L = L

    def close(self):
        if getattr(self, "_r", None) and self._r.value:
            self._L.gpsb_destroy(self._r)
            self._r = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, st):
        _check(self._r, st)

    @property
    def handle(self):
        return self._r

    # ---------------------------------------------------------------- scene / state
    def set_gaussians(self, splats):
        g = _splats(splats)
        self._ck(self._L.gpsb_set_gaussians(self._r, g.ctypes.data_as(C.c_void_p), g.shape[0]))

    def set_gaussians_sh(self, splats, sh_rest, degree):
        g = _splats(splats)
        s = np.ascontiguousarray(sh_rest, dtype=np.float32).reshape(-1)
        self._ck(self._L.gpsb_set_gaussians_sh(self._r, g.ctypes.data_as(C.c_void_p), g.shape[0],
                                               s.ctypes.data_as(C.c_void_p), s.size, int(degree)))

    def set_gaussians_device(self, splats_ptr, n, sh_ptr=None, sh_len=0, degree=0):
        self._ck(self._L.gpsb_set_gaussians_sh_device(self._r, C.c_void_p(splats_ptr), n,
                                                      C.c_void_p(sh_ptr) if sh_ptr else None, sh_len, degree))

    def resize(self, width, height, spp_side):
        self._ck(self._L.gpsb_resize(self._r, width, height, spp_side))

    def reset_accum(self):
        self._ck(self._L.gpsb_reset_accum(self._r))

    def reset_stats(self):
        self._ck(self._L.gpsb_reset_stats(self._r))

    def size(self):
        w, h, s = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._L.gpsb_size(self._r, C.byref(w), C.byref(h), C.byref(s))
        return w.value, h.value

    def spp_side(self):
        w, h, s = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._L.gpsb_size(self._r, C.byref(w), C.byref(h), C.byref(s))
        return s.value

    def gaussian_count(self):
        return self._L.gpsb_gaussian_count(self._r)

    def sh_max_degree(self):
        return self._L.gpsb_sh_max_degree(self._r)

    def sh_bytes(self):
        return self._L.gpsb_sh_bytes(self._r)

    # ---------------------------------------------------------------- rendering
    def render_ensembles(self, cam: OracleCamera, params: RenderParams, first_seed: int, count: int):
        c, p = cam.to_c(), params.to_c()
        self._ck(self._L.gpsb_render_ensembles(self._r, C.byref(c), C.byref(p), first_seed & 0xFFFFFFFF, count))

    def render_trajectory(self, cams: Sequence[OracleCamera], params: RenderParams, first_seed: int,
                          ensembles_per_camera: int, accum_out_ptr: int):
        arr = (abi.Camera * len(cams))(*[c.to_c() for c in cams])
        p = params.to_c()
        self._ck(self._L.gpsb_render_trajectory(self._r, arr, len(cams), C.byref(p), first_seed & 0xFFFFFFFF,
                                                ensembles_per_camera, C.c_void_p(accum_out_ptr)))

    def render_trajectory_graph(self, cams: Sequence[OracleCamera], params: RenderParams, first_seed: int,
                                ensembles_per_camera: int, accum_out_ptr: int):
        """render_trajectory through one captured CUDA graph (captured on the first call, relaunched
        by identical repeats)."""
        arr = (abi.Camera * len(cams))(*[c.to_c() for c in cams])
        p = params.to_c()
        self._ck(self._L.gpsb_render_trajectory_graph(self._r, arr, len(cams), C.byref(p), first_seed & 0xFFFFFFFF,
                                                      ensembles_per_camera, C.c_void_p(accum_out_ptr)))

    def render_sorted(self, cam: OracleCamera, params: RenderParams, as_ensembles: int):
        c, p = cam.to_c(), params.to_c()
        self._ck(self._L.gpsb_render_sorted(self._r, C.byref(c), C.byref(p), as_ensembles))

    def probe_demand(self, cam: OracleCamera, params: RenderParams):
        c, p = cam.to_c(), params.to_c()
        self._ck(self._L.gpsb_probe_demand(self._r, C.byref(c), C.byref(p)))

    # ---------------------------------------------------------------- readback
    def read_accum(self) -> np.ndarray:
        w, h = self.size()
        out = np.zeros((h * w, 4), np.float32)
        self._ck(self._L.gpsb_read_accum(self._r, out.ctypes.data_as(C.c_void_p)))
        return out

    def accum_device_ptr(self) -> int:
        p = C.c_void_p()
        self._ck(self._L.gpsb_accum_device_ptr(self._r, C.byref(p)))
        return p.value

    def read_stats(self) -> GpuStats:
        s = abi.StatsC()
        self._ck(self._L.gpsb_read_stats(self._r, C.byref(s)))
        return GpuStats.from_c(s)

    def request_stats(self):
        self._ck(self._L.gpsb_request_stats(self._r))

    def latest_stats(self) -> GpuStats:
        s = abi.StatsC()
        self._ck(self._L.gpsb_latest_stats(self._r, C.byref(s)))
        return GpuStats.from_c(s)

    def stats_issued(self) -> int:
        return self._L.gpsb_stats_issued(self._r)

    def read_sorted(self):
        n = self.gaussian_count()
        k = np.zeros(n, np.uint32)
        v = np.zeros(n, np.uint32)
        self._ck(self._L.gpsb_read_sorted(self._r, k.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p)))
        return k, v

    def accumulated(self) -> int:
        return self._L.gpsb_accumulated(self._r)

    def submitted(self) -> int:
        return self._L.gpsb_submitted(self._r)

    def wait_idle(self):
        self._ck(self._L.gpsb_sync(self._r))

    def composite(self, params: RenderParams, out_w: Optional[int] = None, out_h: Optional[int] = None) -> np.ndarray:
        w, h = self.size()
        ow, oh = out_w or w, out_h or h
        out = np.zeros((oh * ow, 4), np.uint8)
        p = params.to_c()
        self._ck(self._L.gpsb_composite_rgba8(self._r, C.byref(p), ow, oh, out.ctypes.data_as(C.c_void_p)))
        return out

    # ---------------------------------------------------------------- test hooks
    def debug_counts(self, slot: int) -> np.ndarray:
        out = np.zeros(self.gaussian_count(), np.uint32)
        self._ck(self._L.gpsb_debug_read_counts(self._r, slot, out.ctypes.data_as(C.c_void_p)))
        return out

    def debug_subpixels(self, slot: int) -> np.ndarray:
        w, h = self.size()
        s = self.spp_side()
        out = np.zeros(w * h * s * s, np.uint64)
        self._ck(self._L.gpsb_debug_read_subpixels(self._r, slot, out.ctypes.data_as(C.c_void_p)))
        return out

    def debug_particle_seeds(self, slot: int, first_particle: int, n: int) -> np.ndarray:
        """(n, 3) u32: splat, index within the splat and stream seed of particles first_particle..
        of ensemble `slot` of the last particle-path render, as the particle kernel derives them."""
        out = np.zeros((n, 3), np.uint32)
        self._ck(self._L.gpsb_debug_particle_seeds(self._r, slot, first_particle, n, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_footprint(self, footprint_subpixels=1, adaptive_kappa=0.0, footprint_max=4, compensate_blur=False):
        """Footprint-subpixel Monte-Carlo mode of GPS (MonteCarloOptions of the CPU oracle)."""
        self._ck(self._L.gpsb_set_footprint(self._r, footprint_subpixels, adaptive_kappa, footprint_max,
                                            int(bool(compensate_blur))))

    def set_fast_decisions(self, mode: int = 1):
        """PBVR fast decisions: 0 off, 1 on (outputs bit-identical), 2 validate every particle."""
        self._ck(self._L.gpsb_set_fast_decisions(self._r, int(mode)))

    def debug_fast_counts(self):
        """(particles left to the exact path, fast answers that disagreed) of the last frame."""
        out = np.zeros(2, np.uint64)
        self._ck(self._L.gpsb_debug_fast_counts(self._r, out.ctypes.data_as(C.c_void_p)))
        return int(out[0]), int(out[1])

    def debug_fast_bounds(self) -> np.ndarray:
        """Largest error / bound of each approximation the fast decisions use, over all its inputs."""
        out = np.zeros(6, np.float32)
        self._ck(self._L.gpsb_debug_fast_bounds(self._r, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_feature_accum(self, feat):
        """Denoiser feature sums into `feat` (a zeroed CUDA tensor of W*H*8 float32), or None to stop."""
        self._ck(self._L.gpsb_set_feature_accum(self._r, C.c_void_p(feat.data_ptr()) if feat is not None else None))

    def debug_error_word(self) -> int:
        return self._L.gpsb_debug_error_word(self._r)

    # ---------------------------------------------------------------- profiling
    def profile_enable(self, on: bool = True):
        self._ck(self._L.gpsb_profile_enable(self._r, int(on)))

    def profile(self) -> dict:
        p = abi.ProfileC()
        self._ck(self._L.gpsb_profile_read(self._r, C.byref(p)))
        return {"launches": {n: int(p.launches[i]) for i, n in enumerate(abi.STAGES)},
                "ms": {n: float(p.ms[i]) for i, n in enumerate(abi.STAGES)}, "total_launches": int(p.total_launches)}

    def set_tuning(self, **kw):
        """sort_digit_bits, blend_tile_w, blend_tile_h, particle_items, particle_blocks_per_sm, ensemble_batch."""
        t = abi.TuningC()
        for k, v in kw.items():
            setattr(t, k, int(v))
        self._ck(self._L.gpsb_set_tuning(self._r, C.byref(t)))

    def tuning(self) -> dict:
        t = abi.TuningC()
        self._ck(self._L.gpsb_get_tuning(self._r, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def set_sort_digit_bits(self, bits: int):
        self.set_tuning(sort_digit_bits=bits)

    def set_stream(self, cuda_stream_ptr: int):
        self._ck(self._L.gpsb_set_stream(self._r, C.c_void_p(cuda_stream_ptr) if cuda_stream_ptr else None))


def default_params(**kw) -> RenderParams:
    p = RenderParams()
    return replace(p, **kw)
