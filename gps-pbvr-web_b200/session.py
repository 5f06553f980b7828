"""Python mirror of the frame-loop session (include/gpsb200.h, gpsb_session_*): the reference
viewer's per-tick policy (crates/gps-web/src/lib.rs:437-697) over a GpsRenderer, or over any object
providing the renderer calls (a `backend`, used by the CPU tests)."""
import ctypes as C

from . import abi


class SessionError(RuntimeError):
    pass


def _ck(st, what):
    if st != abi.GPSB_OK:
        raise SessionError(f"{what}: {abi.STATUS_NAMES.get(st, st)}")


class FrameSession:
    """`renderer`: a gps.GpsRenderer; or `backend`: an object with render_ensembles(cam, params,
    first_seed, count), render_sorted(cam, params, n), probe_demand(cam, params), request_stats(),
    latest_stats() -> abi.StatsC, stats_issued(), accumulated(), submitted(), reset_accum(),
    reset_stats(), gaussian_count() (cam / params arrive as abi.Camera / abi.ParamsC; each call
    returns a status code, 0 = OK, or the count)."""

    def __init__(self, renderer=None, backend=None):
        self._L = abi.lib()
        self._s = C.c_void_p()
        self._keep = None
        if renderer is not None:
            _ck(self._L.gpsb_session_create(renderer.handle, C.byref(self._s)), "session_create")
        else:
            b = backend

            def cam_of(p):
                return C.cast(p, C.POINTER(abi.Camera)).contents

            def par_of(p):
                return C.cast(p, C.POINTER(abi.ParamsC)).contents

            def latest(_, out):
                C.cast(out, C.POINTER(abi.StatsC))[0] = b.latest_stats()
                return 0
            fns = abi.SessionBackendC(
                abi.BE_RENDER(lambda _, c, p, s, n: b.render_ensembles(cam_of(c), par_of(p), s, n)),
                abi.BE_SORTED(lambda _, c, p, n: b.render_sorted(cam_of(c), par_of(p), n)),
                abi.BE_PROBE(lambda _, c, p: b.probe_demand(cam_of(c), par_of(p))),
                abi.BE_CALL(lambda _: b.request_stats()), abi.BE_STATS(latest),
                abi.BE_U32(lambda _: b.stats_issued()), abi.BE_U32(lambda _: b.accumulated()),
                abi.BE_U32(lambda _: b.submitted()), abi.BE_CALL(lambda _: b.reset_accum()),
                abi.BE_CALL(lambda _: b.reset_stats()), abi.BE_U32(lambda _: b.gaussian_count()))
            self._keep = fns  # the callbacks must outlive the session
            _ck(self._L.gpsb_session_create_with_backend(C.byref(fns), None, C.byref(self._s)), "session_create")

    def close(self):
        if self._s:
            self._L.gpsb_session_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, params, per_frame=1, target=256):
        pc = params.to_c() if hasattr(params, "to_c") else params
        _ck(self._L.gpsb_session_configure(self._s, C.byref(pc), per_frame, target), "configure")

    def set_lod(self, adaptive, target_ms=33.3, moving_cap=2048):
        _ck(self._L.gpsb_session_set_lod(self._s, int(adaptive), target_ms, moving_cap), "set_lod")

    def set_point_budget(self, millions):
        _ck(self._L.gpsb_session_set_point_budget(self._s, millions), "set_point_budget")

    def set_render_path(self, mode, demand_threshold_millions=30.0):
        _ck(self._L.gpsb_session_set_render_path(self._s, mode, demand_threshold_millions), "set_render_path")

    def set_camera(self, cam, user_input=False):
        cc = cam.to_c() if hasattr(cam, "to_c") else cam
        _ck(self._L.gpsb_session_set_camera(self._s, C.byref(cc), int(user_input)), "set_camera")

    def reset(self):
        _ck(self._L.gpsb_session_reset(self._s), "reset")

    def frame(self, now_ms):
        presented = C.c_int(0)
        _ck(self._L.gpsb_session_frame(self._s, now_ms, C.byref(presented)), "frame")
        return bool(presented.value)

    def state(self):
        st = abi.SessionStateC()
        _ck(self._L.gpsb_session_read_state(self._s, C.byref(st)), "state")
        return {k: getattr(st, k) for k, _ in abi.SessionStateC._fields_}
