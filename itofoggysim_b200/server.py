"""Python side of the solve server (foggy_server_* in include/foggy_gpu.h): submit scenes as they
arrive, poll for their solutions.  Requests run the direct operator on one GPU, several at once
when their device footprints fit the server's budget together; each result equals the result of
the same request solved alone."""
import ctypes as C

import numpy as np

from . import _native as N
from .solver import _params


class SolveServer:
    def __init__(self, max_concurrent=2, memory_budget=0, device=0):
        self.L = N.load()
        h = C.c_void_p()
        N.check(self.L.foggy_server_start(int(device), int(max_concurrent), int(memory_budget), C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, scene, rhs_per_wave=False, init_with_single_sphere=False, pair_tables=0, precision=0):
        """Queue one solve of scene (its plane waves summed into one right-hand side, or one
        right-hand side per wave); precision 1 solves it in mixed precision (FP32 Arnoldi steps,
        FP64 residuals).  Returns the request id."""
        s = scene
        prm = _params(s, False, init_with_single_sphere, 0, pair_tables, precision=precision)
        arrs = dict(params=prm, centres=N.as_f64(s.centres).reshape(-1), pidx=N.as_i32(s.param_index),
                    m=N.as_c128(s.refractive_index), r=N.as_f64(s.radius),
                    nr=N.as_i32(s.n_range_param).reshape(-1), th=N.as_f64(s.wave_theta), ph=N.as_f64(s.wave_phi),
                    jo=N.as_f64(s.jones).reshape(-1), g=N.as_f64(s.wave_g), pa=N.as_f64(s.wave_phase),
                    d0=N.as_f64(s.wave_d0).reshape(-1))
        q = N.FoggyRequest(C.pointer(prm), s.n_spheres, arrs["centres"].ctypes.data, arrs["pidx"].ctypes.data,
                           s.n_param, arrs["m"].ctypes.data, arrs["r"].ctypes.data, arrs["nr"].ctypes.data,
                           s.n_waves, arrs["th"].ctypes.data, arrs["ph"].ctypes.data, arrs["jo"].ctypes.data,
                           arrs["g"].ctypes.data, arrs["pa"].ctypes.data, arrs["d0"].ctypes.data,
                           int(bool(rhs_per_wave)))
        rid = C.c_int64()
        N.check(self.L.foggy_server_submit(self.h, C.byref(q), C.byref(rid)))
        return rid.value

    def poll(self, rid, wait_ms=0):
        """(info dict, x or None, cross-sections or None); x has shape (nrhs, vector length)."""
        info = N.FoggyRequestInfo()
        N.check(self.L.foggy_server_poll(self.h, int(rid), int(wait_ms), C.byref(info), None, 0, None))
        d = {f: getattr(info, f) for f, _ in info._fields_ if f not in ("stats", "error", "reserved")}
        d["stats"] = info.stats.as_dict()
        d["error"] = info.error.decode(errors="replace")
        if info.state != N.REQ_DONE:
            return d, None, None
        x = np.zeros(info.x_len // 2, np.complex128)
        cs = np.zeros(3 * info.nrhs)
        N.check(self.L.foggy_server_poll(self.h, int(rid), 0, C.byref(info), x.ctypes.data, info.x_len,
                                         cs.ctypes.data))
        return d, x.reshape(info.nrhs, -1), cs.reshape(info.nrhs, 3)

    def wait(self, rid):
        return self.poll(rid, wait_ms=-1)

    def cancel(self, rid):
        return int(self.L.foggy_server_cancel(self.h, int(rid)))

    def release(self, rid):
        N.check(self.L.foggy_server_release(self.h, int(rid)))

    def stop(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.foggy_server_stop(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
