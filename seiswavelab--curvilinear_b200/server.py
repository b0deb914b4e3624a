"""Serving in Python: ``Server`` over include/swl_server.h (request loop with memory-budget
admission, concurrent shots on one GPU, records collected per shot)."""
from __future__ import annotations

import ctypes as C
import os

# The server runs every shot on its own CUDA stream.  With the CUDA default of 8 hardware work
# queues, streams beyond 8 share queues and serialise behind one another (measured: the batched
# makespan of the serving mix doubled); 32 queues keep them independent.  This only takes effect
# if it is set before the process creates its CUDA context, so it is set when this module is
# imported (a value the caller already set is kept).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import numpy as np

from . import _check, library
from .session import params2d, params3d

_dp = C.POINTER(C.c_double)


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("memory_budget", C.c_int64), ("max_active", C.c_int32),
                ("batch_steps", C.c_int32), ("build_threads", C.c_int32), ("scheduler_threads", C.c_int32),
                ("persistent", C.c_int32), ("persistent_ctas", C.c_int32)]


class ShotStatus(C.Structure):
    _fields_ = [("id", C.c_int64), ("dim", C.c_int32), ("state", C.c_int32), ("steps_done", C.c_int32),
                ("total_steps", C.c_int32), ("receivers", C.c_int32), ("pad", C.c_int32), ("samples", C.c_int64),
                ("resident_bytes", C.c_int64), ("submit_s", C.c_double), ("start_s", C.c_double),
                ("finish_s", C.c_double), ("run_s", C.c_double), ("error", C.c_char * 256)]


class Stats(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("queued", "building", "running", "done", "failed", "peak_running")] + \
               [(k, C.c_int64) for k in ("resident_bytes", "peak_resident_bytes", "memory_budget")]


STATES = {0: "queued", 1: "building", 2: "running", 3: "done", 4: "failed"}
_bound = False


def _bind():
    global _bound
    L = library()
    if _bound:
        return L
    vp = C.c_void_p
    L.swl_server_config_default.argtypes = [C.POINTER(Config)]
    L.swl_server_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.swl_server_destroy.argtypes = [vp]
    L.swl_server_submit2d.argtypes = [vp, C.c_void_p, C.POINTER(C.c_int64)]
    L.swl_server_submit3d.argtypes = [vp, C.c_void_p, C.POINTER(C.c_int64)]
    L.swl_server_status.argtypes = [vp, C.c_int64, C.POINTER(ShotStatus)]
    L.swl_server_next_finished.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64)]
    L.swl_server_records.argtypes = [vp, C.c_int64, _dp, _dp, _dp]
    L.swl_server_release.argtypes = [vp, C.c_int64]
    L.swl_server_drain.argtypes = [vp]
    L.swl_server_stats_get.argtypes = [vp, C.POINTER(Stats)]
    _bound = True
    return L


class Server:
    def __init__(self, device: int = -1, memory_budget: int = 0, max_active: int = 0, batch_steps: int = 64,
                 build_threads: int = 4, scheduler_threads: int = 4, persistent: int = 0,
                 persistent_ctas: int = -1):
        L = _bind()
        c = Config()
        L.swl_server_config_default(C.byref(c))
        c.device, c.memory_budget, c.max_active = device, int(memory_budget), int(max_active)
        c.batch_steps, c.build_threads = int(batch_steps), int(build_threads)
        c.scheduler_threads = int(scheduler_threads)
        c.persistent = int(persistent)
        c.persistent_ctas = int(persistent_ctas)
        h = C.c_void_p()
        _check(L.swl_server_create(C.byref(c), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().swl_server_destroy(self._h)
            self._h = C.c_void_p()

    __del__ = close

    def submit(self, params: dict, dim: int = 2) -> int:
        L = _bind()
        p, keep = (params2d if dim == 2 else params3d)(params)
        i = C.c_int64()
        _check((L.swl_server_submit2d if dim == 2 else L.swl_server_submit3d)(self._h, C.cast(C.byref(p), C.c_void_p),
                                                                              C.byref(i)))
        return i.value

    def status(self, sid: int) -> dict:
        s = ShotStatus()
        _check(_bind().swl_server_status(self._h, sid, C.byref(s)))
        d = {k: getattr(s, k) for k, _ in ShotStatus._fields_ if k not in ("pad", "error")}
        d["state"] = STATES[s.state]
        d["error"] = s.error.decode()
        return d

    def next_finished(self, timeout_ms: int = 1000):
        i = C.c_int64()
        _check(_bind().swl_server_next_finished(self._h, int(timeout_ms), C.byref(i)))
        return None if i.value < 0 else i.value

    def records(self, sid: int):
        st = self.status(sid)
        shape = (st["receivers"], st["samples"])
        if st["dim"] == 2:
            vx, vz = np.zeros(shape), np.zeros(shape)
            _check(_bind().swl_server_records(self._h, sid, vx.ctypes.data_as(_dp), None, vz.ctypes.data_as(_dp)))
            return [vx, vz]
        t = [np.zeros(shape) for _ in range(3)]
        _check(_bind().swl_server_records(self._h, sid, *(x.ctypes.data_as(_dp) for x in t)))
        return t

    def release(self, sid: int):
        _check(_bind().swl_server_release(self._h, sid))

    def drain(self):
        _check(_bind().swl_server_drain(self._h))

    def stats(self) -> dict:
        s = Stats()
        _check(_bind().swl_server_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}
