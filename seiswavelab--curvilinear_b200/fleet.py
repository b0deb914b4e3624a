"""Multi-GPU serving in Python: ``Fleet`` over include/swl_fleet.h (one request loop per device,
requests placed by device-memory budget), plus the placement rule and the request-size estimate
on their own (no device needed)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, library
from .server import STATES, Config, ShotStatus, Stats, _bind as _bind_server
from .session import params2d, params3d

_dp = C.POINTER(C.c_double)
MAX_DEVICES = 16


class FleetConfig(C.Structure):
    _fields_ = [("n_devices", C.c_int32), ("devices", C.c_int32 * MAX_DEVICES), ("server", Config)]


_bound = False


def _bind():
    global _bound
    L = _bind_server()
    if _bound:
        return L
    vp, i64p = C.c_void_p, C.POINTER(C.c_int64)
    L.swl_request_bytes2d.argtypes = [C.c_void_p, i64p]
    L.swl_request_bytes3d.argtypes = [C.c_void_p, i64p]
    L.swl_fleet_choose.argtypes = [C.c_int32, i64p, i64p, C.c_int64]
    L.swl_fleet_choose.restype = C.c_int32
    L.swl_fleet_config_default.argtypes = [C.POINTER(FleetConfig)]
    L.swl_fleet_create.argtypes = [C.POINTER(FleetConfig), C.POINTER(vp)]
    L.swl_fleet_destroy.argtypes = [vp]
    L.swl_fleet_size.argtypes = [vp]
    L.swl_fleet_size.restype = C.c_int32
    L.swl_fleet_device.argtypes = [vp, C.c_int32]
    L.swl_fleet_device.restype = C.c_int32
    L.swl_fleet_submit2d.argtypes = [vp, C.c_void_p, i64p, C.POINTER(C.c_int32)]
    L.swl_fleet_submit3d.argtypes = [vp, C.c_void_p, i64p, C.POINTER(C.c_int32)]
    L.swl_fleet_status.argtypes = [vp, C.c_int64, C.POINTER(ShotStatus), C.POINTER(C.c_int32)]
    L.swl_fleet_records.argtypes = [vp, C.c_int64, _dp, _dp, _dp]
    L.swl_fleet_release.argtypes = [vp, C.c_int64]
    L.swl_fleet_drain.argtypes = [vp]
    L.swl_fleet_stats.argtypes = [vp, C.c_int32, C.POINTER(Stats), i64p]
    _bound = True
    return L


def request_bytes(params: dict, dim: int = 2) -> int:
    """Device bytes a server charges a request at admission (its resident-memory estimate)."""
    L = _bind()
    p, keep = (params2d if dim == 2 else params3d)(params)
    b = C.c_int64()
    _check((L.swl_request_bytes2d if dim == 2 else L.swl_request_bytes3d)(C.cast(C.byref(p), C.c_void_p), C.byref(b)))
    return b.value


def choose(budgets, charged, charge: int) -> int:
    """The fleet's placement rule: the slot a request of `charge` bytes goes to (-1: none can hold it)."""
    n = len(budgets)
    b = (C.c_int64 * n)(*[int(x) for x in budgets])
    c = (C.c_int64 * n)(*[int(x) for x in charged])
    return int(_bind().swl_fleet_choose(n, b, c, int(charge)))


def plan(requests, budgets):
    """Placement of a request list on devices of the given budgets when no shot finishes in
    between (the charges only grow): the slot of each request, the rule applied in order."""
    charged = [0] * len(budgets)
    slots = []
    for r in requests:
        need = request_bytes(r["params"], r["dim"])
        s = choose(budgets, charged, need)
        slots.append(s)
        if s >= 0:
            charged[s] += need
    return slots


class Fleet:
    def __init__(self, devices=None, memory_budget: int = 0, max_active: int = 0, batch_steps: int = 64,
                 build_threads: int = 4, scheduler_threads: int = 4, persistent: int = 0, persistent_ctas: int = -1):
        L = _bind()
        c = FleetConfig()
        L.swl_fleet_config_default(C.byref(c))
        devs = list(devices or [])
        c.n_devices = len(devs)
        for k, d in enumerate(devs):
            c.devices[k] = int(d)
        s = c.server
        s.memory_budget, s.max_active, s.batch_steps = int(memory_budget), int(max_active), int(batch_steps)
        s.build_threads, s.scheduler_threads = int(build_threads), int(scheduler_threads)
        s.persistent, s.persistent_ctas = int(persistent), int(persistent_ctas)
        h = C.c_void_p()
        _check(L.swl_fleet_create(C.byref(c), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().swl_fleet_destroy(self._h)
            self._h = C.c_void_p()

    __del__ = close

    def size(self) -> int:
        return int(_bind().swl_fleet_size(self._h))

    def device(self, slot: int) -> int:
        return int(_bind().swl_fleet_device(self._h, int(slot)))

    def submit(self, params: dict, dim: int = 2):
        """Returns (fleet id, slot)."""
        L = _bind()
        p, keep = (params2d if dim == 2 else params3d)(params)
        i, s = C.c_int64(), C.c_int32()
        _check((L.swl_fleet_submit2d if dim == 2 else L.swl_fleet_submit3d)(self._h, C.cast(C.byref(p), C.c_void_p),
                                                                            C.byref(i), C.byref(s)))
        return i.value, s.value

    def status(self, sid: int) -> dict:
        st, slot = ShotStatus(), C.c_int32()
        _check(_bind().swl_fleet_status(self._h, sid, C.byref(st), C.byref(slot)))
        d = {k: getattr(st, k) for k, _ in ShotStatus._fields_ if k not in ("pad", "error")}
        d["state"] = STATES[st.state]
        d["error"] = st.error.decode()
        d["slot"] = slot.value
        return d

    def records(self, sid: int):
        st = self.status(sid)
        shape = (st["receivers"], st["samples"])
        if st["dim"] == 2:
            vx, vz = np.zeros(shape), np.zeros(shape)
            _check(_bind().swl_fleet_records(self._h, sid, vx.ctypes.data_as(_dp), None, vz.ctypes.data_as(_dp)))
            return [vx, vz]
        t = [np.zeros(shape) for _ in range(3)]
        _check(_bind().swl_fleet_records(self._h, sid, *(x.ctypes.data_as(_dp) for x in t)))
        return t

    def release(self, sid: int):
        _check(_bind().swl_fleet_release(self._h, sid))

    def drain(self):
        _check(_bind().swl_fleet_drain(self._h))

    def stats(self, slot: int) -> dict:
        s, charged = Stats(), C.c_int64()
        _check(_bind().swl_fleet_stats(self._h, int(slot), C.byref(s), C.byref(charged)))
        d = {k: getattr(s, k) for k, _ in Stats._fields_}
        d["charged"] = charged.value
        return d
