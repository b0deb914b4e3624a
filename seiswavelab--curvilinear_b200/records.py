"""Receiver records in Python over include/swl_records.h: SEG-Y export/import in the reference's
layout (src/common/SegyIo.cpp) and the sessions' receiver CSV / SEG-Y files."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, library

_dp = C.POINTER(C.c_double)
IEEE32, IEEE64, IBM32, COMPATIBLE_IEEE32 = 0, 1, 2, 3


class TraceView(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("source", C.c_double * 3), ("start_time", C.c_double),
                ("channels", _dp * 3)]


class RecordView(C.Structure):
    _fields_ = [("traces", C.POINTER(TraceView)), ("n_traces", C.c_int32), ("n_components", C.c_int32),
                ("n_samples", C.c_int64), ("components", C.c_char_p * 3), ("dt", C.c_double), ("units", C.c_char_p)]


class SegyOptions(C.Structure):
    _fields_ = [("profile", C.c_int32), ("sample_gain", C.c_double), ("sample_interval_s", C.c_double)]


class SegyInfo(C.Structure):
    _fields_ = [("n_traces", C.c_int32), ("max_samples", C.c_int64), ("dt", C.c_double), ("component", C.c_char * 64),
                ("units", C.c_char * 64), ("description", C.c_char * 128)]


_bound = False


def _bind():
    global _bound
    L = library()
    if _bound:
        return L
    vp = C.c_void_p
    L.swl_segy_options_default.argtypes = [C.POINTER(SegyOptions)]
    L.swl_write_segy.argtypes = [C.POINTER(RecordView), C.c_int32, C.c_char_p, C.POINTER(SegyOptions)]
    L.swl_read_segy.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.swl_segy_records_free.argtypes = [vp]
    L.swl_segy_records_info.argtypes = [vp, C.POINTER(SegyInfo)]
    L.swl_segy_records_trace.argtypes = [vp, C.c_int32, _dp, _dp, _dp, _dp, C.c_int64, C.POINTER(C.c_int64)]
    L.swl2d_session_write_segy.argtypes = [vp, C.c_int32, C.c_char_p, C.POINTER(SegyOptions)]
    L.swl3d_session_write_segy.argtypes = [vp, C.c_int32, C.c_char_p, C.POINTER(SegyOptions)]
    L.swl2d_session_write_receivers.argtypes = [vp, C.c_char_p]
    L.swl3d_session_write_receivers.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int32)]
    _bound = True
    return L


def options(profile: int = IEEE32, gain: float = 1.0, interval_s: float = 0.0) -> SegyOptions:
    return SegyOptions(int(profile), float(gain), float(interval_s))


def write_segy(path, channels, components, dt, component=0, positions=None, sources=None, start_times=None,
               units="m/s", profile=IEEE32, gain=1.0, interval_s=0.0):
    """writeSegy of a record set: channels[c] is a (traces x samples) array per component."""
    L = _bind()
    chans = [np.ascontiguousarray(np.asarray(c, dtype=np.float64)) for c in channels]
    n, s = chans[0].shape
    pos = np.zeros((n, 3)) if positions is None else np.asarray(positions, dtype=np.float64)
    src = np.zeros((n, 3)) if sources is None else np.asarray(sources, dtype=np.float64)
    start = np.zeros(n) if start_times is None else np.asarray(start_times, dtype=np.float64)
    tv = (TraceView * max(n, 1))()
    for r in range(n):
        tv[r].position[:] = list(pos[r])
        tv[r].source[:] = list(src[r])
        tv[r].start_time = float(start[r])
        for c, a in enumerate(chans):
            tv[r].channels[c] = a[r].ctypes.data_as(_dp)
    names = (C.c_char_p * 3)(*[x.encode() for x in components] + [None] * (3 - len(components)))
    v = RecordView(tv, n, len(chans), s, names, float(dt), units.encode())
    o = options(profile, gain, interval_s)
    _check(L.swl_write_segy(C.byref(v), int(component), str(path).encode(), C.byref(o)))


def read_segy(path) -> dict:
    """readSegy: dt, component, units, description and per trace position, source, start, samples."""
    L = _bind()
    h = C.c_void_p()
    _check(L.swl_read_segy(str(path).encode(), C.byref(h)))
    try:
        info = SegyInfo()
        _check(L.swl_segy_records_info(h, C.byref(info)))
        traces = []
        for r in range(info.n_traces):
            pos, src, start = (C.c_double * 3)(), (C.c_double * 3)(), C.c_double()
            buf = np.zeros(max(1, info.max_samples))
            n = C.c_int64()
            _check(L.swl_segy_records_trace(h, r, pos, src, C.byref(start), buf.ctypes.data_as(_dp), buf.size, C.byref(n)))
            traces.append({"position": list(pos), "source": list(src), "start": start.value, "samples": buf[:n.value].copy()})
        return {"dt": info.dt, "component": info.component.decode(), "units": info.units.decode(),
                "description": info.description.decode(), "traces": traces}
    finally:
        L.swl_segy_records_free(h)


def session_write_segy(sim, component: int, path, profile=IEEE32, gain=1.0, interval_s=0.0):
    """The session's records (2D: Vz, Vx; 3D: Vz, Vx, Vy) as one SEG-Y file per component."""
    L = _bind()
    o = options(profile, gain, interval_s)
    fn = L.swl3d_session_write_segy if type(sim).__name__ == "Simulation3D" else L.swl2d_session_write_segy
    _check(fn(sim._h, int(component), str(path).encode(), C.byref(o)))


def session_write_receivers(sim, path, selected=(1, 1, 1)):
    """writeReceivers (2D) / writeReceiversCsv (3D, `selected` = Vx, Vy, Vz)."""
    L = _bind()
    if type(sim).__name__ == "Simulation3D":
        sel = (C.c_int32 * 3)(*[int(bool(x)) for x in selected])
        _check(L.swl3d_session_write_receivers(sim._h, str(path).encode(), sel))
    else:
        _check(L.swl2d_session_write_receivers(sim._h, str(path).encode()))
