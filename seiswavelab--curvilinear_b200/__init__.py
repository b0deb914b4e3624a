"""swl_b200: B200-native curvilinear velocity-stress engine (Python view of the C ABI).

The compute path is ``libswl_b200.so`` (hand-written sm_100a kernels behind the C ABI in
``include/swl_b200.h``); this module only marshals arrays through ctypes.  There is no CPU
fallback: importing works anywhere, but creating an engine without the library or without an
sm_100 GPU raises ``SwlError``.

Engine level (drop-in for the reference CUDA engines):
    ``Engine2D(mesh, receivers)``  ~ Seis2D::Curvilinear::CudaEngine (src/two_d/CudaEngine2D.hpp)
    ``Engine3D(mesh, receivers)``  ~ Seis3D::Curvilinear::CudaEngine3D (src/three_d/CudaEngine3D.hpp)
Session level (model build + engine), mirroring Simulation / ISimulationBackend3D, lives in
``session.py``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("SWL_B200_LIBRARY", PKG / "libswl_b200.so"))  # override: an alternative build

SWL_FP64, SWL_FP32 = 0, 1
OK, ERR_INVALID, ERR_CUDA, ERR_MEMORY, ERR_FAULT, ERR_UNAVAILABLE, ERR_STATE = 0, -1, -2, -3, -4, -5, -6
_NAMES = {ERR_INVALID: "invalid", ERR_CUDA: "cuda", ERR_MEMORY: "memory", ERR_FAULT: "fault",
          ERR_UNAVAILABLE: "unavailable", ERR_STATE: "state"}


class SwlError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{_NAMES.get(status, status)}] {message}")
        self.status = status


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)


class Mesh2D(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("nz", C.c_int32), ("count", C.c_int64), ("h", C.c_double),
        ("a", _vp), ("b", _vp), ("jac", _vp), ("normals", _vp), ("lam", _vp), ("mu", _vp), ("rho", _vp),
        ("source", _vp), ("damping", _vp), ("source_direction", C.c_double * 3), ("source_gradient", _vp * 2),
        ("mechanisms", C.c_int32), ("field_count", C.c_int32), ("cpml_x", _vp), ("cpml_z", _vp),
        ("cpml_width_x", C.c_int32), ("cpml_width_z", C.c_int32), ("cpml_count", C.c_int64),
        ("rates", C.c_double * 3), ("delta_p", _vp * 3), ("delta_s", _vp * 3),
        ("precision", C.c_int32), ("array_precision", C.c_int32), ("segment_rule", C.c_int32),
    ]


class Diag2D(C.Structure):
    _fields_ = [("energy", C.c_double), ("peak_energy", C.c_double), ("max_velocity", C.c_double),
                ("traction_relative", C.c_double), ("finite", C.c_int32), ("rhs_registers", C.c_int32),
                ("rhs_local_bytes", C.c_int64), ("resident_bytes", C.c_int64)]


class Mesh3D(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("count", C.c_int64),
        ("h", C.c_double), ("lam", C.c_double), ("mu", C.c_double), ("density", C.c_double),
        ("metrics", _dp), ("normals", _dp), ("jacobian", _dp), ("source", _dp), ("damping", _dp),
        ("material_lambda", _dp), ("material_mu", _dp), ("material_density", _dp),
        ("source_direction", C.c_double * 3), ("source_amplitude", C.c_double), ("source_gradient", _dp * 3),
        ("precision", C.c_int32),
        ("cpml_x", _dp), ("cpml_y", _dp), ("cpml_z", _dp), ("cpml_width_x", C.c_int32), ("cpml_width_y", C.c_int32),
        ("cpml_width_z", C.c_int32), ("cpml_count", C.c_int64),
        ("mechanisms", C.c_int32), ("rates", C.c_double * 3), ("delta_p", _dp * 3), ("delta_s", _dp * 3),
    ]


class Diag3D(C.Structure):
    _fields_ = [("energy", C.c_double), ("peak_energy", C.c_double), ("max_velocity", C.c_double),
                ("traction_rate_relative", C.c_double), ("peaks", C.c_double * 5), ("finite", C.c_int32),
                ("rhs_registers", C.c_int32), ("resident_bytes", C.c_int64)]


class Profile(C.Structure):
    _fields_ = [("stage_ms", C.c_double * 4), ("stats_ms", C.c_double), ("verdict_ms", C.c_double),
                ("step_ms", C.c_double), ("steps", C.c_int64), ("launches_per_step", C.c_int64),
                ("bytes_per_step", C.c_double), ("extra_bytes_per_step", C.c_double)]

    def as_dict(self) -> dict:
        return {"stage_ms": list(self.stage_ms), "stats_ms": self.stats_ms, "verdict_ms": self.verdict_ms,
                "step_ms": self.step_ms, "steps": self.steps, "launches_per_step": self.launches_per_step,
                "bytes_per_step": self.bytes_per_step, "extra_bytes_per_step": self.extra_bytes_per_step}


class Layout2D(C.Structure):
    _fields_ = [("strip_width", C.c_int32), ("block_rows", C.c_int32), ("segment_blocks", C.c_int32),
                ("strips", C.c_int32), ("segments", C.c_int32), ("interior_ctas", C.c_int64),
                ("exact_h", C.c_int32), ("precision", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


_lib = None


def library() -> C.CDLL:
    """Load libswl_b200.so (building it first when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("_swl_build", PKG / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    L = C.CDLL(str(LIB_PATH))
    L.swl_last_error.restype = C.c_char_p
    L.swl_version.restype = C.c_char_p
    L.swl_device_count.restype = C.c_int32
    L.swl2d_create.argtypes = [C.POINTER(Mesh2D), _i64p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.swl2d_destroy.argtypes = [C.c_void_p]
    L.swl2d_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32]
    L.swl2d_advance.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.POINTER(C.c_int32)]
    L.swl2d_rollback.argtypes = [C.c_void_p]
    L.swl2d_reset.argtypes = [C.c_void_p]
    L.swl2d_diagnostics.argtypes = [C.c_void_p, C.POINTER(Diag2D)]
    L.swl2d_step_diagnostics.argtypes = [C.c_void_p, C.POINTER(Diag2D)]
    L.swl2d_sample.argtypes = [C.c_void_p, _dp, _dp]
    L.swl2d_traces.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _dp, _dp]
    L.swl2d_snapshot.argtypes = [C.c_void_p, C.c_int32, _dp]
    L.swl2d_load_field.argtypes = [C.c_void_p, C.c_int32, _dp]
    L.swl2d_probes.argtypes = [C.c_void_p, _i64p, C.c_int32, _dp]
    L.swl2d_resident_bytes.argtypes = [C.c_void_p]
    L.swl2d_resident_bytes.restype = C.c_int64
    L.swl2d_layout.argtypes = [C.c_void_p, C.POINTER(Layout2D)]
    L.swl3d_create.argtypes = [C.POINTER(Mesh3D), _i64p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.swl3d_destroy.argtypes = [C.c_void_p]
    L.swl3d_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int32]
    L.swl3d_advance.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                C.POINTER(C.c_int32)]
    L.swl3d_rollback.argtypes = [C.c_void_p]
    L.swl3d_reset.argtypes = [C.c_void_p]
    L.swl3d_diagnostics.argtypes = [C.c_void_p, C.POINTER(Diag3D)]
    L.swl3d_step_diagnostics.argtypes = [C.c_void_p, C.POINTER(Diag3D)]
    L.swl3d_sample.argtypes = [C.c_void_p, _dp, _dp, _dp]
    L.swl3d_traces.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _dp, _dp, _dp]
    L.swl3d_snapshot.argtypes = [C.c_void_p, C.c_int32, _dp]
    L.swl3d_load_field.argtypes = [C.c_void_p, C.c_int32, _dp]
    L.swl3d_resident_bytes.argtypes = [C.c_void_p]
    L.swl3d_resident_bytes.restype = C.c_int64
    L.swl2d_profile.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                C.POINTER(Profile)]
    L.swl3d_profile.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.POINTER(Profile)]
    L.swl2d_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.swl3d_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.swl2d_reserve.argtypes = [C.c_void_p, C.c_int32]
    L.swl3d_reserve.argtypes = [C.c_void_p, C.c_int32]
    L.swl2d_launch.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double]
    L.swl2d_query.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.swl2d_wait.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
    L.swl2d_queue_create.argtypes = [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.swl2d_queue_destroy.argtypes = [C.c_void_p]
    L.swl2d_queue_launch.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.swl2d_queue_query.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
    L.swl2d_queue_limit.argtypes = [C.c_void_p, C.c_int32]
    L.swl2d_queue_segment.argtypes = [C.c_void_p, C.c_int32]
    L.swl2d_queue_wait.argtypes = [C.c_void_p]
    L.swl3d_launch.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double]
    L.swl3d_query.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.swl3d_wait.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
    _lib = L
    return L


def _check(status: int):
    if status != OK:
        raise SwlError(status, library().swl_last_error().decode())


def device_count() -> int:
    return int(library().swl_device_count())


def layout2d(engine_handle) -> dict:
    """swl2d_layout of an engine handle (Engine2D._h, or a session's engine_handle())."""
    out = Layout2D()
    h = engine_handle if isinstance(engine_handle, C.c_void_p) else C.c_void_p(engine_handle)
    _check(library().swl2d_layout(h, C.byref(out)))
    return out.as_dict()


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Queue2D:
    """Persistent multi-shot launches (swl2d_queue_*): the batches of several Engine2D of one
    precision and GSLS mechanism count advance together in one kernel launch."""

    def __init__(self, precision: int = SWL_FP32, device: int = -1):
        h = C.c_void_p()
        _check(library().swl2d_queue_create(int(device), int(precision), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().swl2d_queue_destroy(self._h)
            self._h = C.c_void_p()

    __del__ = close

    def launch(self, engines, first, count, dt, frequency, scale, growth_after=None):
        """One launch for batches (first[i], count[i], dt[i], ...) of engines[i]; scalars broadcast."""
        n = len(engines)

        def vec(v, ctype, default=None):
            v = default if v is None else v
            v = [v] * n if np.isscalar(v) else list(v)
            return (ctype * n)(*v)
        hs = (C.c_void_p * n)(*[e._h.value for e in engines])
        _check(library().swl2d_queue_launch(self._h, hs, n, vec(first, C.c_int32), vec(count, C.c_int32),
                                            vec(dt, C.c_double), vec(frequency, C.c_double), vec(scale, C.c_double),
                                            vec(growth_after, C.c_double, np.inf)))

    def limit(self, ctas_per_sm: int):
        """Resident CTAs per SM of later launches (0 all, n > 0 at most n, n < 0 all but -n)."""
        _check(library().swl2d_queue_limit(self._h, int(ctas_per_sm)))

    def segment(self, seg: int):
        """Row blocks per work item (1, 2, 4, 8), or 0: chosen per grid."""
        _check(library().swl2d_queue_segment(self._h, int(seg)))

    def query(self) -> bool:
        done = C.c_int32()
        _check(library().swl2d_queue_query(self._h, C.byref(done)))
        return bool(done.value)

    def wait(self):
        _check(library().swl2d_queue_wait(self._h))


class Engine2D:
    """GPU engine for one 2D shot, built from a mesh dictionary.

    Mesh keys follow the reference's MeshT names: nx, nz (padded), h, metricA, metricB,
    jacobian, normals, lambda, mu, density, source, damping, sourceDirection,
    sourceGradientX/Z (moment source), fieldCount, mechanisms, rates, deltaP0.., deltaS0..,
    cpmlX, cpmlZ, cpmlWidthX, cpmlWidthZ, cpmlCount.
    """

    def __init__(self, mesh: dict, receivers=(), precision: int = SWL_FP64, device: int = -1):
        L = library()
        self._keep = []

        def arr(k):
            v = mesh.get(k)
            if v is None:
                return None
            v = _f64(v)
            self._keep.append(v)
            return v.ctypes.data

        g = Mesh2D()
        g.nx, g.nz = int(mesh["nx"]), int(mesh["nz"])
        g.count = g.nx * g.nz
        g.h = float(mesh["h"])
        g.a, g.b, g.jac, g.normals = arr("metricA"), arr("metricB"), arr("jacobian"), arr("normals")
        g.lam, g.mu, g.rho = arr("lambda"), arr("mu"), arr("density")
        g.source, g.damping = arr("source"), arr("damping")
        sd = mesh.get("sourceDirection", (0.0, 0.0, 1.0))
        for a in range(3):
            g.source_direction[a] = float(sd[a])
        g.source_gradient[0], g.source_gradient[1] = arr("sourceGradientX"), arr("sourceGradientZ")
        g.mechanisms = int(mesh.get("mechanisms", 0))
        g.field_count = int(mesh.get("fieldCount", 5))
        g.cpml_x, g.cpml_z = arr("cpmlX"), arr("cpmlZ")
        g.cpml_width_x, g.cpml_width_z = int(mesh.get("cpmlWidthX", 0)), int(mesh.get("cpmlWidthZ", 0))
        g.cpml_count = int(mesh.get("cpmlCount", 0))
        rates = mesh.get("rates", (0, 0, 0))
        for l in range(3):
            g.rates[l] = float(rates[l])
            g.delta_p[l], g.delta_s[l] = arr(f"deltaP{l}"), arr(f"deltaS{l}")
        g.precision, g.array_precision = int(precision), SWL_FP64
        self.field_count, self.count, self.cpml_count = g.field_count, g.count, g.cpml_count
        self.nx, self.nz = g.nx, g.nz
        rec = np.ascontiguousarray(receivers, dtype=np.int64)
        self.nrec = len(rec)
        h = C.c_void_p()
        _check(L.swl2d_create(C.byref(g), rec.ctypes.data_as(_i64p), len(rec), int(device), C.byref(h)))
        self._h = h
        self._keep.clear()

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().swl2d_destroy(self._h)
            self._h = C.c_void_p()

    __del__ = close

    def step(self, dt, frequency, scale, step):
        _check(library().swl2d_step(self._h, step * dt, dt, frequency, scale, step))

    def advance(self, first, count, dt, frequency, scale, growth_after=np.inf):
        acc = C.c_int32()
        st = library().swl2d_advance(self._h, first, count, dt, frequency, scale, growth_after, C.byref(acc))
        if st not in (OK, ERR_FAULT):
            _check(st)
        return acc.value, st == ERR_FAULT

    def launch(self, first, count, dt, frequency, scale, growth_after=np.inf):
        """Enqueue a batch and return at once (see swl2d_launch)."""
        _check(library().swl2d_launch(self._h, first, count, dt, frequency, scale, growth_after))

    def query(self):
        """(done, accepted, faulted) of the batch in flight, without blocking."""
        done, acc = C.c_int32(), C.c_int32()
        st = library().swl2d_query(self._h, C.byref(done), C.byref(acc))
        if st not in (OK, ERR_FAULT):
            _check(st)
        return bool(done.value), acc.value, st == ERR_FAULT

    def wait(self):
        acc = C.c_int32()
        st = library().swl2d_wait(self._h, C.byref(acc))
        if st not in (OK, ERR_FAULT):
            _check(st)
        return acc.value, st == ERR_FAULT

    def rollback(self):
        _check(library().swl2d_rollback(self._h))

    def reset(self):
        _check(library().swl2d_reset(self._h))

    def diagnostics(self) -> dict:
        d = Diag2D()
        _check(library().swl2d_diagnostics(self._h, C.byref(d)))
        return {k: getattr(d, k) for k, _ in Diag2D._fields_}

    def step_diagnostics(self) -> dict:
        """The last accepted step's diagnostics as the device verdict computed them (no kernel)."""
        d = Diag2D()
        _check(library().swl2d_step_diagnostics(self._h, C.byref(d)))
        return {k: getattr(d, k) for k, _ in Diag2D._fields_}

    def sample(self):
        vx, vz = np.zeros(self.nrec), np.zeros(self.nrec)
        _check(library().swl2d_sample(self._h, vx.ctypes.data_as(_dp), vz.ctypes.data_as(_dp)))
        return vx, vz

    def traces(self, first, count):
        vx, vz = np.zeros((self.nrec, count)), np.zeros((self.nrec, count))
        _check(library().swl2d_traces(self._h, first, count, vx.ctypes.data_as(_dp), vz.ctypes.data_as(_dp)))
        return vx, vz

    def field(self, f: int) -> np.ndarray:
        out = np.zeros(self.cpml_count if f == -1 else self.count)
        _check(library().swl2d_snapshot(self._h, f, out.ctypes.data_as(_dp)))
        return out

    def fields(self) -> np.ndarray:
        return np.stack([self.field(f) for f in range(self.field_count)])

    def load(self, f: int, values):
        v = _f64(values)
        _check(library().swl2d_load_field(self._h, f, v.ctypes.data_as(_dp)))

    def probes(self, nodes):
        nodes = np.ascontiguousarray(nodes, dtype=np.int64)
        out = np.zeros((len(nodes), 5))
        _check(library().swl2d_probes(self._h, nodes.ctypes.data_as(_i64p), len(nodes), out.ctypes.data_as(_dp)))
        return out

    def resident_bytes(self) -> int:
        return int(library().swl2d_resident_bytes(self._h))

    def profile(self, first, count, dt, frequency, scale) -> dict:
        p = Profile()
        _check(library().swl2d_profile(self._h, first, count, dt, frequency, scale, C.byref(p)))
        return p.as_dict()

    def layout(self) -> dict:
        """Stage decomposition: strips x segments CTAs, how many run the interior form, exact 1/h."""
        return layout2d(self._h)

    def set_stream(self, stream_handle: int | None):
        _check(library().swl2d_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def reserve(self, steps: int):
        _check(library().swl2d_reserve(self._h, int(steps)))


class Engine3D:
    """GPU engine for one 3D shot.  Mesh keys: nx, ny, nz (padded), h, lambda, mu, density,
    metrics (9 per node), normals (3 per node), jacobian, source, damping, sourceAmplitude,
    sourceDirection, sourceGradient0..2, materialLambda/Mu/Density (layered)."""

    def __init__(self, mesh: dict, receivers=(), precision: int = SWL_FP64, device: int = -1):
        L = library()
        keep = []

        def arr(k):
            v = mesh.get(k)
            if v is None:
                return None
            v = _f64(v)
            keep.append(v)
            return v.ctypes.data_as(_dp)

        g = Mesh3D()
        g.nx, g.ny, g.nz = int(mesh["nx"]), int(mesh["ny"]), int(mesh["nz"])
        g.count = g.nx * g.ny * g.nz
        g.h, g.lam, g.mu, g.density = float(mesh["h"]), float(mesh["lambda"]), float(mesh["mu"]), float(mesh["density"])
        g.metrics, g.normals, g.jacobian = arr("metrics"), arr("normals"), arr("jacobian")
        g.source, g.damping = arr("source"), arr("damping")
        g.material_lambda, g.material_mu, g.material_density = (arr("materialLambda"), arr("materialMu"),
                                                                 arr("materialDensity"))
        sd = mesh.get("sourceDirection", (0.0, 0.0, 1.0))
        for a in range(3):
            g.source_direction[a] = float(sd[a])
            g.source_gradient[a] = arr(f"sourceGradient{a}")
        g.source_amplitude = float(mesh["sourceAmplitude"])
        g.precision = int(precision)
        g.cpml_x, g.cpml_y, g.cpml_z = arr("cpmlX"), arr("cpmlY"), arr("cpmlZ")
        g.cpml_width_x, g.cpml_width_y = int(mesh.get("cpmlWidthX", 0)), int(mesh.get("cpmlWidthY", 0))
        g.cpml_width_z, g.cpml_count = int(mesh.get("cpmlWidthZ", 0)), int(mesh.get("cpmlCount", 0))
        g.mechanisms = int(mesh.get("mechanisms", 0))
        for l in range(g.mechanisms):
            g.rates[l] = float(np.atleast_1d(mesh["rates"])[l])
            g.delta_p[l], g.delta_s[l] = arr(f"deltaP{l}"), arr(f"deltaS{l}")
        self.field_count = 9 + 6 * g.mechanisms
        self.count, self.nrec = g.count, len(receivers)
        self.cpml_count = g.cpml_count
        rec = np.ascontiguousarray(receivers, dtype=np.int64)
        h = C.c_void_p()
        _check(L.swl3d_create(C.byref(g), rec.ctypes.data_as(_i64p), len(rec), int(device), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().swl3d_destroy(self._h)
            self._h = C.c_void_p()

    __del__ = close

    def step(self, dt, frequency, step):
        _check(library().swl3d_step(self._h, step * dt, dt, frequency, step))

    def advance(self, first, count, dt, frequency, growth_after=np.inf):
        acc = C.c_int32()
        st = library().swl3d_advance(self._h, first, count, dt, frequency, growth_after, C.byref(acc))
        if st not in (OK, ERR_FAULT):
            _check(st)
        return acc.value, st == ERR_FAULT

    def rollback(self):
        _check(library().swl3d_rollback(self._h))

    def reset(self):
        _check(library().swl3d_reset(self._h))

    def diagnostics(self) -> dict:
        d = Diag3D()
        _check(library().swl3d_diagnostics(self._h, C.byref(d)))
        out = {k: getattr(d, k) for k, _ in Diag3D._fields_}
        out["peaks"] = list(d.peaks)
        return out

    def step_diagnostics(self) -> dict:
        """The last accepted step's diagnostics as the device verdict computed them (no kernel)."""
        d = Diag3D()
        _check(library().swl3d_step_diagnostics(self._h, C.byref(d)))
        out = {k: getattr(d, k) for k, _ in Diag3D._fields_}
        out["peaks"] = list(d.peaks)
        return out

    def traces(self, first, count):
        t = [np.zeros((self.nrec, count)) for _ in range(3)]
        _check(library().swl3d_traces(self._h, first, count, *(x.ctypes.data_as(_dp) for x in t)))
        return t

    def field(self, f: int) -> np.ndarray:
        """Field f (0..8) of the current state, or f = -1: the CFS-PML memories."""
        out = np.zeros(max(self.cpml_count, 1) if f == -1 else self.count)
        _check(library().swl3d_snapshot(self._h, f, out.ctypes.data_as(_dp)))
        return out[: self.cpml_count] if f == -1 else out

    def fields(self) -> np.ndarray:
        return np.stack([self.field(f) for f in range(9)])

    def load(self, f: int, values):
        v = _f64(values)
        _check(library().swl3d_load_field(self._h, f, v.ctypes.data_as(_dp)))

    def resident_bytes(self) -> int:
        return int(library().swl3d_resident_bytes(self._h))

    def profile(self, first, count, dt, frequency) -> dict:
        p = Profile()
        _check(library().swl3d_profile(self._h, first, count, dt, frequency, C.byref(p)))
        return p.as_dict()

    def set_stream(self, stream_handle: int | None):
        _check(library().swl3d_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def reserve(self, steps: int):
        _check(library().swl3d_reserve(self._h, int(steps)))
