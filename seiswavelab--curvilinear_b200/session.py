"""Session level in Python: ``Simulation2D`` / ``Simulation3D`` over include/swl_session.h.

Parameters are dictionaries in the reference's vocabulary (the same keys as its Parameters /
SimulationParameters members, e.g. ``nx, nz, spacing, relief, wavelength, frequency, duration,
cfl, sourceX, sourceZ, sourceKind, absorber, spongeX, externalAbsorption, receiverStart,
receiverCount, layered, layers, attenuation, mechanisms, qp, qs, importedSurface, surface``).
2D layer rows are (thickness, vp, vs, density, qp, qs); 3D rows are (thickness, vp, vs, density).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import SWL_FP64, SwlError, _check, library

MODEL_ONLY = -2
_dp = C.POINTER(C.c_double)


class Layer2D(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("thickness", "vp", "vs", "density", "qp", "qs")]


class Params2D(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("nx", C.c_int32), ("nz", C.c_int32),
        *[(k, C.c_double) for k in ("spacing", "vp", "vs", "density", "relief", "wavelength", "flatten_depth",
                                   "frequency", "duration", "cfl", "force_per_length")],
        ("source_x", C.c_int32), ("source_z", C.c_int32), ("max_steps", C.c_int32), ("source_kind", C.c_int32),
        ("source_direction", C.c_double * 3),
        ("moment_per_length", C.c_double), ("source_sigma_m", C.c_double), ("source_radius_m", C.c_double),
        ("absorbing", C.c_int32), ("sponge_x", C.c_int32), ("sponge_z", C.c_int32), ("sponge_strength", C.c_double),
        ("absorber", C.c_int32), ("cpml_reflection", C.c_double), ("cpml_kappa_max", C.c_double),
        ("cpml_frequency", C.c_double), ("external_absorption", C.c_int32),
        ("receiver_start", C.c_int32), ("receiver_count", C.c_int32), ("receiver_stride", C.c_int32),
        ("receiver_depth", C.c_int32), ("sample_interval_ms", C.c_double),
        ("layered", C.c_int32), ("n_layers", C.c_int32), ("layers", C.POINTER(Layer2D)),
        ("attenuation", C.c_int32), ("mechanisms", C.c_int32),
        *[(k, C.c_double) for k in ("q_min_frequency", "q_max_frequency", "q_reference_frequency", "qp", "qs")],
        ("imported_surface", C.c_int32), ("n_surface", C.c_int32), ("surface_datum", C.c_double),
        ("surface_xz", _dp), ("device_geometry", C.c_int32), ("segment_rule", C.c_int32),
    ]


class Info2D(C.Structure):
    _fields_ = [*[(k, C.c_int32) for k in ("nx", "nz", "model_offset_x", "total_steps", "step", "field_count",
                                           "receivers", "completed", "finite", "mechanisms")],
                *[(k, C.c_int64) for k in ("count", "samples", "cpml_count", "resident_bytes")],
                *[(k, C.c_double) for k in ("dt", "record_dt", "h", "flatten_depth", "max_metric", "min_jacobian",
                                            "max_edge", "ppw", "wave_dt", "damping_dt", "source_dt", "relaxation_dt",
                                            "cpml_dt", "max_relative_q_error", "energy", "peak_energy", "max_velocity",
                                            "traction_relative", "init_ms", "total_step_ms", "last_step_ms")]]


class Layer3D(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("thickness", "vp", "vs", "density")]


class Params3D(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        *[(k, C.c_double) for k in ("spacing", "vp", "vs", "density")],
        ("layered", C.c_int32), ("layer_depth_mode", C.c_int32), ("n_layers", C.c_int32), ("layers", C.POINTER(Layer3D)),
        ("frequency", C.c_double),
        *[(k, C.c_int32) for k in ("source_x", "source_y", "source_z", "source_kind")],
        ("source_direction", C.c_double * 3), ("source_force", C.c_double), ("source_moment", C.c_double),
        ("duration", C.c_double), ("max_steps", C.c_int32),
        *[(k, C.c_double) for k in ("cfl", "relief", "wavelength", "flatten_depth")],
        ("dem_nx", C.c_int32), ("dem_ny", C.c_int32),
        *[(k, C.c_double) for k in ("dem_spacing", "dem_origin_x", "dem_origin_y", "dem_datum")],
        ("dem_elevations", _dp),
        *[(k, C.c_int32) for k in ("receiver_kind", "receiver_start_x", "receiver_start_y", "receiver_z",
                                   "receiver_count_x", "receiver_count_y", "receiver_stride_x", "receiver_stride_y",
                                   "receiver_limit")],
        ("absorbing", C.c_int32), ("absorbing_cells", C.c_int32 * 3), ("absorbing_strength", C.c_double),
        ("device_geometry", C.c_int32), ("layer_names", C.POINTER(C.c_char_p)),
        ("absorber", C.c_int32), ("cpml_reflection", C.c_double), ("cpml_kappa_max", C.c_double),
        ("cpml_frequency", C.c_double),
        ("attenuation", C.c_int32), ("mechanisms", C.c_int32),
        *[(k, C.c_double) for k in ("q_min_frequency", "q_max_frequency", "q_reference_frequency", "qp", "qs")],
        ("layer_q", _dp),
    ]


class Info3D(C.Structure):
    _fields_ = [*[(k, C.c_int32) for k in ("nx", "ny", "nz", "total_steps", "step", "receivers", "completed", "finite")],
                *[(k, C.c_int64) for k in ("count", "resident_bytes")],
                *[(k, C.c_double) for k in ("dt", "h", "flatten_depth", "min_jacobian", "max_metric_norm",
                                            "min_cell_length", "max_cell_edge", "wave_dt", "damping_dt", "source_dt",
                                            "ppw", "energy", "peak_energy", "max_velocity", "traction_rate_relative",
                                            "init_ms", "total_step_ms", "last_step_ms")]]


_bound = False


class ModelCompute(C.Structure):
    _fields_ = [("backend", C.c_int32), ("cpu_threads", C.c_int32), ("cuda_device", C.c_int32)]


def _bind():
    global _bound
    L = library()
    if _bound:
        return L
    vp = C.c_void_p
    L.swl2d_params_default.argtypes = [C.POINTER(Params2D)]
    L.swl2d_session_create.argtypes = [C.POINTER(Params2D), C.c_int32, C.POINTER(vp)]
    L.swl2d_session_destroy.argtypes = [vp]
    L.swl2d_session_advance.argtypes = [vp, C.c_int32]
    L.swl2d_session_reset.argtypes = [vp]
    L.swl2d_session_info.argtypes = [vp, C.POINTER(Info2D)]
    L.swl2d_session_records.argtypes = [vp, _dp, _dp]
    L.swl2d_session_receiver_positions.argtypes = [vp, _dp]
    L.swl2d_session_snapshot.argtypes = [vp, C.c_int32, _dp]
    L.swl2d_session_model.argtypes = [vp, C.c_char_p, _dp, C.POINTER(C.c_int64)]
    L.swl2d_session_engine.argtypes = [vp]
    L.swl2d_session_engine.restype = vp
    L.swl2d_session_write_snapshot.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int32), C.c_int32]
    L.swl2d_session_write_model.argtypes = [vp, C.c_char_p, C.POINTER(ModelCompute)]
    L.swl2d_read_model.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.swl2d_model_document_params.argtypes = [vp, C.POINTER(Params2D), C.POINTER(ModelCompute), _dp]
    L.swl2d_model_document_free.argtypes = [vp]
    L.swl2d_session_read_probes.argtypes = [vp, C.POINTER(C.c_int32), C.c_int32, _dp]
    L.swl3d_params_default.argtypes = [C.POINTER(Params3D)]
    L.swl3d_session_create.argtypes = [C.POINTER(Params3D), C.c_int32, C.POINTER(vp)]
    L.swl3d_session_destroy.argtypes = [vp]
    L.swl3d_session_advance.argtypes = [vp, C.c_int32]
    L.swl3d_session_reset.argtypes = [vp]
    L.swl3d_session_info.argtypes = [vp, C.POINTER(Info3D)]
    L.swl3d_session_records.argtypes = [vp, _dp, _dp, _dp]
    L.swl3d_session_snapshot.argtypes = [vp, C.c_int32, _dp]
    L.swl3d_session_model.argtypes = [vp, C.c_char_p, _dp, C.POINTER(C.c_int64)]
    L.swl3d_session_engine.argtypes = [vp]
    L.swl3d_session_engine.restype = vp
    L.swl3d_session_write_snapshot.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int32), C.c_int32, C.c_int32]
    L.swl3d_session_write_model.argtypes = [vp, C.c_char_p, C.POINTER(ModelCompute)]
    L.swl3d_read_model.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.swl3d_model_document_params.argtypes = [vp, C.POINTER(Params3D), C.POINTER(ModelCompute), _dp]
    L.swl3d_model_document_free.argtypes = [vp]
    _bound = True
    return L


# reference parameter name -> C field (2D)
_MAP2D = {
    "precision": "precision", "nx": "nx", "nz": "nz", "spacing": "spacing", "vp": "vp", "vs": "vs",
    "density": "density", "relief": "relief", "wavelength": "wavelength", "flattenDepth": "flatten_depth",
    "frequency": "frequency", "duration": "duration", "cfl": "cfl", "forcePerLength": "force_per_length",
    "sourceX": "source_x", "sourceZ": "source_z", "maxSteps": "max_steps", "sourceKind": "source_kind",
    "momentPerLength": "moment_per_length", "sourceSigmaM": "source_sigma_m", "sourceRadiusM": "source_radius_m",
    "absorbing": "absorbing", "spongeX": "sponge_x", "spongeZ": "sponge_z", "spongeStrength": "sponge_strength",
    "absorber": "absorber", "cpmlReflection": "cpml_reflection", "cpmlKappaMax": "cpml_kappa_max",
    "cpmlFrequency": "cpml_frequency", "externalAbsorption": "external_absorption",
    "receiverStart": "receiver_start", "receiverCount": "receiver_count", "receiverStride": "receiver_stride",
    "receiverDepth": "receiver_depth", "sampleIntervalMs": "sample_interval_ms", "layered": "layered",
    "attenuation": "attenuation", "mechanisms": "mechanisms", "qMinFrequency": "q_min_frequency",
    "qMaxFrequency": "q_max_frequency", "qReferenceFrequency": "q_reference_frequency", "qp": "qp", "qs": "qs",
    "importedSurface": "imported_surface", "surfaceDatum": "surface_datum",
    "deviceGeometry": "device_geometry", "segmentRule": "segment_rule",
}
_MAP3D = {
    "precision": "precision", "nx": "nx", "ny": "ny", "nz": "nz", "spacing": "spacing", "vp": "vp", "vs": "vs",
    "density": "density", "layered": "layered", "layerDepthMode": "layer_depth_mode", "frequency": "frequency",
    "sourceX": "source_x", "sourceY": "source_y", "sourceZ": "source_z", "sourceKind": "source_kind",
    "sourceForce": "source_force", "sourceMoment": "source_moment", "duration": "duration", "maxSteps": "max_steps",
    "cfl": "cfl", "relief": "relief", "wavelength": "wavelength", "flattenDepth": "flatten_depth",
    "absorbing": "absorbing", "absorbingStrength": "absorbing_strength", "receiverLimit": "receiver_limit",
    "deviceGeometry": "device_geometry", "absorber": "absorber", "cpmlReflection": "cpml_reflection",
    "cpmlKappaMax": "cpml_kappa_max", "cpmlFrequency": "cpml_frequency", "attenuation": "attenuation",
    "mechanisms": "mechanisms", "qMinFrequency": "q_min_frequency", "qMaxFrequency": "q_max_frequency",
    "qReferenceFrequency": "q_reference_frequency", "qp": "qp", "qs": "qs",
}


def _set(struct, field, value):
    t = dict(struct._fields_)[field]
    setattr(struct, field, int(value) if t in (C.c_int32, C.c_int64) else float(value))


def params2d(params: dict):
    """swl_params2d from a parameter dictionary; returns (struct, arrays to keep alive)."""
    L = _bind()
    p = Params2D()
    L.swl2d_params_default(C.byref(p))
    keep = []
    for k, v in params.items():
        if k in _MAP2D:
            _set(p, _MAP2D[k], v)
    if "sourceDirection" in params:
        for a in range(3):
            p.source_direction[a] = float(params["sourceDirection"][a])
    if "layers" in params:
        rows = np.asarray(params["layers"], dtype=np.float64).reshape(-1, 6)
        arr = (Layer2D * len(rows))(*[Layer2D(*r) for r in rows])
        keep.append(arr)
        p.layers, p.n_layers = arr, len(rows)
    if "surface" in params:
        xz = np.ascontiguousarray(params["surface"], dtype=np.float64).ravel()
        keep.append(xz)
        p.surface_xz, p.n_surface = xz.ctypes.data_as(_dp), len(xz) // 2
    return p, keep


def params3d(params: dict):
    """swl_params3d from a parameter dictionary; returns (struct, arrays to keep alive)."""
    L = _bind()
    p = Params3D()
    L.swl3d_params_default(C.byref(p))
    keep = []
    for k, v in params.items():
        if k in _MAP3D:
            _set(p, _MAP3D[k], v)
    if "sourceDirection" in params:
        for a in range(3):
            p.source_direction[a] = float(params["sourceDirection"][a])
    if "layers" in params:
        # rows of (thickness, vp, vs, density), or of six with the layer's GSLS qp, qs
        flat = np.asarray(params["layers"], dtype=np.float64)
        cols = 6 if params.get("layerColumns", 4) == 6 else 4
        rows = flat.reshape(-1, cols)
        arr = (Layer3D * len(rows))(*[Layer3D(*r[:4]) for r in rows])
        keep.append(arr)
        p.layers, p.n_layers = arr, len(rows)
        if cols == 6:
            q = np.ascontiguousarray(rows[:, 4:6]).ravel()
            keep.append(q)
            p.layer_q = q.ctypes.data_as(_dp)
    if "layerNames" in params:
        names = (C.c_char_p * len(params["layerNames"]))(*[n.encode() for n in params["layerNames"]])
        keep.append(names)
        p.layer_names = C.cast(names, C.POINTER(C.c_char_p))
    if "receiverArray" in params:  # kind startX startY z countX countY strideX strideY
        r = [int(x) for x in params["receiverArray"]]
        (p.receiver_kind, p.receiver_start_x, p.receiver_start_y, p.receiver_z, p.receiver_count_x,
         p.receiver_count_y, p.receiver_stride_x, p.receiver_stride_y) = r
    if "absorbingCells" in params:
        for a in range(3):
            p.absorbing_cells[a] = int(params["absorbingCells"][a])
    if "demShape" in params:  # nx ny spacing originX originY datum
        d = params["demShape"]
        p.dem_nx, p.dem_ny = int(d[0]), int(d[1])
        p.dem_spacing, p.dem_origin_x, p.dem_origin_y, p.dem_datum = map(float, d[2:6])
        e = np.ascontiguousarray(params["demElevations"], dtype=np.float64)
        keep.append(e)
        p.dem_elevations = e.ctypes.data_as(_dp)
    return p, keep


class Simulation2D:
    """Seis2D::Curvilinear::Simulation on the B200 engine."""

    def __init__(self, params: dict, device: int = -1):
        L = _bind()
        p, keep = params2d(params)
        h = C.c_void_p()
        _check(L.swl2d_session_create(C.byref(p), int(device), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().swl2d_session_destroy(self._h)
            self._h = C.c_void_p()

    __del__ = close

    def advance(self, count: int) -> bool:
        """Simulation::advance: True when every requested step was accepted; raises on a fault."""
        _check(library().swl2d_session_advance(self._h, int(count)))
        return True

    def reset(self):
        _check(library().swl2d_session_reset(self._h))

    def info(self) -> dict:
        i = Info2D()
        _check(library().swl2d_session_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in Info2D._fields_}

    def records(self):
        i = self.info()
        vx, vz = np.zeros((i["receivers"], i["samples"])), np.zeros((i["receivers"], i["samples"]))
        _check(library().swl2d_session_records(self._h, vx.ctypes.data_as(_dp), vz.ctypes.data_as(_dp)))
        return vx, vz

    def receiver_positions(self):
        n = self.info()["receivers"]
        xz = np.zeros((n, 2))
        _check(library().swl2d_session_receiver_positions(self._h, xz.ctypes.data_as(_dp)))
        return xz

    def field(self, f: int) -> np.ndarray:
        i = self.info()
        out = np.zeros(i["cpml_count"] if f == -1 else i["count"])
        _check(library().swl2d_session_snapshot(self._h, f, out.ctypes.data_as(_dp)))
        return out

    def model(self, name: str) -> np.ndarray:
        n = C.c_int64()
        _check(library().swl2d_session_model(self._h, name.encode(), None, C.byref(n)))
        out = np.zeros(n.value)
        _check(library().swl2d_session_model(self._h, name.encode(), out.ctypes.data_as(_dp), C.byref(n)))
        return out

    def engine_handle(self) -> int:
        return library().swl2d_session_engine(self._h)

    def write_snapshot(self, path, components=(1, 1, 0, 0, 1, 1, 1), include_material=True):
        """writeSnapshot: the wavefield as a .vts file (Vx, Vz, |V|, pressure, Sxx, Szz, Sxz)."""
        comp = (C.c_int32 * 7)(*[int(bool(c)) for c in components])
        _check(library().swl2d_session_write_snapshot(self._h, str(path).encode(), comp, int(bool(include_material))))

    def write_model(self, path, backend=1, cpu_threads=0, cuda_device=-1):
        """writeModelVts: the session's model as the reference's versioned model file."""
        c = ModelCompute(int(backend), int(cpu_threads), int(cuda_device))
        _check(library().swl2d_session_write_model(self._h, str(path).encode(), C.byref(c)))

    def read_probes(self, nodes) -> np.ndarray:
        """Simulation::readProbes: Vx, Vz, Sxx, Szz, Sxz at logical nodes (i, k)."""
        ik = np.ascontiguousarray(np.asarray(nodes, dtype=np.int32).reshape(-1, 2))
        out = np.zeros((ik.shape[0], 5))
        _check(library().swl2d_session_read_probes(self._h, ik.ctypes.data_as(C.POINTER(C.c_int32)), ik.shape[0],
                                                   out.ctypes.data_as(_dp)))
        return out


def read_model(path):
    """readModelVts: (parameters with the reference's names, compute settings, planned dt) of a 2D
    model file; the parameters build a Simulation2D."""
    L = _bind()
    h = C.c_void_p()
    _check(L.swl2d_read_model(str(path).encode(), C.byref(h)))
    try:
        p, c, dt = Params2D(), ModelCompute(), C.c_double()
        _check(L.swl2d_model_document_params(h, C.byref(p), C.byref(c), C.byref(dt)))
        out = {k: getattr(p, f) for k, f in _MAP2D.items() if k not in ("deviceGeometry", "segmentRule")}
        out["sourceDirection"] = list(p.source_direction)
        out["layers"] = [[p.layers[i].thickness, p.layers[i].vp, p.layers[i].vs, p.layers[i].density, p.layers[i].qp,
                          p.layers[i].qs] for i in range(p.n_layers)]
        if p.n_surface:
            out["surface"] = [[p.surface_xz[2 * i], p.surface_xz[2 * i + 1]] for i in range(p.n_surface)]
        compute = {"backend": c.backend, "cpuThreads": c.cpu_threads, "cudaDevice": c.cuda_device}
        return out, compute, dt.value
    finally:
        L.swl2d_model_document_free(h)


class Simulation3D:
    """Seis3D::Curvilinear::ISimulationBackend3D on the B200 engine."""

    def __init__(self, params: dict, device: int = -1):
        L = _bind()
        p, keep = params3d(params)
        h = C.c_void_p()
        _check(L.swl3d_session_create(C.byref(p), int(device), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            library().swl3d_session_destroy(self._h)
            self._h = C.c_void_p()

    __del__ = close

    def advance(self, count: int) -> bool:
        _check(library().swl3d_session_advance(self._h, int(count)))
        return True

    def reset(self):
        _check(library().swl3d_session_reset(self._h))

    def info(self) -> dict:
        i = Info3D()
        _check(library().swl3d_session_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in Info3D._fields_}

    def records(self):
        i = self.info()
        shape = (i["receivers"], i["step"] + 1)
        t = [np.zeros(shape) for _ in range(3)]
        _check(library().swl3d_session_records(self._h, *(x.ctypes.data_as(_dp) for x in t)))
        return t

    def field(self, f: int) -> np.ndarray:
        """Field f (0..8), or f = -1: the CFS-PML memories (model('cpmlShape')[3] of them)."""
        if f == -1:
            n = int(self.model("cpmlShape")[3])
            out = np.zeros(max(n, 1))
            _check(library().swl3d_session_snapshot(self._h, f, out.ctypes.data_as(_dp)))
            return out[:n]
        out = np.zeros(self.info()["count"])
        _check(library().swl3d_session_snapshot(self._h, f, out.ctypes.data_as(_dp)))
        return out

    def model(self, name: str) -> np.ndarray:
        n = C.c_int64()
        _check(library().swl3d_session_model(self._h, name.encode(), None, C.byref(n)))
        out = np.zeros(n.value)
        _check(library().swl3d_session_model(self._h, name.encode(), out.ctypes.data_as(_dp), C.byref(n)))
        return out

    def engine_handle(self) -> int:
        return library().swl3d_session_engine(self._h)

    def write_snapshot(self, path, fields=(1,) * 11, include_material=True, include_velocity_vector=True):
        """writeVts: Vx, Vy, Vz, |V|, mean normal stress, Sxx, Syy, Szz, Sxy, Sxz, Syz as a .vts file."""
        sel = (C.c_int32 * 11)(*[int(bool(c)) for c in fields])
        _check(library().swl3d_session_write_snapshot(self._h, str(path).encode(), sel, int(bool(include_material)),
                                                      int(bool(include_velocity_vector))))

    def write_model(self, path, backend=1, cpu_threads=0, cuda_device=-1):
        """writeModelVts3D: the session's model as the reference's versioned 3D model file."""
        c = ModelCompute(int(backend), int(cpu_threads), int(cuda_device))
        _check(library().swl3d_session_write_model(self._h, str(path).encode(), C.byref(c)))


def read_model3d(path):
    """readModelVts3D: (parameters with the reference's names, compute settings, planned dt) of a 3D
    model file; the parameters build a Simulation3D."""
    L = _bind()
    h = C.c_void_p()
    _check(L.swl3d_read_model(str(path).encode(), C.byref(h)))
    try:
        p, c, dt = Params3D(), ModelCompute(), C.c_double()
        _check(L.swl3d_model_document_params(h, C.byref(p), C.byref(c), C.byref(dt)))
        out = {k: getattr(p, f) for k, f in _MAP3D.items()
               if k not in ("deviceGeometry", "precision", "receiverLimit", "absorber", "cpmlReflection", "cpmlKappaMax",
                            "cpmlFrequency", "attenuation", "mechanisms", "qMinFrequency", "qMaxFrequency",
                            "qReferenceFrequency", "qp", "qs")}
        out["sourceDirection"] = list(p.source_direction)
        out["layers"] = [[p.layers[i].thickness, p.layers[i].vp, p.layers[i].vs, p.layers[i].density]
                         for i in range(p.n_layers)]
        if p.n_layers:
            out["layerNames"] = [p.layer_names[i].decode() for i in range(p.n_layers)]
        out["receiverArray"] = [p.receiver_kind, p.receiver_start_x, p.receiver_start_y, p.receiver_z,
                                p.receiver_count_x, p.receiver_count_y, p.receiver_stride_x, p.receiver_stride_y]
        out["absorbingCells"] = list(p.absorbing_cells)
        if p.dem_nx:
            out["demShape"] = [p.dem_nx, p.dem_ny, p.dem_spacing, p.dem_origin_x, p.dem_origin_y, p.dem_datum]
            out["demElevations"] = np.ctypeslib.as_array(p.dem_elevations, shape=(p.dem_nx * p.dem_ny,)).copy()
        compute = {"backend": c.backend, "cpuThreads": c.cpu_threads, "cudaDevice": c.cuda_device}
        return out, compute, dt.value
    finally:
        L.swl3d_model_document_free(h)
