"""Test infrastructure only: Python access to the oracle.

* ``Oracle`` wraps ``liboracle.so`` (the C restatement in ``swl_oracle.c``).
* ``run_reference_2d`` / ``run_reference_3d`` run the reference's own CPU solver
  (``_ref/ref2d``, ``_ref/ref3d``, built from the reference sources by the Makefile)
  on a case dictionary and load its dumps.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF2D = HERE / "_ref" / "ref2d"
REF3D = HERE / "_ref" / "ref3d"
REF2D_CUDA = HERE / "_ref" / "ref2d_cuda"  # the 2D driver with the reference's own CUDA engine
LIB = HERE / "liboracle.so"

_dp = C.POINTER(C.c_double)


class Mesh2D(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("nz", C.c_int32), ("count", C.c_int64), ("h", C.c_double),
        ("a", _dp), ("b", _dp), ("jac", _dp), ("normals", _dp), ("lam", _dp), ("mu", _dp),
        ("rho", _dp), ("source", _dp), ("damping", _dp),
        ("source_direction", C.c_double * 3), ("source_gradient", _dp * 2),
        ("mechanisms", C.c_int32), ("field_count", C.c_int32),
        ("cpml_x", _dp), ("cpml_z", _dp), ("cpml_width_x", C.c_int32), ("cpml_width_z", C.c_int32),
        ("cpml_count", C.c_int64), ("rates", C.c_double * 3), ("delta_p", _dp * 3), ("delta_s", _dp * 3),
    ]


class Mesh3D(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("count", C.c_int64),
        ("h", C.c_double), ("lam", C.c_double), ("mu", C.c_double), ("density", C.c_double),
        ("metrics", _dp), ("normals", _dp), ("jacobian", _dp), ("source", _dp), ("damping", _dp),
        ("material_lambda", _dp), ("material_mu", _dp), ("material_density", _dp),
        ("source_direction", C.c_double * 3), ("source_amplitude", C.c_double), ("source_gradient", _dp * 3),
        ("cpml_x", _dp), ("cpml_y", _dp), ("cpml_z", _dp), ("cpml_width_x", C.c_int32), ("cpml_width_y", C.c_int32),
        ("cpml_width_z", C.c_int32), ("cpml_count", C.c_int64),
        ("mechanisms", C.c_int32), ("field_count", C.c_int32), ("rates", C.c_double * 3), ("delta_p", _dp * 3),
        ("delta_s", _dp * 3),
    ]


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def reference_root() -> Path | None:
    """The reference checkout the Makefile compiles from (SWL_REFERENCE_ROOT or the recipe's
    default), or None when its sources are not on this machine."""
    out = subprocess.run(["make", "-s", "-C", str(HERE), "print-ref"], capture_output=True, text=True)
    root = Path(out.stdout.strip()) if out.returncode == 0 and out.stdout.strip() else None
    return root if root is not None and (root / "src").is_dir() else None


def build():
    """Compile liboracle.so (and the reference binaries when its sources are present)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    if reference_root() is not None:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)


class Oracle:
    def __init__(self):
        if not LIB.exists():
            build()
        self.lib = C.CDLL(str(LIB))
        L = self.lib
        L.swlo_direction.argtypes = [C.c_int, C.c_int, C.c_int]
        L.swlo2d_run.argtypes = [C.POINTER(Mesh2D), _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(C.c_int64), C.c_int, _dp, _dp]
        L.swlo2d_rhs.argtypes = [C.POINTER(Mesh2D), C.POINTER(_dp), _dp, C.POINTER(_dp), _dp, C.c_double, C.c_int,
                                 C.c_int]
        L.swlo2d_project.argtypes = [C.POINTER(Mesh2D), C.POINTER(_dp)]
        L.swlo3d_run.argtypes = [C.POINTER(Mesh3D), _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.POINTER(C.c_int64), C.c_int, _dp, _dp, _dp]
        L.swlo3d_rhs.argtypes = [C.POINTER(Mesh3D), C.POINTER(_dp), _dp, C.POINTER(_dp), _dp, C.c_double, C.c_int, C.c_int]

    # -- 2D ---------------------------------------------------------------------------------
    @staticmethod
    def mesh2d(m: dict):
        """Build the C mesh from a dict of float64 arrays (keys as in the reference dump)."""
        keep = []

        def arr(k):
            a = m.get(k)
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return _ptr(a)

        g = Mesh2D()
        g.nx, g.nz = int(m["nx"]), int(m["nz"])
        g.count = g.nx * g.nz
        g.h = float(m["h"])
        g.a, g.b, g.jac, g.normals = arr("metricA"), arr("metricB"), arr("jacobian"), arr("normals")
        g.lam, g.mu, g.rho, g.source, g.damping = arr("lambda"), arr("mu"), arr("density"), arr("source"), arr("damping")
        for a in range(3):
            g.source_direction[a] = float(m.get("sourceDirection", (0, 0, 1))[a])
        g.source_gradient[0] = arr("sourceGradientX")
        g.source_gradient[1] = arr("sourceGradientZ")
        g.mechanisms = int(m.get("mechanisms", 0))
        g.field_count = int(m.get("fieldCount", 5))
        g.cpml_x, g.cpml_z = arr("cpmlX"), arr("cpmlZ")
        g.cpml_width_x, g.cpml_width_z = int(m.get("cpmlWidthX", 0)), int(m.get("cpmlWidthZ", 0))
        g.cpml_count = int(m.get("cpmlCount", 0))
        for l in range(3):
            g.rates[l] = float(m.get("rates", (0, 0, 0))[l])
            g.delta_p[l] = arr(f"deltaP{l}")
            g.delta_s[l] = arr(f"deltaS{l}")
        return g, keep

    def run2d(self, m: dict, steps: int, first: int = 0, state=None, pml=None, receivers=()):
        g, keep = self.mesh2d(m)
        n, fc = g.count, g.field_count
        state = np.zeros(fc * n) if state is None else np.array(state, dtype=np.float64, copy=True)
        pml = np.zeros(max(g.cpml_count, 1)) if pml is None else np.array(pml, dtype=np.float64, copy=True)
        rec = np.ascontiguousarray(receivers, dtype=np.int64)
        vx = np.zeros((len(rec), steps))
        vz = np.zeros((len(rec), steps))
        rc = self.lib.swlo2d_run(C.byref(g), _ptr(state), _ptr(pml), first, steps, float(m["dt"]),
                                 float(m["frequency"]), float(m["scale"]), rec.ctypes.data_as(C.POINTER(C.c_int64)),
                                 len(rec), _ptr(vx), _ptr(vz))
        if rc:
            raise MemoryError("oracle 2D run failed")
        return state.reshape(fc, n), pml[: g.cpml_count], vx, vz

    def rhs2d(self, m: dict, state, pml, forcing, step, stage):
        g, keep = self.mesh2d(m)
        n, fc = g.count, g.field_count
        state = np.ascontiguousarray(state, dtype=np.float64).reshape(fc, n)
        out = np.zeros((fc, n))
        pml = np.ascontiguousarray(pml if pml is not None and len(pml) else np.zeros(1), dtype=np.float64)
        out_pml = np.zeros(max(g.cpml_count, 1))
        ins = (_dp * 18)(*[_ptr(state[f]) for f in range(fc)])
        outs = (_dp * 18)(*[_ptr(out[f]) for f in range(fc)])
        self.lib.swlo2d_rhs(C.byref(g), ins, _ptr(pml), outs, _ptr(out_pml), float(forcing), step, stage)
        return out, out_pml[: g.cpml_count]

    # -- 3D ---------------------------------------------------------------------------------
    @staticmethod
    def mesh3d(m: dict):
        keep = []

        def arr(k):
            a = m.get(k)
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return _ptr(a)

        g = Mesh3D()
        g.nx, g.ny, g.nz = int(m["nx"]), int(m["ny"]), int(m["nz"])
        g.count = g.nx * g.ny * g.nz
        g.h, g.lam, g.mu, g.density = float(m["h"]), float(m["lambda"]), float(m["mu"]), float(m["density"])
        g.metrics, g.normals, g.jacobian = arr("metrics"), arr("normals"), arr("jacobian")
        g.source, g.damping = arr("source"), arr("damping")
        g.material_lambda, g.material_mu, g.material_density = arr("materialLambda"), arr("materialMu"), arr("materialDensity")
        for a in range(3):
            g.source_direction[a] = float(m.get("sourceDirection", (0, 0, 1))[a])
            g.source_gradient[a] = arr(f"sourceGradient{a}")
        g.source_amplitude = float(m["sourceAmplitude"])
        # CFS-PML (keys as the 3D session's model names them; absent: no CFS-PML)
        g.cpml_x, g.cpml_y, g.cpml_z = arr("cpmlX"), arr("cpmlY"), arr("cpmlZ")
        g.cpml_width_x, g.cpml_width_y = int(m.get("cpmlWidthX", 0)), int(m.get("cpmlWidthY", 0))
        g.cpml_width_z, g.cpml_count = int(m.get("cpmlWidthZ", 0)), int(m.get("cpmlCount", 0))
        # GSLS (absent: elastic, nine fields)
        g.mechanisms = int(m.get("mechanisms", 0))
        g.field_count = 9 + 6 * g.mechanisms
        for l in range(3):
            g.rates[l] = float(np.atleast_1d(m.get("rates", (0, 0, 0)))[l]) if l < g.mechanisms else 0.0
            g.delta_p[l] = arr(f"deltaP{l}") if l < g.mechanisms else None
            g.delta_s[l] = arr(f"deltaS{l}") if l < g.mechanisms else None
        return g, keep

    def run3d(self, m: dict, steps: int, first: int = 0, state=None, receivers=(), pml=None, with_pml=False):
        g, keep = self.mesh3d(m)
        n, fc = g.count, g.field_count
        state = np.zeros(fc * n) if state is None else np.array(state, dtype=np.float64, copy=True)
        pml = np.zeros(max(g.cpml_count, 1)) if pml is None else np.array(pml, dtype=np.float64, copy=True)
        rec = np.ascontiguousarray(receivers, dtype=np.int64)
        tr = [np.zeros((len(rec), steps)) for _ in range(3)]
        rc = self.lib.swlo3d_run(C.byref(g), _ptr(state), _ptr(pml), first, steps, float(m["dt"]), float(m["frequency"]),
                                 rec.ctypes.data_as(C.POINTER(C.c_int64)), len(rec), *(_ptr(t) for t in tr))
        if rc:
            raise MemoryError("oracle 3D run failed")
        if with_pml:
            return state.reshape(fc, n), tr, pml[: g.cpml_count]
        return state.reshape(fc, n), tr

    def rhs3d(self, m: dict, state, source, step, stage, pml=None):
        g, keep = self.mesh3d(m)
        n, fc = g.count, g.field_count
        state = np.ascontiguousarray(state, dtype=np.float64).reshape(fc, n)
        out = np.zeros((fc, n))
        pml = np.ascontiguousarray(pml if pml is not None and len(pml) else np.zeros(max(g.cpml_count, 1)), dtype=np.float64)
        out_pml = np.zeros(max(g.cpml_count, 1))
        ins = (_dp * fc)(*[_ptr(state[f]) for f in range(fc)])
        outs = (_dp * fc)(*[_ptr(out[f]) for f in range(fc)])
        self.lib.swlo3d_rhs(C.byref(g), ins, _ptr(pml), outs, _ptr(out_pml), float(source), step, stage)
        return out


# -- receiver records ------------------------------------------------------------------------------
def lerp(a: float, b: float, t: float) -> float:
    """std::lerp as libstdc++ implements C++20 P0811R3 (exact at t=0 and t=1, monotonic)."""
    if (a <= 0 and b >= 0) or (a >= 0 and b <= 0):
        return t * b + (1 - t) * a
    if t == 1:
        return b
    x = a + t * (b - a)
    return (x if b < x else b) if (t > 1) == (b > a) else (x if b > x else b)


def records_from_raw(raw, dt: float, interval_ms: float = 0.0):
    """Resample raw per-step receiver values (receivers x steps, the value after each step)
    onto the record axis, restating Simulation::Impl::sample
    (src/two_d/CurvilinearSolver2D.cpp:120-147): t=0 sample 0, then linear interpolation
    between consecutive accepted steps at n*interval."""
    raw = np.asarray(raw, dtype=np.float64)
    nrec, steps = raw.shape
    interval = interval_ms * .001 if interval_ms > 0 else dt
    out = [[0.0] for _ in range(nrec)]
    prev = [0.0] * nrec
    for step in range(steps):
        end = (step + 1) * dt
        n = len(out[0])
        while n * interval <= end + 1e-9 * dt:
            a = min(max((n * interval - step * dt) / dt, 0.0), 1.0)
            for r in range(nrec):
                out[r].append(lerp(prev[r], float(raw[r, step]), a))
            n += 1
        for r in range(nrec):
            prev[r] = float(raw[r, step])
    return np.array(out)


def probe_nodes_2d(r: dict):
    """Padded node indices of the reference's receiver probes from a 2D dump."""
    nx = int(r["nx"])
    xs = np.atleast_1d(r["probeX"]).astype(np.int64)
    zs = np.atleast_1d(r["probeZ"]).astype(np.int64)
    return (xs + 3) + nx * (zs + 3)


# -- running the reference's own CPU solver --------------------------------------------------------
def write_case(case: dict, path: Path):
    """Write a case dict as the key/value text the reference drivers read."""
    with open(path, "w") as f:
        for k, v in case.items():
            if isinstance(v, (list, tuple, np.ndarray)):
                vals = np.asarray(v, dtype=np.float64).ravel()
                f.write(k + " " + " ".join(repr(float(x)) for x in vals) + "\n")
            else:
                f.write(f"{k} {float(v)!r}\n")


def _meta(path: Path) -> dict:
    out = {}
    for line in open(path):
        parts = line.split()
        if not parts:
            continue
        vals = []
        for p in parts[1:]:
            try:
                vals.append(float(p))
            except ValueError:
                vals.append(p)
        out[parts[0]] = vals[0] if len(vals) == 1 else vals
    return out


def _load_dir(d: Path) -> dict:
    res = _meta(d / "meta.txt")
    for f in d.glob("*.bin"):
        res[f.stem] = np.fromfile(f, dtype=np.float64)
    for f in d.glob("*.csv"):  # the reference's receiver CSV files, as text
        res["csv:" + f.stem] = f.read_text()
    for f in d.glob("*.sgy"):  # its SEG-Y exports of the session records, as bytes
        res["sgy:" + f.stem] = f.read_bytes()
    for f in d.glob("*.vts"):  # its wavefield snapshots and model files, as text
        res["vts:" + f.stem] = f.read_text()
    return res


def run_reference(dim: int, case: dict, steps: int = -1, threads: int = 1, dump_mesh: bool = True,
                  workdir: Path | None = None, timeout: float | None = None, warmup: int = 0,
                  backend: str = "cpu", files: bool = False) -> dict:
    """Run the reference solver built from its sources: its CPU loops, or (2D, backend="cuda")
    its own CUDA engine."""
    exe = REF2D_CUDA if backend == "cuda" else REF2D if dim == 2 else REF3D
    if not exe.exists():
        raise FileNotFoundError(f"{exe} is not built (make -C oracle ref ref-cuda)")
    tmp = None
    if workdir is None:
        tmp = tempfile.TemporaryDirectory()
        workdir = Path(tmp.name)
    workdir = Path(workdir)
    workdir.mkdir(parents=True, exist_ok=True)
    write_case(case, workdir / "case.txt")
    out = workdir / "out"
    proc = subprocess.run([str(exe), str(workdir / "case.txt"), str(out), str(steps), str(threads),
                           "1" if dump_mesh else "0", str(int(warmup)), backend] + (["files"] if files else []),
                          capture_output=True, text=True,
                          timeout=timeout)
    if proc.returncode != 0:
        raise RuntimeError(f"reference {dim}D run failed ({proc.returncode}): {proc.stderr.strip()}")
    res = _load_dir(out)
    if tmp is not None:
        tmp.cleanup()
    return res


def run_reference_2d(case: dict, steps: int = -1, threads: int = 1, **kw) -> dict:
    return run_reference(2, case, steps, threads, **kw)


def run_reference_3d(case: dict, steps: int = -1, threads: int = 1, **kw) -> dict:
    return run_reference(3, case, steps, threads, **kw)


def mesh_from_reference_2d(r: dict, case: dict) -> dict:
    """Oracle mesh dict from a reference 2D dump (model arrays as the reference built them)."""
    m = dict(r)
    m["sourceDirection"] = r["sourceDirection"]
    kind = int(case.get("sourceKind", 0))
    amp = case.get("momentPerLength", 2e6) if kind else case.get("forcePerLength", 2e5)
    h = float(r["h"])
    m["scale"] = amp / (h * h)
    m["frequency"] = case.get("frequency", 30.0)
    return m


def mesh_from_reference_3d(r: dict, case: dict) -> dict:
    m = dict(r)
    m["h"] = r["h"]
    kind = int(case.get("sourceKind", 0))
    m["sourceAmplitude"] = case.get("sourceMoment", 2e9) if kind else case.get("sourceForce", 2e8)
    d = np.asarray(case.get("sourceDirection", (0, 0, 1)), dtype=np.float64)
    m["sourceDirection"] = (0.0, 0.0, 0.0) if kind else tuple(d / np.linalg.norm(d))
    m["frequency"] = case.get("frequency", 12.0)
    return m
