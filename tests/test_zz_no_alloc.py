"""swl2d_stats_noalloc: the 2D diagnostics for callers that cannot allocate device memory.

Such callers (a process whose device memory is owned entirely by its own allocator or a
pre-sized arena, or a latency-critical loop where an allocation could synchronise the device)
hand the library device arrays they already own and get the energy, peak |v|, peak surface
traction ratio and finiteness back in device memory, with no allocation by the library: its
per-block scratch is a fixed device array inside the library.  This test calls the entry point
through the C ABI on device buffers the test owns and checks it against swl2d_diagnostics (the
engine's own, allocating, reduction) on the same state, for two calls in a row.  The file is
named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import load_2d, receivers_2d

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative; the two reductions sum the energy in different orders
# The surface traction ratio after the free-surface projection is a round-off residual
# (~1e-17); it is compared absolutely, far below the 1e-9 FP64 traction bar of the reference's
# own validation (src/two_d/PrecisionValidation2D.cpp:38).
TRACTION_ABS = 1e-15


class StateView(C.Structure):
    _fields_ = [("nx", C.c_int32), ("nz", C.c_int32), ("h", C.c_double),
                ("vx", C.c_void_p), ("vz", C.c_void_p), ("sxx", C.c_void_p), ("szz", C.c_void_p), ("sxz", C.c_void_p),
                ("lam", C.c_void_p), ("mu", C.c_void_p), ("rho", C.c_void_p), ("jac", C.c_void_p),
                ("normals", C.c_void_p), ("pml", C.c_void_p), ("cpml_width_x", C.c_int32), ("cpml_width_z", C.c_int32)]


@pytest.mark.parametrize("name", ["cpml_external_moment_layers", "sponge_force"])
def test_noalloc_diagnostics_match_engine_diagnostics(name, swl):
    import torch

    case, res, mesh = load_2d(name)
    eng = swl.Engine2D(mesh, receivers_2d(res), precision=swl.SWL_FP64, device=0)
    acc, fault = eng.advance(0, int(res["steps"]), float(res["dt"]), mesh["frequency"], mesh["scale"])
    assert acc == int(res["steps"]) and not fault
    want = eng.diagnostics()
    fields = eng.fields()
    dev = torch.device("cuda:0")

    def on_device(a):
        return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

    buffers = {f: on_device(fields[i]) for i, f in enumerate(["vx", "vz", "sxx", "szz", "sxz"])}
    for key, src in (("lam", "lambda"), ("mu", "mu"), ("rho", "density"), ("jac", "jacobian"), ("normals", "normals")):
        buffers[key] = on_device(mesh[src])
    v = StateView()
    v.nx, v.nz, v.h = int(res["nx"]), int(res["nz"]), float(res["h"])
    for k, t in buffers.items():
        setattr(v, k, t.data_ptr())
    if int(res["cpmlCount"]):
        buffers["pml"] = on_device(eng.field(-1))
        v.pml = buffers["pml"].data_ptr()
        v.cpml_width_x, v.cpml_width_z = int(res["cpmlWidthX"]), int(res["cpmlWidthZ"])
    out = torch.empty(4, dtype=torch.float64, device=dev)
    lib = swl.library()
    lib.swl2d_stats_noalloc.argtypes = [C.POINTER(StateView), C.c_void_p, C.c_void_p]
    lib.swl2d_stats_noalloc.restype = C.c_int32
    for call in range(2):  # the shared scratch keeps the previous call's contents
        out.fill_(float("nan"))
        st = lib.swl2d_stats_noalloc(C.byref(v), C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == swl.OK, lib.swl_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[0] == pytest.approx(want["energy"], rel=TOL), call
        assert got[1] == pytest.approx(want["max_velocity"], rel=TOL), call
        assert got[2] == pytest.approx(want["traction_relative"], rel=TOL, abs=TRACTION_ABS), call
        assert got[2] < 1e-9, call
        assert got[3] == 1.0 and want["finite"] == 1


def test_noalloc_rejects_states_beyond_its_scratch(swl):
    lib = swl.library()
    lib.swl2d_stats_noalloc.argtypes = [C.POINTER(StateView), C.c_void_p, C.c_void_p]
    v = StateView()
    v.nx, v.nz, v.h = 40000, 20000, 1.0  # 1250 x 2500 blocks > 65,536
    for k in ("vx", "vz", "sxx", "szz", "sxz", "lam", "mu", "rho", "jac", "normals"):
        setattr(v, k, 16)  # never dereferenced: the size check fails before any launch
    assert lib.swl2d_stats_noalloc(C.byref(v), C.c_void_p(16), None) == swl.ERR_INVALID
    assert b"too large" in lib.swl_last_error()


def test_noalloc_rejects_cpml_widths_beyond_the_grid(swl):
    lib = swl.library()
    lib.swl2d_stats_noalloc.argtypes = [C.POINTER(StateView), C.c_void_p, C.c_void_p]
    v = StateView()
    v.nx, v.nz, v.h = 46, 36, 5.0
    for k in ("vx", "vz", "sxx", "szz", "sxz", "lam", "mu", "rho", "jac", "normals", "pml"):
        setattr(v, k, 16)  # never dereferenced: the width check fails before any launch
    for wx, wz in ((21, 6), (6, 31)):  # 2*wx > nx-6, wz > nz-6
        v.cpml_width_x, v.cpml_width_z = wx, wz
        assert lib.swl2d_stats_noalloc(C.byref(v), C.c_void_p(16), None) == swl.ERR_INVALID
        assert b"widths exceed" in lib.swl_last_error()
