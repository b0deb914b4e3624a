"""The C-ABI library loads and exports every entry point declared in include/*.h; calls that
need a device fail loudly with a status (no CPU fallback) when there is none."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(swl[0-9a-z_]*)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_engine_surface():
    names = declared_functions()
    for want in ("swl2d_create", "swl2d_step", "swl2d_advance", "swl2d_rollback", "swl2d_reset", "swl2d_diagnostics",
                 "swl2d_sample", "swl2d_snapshot", "swl2d_probes", "swl2d_resident_bytes", "swl2d_destroy",
                 "swl3d_create", "swl3d_step", "swl3d_advance", "swl3d_snapshot", "swl_last_error"):
        assert want in names


def test_library_exports_every_declared_symbol(swl):
    lib = swl.library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_build_targets_sm100a_only():
    text = (ROOT / "seiswavelab--curvilinear_b200" / "build.py").read_text()
    assert "arch=compute_100a,code=sm_100a" in text
    assert re.findall(r"arch=compute_\d+a?", text) == ["arch=compute_100a"]


def test_create_without_device_fails_loudly(swl):
    if swl.device_count() > 0:
        pytest.skip("a GPU is present; covered by the gpu tests")
    mesh = {"nx": 20, "nz": 20, "h": 1.0}
    for k in ("metricA", "metricB", "jacobian", "lambda", "mu", "density", "source", "damping"):
        mesh[k] = np.ones(400)
    mesh["normals"] = np.ones(800)
    with pytest.raises(swl.SwlError) as e:
        swl.Engine2D(mesh)
    assert e.value.status in (swl.ERR_UNAVAILABLE, swl.ERR_CUDA)


def test_null_arguments_are_rejected(swl):
    lib = swl.library()
    assert lib.swl2d_create(None, None, 0, -1, None) == swl.ERR_INVALID
    assert b"null" in lib.swl_last_error()
    assert lib.swl2d_step(None, 0.0, 1e-3, 10.0, 1.0, 0) == swl.ERR_INVALID
    assert lib.swl3d_create(None, None, 0, -1, None) == swl.ERR_INVALID
    assert lib.swl2d_resident_bytes(None) == 0


def test_queue_needs_a_device_and_valid_arguments(swl):
    lib = swl.library()
    h = C.c_void_p()
    assert lib.swl2d_queue_create(-1, 7, C.byref(h)) == swl.ERR_INVALID  # precision
    assert b"precision" in lib.swl_last_error()
    assert lib.swl2d_queue_launch(None, None, 0, None, None, None, None, None, None) == swl.ERR_INVALID
    assert lib.swl2d_queue_segment(None, 8) == swl.ERR_INVALID
    if swl.device_count() == 0:  # no CPU fallback: a queue needs a device
        assert lib.swl2d_queue_create(-1, swl.SWL_FP32, C.byref(h)) == swl.ERR_UNAVAILABLE
