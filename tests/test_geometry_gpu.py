"""FP64 node geometry built on the GPU (swl2d_build_geometry) against the reference's own arrays.

With deviceGeometry the session computes the node coordinates, metrics, Jacobian and normals of
the terrain-following map on the GPU in FP64 (the host still evaluates the surface profile).
They must match the reference build to <= 1e-14 relative (CUDA's pow/hypot may differ from
glibc's by an ulp, so this is not a bitwise check), and the FP64 run on that geometry must match
the reference's records to <= 1e-11 relative L2.
"""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import golden_2d, load_2d, records_2d

pytestmark = pytest.mark.gpu

GEOMETRY_TOL = 1e-14
TRACE_TOL = 1e-11


def max_rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def S(swl):
    import importlib
    return importlib.import_module("swl_b200.session")


@pytest.mark.parametrize("name", golden_2d())
def test_device_geometry_matches_reference(name, S):
    case, res, _ = load_2d(name)
    sim = S.Simulation2D(dict(case, deviceGeometry=1), device=0)
    for key in ("metricA", "metricB", "jacobian", "normals", "coordinates"):
        assert max_rel(sim.model(key), res[key]) <= GEOMETRY_TOL, key
    info = sim.info()
    assert info["max_metric"] == pytest.approx(float(res["maxMetric"]), rel=GEOMETRY_TOL)
    assert info["dt"] == pytest.approx(float(res["dt"]), rel=1e-14)
    sim.advance(info["total_steps"])
    vx, vz = sim.records()
    rvx, rvz = records_2d(res)
    assert rel_l2(vz, rvz) <= TRACE_TOL and rel_l2(vx, rvx) <= TRACE_TOL


def test_device_geometry_needs_a_device(S, swl):
    case, _, _ = load_2d("sponge_force")
    with pytest.raises(swl.SwlError):
        S.Simulation2D(dict(case, deviceGeometry=1), device=S.MODEL_ONLY)


@pytest.mark.parametrize("name", ["moment_layered", "force"])
def test_device_geometry_3d_matches_reference(name, S):
    from helpers import fields_3d, load_3d
    case, res, _ = load_3d(name)
    sim = S.Simulation3D(dict(case, deviceGeometry=1), device=0)
    for key in ("metrics", "jacobian", "normals"):
        assert max_rel(sim.model(key), res[key]) <= GEOMETRY_TOL, key
    sim.advance(sim.info()["total_steps"])
    for f in range(9):
        assert rel_l2(sim.field(f), fields_3d(res)[f]) <= TRACE_TOL, f
