"""Model build on the terrain inputs the benchmark workloads use, against the reference's own CPU
solver run live (oracle/_ref, built from its sources; no GPU needed).

* 2D imported surface: samples of a seeded terrain profile interpolated by PCHIP
  (src/two_d/SurfaceProfile.cpp:8-49, used by CurvilinearSolver2D.cpp:289-330), the input of the
  5001x2001 curvilinear shot and of every 2D request of the serving mix.
* 3D DEM: a Gaussian-random-field elevation lattice sampled bilinearly
  (include/Seis3D/SurfaceGrid3D.hpp:44-51), the input of the 400x288x200 shot.

Sessions are created with SWL_MODEL_ONLY.  Every array the engine consumes, the node coordinates
and the dt plan must equal the reference's bit for bit (the stated bar for metrics and Jacobian
is relative 1e-14; the build follows the reference expression by expression).
"""
import importlib

import numpy as np
import pytest

from conftest import has_reference_binaries

ARRAYS_2D = ["metricA", "metricB", "jacobian", "normals", "coordinates", "lambda", "mu", "density", "vp", "vs",
             "source", "damping", "sourceGradientX", "sourceGradientZ", "cpmlX", "cpmlZ",
             "deltaP0", "deltaP1", "deltaP2", "deltaS0", "deltaS1", "deltaS2"]
ARRAYS_3D = ["metrics", "jacobian", "normals", "coordinates", "source", "damping", "sourceGradient0",
             "sourceGradient1", "sourceGradient2", "materialLambda", "materialMu", "materialDensity"]


@pytest.fixture(scope="module")
def S(swl, oracle_mod):
    if not has_reference_binaries(oracle_mod):
        pytest.skip("reference binaries not built (make -C oracle ref)")
    return importlib.import_module("swl_b200.session")


@pytest.fixture(scope="module")
def W(swl):
    return importlib.import_module("swl_b200.workloads")


def stored(a, precision):
    """A model array as a session of `precision` stores it: an FP32 session keeps each FP64-built
    value rounded once to FP32, as the reference's FP32 arrays do (the dump promotes them back)."""
    a = np.asarray(a, dtype=np.float64)
    return a.astype(np.float32).astype(np.float64) if precision == 1 else a


def compare_2d(S, oracle_mod, params):
    r = oracle_mod.run_reference_2d(params, steps=0, threads=4)
    sim = S.Simulation2D(params, device=S.MODEL_ONLY)
    prec = int(params.get("precision", 0))
    info = sim.info()
    assert (info["nx"], info["nz"]) == (int(r["nx"]), int(r["nz"]))
    assert info["dt"] == float(r["dt"]) and info["total_steps"] == int(r["total"])
    assert info["max_metric"] == float(r["maxMetric"]) and info["min_jacobian"] == float(r["minJacobian"])
    checked = []
    for k in ARRAYS_2D:
        if k in r:
            np.testing.assert_array_equal(stored(sim.model(k), prec), r[k], err_msg=k)
            checked.append(k)
    assert {"metricA", "metricB", "jacobian", "normals", "coordinates"} <= set(checked)
    return checked


@pytest.mark.parametrize("nz,attenuation", [(200, 0), (160, 1)])
def test_imported_surface_model_matches_reference(S, W, oracle_mod, nz, attenuation):
    # the 5001x2001 shot's generator (6 sinusoids + 2 gullies, 60 m relief, samples every 1 m,
    # blend depth 300 m) on a 300-wide grid at h = 2
    p = W.curvilinear_large(nx=300, nz=nz, steps=10)
    if attenuation:
        p.update(attenuation=1, mechanisms=3, qMinFrequency=5.0, qMaxFrequency=60.0, qReferenceFrequency=25.0,
                 flattenDepth=250.0)
    checked = compare_2d(S, oracle_mod, p)
    if attenuation:
        assert {"deltaP2", "deltaS2"} <= set(checked)


def test_serving_mix_models_match_reference(S, W, oracle_mod):
    # 2D requests of the seeded serving mix (h in {1, 2, 4}, elastic and GSLS, force and moment
    # sources, imported terrain sampled every h) at reduced grid edges
    reqs = [r for r in W.serving_mix(n=24, scale=0.25, steps_scale=0.01) if r["dim"] == 2][:6]
    assert len({r["params"]["spacing"] for r in reqs}) >= 2
    for r in reqs:
        for precision in (1, 0):  # the mix is served in FP32; its FP64 baseline builds the same model
            compare_2d(S, oracle_mod, dict(r["params"], precision=precision))


def test_dem_terrain_model_matches_reference(S, W, oracle_mod):
    # the 400x288x200 shot's DEM generator (correlation 500 m on a 25 m lattice) on a reduced grid
    p = W.elastic_3d(nx=60, ny=48, nz=40, steps=6, receivers=8, relief=30.0, flatten_depth=300.0)
    r = oracle_mod.run_reference_3d(p, steps=0, threads=4)
    sim = S.Simulation3D(p, device=S.MODEL_ONLY)
    info = sim.info()
    assert (info["nx"], info["ny"], info["nz"]) == (int(r["nx"]), int(r["ny"]), int(r["nz"]))
    assert info["dt"] == float(r["dt"]) and info["total_steps"] == int(r["total"])
    assert info["min_jacobian"] == float(r["minJacobian"]) and info["max_metric_norm"] == float(r["maxMetricNorm"])
    for k in ARRAYS_3D:
        if k in r:
            np.testing.assert_array_equal(sim.model(k), r[k], err_msg=k)
    # the terrain is really curved: the surface row's vertical coordinates vary
    z = np.asarray(r["coordinates"]).reshape(-1, 3)[:, 2]
    assert np.ptp(z) > 0
