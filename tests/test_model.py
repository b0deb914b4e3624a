"""The C++20 host model build against the reference's own model arrays (no GPU needed).

Sessions are created with SWL_MODEL_ONLY; every array the engine consumes (metrics,
Jacobian, normals, materials, GSLS strengths, sponge, CFS-PML profiles, source kernel and
moment pattern) and the dt plan must equal the reference's bit for bit (the metric/Jacobian bar
is <= 1e-14; the construction follows the reference expression by expression).
"""
import importlib

import numpy as np
import pytest

from helpers import golden_2d, golden_3d, load_2d, load_3d

ARRAYS_2D = ["metricA", "metricB", "jacobian", "normals", "coordinates", "lambda", "mu", "density", "vp", "vs",
             "source", "damping", "sourceGradientX", "sourceGradientZ", "cpmlX", "cpmlZ",
             "deltaP0", "deltaP1", "deltaP2", "deltaS0", "deltaS1", "deltaS2"]
ARRAYS_3D = ["metrics", "jacobian", "normals", "source", "damping", "sourceGradient0", "sourceGradient1",
             "sourceGradient2", "materialLambda", "materialMu", "materialDensity"]


@pytest.fixture(scope="module")
def session_mod(swl):
    return importlib.import_module("swl_b200.session")


@pytest.mark.parametrize("name", golden_2d())
def test_model2d_matches_reference(name, session_mod):
    case, res, _ = load_2d(name)
    sim = session_mod.Simulation2D(case, device=session_mod.MODEL_ONLY)
    info = sim.info()
    assert info["nx"] == int(res["nx"]) and info["nz"] == int(res["nz"])
    assert info["dt"] == float(res["dt"]) and info["total_steps"] == int(res["total"])
    assert info["cpml_count"] == int(res["cpmlCount"]) and info["field_count"] == int(res["fieldCount"])
    for k in ("maxMetric", "minJacobian", "maxEdge", "flattenDepth"):
        snake = {"maxMetric": "max_metric", "minJacobian": "min_jacobian", "maxEdge": "max_edge",
                 "flattenDepth": "flatten_depth"}[k]
        assert info[snake] == float(res[k]), k
    checked = 0
    for k in ARRAYS_2D:
        if k in res:
            np.testing.assert_array_equal(sim.model(k), res[k], err_msg=k)
            checked += 1
    assert checked >= 12
    pos = sim.receiver_positions()
    assert pos.shape == (int(res["receivers"]), 2)


@pytest.mark.parametrize("name", golden_3d())
def test_model3d_matches_reference(name, session_mod):
    case, res, _ = load_3d(name)
    sim = session_mod.Simulation3D(case, device=session_mod.MODEL_ONLY)
    info = sim.info()
    assert (info["nx"], info["ny"], info["nz"]) == (int(res["nx"]), int(res["ny"]), int(res["nz"]))
    assert info["dt"] == float(res["dt"]) and info["total_steps"] == int(res["total"])
    for k, snake in (("minJacobian", "min_jacobian"), ("maxMetricNorm", "max_metric_norm"),
                     ("minCellLength", "min_cell_length"), ("maxCellEdge", "max_cell_edge")):
        assert info[snake] == float(res[k]), k
    for k in ARRAYS_3D:
        if k in res:
            np.testing.assert_array_equal(sim.model(k), res[k], err_msg=k)


def test_invalid_parameters_report_reference_messages(swl, session_mod):
    with pytest.raises(swl.SwlError, match="2D dimensions must be in 8..16384"):
        session_mod.Simulation2D({"nx": 4, "nz": 40}, device=session_mod.MODEL_ONLY)
    with pytest.raises(swl.SwlError, match="Isotropic moment needs 11"):
        session_mod.Simulation2D({"nx": 40, "nz": 40, "sourceKind": 1, "sourceZ": 2}, device=session_mod.MODEL_ONLY)
    with pytest.raises(swl.SwlError, match="Source must stay two nodes"):
        session_mod.Simulation3D({"nx": 16, "ny": 16, "nz": 16, "sourceZ": 0}, device=session_mod.MODEL_ONLY)


def test_model_only_session_refuses_to_step(swl, session_mod):
    sim = session_mod.Simulation2D({"nx": 40, "nz": 30, "spacing": 5, "relief": 0, "sourceZ": 5, "receiverCount": 8},
                                   device=session_mod.MODEL_ONLY)
    with pytest.raises(swl.SwlError):
        sim.advance(1)
