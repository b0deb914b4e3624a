"""Whole sessions on the GPU (host model build -> engine -> receiver records) against the
reference's own CPU solver: records and final wavefields of the plain FP64 path must match to
relative L2 <= 1e-11 (they are constructed to be identical); the FP32 form to <= 1e-4 on traces."""
import importlib

import numpy as np
import pytest

from conftest import rel_l2
from helpers import fields_2d, fields_3d, golden_2d, golden_3d, load_2d, load_3d, records_2d, records_3d

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S(swl):
    return importlib.import_module("swl_b200.session")


@pytest.mark.parametrize("name", golden_2d())
def test_session2d_fp64_records_match_reference(name, S):
    case, res, _ = load_2d(name)
    sim = S.Simulation2D(case, device=0)
    assert sim.advance(int(res["steps"]))
    vx, vz = sim.records()
    rvx, rvz = records_2d(res)
    assert rel_l2(vx, rvx) <= 1e-11 and rel_l2(vz, rvz) <= 1e-11
    np.testing.assert_array_equal(vz, rvz)
    want = fields_2d(res)
    for f in range(want.shape[0]):
        assert rel_l2(sim.field(f), want[f]) <= 1e-11
    info = sim.info()
    assert info["step"] == int(res["steps"]) and info["finite"] == 1
    assert info["energy"] == pytest.approx(float(res["energy"]), rel=1e-9)


@pytest.mark.parametrize("name", golden_2d())
def test_session2d_fp32_traces_within_tolerance(name, S):
    case, res, _ = load_2d(name)
    sim = S.Simulation2D(dict(case, precision=1), device=0)
    sim.advance(int(res["steps"]))
    vx, vz = sim.records()
    rvx, rvz = records_2d(res)
    assert rel_l2(vz, rvz) <= 1e-4 and rel_l2(vx, rvx) <= 1e-4


@pytest.mark.parametrize("name", golden_3d())
def test_session3d_fp64_records_match_reference(name, S):
    case, res, _ = load_3d(name)
    sim = S.Simulation3D(case, device=0)
    sim.advance(int(res["steps"]))
    for got, want in zip(sim.records(), records_3d(res)):
        np.testing.assert_array_equal(got, want)
    want = fields_3d(res)
    for f in range(9):
        np.testing.assert_array_equal(sim.field(f), want[f])


def test_session_reset_reproduces_bitwise(S):
    case, res, _ = load_2d("gsls3_cpml_surface_force")
    sim = S.Simulation2D(case, device=0)
    sim.advance(15)
    a = sim.records()
    sim.reset()
    assert sim.info()["step"] == 0
    sim.advance(15)
    b = sim.records()
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_session_advance_in_pieces_equals_one_call(S):
    case, res, _ = load_2d("cpml_internal_steep")
    one = S.Simulation2D(case, device=0)
    one.advance(int(res["steps"]))
    parts = S.Simulation2D(case, device=0)
    for n in (1, 7, 3, 13, 100):
        parts.advance(n)
    np.testing.assert_array_equal(one.records()[1], parts.records()[1])
    assert parts.info()["completed"] == 1


def test_record_interval_resampling_matches_reference(S, oracle_mod):
    # sampleIntervalMs > 0 resamples onto a uniform record axis (CurvilinearSolver2D.cpp:135-146)
    from conftest import has_reference_binaries
    if not has_reference_binaries(oracle_mod):
        pytest.skip("reference binaries not built")
    from cases import case2d
    case = case2d(absorber=1, spongeX=6, spongeZ=6, sampleIntervalMs=0.35, maxSteps=30)
    r = oracle_mod.run_reference_2d(case, steps=30)
    sim = S.Simulation2D(case, device=0)
    sim.advance(30)
    vx, vz = sim.records()
    R, Sm = int(r["receivers"]), int(r["samples"])
    np.testing.assert_array_equal(vz, r["tracesVz"].reshape(R, Sm))
    np.testing.assert_array_equal(vx, r["tracesVx"].reshape(R, Sm))
