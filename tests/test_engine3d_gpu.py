"""3D nine-field engine on the GPU against the reference (golden fixtures)."""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import fields_3d, golden_3d, load_3d, receivers_3d, records_3d

pytestmark = pytest.mark.gpu


def run(swl, mesh, res, precision, batch=None):
    steps = int(res["steps"])
    e = swl.Engine3D(mesh, receivers_3d(res), precision=precision)
    batch = batch or steps
    tr, done = [[], [], []], 0
    while done < steps:
        n = min(batch, steps - done)
        acc, fault = e.advance(done, n, float(res["dt"]), mesh["frequency"], 3.0 / mesh["frequency"])
        assert not fault and acc == n
        for c, t in enumerate(e.traces(done, n)):
            tr[c].append(t)
        done += n
    return e, [np.concatenate(t, axis=1) for t in tr]


@pytest.mark.parametrize("name", golden_3d())
def test_fp64_matches_reference(name, swl):
    case, res, mesh = load_3d(name)
    e, tr = run(swl, mesh, res, swl.SWL_FP64, batch=5)
    want, got = fields_3d(res), e.fields()
    for f in range(9):
        assert rel_l2(got[f], want[f]) <= 1e-11, (name, f)
    for t, w in zip(tr, records_3d(res)):
        assert rel_l2(t, w[:, 1:]) <= 1e-11
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("name", golden_3d())
def test_fp32_within_tolerance(name, swl):
    case, res, mesh = load_3d(name)
    e, tr = run(swl, mesh, res, swl.SWL_FP32)
    for t, w in zip(tr, records_3d(res)):
        assert rel_l2(t, w[:, 1:]) <= 1e-4


def test_eager_step_matches_advance(swl):
    case, res, mesh = load_3d("moment_layered")
    dt = float(res["dt"])
    a = swl.Engine3D(mesh, receivers_3d(res))
    for s in range(6):
        a.step(dt, mesh["frequency"], s)
    b = swl.Engine3D(mesh, receivers_3d(res))
    b.advance(0, 6, dt, mesh["frequency"], 3.0 / mesh["frequency"])
    np.testing.assert_array_equal(a.fields(), b.fields())


def test_fp32_rollback_restores_compensation(swl):
    # the FP32 Kahan compensation terms roll back with the state
    case, res, mesh = load_3d("moment_layered")
    dt, f, g = float(res["dt"]), mesh["frequency"], 3.0 / mesh["frequency"]
    a = swl.Engine3D(mesh, receivers_3d(res), precision=swl.SWL_FP32)
    a.advance(0, 5, dt, f, g)
    a.advance(5, 1, dt, f, g)
    a.rollback()
    a.advance(5, 4, dt, f, g)
    b = swl.Engine3D(mesh, receivers_3d(res), precision=swl.SWL_FP32)
    b.advance(0, 9, dt, f, g)
    np.testing.assert_array_equal(a.fields(), b.fields())


def test_diagnostics(swl):
    case, res, mesh = load_3d("force")
    e, _ = run(swl, mesh, res, swl.SWL_FP64)
    d = e.diagnostics()
    assert d["finite"] == 1
    assert d["energy"] == pytest.approx(float(res["energy"]), rel=1e-9)
    assert d["max_velocity"] == pytest.approx(float(res["maxAbsVelocity"]), rel=1e-12)


def test_step_diagnostics_match_full_diagnostics(swl):
    # the verdict's per-step numbers, read back with the batch, agree with a full pass over the state
    case, res, mesh = load_3d("force")
    e, _ = run(swl, mesh, res, swl.SWL_FP64)
    quick, full = e.step_diagnostics(), e.diagnostics()
    assert quick["finite"] == full["finite"] == 1
    assert quick["energy"] == pytest.approx(full["energy"], rel=1e-12)
    assert quick["max_velocity"] == pytest.approx(full["max_velocity"], rel=1e-14)
    assert quick["traction_rate_relative"] == pytest.approx(full["traction_rate_relative"], rel=1e-14)
    assert quick["peaks"] == pytest.approx(full["peaks"], rel=1e-14)
