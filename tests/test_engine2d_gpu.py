"""2D engine on the GPU against the reference (golden fixtures) and the oracle.

Plain FP64: wavefields, CFS-PML/GSLS memories and receiver records must match the reference to
relative L2 <= 1e-11 (the path is built to reproduce the reference arithmetic; the bitwise
check is reported separately).  FP32: trace relative L2 <= 1e-4 against the FP64 reference.
"""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import fields_2d, golden_2d, load_2d, receivers_2d, records_2d

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11
FP32_TRACE_TOL = 1e-4


def run_engine(swl, mesh, res, precision, steps=None, batch=None):
    steps = int(res["steps"]) if steps is None else steps
    eng = swl.Engine2D(mesh, receivers_2d(res), precision=precision)
    batch = batch or steps
    vx, vz = [], []
    done = 0
    while done < steps:
        n = min(batch, steps - done)
        acc, fault = eng.advance(done, n, float(res["dt"]), mesh["frequency"], mesh["scale"])
        assert not fault and acc == n
        tx, tz = eng.traces(done, n)
        vx.append(tx)
        vz.append(tz)
        done += n
    return eng, np.concatenate(vx, axis=1), np.concatenate(vz, axis=1)


@pytest.mark.parametrize("name", golden_2d())
def test_fp64_matches_reference(name, swl, oracle_mod):
    case, res, mesh = load_2d(name)
    eng, vx, vz = run_engine(swl, mesh, res, swl.SWL_FP64)
    want = fields_2d(res)
    got = eng.fields()
    for f in range(want.shape[0]):
        assert rel_l2(got[f], want[f]) <= FP64_TOL, (name, f, rel_l2(got[f], want[f]))
    if int(res["cpmlCount"]):
        assert rel_l2(eng.field(-1), res["pml"]) <= FP64_TOL
    rvx, rvz = records_2d(res)
    dt = float(res["dt"])
    assert rel_l2(oracle_mod.records_from_raw(vx, dt), rvx) <= FP64_TOL
    assert rel_l2(oracle_mod.records_from_raw(vz, dt), rvz) <= FP64_TOL


@pytest.mark.parametrize("name", golden_2d())
def test_fp64_bitwise(name, swl):
    case, res, mesh = load_2d(name)
    eng, vx, vz = run_engine(swl, mesh, res, swl.SWL_FP64, batch=11)  # graph batches + eager remainder
    np.testing.assert_array_equal(eng.fields(), fields_2d(res))


@pytest.mark.parametrize("name", golden_2d())
def test_fp32_within_tolerance(name, swl, oracle_mod):
    case, res, mesh = load_2d(name)
    eng, vx, vz = run_engine(swl, mesh, res, swl.SWL_FP32)
    rvx, rvz = records_2d(res)
    dt = float(res["dt"])
    assert rel_l2(oracle_mod.records_from_raw(vz, dt), rvz) <= FP32_TRACE_TOL
    assert rel_l2(oracle_mod.records_from_raw(vx, dt), rvx) <= FP32_TRACE_TOL
    assert rel_l2(eng.field(1), res["field1"]) <= 1e-3


def test_eager_steps_equal_batched_advance(swl):
    case, res, mesh = load_2d("cpml_external_moment_layers")
    dt = float(res["dt"])
    a = swl.Engine2D(mesh, receivers_2d(res))
    for s in range(10):
        a.step(dt, mesh["frequency"], mesh["scale"], s)
    b, _, _ = run_engine(swl, mesh, res, swl.SWL_FP64, steps=10)
    np.testing.assert_array_equal(a.fields(), b.fields())
    np.testing.assert_array_equal(a.field(-1), b.field(-1))
    vx, vz = a.sample()
    pv = a.probes(receivers_2d(res))
    np.testing.assert_array_equal(vx, pv[:, 0])
    np.testing.assert_array_equal(vz, pv[:, 1])


def test_rollback_restores_previous_step(swl):
    case, res, mesh = load_2d("sponge_force")
    dt = float(res["dt"])
    e = swl.Engine2D(mesh, receivers_2d(res))
    e.advance(0, 12, dt, mesh["frequency"], mesh["scale"])
    before = e.fields()
    e.advance(12, 1, dt, mesh["frequency"], mesh["scale"])
    assert not np.array_equal(e.fields(), before)
    e.rollback()
    np.testing.assert_array_equal(e.fields(), before)


@pytest.mark.parametrize("name", ["sponge_force", "cpml_external_moment_layers"])
def test_fp32_rollback_restores_compensation(name, swl):
    # FP32 keeps a Kahan compensation term per value beside the state; a rolled-back step must
    # restore it with the state, so the run continues bit for bit as if the step never happened.
    case, res, mesh = load_2d(name)
    dt, f, s = float(res["dt"]), mesh["frequency"], mesh["scale"]
    a = swl.Engine2D(mesh, receivers_2d(res), precision=swl.SWL_FP32)
    a.advance(0, 12, dt, f, s)
    a.advance(12, 1, dt, f, s)
    a.rollback()
    a.advance(12, 8, dt, f, s)
    b = swl.Engine2D(mesh, receivers_2d(res), precision=swl.SWL_FP32)
    b.advance(0, 20, dt, f, s)
    np.testing.assert_array_equal(a.fields(), b.fields())
    np.testing.assert_array_equal(a.field(-1), b.field(-1))


def test_reset_clears_state(swl):
    case, res, mesh = load_2d("gsls3_cpml_surface_force")
    e = swl.Engine2D(mesh, receivers_2d(res))
    e.advance(0, 9, float(res["dt"]), mesh["frequency"], mesh["scale"])
    assert np.abs(e.fields()).max() > 0
    e.reset()
    assert np.abs(e.fields()).max() == 0 and np.abs(e.field(-1)).max() == 0


def test_nonfinite_step_is_rejected_and_state_kept(swl):
    # Host-side fault injection (cf. src/three_d/BackendValidation.cpp:55-63): a density of
    # 1e-300 near the source overflows the velocity rates to infinity within a few steps.
    case, res, mesh = load_2d("sponge_force")
    mesh = dict(mesh)
    rho = np.array(mesh["density"])
    nx = int(res["nx"])
    q = (int(case["sourceX"]) + 3) + nx * (int(case["sourceZ"]) + 3)
    rho[q] = 1e-300
    mesh["density"] = rho
    dt = float(res["dt"])
    e = swl.Engine2D(mesh, receivers_2d(res))
    acc, fault = e.advance(0, 30, dt, mesh["frequency"], mesh["scale"])
    assert fault and acc < 30
    state = e.fields()
    assert np.all(np.isfinite(state))
    with pytest.raises(swl.SwlError):
        e.advance(acc, 1, dt, mesh["frequency"], mesh["scale"])
    e.reset()
    e.advance(0, 1, dt, mesh["frequency"], mesh["scale"])


def test_diagnostics_report_energy_and_finiteness(swl):
    case, res, mesh = load_2d("flat_surface_force")
    e = swl.Engine2D(mesh, receivers_2d(res))
    e.advance(0, int(res["steps"]), float(res["dt"]), mesh["frequency"], mesh["scale"])
    d = e.diagnostics()
    assert d["finite"] == 1
    assert d["energy"] == pytest.approx(float(res["energy"]), rel=1e-9)
    assert d["max_velocity"] == pytest.approx(float(res["maxVelocity"]), rel=1e-12)
    assert d["resident_bytes"] > 0 and d["rhs_registers"] > 0


@pytest.mark.parametrize("precision", ["SWL_FP32", "SWL_FP64"])
def test_identical_engines_give_identical_results(precision, swl):
    # The per-grid segment choice is kept per grid shape, so two engines of one shot use the same
    # decomposition and agree bit for bit (FP32 rounding would otherwise depend on it).
    case, res, mesh = load_2d("cpml_external_moment_layers")
    dt, f, s = float(res["dt"]), mesh["frequency"], mesh["scale"]
    out = []
    for _ in range(2):
        e = swl.Engine2D(mesh, receivers_2d(res), precision=getattr(swl, precision))
        e.advance(0, 24, dt, f, s)
        out.append((e.fields(), e.traces(0, 24)))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1][0], out[1][1][0])


@pytest.mark.parametrize("precision", ["SWL_FP32", "SWL_FP64"])
def test_step_diagnostics_match_full_diagnostics(precision, swl):
    # The verdict's per-step numbers (read back with the batch) agree with a full pass over the
    # state; only the order of the energy sum differs.
    case, res, mesh = load_2d("gsls3_cpml_surface_force")
    dt, f, s = float(res["dt"]), mesh["frequency"], mesh["scale"]
    e = swl.Engine2D(mesh, receivers_2d(res), precision=getattr(swl, precision))
    before = e.step_diagnostics()
    assert before["energy"] == e.diagnostics()["energy"]
    e.advance(0, 20, dt, f, s)
    quick, full = e.step_diagnostics(), e.diagnostics()
    assert quick["finite"] == full["finite"] == 1
    assert quick["energy"] == pytest.approx(full["energy"], rel=1e-12)
    assert quick["max_velocity"] == pytest.approx(full["max_velocity"], rel=1e-14)
    assert quick["traction_relative"] == pytest.approx(full["traction_relative"], rel=1e-14)
    assert quick["peak_energy"] == full["peak_energy"]
