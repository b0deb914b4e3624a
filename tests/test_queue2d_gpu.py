"""Persistent multi-shot launches (swl2d_queue_*) on the GPU.

Shots of uneven grid sizes and batch lengths advance together in one kernel launch driven by a
(shot, tile, stage) work queue.  The FP64 results must equal the reference's bit for bit (as the
per-shot path does); a shot's results must be the same alone and in a mix; a rejected step in
one shot must not disturb the others.
"""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import fields_2d, golden_2d, load_2d, receivers_2d, records_2d

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11
FP32_TRACE_TOL = 1e-4
BATCHES = (7, 11, 5, 13, 9, 6)  # steps per launch of each shot: uneven on purpose


class Shot:
    def __init__(self, swl, name, precision, batch, mesh_edit=None):
        self.case, self.res, mesh = load_2d(name)
        if mesh_edit:
            mesh = mesh_edit(self.case, self.res, dict(mesh))
        self.name, self.mesh, self.batch = name, mesh, batch
        self.steps, self.dt = int(self.res["steps"]), float(self.res["dt"])
        self.eng = swl.Engine2D(mesh, receivers_2d(self.res), precision=precision)
        self.done, self.vx, self.vz, self.fault = 0, [], [], False

    def next_count(self):
        return 0 if self.fault else min(self.batch, self.steps - self.done)

    def collect(self, n):
        acc, fault = self.eng.wait()
        if acc:
            tx, tz = self.eng.traces(self.done, acc)
            self.vx.append(tx)
            self.vz.append(tz)
        self.done += acc
        self.fault = self.fault or fault
        if not fault:
            assert acc == n

    def traces(self):
        return np.concatenate(self.vx, axis=1), np.concatenate(self.vz, axis=1)


def run_queued(swl, shots, precision):
    """Launch rounds until every shot finished: one queued launch per GSLS mechanism count."""
    queues = {}
    while True:
        pending = [s for s in shots if s.next_count() > 0]
        if not pending:
            break
        for mech in sorted({int(s.mesh.get("mechanisms", 0)) for s in pending}):
            group = [s for s in pending if int(s.mesh.get("mechanisms", 0)) == mech]
            q = queues.setdefault(mech, swl.Queue2D(precision))
            counts = [s.next_count() for s in group]
            q.launch([s.eng for s in group], [s.done for s in group], counts, [s.dt for s in group],
                     [s.mesh["frequency"] for s in group], [s.mesh["scale"] for s in group])
            q.wait()
            for s, n in zip(group, counts):
                s.collect(n)
    for q in queues.values():
        q.close()


def test_fp64_queue_matches_reference_bitwise(swl, oracle_mod):
    names = golden_2d()
    shots = [Shot(swl, n, swl.SWL_FP64, BATCHES[i % len(BATCHES)]) for i, n in enumerate(names)]
    run_queued(swl, shots, swl.SWL_FP64)
    for s in shots:
        assert s.done == s.steps and not s.fault
        np.testing.assert_array_equal(s.eng.fields(), fields_2d(s.res), err_msg=s.name)
        if int(s.res["cpmlCount"]):
            assert rel_l2(s.eng.field(-1), s.res["pml"]) <= FP64_TOL
        vx, vz = s.traces()
        rvx, rvz = records_2d(s.res)
        assert rel_l2(oracle_mod.records_from_raw(vx, s.dt), rvx) <= FP64_TOL, s.name
        assert rel_l2(oracle_mod.records_from_raw(vz, s.dt), rvz) <= FP64_TOL, s.name


def test_fp32_queue_within_tolerance(swl, oracle_mod):
    shots = [Shot(swl, n, swl.SWL_FP32, BATCHES[i % len(BATCHES)]) for i, n in enumerate(golden_2d())]
    run_queued(swl, shots, swl.SWL_FP32)
    for s in shots:
        vx, vz = s.traces()
        rvx, rvz = records_2d(s.res)
        assert rel_l2(oracle_mod.records_from_raw(vz, s.dt), rvz) <= FP32_TRACE_TOL, s.name
        assert rel_l2(oracle_mod.records_from_raw(vx, s.dt), rvx) <= FP32_TRACE_TOL, s.name


@pytest.mark.parametrize("precision", ["SWL_FP32", "SWL_FP64"])
def test_shot_is_the_same_alone_and_in_the_mix(precision, swl):
    prec = getattr(swl, precision)
    elastic = [n for n in golden_2d() if not n.startswith("gsls")]
    alone = Shot(swl, elastic[0], prec, 8)
    run_queued(swl, [alone], prec)
    mix = [Shot(swl, n, prec, BATCHES[i % len(BATCHES)]) for i, n in enumerate(elastic)]
    run_queued(swl, mix, prec)
    np.testing.assert_array_equal(alone.eng.fields(), mix[0].eng.fields())
    np.testing.assert_array_equal(alone.traces()[1], mix[0].traces()[1])
    # and against the engine's own batches (same tiles, same arithmetic)
    own = Shot(swl, elastic[0], prec, 8)
    while own.next_count():
        n = own.next_count()
        own.eng.launch(own.done, n, own.dt, own.mesh["frequency"], own.mesh["scale"])
        own.collect(n)
    got, want = mix[0].eng.fields(), own.eng.fields()
    assert max(rel_l2(got[f], want[f]) for f in range(got.shape[0])) <= (0 if prec == swl.SWL_FP64 else 1e-5)


def test_rejected_step_stops_only_its_shot(swl):
    def heavy(case, res, mesh):  # a density of 1e-300 at the source overflows within a few steps
        rho = np.array(mesh["density"])
        rho[(int(case["sourceX"]) + 3) + int(res["nx"]) * (int(case["sourceZ"]) + 3)] = 1e-300
        mesh["density"] = rho
        return mesh

    bad = Shot(swl, "sponge_force", swl.SWL_FP64, 30, heavy)
    good = Shot(swl, "flat_surface_force", swl.SWL_FP64, 9)
    run_queued(swl, [bad, good], swl.SWL_FP64)
    assert bad.fault and bad.done < bad.steps
    assert np.all(np.isfinite(bad.eng.fields()))
    np.testing.assert_array_equal(good.eng.fields(), fields_2d(good.res))


def test_queue_rejects_mixed_engines(swl):
    _, res, mesh = load_2d("sponge_force")
    a = swl.Engine2D(mesh, receivers_2d(res), precision=swl.SWL_FP32)
    b = swl.Engine2D(mesh, receivers_2d(res), precision=swl.SWL_FP64)
    q = swl.Queue2D(swl.SWL_FP32)
    dt = float(res["dt"])
    with pytest.raises(swl.SwlError, match="precision"):
        q.launch([a, b], 0, 4, dt, mesh["frequency"], mesh["scale"])
    with pytest.raises(swl.SwlError, match="twice"):
        q.launch([a, a], 0, 4, dt, mesh["frequency"], mesh["scale"])
    q.launch([a], 0, 4, dt, mesh["frequency"], mesh["scale"])
    q.wait()
    assert a.wait() == (4, False)
