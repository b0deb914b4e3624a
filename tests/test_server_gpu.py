"""Serving on the GPU: many shots run concurrently through the request loop.

Each shot's records must be the same when it runs alone (session API) and when it runs in a mix
with other shots of different sizes, physics and precisions (here they are identical bit for
bit: every shot owns its state and the kernels are deterministic).  Admission respects the
device-memory budget; an invalid request fails alone without disturbing the others.
"""
import importlib
import time

import numpy as np
import pytest

from cases import CASES_2D, CASES_3D

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(swl):
    return importlib.import_module("swl_b200.session"), importlib.import_module("swl_b200.server")


def mix():
    long2 = dict(duration=1.0, maxSteps=300)
    long3 = dict(duration=1.0, maxSteps=60)
    shots = [
        (2, dict(CASES_2D["cpml_external_moment_layers"], precision=1, **long2)),
        (2, dict(CASES_2D["gsls3_cpml_surface_force"], precision=1, **long2)),
        (2, dict(CASES_2D["sponge_force"], precision=0, **long2)),
        (2, dict(CASES_2D["cpml_internal_steep"], precision=1, **long2)),
        (3, dict(CASES_3D["moment_layered"], precision=1, **long3)),
        (3, dict(CASES_3D["force"], precision=0, **long3)),
        (2, dict(CASES_2D["gsls1_layers_sponge"], precision=1, **long2)),
    ]
    return shots


def alone(S, dim, params):
    # the same shot in the same form, alone: the server picks 2D stage segments by rule (no timing
    # runs while other shots run), and so does this session
    sim = (S.Simulation2D(dict(params, segmentRule=1), device=0) if dim == 2 else S.Simulation3D(params, device=0))
    sim.advance(sim.info()["total_steps"])
    return sim.records()


def alone_persistent(V, dim, params):
    # the persistent form alone: the shot is the only one in its multi-shot launches
    srv = V.Server(device=0, batch_steps=7, persistent=True)
    sid = srv.submit(params, dim)
    srv.drain()
    out = srv.records(sid)
    srv.close()
    return out


@pytest.mark.parametrize("persistent", [False, True])
def test_each_result_is_the_same_alone_and_in_the_mix(persistent, mods):
    S, V = mods
    shots = mix()
    srv = V.Server(device=0, batch_steps=7, persistent=persistent)
    ids = [srv.submit(p, dim) for dim, p in shots]
    srv.drain()
    st = srv.stats()
    assert st["done"] == len(shots) and st["failed"] == 0
    assert st["peak_running"] >= 2  # shots really overlapped
    for (dim, p), sid in zip(shots, ids):
        got = srv.records(sid)
        want = alone_persistent(V, dim, p) if persistent and dim == 2 else alone(S, dim, p)
        assert len(got) == len(want)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)
        s = srv.status(sid)
        assert s["state"] == "done" and s["steps_done"] == s["total_steps"] > 0
        assert s["finish_s"] >= s["start_s"] >= s["submit_s"]


def test_admission_respects_memory_budget(mods):
    S, V = mods
    # large enough that the device bytes, not the fixed per-shot allowance, dominate
    p = dict(CASES_2D["cpml_external_moment_layers"], precision=1, nx=1000, nz=400, maxSteps=60, duration=1.0)
    one = S.Simulation2D(p, device=0).info()["resident_bytes"]
    charge = one + (16 << 20)  # a built shot is charged its resident bytes plus a margin
    budget = int(2.5 * (one + (80 << 20)))
    srv = V.Server(device=0, memory_budget=budget, batch_steps=5)
    ids = [srv.submit(p, 2) for _ in range(6)]
    srv.drain()
    st = srv.stats()
    assert st["done"] == 6 and st["peak_resident_bytes"] <= budget
    assert st["peak_running"] <= budget // charge < 6  # the budget, not the queue, limited concurrency
    ref = srv.records(ids[0])
    for sid in ids[1:]:
        np.testing.assert_array_equal(srv.records(sid)[1], ref[1])


def test_invalid_request_fails_alone(mods):
    S, V = mods
    srv = V.Server(device=0)
    bad = srv.submit({"nx": 4, "nz": 40}, 2)
    good = srv.submit(dict(CASES_2D["sponge_force"], precision=1), 2)
    too_big = V.Server(device=0, memory_budget=1 << 20)
    huge = too_big.submit(dict(CASES_2D["sponge_force"], precision=1), 2)
    srv.drain()
    too_big.drain()
    assert srv.status(bad)["state"] == "failed" and "2D dimensions" in srv.status(bad)["error"]
    assert srv.status(good)["state"] == "done"
    assert too_big.status(huge)["state"] == "failed" and "budget" in too_big.status(huge)["error"]


def test_next_finished_streams_completions(mods):
    S, V = mods
    srv = V.Server(device=0, batch_steps=4)
    ids = {srv.submit(dict(CASES_2D["flat_surface_force"], precision=1), 2) for _ in range(3)}
    seen = set()
    t0 = time.time()
    while len(seen) < 3 and time.time() - t0 < 60:
        sid = srv.next_finished(2000)
        if sid is not None:
            seen.add(sid)
    assert seen == ids


def test_engine_async_batches_match_blocking_advance(swl):
    from helpers import load_2d, receivers_2d
    case, res, mesh = load_2d("gsls3_cpml_surface_force")
    dt = float(res["dt"])
    a = swl.Engine2D(mesh, receivers_2d(res))
    a.advance(0, 20, dt, mesh["frequency"], mesh["scale"])
    b = swl.Engine2D(mesh, receivers_2d(res))
    b.launch(0, 20, dt, mesh["frequency"], mesh["scale"])
    while not b.query()[0]:
        time.sleep(0.001)
    np.testing.assert_array_equal(a.fields(), b.fields())


def test_fleet_places_by_budget_and_each_result_is_the_same_alone(mods):
    # Two device slots on the one GPU of the test box: each slot is its own request loop, the front
    # places every shot by budget, and every shot's records equal those of the shot run alone.  The
    # slots' shots never wait on one another (shots are independent), so sharing one GPU is safe.
    S, V = mods
    F = importlib.import_module("swl_b200.fleet")
    shots = mix()
    fleet = F.Fleet(devices=[0, 0], batch_steps=7)
    assert fleet.size() == 2 and fleet.device(0) == fleet.device(1) == 0
    placed = [fleet.submit(p, dim) for dim, p in shots]
    assert {slot for _, slot in placed} == {0, 1}  # the front spread the mix over both slots
    fleet.drain()
    for (dim, p), (sid, slot) in zip(shots, placed):
        st = fleet.status(sid)
        assert st["state"] == "done" and st["slot"] == slot
        for g, w in zip(fleet.records(sid), alone(S, dim, p)):
            np.testing.assert_array_equal(g, w)
    for slot in (0, 1):
        s = fleet.stats(slot)
        assert s["failed"] == 0 and s["charged"] == 0  # finished shots no longer count
    fleet.close()
