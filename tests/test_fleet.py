"""The multi-GPU front's placement on CPU (no device needed): the rule, the request-size
estimate it charges, and the plan it makes for the seeded serving mix.

Shots are independent, so a request stream shards over GPUs by placement alone: every request is
charged its estimated resident bytes against one device and runs there whole.  The rule sends a
request to the device with the most budget left (ties to the lower slot) and refuses one larger
than every device's whole budget.
"""
import importlib

import pytest


@pytest.fixture(scope="module")
def F(swl):
    return importlib.import_module("swl_b200.fleet")


@pytest.fixture(scope="module")
def W(swl):
    return importlib.import_module("swl_b200.workloads")


def test_rule_takes_the_device_with_most_budget_left(F):
    assert F.choose([100, 100], [0, 30], 50) == 0
    assert F.choose([100, 200], [0, 150], 50) == 0      # 100 left beats 50 left
    assert F.choose([100, 200], [0, 50], 50) == 1       # 150 left beats 100 left
    assert F.choose([100, 100], [40, 40], 10) == 0      # ties go to the lower slot
    assert F.choose([100, 100], [90, 95], 50) == 0      # none fits now: it queues where most frees
    assert F.choose([100, 300], [0, 290], 150) == 1     # only slot 1 can ever hold it
    assert F.choose([100, 100], [0, 0], 150) == -1      # larger than every budget: refused
    assert F.choose([], [], 1) == -1


def test_request_estimate_grows_with_the_shot(F, W):
    small = W.curvilinear_large(nx=300, nz=200, steps=10)
    big = W.curvilinear_large(nx=600, nz=400, steps=10)
    b_small, b_big = F.request_bytes(small), F.request_bytes(big)
    assert 0 < b_small < b_big
    # FP32 holds six state sets of 4-byte words against four of 8 bytes
    assert F.request_bytes(dict(small, precision=1)) < b_small
    gsls = dict(big, attenuation=1, mechanisms=3, qMinFrequency=5.0, qMaxFrequency=60.0, qReferenceFrequency=25.0)
    assert F.request_bytes(gsls) > 1.5 * b_big     # 18 fields instead of 5 (beside a fixed allowance)
    d3 = W.elastic_3d(nx=60, ny=48, nz=40, steps=6, receivers=8, relief=30.0, flatten_depth=300.0)
    assert F.request_bytes(d3, 3) > 0


@pytest.mark.parametrize("devices", [2, 8])
def test_serving_mix_plan_spreads_the_load(F, W, devices):
    reqs = W.serving_mix(n=64, scale=0.5, steps_scale=0.01)
    need = [F.request_bytes(r["params"], r["dim"]) for r in reqs]
    budget = 4 * max(need)
    slots = F.plan(reqs, [budget] * devices)
    assert all(0 <= s < devices for s in slots)
    charged = [sum(n for n, s in zip(need, slots) if s == d) for d in range(devices)]
    # worst fit in arrival order keeps the devices within one request of each other
    assert max(charged) - min(charged) <= max(need)
    assert all(sum(1 for s in slots if s == d) > 0 for d in range(devices))


def test_a_request_no_device_can_hold_is_refused(F, W):
    reqs = [{"dim": 2, "params": W.curvilinear_large(nx=300, nz=200, steps=10)}]
    need = F.request_bytes(reqs[0]["params"])
    assert F.plan(reqs, [need - 1, need - 1]) == [-1]
    assert F.plan(reqs, [need - 1, need]) == [1]
