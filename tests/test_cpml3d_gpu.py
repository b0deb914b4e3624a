"""3D CFS-PML on the GPU against the oracle's restatement (the reference has no 3D CFS-PML).

The session builds the model with CFS-PML slabs; the oracle runs the same model arrays
(swlo3d_run with memories).  FP64: wavefields, memories and records bit for bit (the stated bar,
relative L2 <= 1e-11, is asserted as well).  FP32: traces within 1e-4 of the FP64 oracle.
"""
import importlib

import numpy as np
import pytest

from conftest import rel_l2
from cpml3d import cpml_case, mesh_from_session, receiver_nodes

pytestmark = pytest.mark.gpu
STEPS = 80


@pytest.fixture(scope="module")
def S(swl):
    return importlib.import_module("swl_b200.session")


@pytest.fixture(scope="module")
def want(S, orc):
    p = cpml_case(maxSteps=STEPS, duration=1.0)
    model = S.Simulation3D(p, device=S.MODEL_ONLY)
    m = mesh_from_session(S, model, p)
    st, tr, pml = orc.run3d(m, STEPS, receivers=receiver_nodes(S, model), with_pml=True)
    return p, st, tr, pml


def test_fp64_cpml_matches_oracle_bitwise(S, want):
    p, st, tr, pml = want
    sim = S.Simulation3D(dict(p, precision=0), device=0)
    sim.advance(STEPS)
    for f in range(9):
        got = sim.field(f)
        assert rel_l2(got, st[f]) <= 1e-11, f
        np.testing.assert_array_equal(got, st[f], err_msg=f"field {f}")
    mem = sim.field(-1)
    assert mem.size == pml.size and np.any(pml)
    np.testing.assert_array_equal(mem, pml)
    for got, w in zip(sim.records(), tr):
        np.testing.assert_array_equal(got[:, 1:], w)   # the records start with the t = 0 sample


def test_fp32_cpml_traces_within_tolerance(S, want):
    p, st, tr, pml = want
    sim = S.Simulation3D(dict(p, precision=1), device=0)
    sim.advance(STEPS)
    vz = sim.records()[2][:, 1:]
    assert np.max(np.abs(tr[2])) > 0
    assert rel_l2(vz, tr[2]) <= 1e-4
    assert rel_l2(sim.field(-1), pml) <= 1e-3


def test_cpml_reset_and_rollback_carry_the_memories(S, want):
    p, st, tr, pml = want
    sim = S.Simulation3D(dict(p, precision=0), device=0)
    sim.advance(STEPS)
    first = sim.field(-1)
    sim.reset()
    assert not np.any(sim.field(-1))
    sim.advance(STEPS)
    np.testing.assert_array_equal(sim.field(-1), first)
