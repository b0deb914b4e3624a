"""3D GSLS on the GPU against the oracle's restatement (the reference's 3D path is elastic).

FP64: the nine fields, the 18 memory fields, and the records bit for bit, with the sponge and with
CFS-PML slabs; FP32: traces within 1e-4 of the FP64 oracle.
"""
import importlib

import numpy as np
import pytest

from conftest import rel_l2
from cpml3d import mesh_from_session
from test_gsls3d import gsls_case

pytestmark = pytest.mark.gpu
STEPS = 60


@pytest.fixture(scope="module")
def S(swl):
    return importlib.import_module("swl_b200.session")


def receivers(sim):
    info = sim.info()
    nx, ny = info["nx"], info["ny"]
    return np.array([(2 + r + 3) + nx * ((10 + 3) + ny * 3) for r in range(info["receivers"])], dtype=np.int64)


def oracle_run(S, orc, p):
    model = S.Simulation3D(p, device=S.MODEL_ONLY)
    return orc.run3d(mesh_from_session(S, model, p), STEPS, receivers=receivers(model), with_pml=True)


@pytest.mark.parametrize("absorber", [0, 1], ids=["sponge", "cpml"])
def test_fp64_gsls3d_matches_oracle_bitwise(S, orc, absorber):
    p = gsls_case(maxSteps=STEPS, absorber=absorber)
    st, tr, pml = oracle_run(S, orc, p)
    sim = S.Simulation3D(dict(p, precision=0), device=0)
    sim.advance(STEPS)
    assert st.shape[0] == 27 and np.any(st[9:])
    for f in range(27):
        got = sim.field(f)
        assert rel_l2(got, st[f]) <= 1e-11 or not np.any(st[f]), f
        np.testing.assert_array_equal(got, st[f], err_msg=f"field {f}")
    if absorber:
        np.testing.assert_array_equal(sim.field(-1), pml)
    for got, w in zip(sim.records(), tr):
        np.testing.assert_array_equal(got[:, 1:], w)


def test_fp32_gsls3d_traces_within_tolerance(S, orc):
    p = gsls_case(maxSteps=STEPS)
    st, tr, pml = oracle_run(S, orc, p)
    sim = S.Simulation3D(dict(p, precision=1), device=0)
    sim.advance(STEPS)
    assert np.max(np.abs(tr[2])) > 0
    assert rel_l2(sim.records()[2][:, 1:], tr[2]) <= 1e-4
