"""3D GSLS viscoelasticity on the CPU: the model build and the oracle's own properties.

The reference's 3D path is elastic; this library carries its 2D GSLS (the fit of
src/common/Gsls.cpp and the relaxation of src/two_d/PointKernels2D.hpp:161-168) over to 3D with all six
stress components: per mechanism, six memory fields with rate_l (drive - memory), the stresses
subtract the memories, and the traction-free surface solve subtracts the memories' traction.
Without a reference to compare with, the restatement is pinned by properties:
* the fit is the reference-pinned 2D fit: the 3D strengths and unrelaxed moduli of a layer equal the
  2D session's for the same layer;
* with zero strengths the memories stay zero and the run equals the elastic run with the same moduli
  bit for bit;
* lower Q attenuates more: the energy left after the pulse decreases with Q.
"""
import importlib

import numpy as np
import pytest

from cases import case2d, case3d
from cpml3d import mesh_from_session


@pytest.fixture(scope="module")
def S(swl):
    return importlib.import_module("swl_b200.session")


def gsls_case(qp=60.0, qs=30.0, **kw):
    c = case3d(nx=24, ny=20, nz=22, relief=5, wavelength=100, duration=0.3, maxSteps=60, sourceX=12, sourceY=10, sourceZ=6,
               absorbingCells=[4, 4, 4], receiverArray=[1, 2, 10, 0, 20, 1, 1, 1], attenuation=1, mechanisms=3,
               qMinFrequency=2.0, qMaxFrequency=40.0, qReferenceFrequency=12.0, qp=qp, qs=qs)
    c.update(kw)
    return c


def test_fit_and_moduli_equal_the_2d_fit(S):
    p3 = gsls_case()
    sim3 = S.Simulation3D(p3, device=S.MODEL_ONLY)
    p2 = case2d(attenuation=1, mechanisms=3, qMinFrequency=2.0, qMaxFrequency=40.0, qReferenceFrequency=12.0, qp=60.0,
                qs=30.0, vp=3000.0, vs=1700.0, density=2200.0)
    sim2 = S.Simulation2D(p2, device=S.MODEL_ONLY)
    rates = sim3.model("gslsRates")
    assert rates.size == 3
    q3, q2 = 1000, 400  # interior nodes
    for l in range(3):
        assert sim3.model(f"deltaP{l}")[q3] == sim2.model(f"deltaP{l}")[q2]
        assert sim3.model(f"deltaS{l}")[q3] == sim2.model(f"deltaS{l}")[q2]
    assert sim3.model("materialMu")[q3] == sim2.model("mu")[q2]
    assert sim3.model("materialLambda")[q3] == sim2.model("lambda")[q2]
    # the dt plan holds the relaxation bound 0.25 / fastest rate
    assert sim3.info()["dt"] <= 0.25 / rates[-1]


def test_zero_strengths_reduce_to_the_elastic_run(S, orc):
    p = gsls_case(maxSteps=40)
    sim = S.Simulation3D(p, device=S.MODEL_ONLY)
    m = mesh_from_session(S, sim, p)
    for l in range(3):
        m[f"deltaP{l}"] = np.zeros_like(m[f"deltaP{l}"])
        m[f"deltaS{l}"] = np.zeros_like(m[f"deltaS{l}"])
    st, _ = orc.run3d(m, 40)
    elastic = {k: v for k, v in m.items() if not k.startswith("delta") and k not in ("mechanisms", "rates")}
    ref, _ = orc.run3d(elastic, 40)
    assert st.shape[0] == 27 and not np.any(st[9:])
    np.testing.assert_array_equal(st[:9], ref)
    assert np.any(ref[2])


def test_lower_q_attenuates_more(S, orc):
    steps = 200
    energy = {}
    for name, params in (("q20", gsls_case(20.0, 10.0, maxSteps=steps, duration=1.0)),
                         ("q200", gsls_case(200.0, 100.0, maxSteps=steps, duration=1.0)),
                         ("elastic", dict(gsls_case(maxSteps=steps, duration=1.0), attenuation=0))):
        sim = S.Simulation3D(params, device=S.MODEL_ONLY)
        st, _ = orc.run3d(mesh_from_session(S, sim, params), steps)
        energy[name] = float(np.sum(st[:3] ** 2))
    assert energy["q20"] < 0.8 * energy["q200"] and energy["q200"] < energy["elastic"] * 1.05, energy


def test_benchmark_workload_builds_with_three_mechanisms(S):
    # the 3D GSLS benchmark workload (bench.py --workload gsls_3d) at a reduced grid: three relaxation
    # rates, a strength per node and mechanism, and the relaxation bound in the dt plan
    W = importlib.import_module("swl_b200.workloads")
    p = W.elastic_3d(mechanisms=3, nx=40, ny=36, nz=30, relief=10.0, flatten_depth=100.0, receivers=8)
    sim = S.Simulation3D(p, device=S.MODEL_ONLY)
    rates = sim.model("gslsRates")
    assert rates.size == 3 and np.all(np.diff(rates) > 0)
    count = 46 * 42 * 36  # padded grid: three ghost nodes either side
    for l in range(3):
        assert sim.model(f"deltaP{l}").size == count and sim.model(f"deltaS{l}").size == count
        assert np.all(sim.model(f"deltaS{l}") >= 0)
    assert sim.info()["dt"] <= 0.25 / rates[-1]
    elastic = S.Simulation3D(W.elastic_3d(nx=40, ny=36, nz=30, relief=10.0, flatten_depth=100.0, receivers=8),
                             device=S.MODEL_ONLY)
    assert elastic.model("gslsRates").size == 0
