"""3D CFS-PML on the CPU: the model build and the oracle's own properties.

The reference's 3D path has only the quadratic sponge (include/Seis3D/AbsorbingBoundary3D.hpp:17-21);
this library carries its 2D ADE (src/two_d/PointKernels2D.hpp:50-64, profiles of
src/two_d/CfsPml2D.hpp:31-41) over to 3D, axis by axis.  With no reference to compare with, the
oracle's restatement is pinned by properties:
* with zero profiles (d = 0, kappa = 1, alpha = 0) the memories stay zero and the run equals the run
  without an absorber up to rounding (a slab node sums its momentum per axis, x/rho + y/rho + z/rho,
  where the plain form takes one quotient);
* with the profiles the session builds, waves that reach the boundary leave: the energy left after
  they have crossed it is far below that of the same shot without an absorber.
"""
import importlib

import numpy as np
import pytest

from cpml3d import cpml_case, mesh_from_session, receiver_nodes


@pytest.fixture(scope="module")
def S(swl):
    return importlib.import_module("swl_b200.session")


def profile(nodes, width, h, vp, reflection, kappa, frequency, both):
    # src/two_d/CfsPml2D.hpp:31-41, restated
    out = np.zeros((nodes, 3))
    d0 = -3 * vp * np.log(reflection) / (2 * width * h)
    for i in range(nodes):
        dist = min(i, nodes - 1 - i) if both else nodes - 1 - i
        t = min(max(1.0 - dist / width, 0.0), 1.0)
        out[i] = (d0 * t * t, 1 + (kappa - 1) * t * t, np.pi * frequency * (1 - t) if t > 0 else 0.0)
    return out.ravel()


def test_model_builds_slabs_instead_of_the_sponge(S):
    p = cpml_case()
    sim = S.Simulation3D(p, device=S.MODEL_ONLY)
    assert not np.any(sim.model("damping"))              # no sponge
    wx, wy, wz, count = sim.model("cpmlShape")
    assert (wx, wy, wz) == (6, 5, 6)
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    assert count == 6 * (2 * wx * ny * nz + 2 * wy * nx * nz + wz * nx * ny)
    vpmax = 3000.0                                        # uniform default model
    for key, n, w, both in (("cpmlX", nx, 6, True), ("cpmlY", ny, 5, True), ("cpmlZ", nz, 6, False)):
        np.testing.assert_allclose(sim.model(key), profile(n, w, 10.0, vpmax, 1e-4, 3.0, 12.0, both), rtol=1e-15, atol=0)
    sponge = S.Simulation3D(cpml_case(absorber=0), device=S.MODEL_ONLY)
    assert np.any(sponge.model("damping")) and sponge.model("cpmlShape")[3] == 0
    # the dt plan includes the ADE rate bound (0.5 over the largest d/kappa + alpha)
    none = S.Simulation3D(cpml_case(absorbing=0), device=S.MODEL_ONLY)
    rate = max(max(sim.model(k)[0::3] / sim.model(k)[1::3] + sim.model(k)[2::3]) for k in ("cpmlX", "cpmlY", "cpmlZ"))
    assert sim.info()["dt"] <= min(none.info()["dt"], 0.5 / rate) * (1 + 1e-12)


def test_zero_profiles_reduce_to_the_run_without_absorber(S, orc):
    p = cpml_case(maxSteps=30)
    sim = S.Simulation3D(p, device=S.MODEL_ONLY)
    m = mesh_from_session(S, sim, p)
    for k in ("cpmlX", "cpmlY", "cpmlZ"):
        z = np.zeros_like(m[k])
        z[1::3] = 1.0                                      # d = 0, kappa = 1, alpha = 0
        m[k] = z
    st, _, pml = orc.run3d(m, 30, with_pml=True)
    plain = {k: v for k, v in m.items() if not k.startswith("cpml")}
    ref, _ = orc.run3d(plain, 30)
    assert not np.any(pml)
    for f in range(9):
        den = np.linalg.norm(ref[f])
        assert den > 0 and np.linalg.norm(st[f] - ref[f]) / den < 1e-12, f


def test_slabs_absorb_the_outgoing_waves(S, orc):
    # 280 steps (0.37 s): the pulse (12 Hz, peak at 0.125 s) has crossed the 280 m box several
    # times.  Measured: sum of v^2 4e-9 with CFS-PML against 1.7e-5 with the reference's sponge of
    # the same widths (and 1.5e-5 without an absorber).
    steps = 280
    p = cpml_case(maxSteps=steps, duration=2.0)
    out = {}
    for name, params in (("cpml", p), ("sponge", dict(p, absorber=0))):
        sim = S.Simulation3D(params, device=S.MODEL_ONLY)
        st, _, pml = orc.run3d(mesh_from_session(S, sim, params), steps, with_pml=True)
        out[name] = float(np.sum(st[:3] ** 2))
        if name == "cpml":
            assert np.any(pml) and np.all(np.isfinite(pml))
    assert out["cpml"] < 1e-2 * out["sponge"], out


def test_receivers_of_the_case_sit_on_the_surface(S):
    sim = S.Simulation3D(cpml_case(), device=S.MODEL_ONLY)
    assert len(receiver_nodes(S, sim)) == sim.info()["receivers"] == 24
