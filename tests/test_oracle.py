"""The oracle (C restatement in oracle/swl_oracle.c) pinned against the reference.

Against the committed golden fixtures (outputs of the reference's own CPU solver, see
tests/golden/make_golden.py) the oracle must reproduce the final wavefields, CFS-PML and GSLS
memories bit for bit, and the receiver records after the reference's record resampling.
When the reference binaries are built (oracle/_ref), extra cases run live.
"""
import numpy as np
import pytest

from conftest import has_reference_binaries, load_oracle
from helpers import (fields_2d, fields_3d, golden_2d, golden_3d, load_2d, load_3d, receivers_2d, receivers_3d,
                     records_2d, records_3d)


@pytest.mark.parametrize("name", golden_2d())
def test_oracle_2d_matches_reference_bitwise(name, orc, oracle_mod):
    case, res, mesh = load_2d(name)
    steps = int(res["steps"])
    st, pml, vx, vz = orc.run2d(mesh, steps, receivers=receivers_2d(res))
    np.testing.assert_array_equal(st, fields_2d(res))
    if int(res["cpmlCount"]):
        np.testing.assert_array_equal(pml, res["pml"])
    rvx, rvz = records_2d(res)
    np.testing.assert_array_equal(oracle_mod.records_from_raw(vx, float(res["dt"])), rvx)
    np.testing.assert_array_equal(oracle_mod.records_from_raw(vz, float(res["dt"])), rvz)
    assert np.max(np.abs(st[1])) > 0  # the case actually propagated something


@pytest.mark.parametrize("name", golden_3d())
def test_oracle_3d_matches_reference_bitwise(name, orc):
    case, res, mesh = load_3d(name)
    steps = int(res["steps"])
    st, tr = orc.run3d(mesh, steps, receivers=receivers_3d(res))
    np.testing.assert_array_equal(st, fields_3d(res))
    for got, want in zip(tr, records_3d(res)):
        np.testing.assert_array_equal(got, want[:, 1:])
        assert np.all(want[:, 0] == 0)
    assert np.max(np.abs(st[2])) > 0


def test_direction_table_matches_reference_schedule(orc):
    # include/SeisCommon/FiniteDifference.hpp:9-13, spot values
    got = [[orc.lib.swlo_direction(s, g, a) for a in range(3)] for s in range(8) for g in range(4)]
    assert got[0] == [0, 0, 0] and got[1] == [1, 1, 1]
    assert got[4 * 2] == [1, 1, 1] and got[4 * 2 + 1] == [0, 0, 0]
    assert got[4 * 7 + 3] == [1, 0, 0]


def test_records_resampling_identity_at_native_interval(oracle_mod):
    raw = np.array([[1.0, -2.0, 3.5, 0.25]])
    rec = oracle_mod.records_from_raw(raw, 1e-3)
    assert rec.shape == (1, 5) and rec[0, 0] == 0
    np.testing.assert_allclose(rec[0, 1:], raw[0], rtol=1e-15)


@pytest.mark.skipif(not has_reference_binaries(load_oracle()), reason="reference binaries not built")
def test_oracle_live_against_reference_extra_case(orc, oracle_mod):
    from cases import case2d
    case = case2d(nx=36, nz=28, relief=4, wavelength=90, absorber=1, spongeX=5, spongeZ=5, attenuation=1, mechanisms=2,
                  qMinFrequency=4, qMaxFrequency=40, qReferenceFrequency=10, qp=50, qs=25, sourceKind=1,
                  externalAbsorption=1, maxSteps=25, sourceX=18, sourceZ=9)
    r = oracle_mod.run_reference_2d(case, steps=25)
    m = oracle_mod.mesh_from_reference_2d(r, case)
    st, pml, vx, vz = orc.run2d(m, 25, receivers=oracle_mod.probe_nodes_2d(r))
    for f in range(int(r["fieldCount"])):
        np.testing.assert_array_equal(st[f], r[f"field{f}"])
    np.testing.assert_array_equal(pml, r["pml"])
