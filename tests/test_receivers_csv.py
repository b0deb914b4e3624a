"""Receiver CSV files of the sessions against the reference's own writers.

tests/golden/receivers_csv.json (made by tests/golden/make_csv.py) holds the files that
writeReceivers (src/two_d/CurvilinearSolver2D.cpp:811-855) and writeReceiversCsv
(src/three_d/ReceiverIo.cpp) wrote for the cases of tests/cases.py.  After zero steps (a model-only
session, no GPU) the files must be identical but for the backend line, which names the device;
after the cases' steps (GPU) the header is identical and the samples equal the reference's records.
"""
import importlib
import json
from pathlib import Path

import numpy as np
import pytest

from cases import CASES_2D, CASES_3D
from conftest import rel_l2
from helpers import load_2d, load_3d, records_2d, records_3d

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "receivers_csv.json").read_text())
MODEL_ONLY = -2


@pytest.fixture(scope="module")
def S(swl):
    return importlib.import_module("swl_b200.session")


@pytest.fixture(scope="module")
def R(swl):
    return importlib.import_module("swl_b200.records")


def same_but_backend(got: str, want: str):
    g, w = got.splitlines(), want.splitlines()
    assert len(g) == len(w)
    for a, b in zip(g, w):
        if b.startswith("# backend="):
            assert a.startswith("# backend=")
        else:
            assert a == b


@pytest.mark.parametrize("name", list(CASES_2D))
def test_2d_csv_after_zero_steps_matches_reference(name, S, R, tmp_path):
    sim = S.Simulation2D(CASES_2D[name], device=MODEL_ONLY)
    R.session_write_receivers(sim, tmp_path / "r.csv")
    same_but_backend((tmp_path / "r.csv").read_text(), GOLDEN[f"2/{name}/receivers/0"])


@pytest.mark.parametrize("name", list(CASES_3D))
@pytest.mark.parametrize("which,selected", [("receivers", (1, 1, 1)), ("receivers_xz", (1, 0, 1))])
def test_3d_csv_after_zero_steps_matches_reference(name, which, selected, S, R, tmp_path):
    sim = S.Simulation3D(CASES_3D[name], device=MODEL_ONLY)
    R.session_write_receivers(sim, tmp_path / "r.csv", selected)
    assert (tmp_path / "r.csv").read_text() == GOLDEN[f"3/{name}/{which}/0"]


def test_3d_csv_needs_a_component(S, R, swl, tmp_path):
    sim = S.Simulation3D(CASES_3D["force"], device=MODEL_ONLY)
    with pytest.raises(swl.SwlError, match="Select at least one receiver component."):
        R.session_write_receivers(sim, tmp_path / "r.csv", (0, 0, 0))


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES_2D))
def test_2d_csv_after_steps_matches_reference(name, S, R, tmp_path):
    case, res, _ = load_2d(name)
    want = GOLDEN[f"2/{name}/receivers/n"]
    sim = S.Simulation2D(case, device=0)
    sim.advance(want["steps"])
    R.session_write_receivers(sim, tmp_path / "r.csv")
    lines = (tmp_path / "r.csv").read_text().splitlines()
    head = len(want["header"])
    same_but_backend("\n".join(lines[:head]), "\n".join(want["header"]))
    rows = [line.split(",") for line in lines[head:]]
    rvx, rvz = records_2d(res)
    n = rvx.shape[1]
    assert len(rows) == rvx.shape[0] * n
    vx = np.array([float(r[4]) for r in rows]).reshape(rvx.shape)
    vz = np.array([float(r[5]) for r in rows]).reshape(rvz.shape)
    assert [int(r[0]) for r in rows[::n]] == list(range(rvx.shape[0]))
    assert rel_l2(vx, rvx) <= 1e-11 and rel_l2(vz, rvz) <= 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES_3D))
def test_3d_csv_after_steps_matches_reference(name, S, R, tmp_path):
    case, res, _ = load_3d(name)
    want = GOLDEN[f"3/{name}/receivers/n"]
    sim = S.Simulation3D(case, device=0)
    sim.advance(want["steps"])
    R.session_write_receivers(sim, tmp_path / "r.csv", (1, 1, 1))
    lines = (tmp_path / "r.csv").read_text().splitlines()
    head = len(want["header"])
    assert lines[:head] == want["header"]
    values = np.array([[float(v) for v in line.split(",")] for line in lines[head:]])
    rx, ry, rz = records_3d(res)
    assert values.shape == (rx.shape[1], 1 + 3 * rx.shape[0])
    for c, rec in enumerate((rx, ry, rz)):
        np.testing.assert_array_equal(values[:, 1 + c::3].T, rec)


SEGY = np.load(Path(__file__).resolve().parent / "golden" / "session_segy.npz")
# (component, profile) of each file: Vz as IEEE32; Vx (2D, component 1) / Vy (3D, component 2) as IEEE64
SEGY_FILES = {2: [("vz_ieee32", 0, 0), ("vx_ieee64", 1, 1)], 3: [("vz_ieee32", 0, 0), ("vy_ieee64", 2, 1)]}


@pytest.mark.parametrize("dim,name", [(2, n) for n in CASES_2D] + [(3, n) for n in CASES_3D])
def test_session_segy_after_zero_steps_matches_reference(dim, name, S, R, tmp_path):
    sim = (S.Simulation2D if dim == 2 else S.Simulation3D)((CASES_2D if dim == 2 else CASES_3D)[name], device=MODEL_ONLY)
    for f, comp, profile in SEGY_FILES[dim]:
        R.session_write_segy(sim, comp, tmp_path / f"{f}.sgy", profile=profile)
        assert (tmp_path / f"{f}.sgy").read_bytes() == bytes(SEGY[f"{dim}/{name}/{f}/0"]), f


@pytest.mark.gpu
@pytest.mark.parametrize("dim,name", [(2, n) for n in CASES_2D] + [(3, n) for n in CASES_3D])
def test_session_segy_after_steps_matches_reference(dim, name, S, R, tmp_path):
    # the FP64 session records equal the reference's, so the exported files are identical
    sim = (S.Simulation2D if dim == 2 else S.Simulation3D)((CASES_2D if dim == 2 else CASES_3D)[name], device=0)
    sim.advance(GOLDEN[f"{dim}/{name}/receivers/n"]["steps"])
    for f, comp, profile in SEGY_FILES[dim]:
        R.session_write_segy(sim, comp, tmp_path / f"{f}.sgy", profile=profile)
        assert (tmp_path / f"{f}.sgy").read_bytes() == bytes(SEGY[f"{dim}/{name}/{f}/n"]), f


def check_snapshot(text: str, want: dict):
    got = text.encode()
    head = text[:text.index("<PointData")] if "<PointData" in text else text[:2000]
    assert head == want["head"]
    assert len(got) == want["size"]
    import hashlib
    assert hashlib.sha256(got).hexdigest() == want["sha256"]


ALL = (1, 1, 1, 1, 1, 1, 1)


@pytest.mark.parametrize("name", list(CASES_2D))
def test_2d_snapshot_after_zero_steps_matches_reference(name, S, tmp_path):
    sim = S.Simulation2D(CASES_2D[name], device=MODEL_ONLY)
    sim.write_snapshot(tmp_path / "s.vts")
    check_snapshot((tmp_path / "s.vts").read_text(), GOLDEN[f"2/{name}/snapshot/0"])
    sim.write_snapshot(tmp_path / "a.vts", ALL)
    check_snapshot((tmp_path / "a.vts").read_text(), GOLDEN[f"2/{name}/snapshot_all/0"])


def test_2d_snapshot_needs_a_component(S, swl, tmp_path):
    sim = S.Simulation2D(CASES_2D["sponge_force"], device=MODEL_ONLY)
    with pytest.raises(swl.SwlError, match="Select at least one wavefield export component."):
        sim.write_snapshot(tmp_path / "s.vts", (0,) * 7)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES_2D))
def test_2d_snapshot_and_probes_after_steps_match_reference(name, S, swl, tmp_path):
    case = CASES_2D[name]
    sim = S.Simulation2D(case, device=0)
    sim.advance(GOLDEN[f"2/{name}/receivers/n"]["steps"])
    sim.write_snapshot(tmp_path / "s.vts")
    check_snapshot((tmp_path / "s.vts").read_text(), GOLDEN[f"2/{name}/snapshot/n"])
    sim.write_snapshot(tmp_path / "a.vts", ALL)
    check_snapshot((tmp_path / "a.vts").read_text(), GOLDEN[f"2/{name}/snapshot_all/n"])
    nx, nz = int(case["nx"]), int(case["nz"])
    got = sim.read_probes([(0, 0), (nx // 2, nz // 3), (nx - 1, nz - 1), (nx // 3, 0)])
    want = np.array([float(v) for v in GOLDEN[f"2/{name}/probes/n"]]).reshape(4, 5)
    np.testing.assert_array_equal(got, want)
    with pytest.raises(swl.SwlError, match="Probe outside logical model."):
        sim.read_probes([(nx, 0)])


SOME3D = (0, 0, 1, 0, 1, 0, 0, 0, 1, 0, 0)


@pytest.mark.parametrize("name", list(CASES_3D))
def test_3d_snapshot_after_zero_steps_matches_reference(name, S, tmp_path):
    sim = S.Simulation3D(CASES_3D[name], device=MODEL_ONLY)
    sim.write_snapshot(tmp_path / "s.vts")
    check_snapshot((tmp_path / "s.vts").read_text(), GOLDEN[f"3/{name}/snapshot/0"])
    sim.write_snapshot(tmp_path / "t.vts", SOME3D, include_material=False, include_velocity_vector=False)
    check_snapshot((tmp_path / "t.vts").read_text(), GOLDEN[f"3/{name}/snapshot_some/0"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES_3D))
def test_3d_snapshot_after_steps_matches_reference(name, S, tmp_path):
    sim = S.Simulation3D(CASES_3D[name], device=0)
    sim.advance(GOLDEN[f"3/{name}/receivers/n"]["steps"])
    sim.write_snapshot(tmp_path / "s.vts")
    check_snapshot((tmp_path / "s.vts").read_text(), GOLDEN[f"3/{name}/snapshot/n"])
    sim.write_snapshot(tmp_path / "t.vts", SOME3D, include_material=False, include_velocity_vector=False)
    check_snapshot((tmp_path / "t.vts").read_text(), GOLDEN[f"3/{name}/snapshot_some/n"])


# ---------------------------------------------------------------- model files (writeModelVts)
REF_COMPUTE = dict(backend=0, cpu_threads=1, cuda_device=-1)  # the reference runs' settings


@pytest.mark.parametrize("name", list(CASES_2D))
def test_2d_model_file_matches_reference_and_reads_back(name, S, tmp_path):
    sim = S.Simulation2D(CASES_2D[name], device=MODEL_ONLY)
    sim.write_model(tmp_path / "m.vts", **REF_COMPUTE)
    check_snapshot((tmp_path / "m.vts").read_text(), GOLDEN[f"2/{name}/model"])
    params, compute, dt = S.read_model(tmp_path / "m.vts")
    assert compute == {"backend": 0, "cpuThreads": 1, "cudaDevice": -1}
    assert dt == sim.info()["dt"]
    again = S.Simulation2D(params, device=MODEL_ONLY)  # the file's parameters rebuild the same model
    again.write_model(tmp_path / "m2.vts", **REF_COMPUTE)
    assert (tmp_path / "m2.vts").read_bytes() == (tmp_path / "m.vts").read_bytes()


def test_2d_model_file_rejects_damage(S, swl, tmp_path):
    sim = S.Simulation2D(CASES_2D["gsls3_cpml_surface_force"], device=MODEL_ONLY)
    sim.write_model(tmp_path / "m.vts", **REF_COMPUTE)
    text = (tmp_path / "m.vts").read_text()
    i = text.index('Name="Vp"')
    j = text.index("\n", i) + 1  # first Vp value
    k = text.index(" ", j)
    (tmp_path / "bad.vts").write_text(text[:j] + repr(float(text[j:k]) + 1.0) + text[k:])
    with pytest.raises(swl.SwlError, match="Model checksum mismatch"):
        S.read_model(tmp_path / "bad.vts")
    (tmp_path / "cut.vts").write_text(text[: len(text) // 2])
    with pytest.raises(swl.SwlError):
        S.read_model(tmp_path / "cut.vts")


def named_layers(case: dict) -> dict:
    """The 3D reference driver names its layers "layer0", "layer1", ... (MaterialLayer3D::name)."""
    p = dict(case)
    if "layers" in p:
        p["layerNames"] = [f"layer{i}" for i in range(len(p["layers"]) // 4)]
    return p


@pytest.mark.parametrize("name", list(CASES_3D))
def test_3d_model_file_matches_reference_and_reads_back(name, S, tmp_path):
    sim = S.Simulation3D(named_layers(CASES_3D[name]), device=MODEL_ONLY)
    sim.write_model(tmp_path / "m.vts", **REF_COMPUTE)
    check_snapshot((tmp_path / "m.vts").read_text(), GOLDEN[f"3/{name}/model"])
    params, compute, dt = S.read_model3d(tmp_path / "m.vts")
    assert compute == {"backend": 0, "cpuThreads": 1, "cudaDevice": -1}
    assert dt == sim.info()["dt"]
    if "layers" in CASES_3D[name]:
        assert params["layerNames"] == [f"layer{i}" for i in range(3)]
    again = S.Simulation3D(params, device=MODEL_ONLY)  # the file's parameters rebuild the same model
    again.write_model(tmp_path / "m2.vts", **REF_COMPUTE)
    assert (tmp_path / "m2.vts").read_bytes() == (tmp_path / "m.vts").read_bytes()


def test_3d_model_file_with_dem_round_trips(S, tmp_path):
    """Schema 2: the embedded DEM (SurfaceGridGeometry / SurfaceGridElevations) survives a round trip."""
    nx, ny = 7, 6
    y, x = np.mgrid[0:ny, 0:nx]
    elev = 100.0 + 4.0 * np.sin(0.7 * x) * np.cos(0.5 * y)
    case = dict(CASES_3D["force"], demShape=[nx, ny, 60.0, -30.0, -30.0, 104.0], demElevations=elev.ravel())
    sim = S.Simulation3D(case, device=MODEL_ONLY)
    sim.write_model(tmp_path / "m.vts", **REF_COMPUTE)
    text = (tmp_path / "m.vts").read_text()
    assert 'Name="SeisWaveModel3DVersion" NumberOfComponents="1" NumberOfTuples="1" format="ascii">2 ' in text
    params, _, _ = S.read_model3d(tmp_path / "m.vts")
    assert params["demShape"] == [nx, ny, 60.0, -30.0, -30.0, 104.0]
    np.testing.assert_array_equal(params["demElevations"], elev.ravel())
    again = S.Simulation3D(params, device=MODEL_ONLY)
    again.write_model(tmp_path / "m2.vts", **REF_COMPUTE)
    assert (tmp_path / "m2.vts").read_bytes() == (tmp_path / "m.vts").read_bytes()


def test_3d_model_file_rejects_damage(S, swl, tmp_path):
    sim = S.Simulation3D(named_layers(CASES_3D["moment_layered"]), device=MODEL_ONLY)
    sim.write_model(tmp_path / "m.vts", **REF_COMPUTE)
    text = (tmp_path / "m.vts").read_text()
    i = text.index('Name="Jacobian"')
    j = text.index("\n", i) + 1  # first Jacobian value
    k = text.index(" ", j)
    (tmp_path / "bad.vts").write_text(text[:j] + repr(float(text[j:k]) * 1.5) + text[k:])
    with pytest.raises(swl.SwlError, match="Model checksum mismatch"):
        S.read_model3d(tmp_path / "bad.vts")
    (tmp_path / "cut.vts").write_text(text[: len(text) // 2])
    with pytest.raises(swl.SwlError):
        S.read_model3d(tmp_path / "cut.vts")
    (tmp_path / "two.vts").write_text(text.replace('type="StructuredGrid"', 'type="UnstructuredGrid"', 1))
    with pytest.raises(swl.SwlError, match="Expected a 3D StructuredGrid model VTS."):
        S.read_model3d(tmp_path / "two.vts")
    with pytest.raises(swl.SwlError, match="Cannot open 3D model VTS."):
        S.read_model3d(tmp_path / "missing.vts")
