"""SEG-Y record export and import against the reference's own writer and reader (CPU only).

The fixtures (tests/golden/segy.npz, made by tests/golden/make_segy.py) hold the files that the
reference's src/common/SegyIo.cpp wrote for seeded record sets, profiles, multipliers and
resampling intervals, its refusals, and what its reader returned for those files and for
hand-built files of the other formats it imports.  The export must match byte for byte; the
import must return the same dt, component, units, description, geometry and samples.
"""
import importlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "segy.npz"


@pytest.fixture(scope="module")
def fixtures():
    z = np.load(GOLDEN)
    return z, json.loads(bytes(z["index"]).decode())


@pytest.fixture(scope="module")
def R(swl):
    return importlib.import_module("swl_b200.records")


def record_set(z, case):
    key = f"set/{case['set']}"
    channels = [z[f"{key}/channel{c}"] for c in range(len(case["components"]))]
    return dict(channels=channels, components=case["components"], dt=case["dt"], units=case["units"],
                positions=z[f"{key}/positions"], sources=z[f"{key}/sources"], start_times=z[f"{key}/starts"])


def parse_dump(text):
    lines = text.splitlines()
    if lines[0] != "ok":
        return {"error": lines[0][len("error "):]}
    out = {"dt": float(lines[1]), "component": lines[2], "units": lines[3], "description": lines[4], "traces": []}
    n = int(lines[5])
    for r in range(n):
        head = [float(v) for v in lines[6 + 2 * r].split()]
        samples = [float(v) for v in lines[7 + 2 * r].split()]
        out["traces"].append({"position": head[0:3], "source": head[3:6], "start": head[6], "samples": samples})
        assert int(head[7]) == len(samples)
    return out


def export_cases():
    z = np.load(GOLDEN)
    return json.loads(bytes(z["index"]).decode())["export"]


def import_cases():
    z = np.load(GOLDEN)
    return json.loads(bytes(z["index"]).decode())["import"]


@pytest.mark.parametrize("case", export_cases(), ids=lambda c: c["name"])
def test_export_matches_reference_bytes(case, fixtures, R, swl, tmp_path):
    z, _ = fixtures
    path = tmp_path / "out.sgy"
    kw = record_set(z, case)
    args = dict(component=case["component"], profile=case["profile"], gain=case["gain"], interval_s=case["interval"])
    if case["status"] != "ok":
        with pytest.raises(swl.SwlError) as e:
            R.write_segy(path, **kw, **args)
        assert str(e.value).endswith(case["status"][len("error "):]), (str(e.value), case["status"])
        assert not path.exists()
        return
    R.write_segy(path, **kw, **args)
    want = bytes(z[f"file/{case['name']}"])
    got = path.read_bytes()
    assert len(got) == len(want)
    if got != want:
        first = next(i for i in range(len(got)) if got[i] != want[i])
        pytest.fail(f"first differing byte at {first}")


@pytest.mark.parametrize("case", import_cases(), ids=lambda c: c["name"])
def test_import_matches_reference_reader(case, fixtures, R, swl, tmp_path):
    z, _ = fixtures
    path = tmp_path / "in.sgy"
    path.write_bytes(bytes(z[f"file/{case['name']}"]))
    want = parse_dump(case["dump"])
    if "error" in want:
        with pytest.raises(swl.SwlError) as e:
            R.read_segy(path)
        assert str(e.value).endswith(want["error"]), (str(e.value), want["error"])
        return
    got = R.read_segy(path)
    for k in ("dt", "component", "units", "description"):
        assert got[k] == want[k], k
    assert len(got["traces"]) == len(want["traces"])
    for g, w in zip(got["traces"], want["traces"]):
        assert g["position"] == w["position"] and g["source"] == w["source"] and g["start"] == w["start"]
        np.testing.assert_array_equal(g["samples"], np.array(w["samples"]))


def test_round_trip_and_transactional_failure(R, swl, tmp_path):
    # src/common/RecordIoValidation.cpp: two components, IEEE32/64, exact fractional-us dt, signed mm
    # geometry, trace delays; a refused export leaves an existing file untouched; a broken file fails
    a, b = [.125, -.5, 1.25, 0], [-.25, 1, -2.5, 0]
    kw = dict(channels=[np.array([a, a]), np.array([b, b])], components=["Vz", "Vx"], dt=.000423370123456789,
              positions=[[-1.234, 23.456, 10.234], [0.766, 23.456, 10.234]], sources=[[12.345, -6.789, 8.765]] * 2,
              start_times=[0.0, 0.005])
    for profile in (R.IEEE32, R.IEEE64):
        for comp in (0, 1):
            path = tmp_path / f"p{profile}_c{comp}.sgy"
            R.write_segy(path, component=comp, profile=profile, **kw)
            got = R.read_segy(path)
            assert abs(got["dt"] - kw["dt"]) < 1e-18 and got["component"] == kw["components"][comp] and got["units"] == "m/s"
            for r in range(2):
                assert got["traces"][r]["start"] == kw["start_times"][r]
                np.testing.assert_allclose(got["traces"][r]["position"], kw["positions"][r], atol=1e-10)
                np.testing.assert_allclose(got["traces"][r]["source"], kw["sources"][r], atol=1e-10)
                np.testing.assert_array_equal(got["traces"][r]["samples"], kw["channels"][comp][r])
    existing = tmp_path / "p0_c0.sgy"
    before = existing.read_bytes()
    with pytest.raises(swl.SwlError):
        R.write_segy(existing, **dict(kw, dt=0.0))
    assert existing.read_bytes() == before
    broken = tmp_path / "broken.sgy"
    broken.write_bytes(b"not segy")
    with pytest.raises(swl.SwlError, match="shorter than its file headers"):
        R.read_segy(broken)


def test_ebcdic_header_is_code_page_037(R, tmp_path):
    # the legacy IBM profile writes its textual header in EBCDIC (IBM code page 037)
    path = tmp_path / "ibm.sgy"
    R.write_segy(path, channels=[np.array([[1.0, -2.0]])], components=["Vz"], dt=.001, profile=R.IBM32)
    text = path.read_bytes()[:3200]
    assert text.decode("cp037").startswith("C 1 SEISWAVE LAB - ELASTIC WAVE RECEIVER RECORDS")
