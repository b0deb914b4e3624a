"""Generates the SEG-Y golden fixtures from the reference's own writer and reader.

Runs oracle/_ref/ref_segy (src/common/SegyIo.cpp compiled from the reference's sources by
oracle/Makefile) on seeded record sets and on hand-built files of the formats the importer reads,
and stores everything the tests need in tests/golden/segy.npz:
  - per export case: the record set, the options, and the reference's file bytes or its error;
  - per import case: the file bytes and the reference reader's result (or its error).
The record sets follow src/common/RecordIoValidation.cpp (two traces, Vz/Vx, fractional-us dt,
signed millimetre geometry, trace delays; legacy IBM/IEEE with gain 1 and 1e6; resampling) plus a
seeded 24-trace set with values across many magnitudes.

Usage: python tests/golden/make_segy.py   (needs oracle/_ref/ref_segy: make -C oracle ref)
"""
from __future__ import annotations

import json
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF = ROOT / "oracle" / "_ref" / "ref_segy"
OUT = Path(__file__).resolve().parent / "segy.npz"


def records_text(rec) -> str:
    lines = [f"dt {rec['dt']!r}", f"units {rec['units']}",
             "components %d %s" % (len(rec["components"]), " ".join(rec["components"])),
             "traces %d %d" % rec["channels"][0].shape]
    for r in range(rec["channels"][0].shape[0]):
        geo = list(rec["positions"][r]) + list(rec["sources"][r]) + [rec["starts"][r]]
        lines.append(" ".join(repr(float(v)) for v in geo))
        for ch in rec["channels"]:
            lines.append(" ".join(repr(float(v)) for v in ch[r]))
    return "\n".join(lines) + "\n"


def validation_set(dt):
    a, b = [.125, -.5, 1.25, 0], [-.25, 1, -2.5, 0]
    return {"dt": dt, "units": "m/s", "components": ["Vz", "Vx"],
            "channels": [np.array([a, a]), np.array([b, b])],
            "positions": np.array([[-1.234 + r * 2, 23.456, 10.234] for r in range(2)]),
            "sources": np.array([[12.345, -6.789, 8.765]] * 2), "starts": np.array([0.0, 0.005])}


def seeded_set(seed=7, traces=12, samples=96):
    g = np.random.default_rng(seed)
    mag = 10.0 ** g.uniform(-12, 2, size=(traces, samples))
    vz = mag * g.choice([-1.0, 1.0], size=mag.shape)
    vz[:, 0] = 0.0
    vz[0, 5] = -0.0
    vz[1, 7] = 1e-80  # underflows IEEE32 and IBM32
    vx = np.sin(np.linspace(0, 30, samples))[None, :] * g.uniform(1e-6, 1e-2, size=(traces, 1))
    x = np.arange(traces) * 10.0 - 115.0
    return {"dt": 2.5e-4, "units": "m/s", "components": ["Vz", "Vx"], "channels": [vz, vx],
            "positions": np.stack([x, np.zeros(traces), np.full(traces, 2.0)], 1),
            "sources": np.array([[0.5, 0.0, 4.0]] * traces), "starts": np.zeros(traces)}


def export_cases():
    cases = []
    val = validation_set(.000423370123456789)
    val["name"] = "validation"
    for profile in (0, 1):
        for comp in (0, 1):
            cases.append((f"validation_p{profile}_c{comp}", val, comp, profile, 1.0, 0.0))
    legacy = validation_set(.0005)
    legacy["name"] = "legacy"
    for profile in (2, 3):
        for gain in (1.0, 1e6):
            cases.append((f"legacy_p{profile}_g{int(gain)}", legacy, 0, profile, gain, 0.0))
    cases.append(("resampled_legacy", val, 0, 3, 1.0, .0005))
    cases.append(("resampled_ieee32", val, 1, 0, 1.0, .0001))
    seeded = seeded_set()
    seeded["name"] = "seeded"
    for profile in range(4):
        for gain in (1.0, 1e3):
            cases.append((f"seeded_p{profile}_g{int(gain)}", seeded, profile % 2, profile, gain, 0.0))
    cases.append(("seeded_resampled_p1", seeded, 0, 1, 1.0, 1e-4))
    # the reference's refusals
    cases.append(("error_negative_gain", legacy, 0, 2, -1.0, 0.0))
    cases.append(("error_fractional_us_legacy", val, 0, 3, 1.0, 0.0))
    cases.append(("error_bad_component", val, 2, 0, 1.0, 0.0))
    big = validation_set(.0005)
    big["channels"] = [c * 1e60 for c in big["channels"]]
    big["name"] = "huge"
    cases.append(("error_ieee32_overflow", big, 0, 0, 1.0, 0.0))
    cases.append(("error_ibm_overflow", big, 0, 2, 1e30, 0.0))
    return cases


def handmade_files():
    """Files of the formats the importer accepts that this writer never produces."""
    files = {}

    def build(little, rev, fmt, samples, ns=3, interval=500, ext=0, feet=False, weighting=0, extra=None):
        e = "<" if little else ">"
        text = bytearray(b" " * 3200)
        text[0:40] = b"C 1 HAND-MADE TEST FILE".ljust(40)
        binary = bytearray(400)
        struct.pack_into(e + "H", binary, 16, interval)
        struct.pack_into(e + "H", binary, 20, ns)
        struct.pack_into(e + "H", binary, 24, fmt)
        struct.pack_into(e + "H", binary, 54, 2 if feet else 1)
        binary[300] = rev
        struct.pack_into(e + "h", binary, 304, ext)
        body = bytearray(b" " * 3200 * ext)
        codes = {1: "I", 2: "i", 3: "h", 4: "i", 5: "f", 6: "d", 8: "b"}
        for r, trace in enumerate(samples):
            h = bytearray(240)
            struct.pack_into(e + "H", h, 28, 1)
            struct.pack_into(e + "i", h, 80, 1000 * (r + 1))
            struct.pack_into(e + "i", h, 84, -250)
            struct.pack_into(e + "i", h, 40, -30)
            struct.pack_into(e + "h", h, 70, -10)
            struct.pack_into(e + "h", h, 68, 1)
            struct.pack_into(e + "h", h, 108, 4)
            struct.pack_into(e + "H", h, 114, len(trace))
            struct.pack_into(e + "H", h, 116, interval)
            struct.pack_into(e + "h", h, 168, weighting)
            if extra:
                extra(h, e)
            body += h
            for v in trace:
                body += struct.pack(e + codes[fmt], v)
        return bytes(text + binary + body)

    files["rev0_le_int16"] = build(True, 0, 3, [[1, -2, 3], [32767, -32768, 0]])
    files["rev1_be_int32_weighted"] = build(False, 1, 2, [[7, -9, 1 << 20]], weighting=3)
    files["rev1_be_int8_feet_ext"] = build(False, 1, 8, [[1, -1, 127]], ext=1, feet=True)
    files["rev1_be_ieee64"] = build(False, 1, 6, [[0.5, -1e-300, 3.25]])
    files["rev1_le_ieee32"] = build(True, 1, 5, [[0.125, -7.5, 1e-30]])
    files["rev1_be_ibm_bits"] = build(False, 1, 1, [[0x41100000, 0xC2640000, 0]])  # 1.0, -100.0, 0
    files["error_format4"] = build(False, 1, 4, [[1]])
    files["error_short"] = b"not segy"
    return files


def run_write(rec, comp, profile, gain, interval, tmp: Path):
    src, out = tmp / "records.txt", tmp / "out.sgy"
    src.write_text(records_text(rec))
    if out.exists():
        out.unlink()
    r = subprocess.run([str(REF), "write", str(src), str(comp), str(profile), repr(gain), repr(interval), str(out)],
                       capture_output=True, text=True, check=True)
    status = r.stdout.strip()
    return status, (out.read_bytes() if status == "ok" else b"")


def run_read(data: bytes, tmp: Path):
    f, dump = tmp / "in.sgy", tmp / "dump.txt"
    f.write_bytes(data)
    subprocess.run([str(REF), "read", str(f), str(dump)], check=True)
    return dump.read_text()


def main():
    arrays, index = {}, {"export": [], "import": []}
    with tempfile.TemporaryDirectory() as d:
        tmp = Path(d)
        for name, rec, comp, profile, gain, interval in export_cases():
            status, data = run_write(rec, comp, profile, gain, interval, tmp)
            key = f"set/{rec['name']}"
            for c, ch in enumerate(rec["channels"]):
                arrays[f"{key}/channel{c}"] = ch
            arrays[f"{key}/positions"] = rec["positions"]
            arrays[f"{key}/sources"] = rec["sources"]
            arrays[f"{key}/starts"] = rec["starts"]
            if status == "ok":
                arrays[f"file/{name}"] = np.frombuffer(data, dtype=np.uint8)
            index["export"].append({"name": name, "set": rec["name"], "dt": rec["dt"], "units": rec["units"],
                                    "components": rec["components"], "component": comp, "profile": profile,
                                    "gain": gain, "interval": interval, "status": status})
            if status == "ok":
                index["import"].append({"name": name, "dump": run_read(data, tmp)})
        for name, data in handmade_files().items():
            arrays[f"file/{name}"] = np.frombuffer(data, dtype=np.uint8)
            index["import"].append({"name": name, "dump": run_read(data, tmp)})
    arrays["index"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes): {len(index['export'])} export, {len(index['import'])} import cases")


if __name__ == "__main__":
    main()
