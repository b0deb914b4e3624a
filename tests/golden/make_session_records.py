"""Generates the receiver-CSV and session SEG-Y golden fixtures from the reference's own writers.

Runs oracle/_ref/ref2d and ref3d (built from the reference's sources by oracle/Makefile, which
call writeReceivers, src/two_d/CurvilinearSolver2D.cpp:811-855, and writeReceiversCsv,
src/three_d/ReceiverIo.cpp) on every case of tests/cases.py, after zero steps and after the
case's steps, and stores the files' text in tests/golden/receivers_csv.json:
  - "<dim>/<case>/0": the whole file after zero steps (header and the t = 0 rows);
  - "<dim>/<case>/n": the comment and column-header lines after the case's steps, and the steps.
The data rows after n steps are checked against the golden records of the same runs.
The drivers also export the sessions' record views (src/two_d/ui/Workbench2D.cpp:251-268,
src/three_d/ui/RecordView3D.cpp:5-6) with writeSegy (src/common/SegyIo.cpp): Vz as IEEE32 and
Vx (2D) / Vy (3D) as IEEE64, after zero and after n steps; their bytes go to
tests/golden/session_segy.npz as "<dim>/<case>/<file>/<0|n>".

The 2D drivers also call writeSnapshot (src/two_d/CurvilinearSolver2D.cpp:725-810) with the
default options and with every component, and readProbes (:710-724) at four logical nodes; the
snapshots are stored as their SHA-256, size and header (through "<PointData"), the probes as values,
in receivers_csv.json under "2/<case>/snapshot[_all]/<0|n>" and "2/<case>/probes/n".  The 3D
drivers call writeVts (src/three_d/VtsWriter.cpp) with the default options and with a reduced set
("3/<case>/snapshot[_some]/<0|n>").  The drivers also save the model with writeModelVts
(src/two_d/ModelIo2D.cpp:75-145) and writeModelVts3D (src/three_d/ModelIo3D.cpp:87-170) as a CPU
run with one thread ("<dim>/<case>/model"); the 3D driver names its layers "layer0", "layer1", ...

Usage: python tests/golden/make_session_records.py   (needs oracle/_ref/ref2d and ref3d: make -C oracle ref)
"""
from __future__ import annotations

import hashlib
import json
import sys

import numpy as np
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE.parent))

import oracle as O  # noqa: E402
from cases import CASES_2D, CASES_3D  # noqa: E402


def header(text: str) -> list[str]:
    lines = text.splitlines()
    n = next(i for i, line in enumerate(lines) if not line.startswith("#")) + 1  # comments + column names
    return lines[:n]


def main():
    out, segy = {}, {}
    for dim, cases, run in ((2, CASES_2D, O.run_reference_2d), (3, CASES_3D, O.run_reference_3d)):
        for name, case in cases.items():
            zero = run(case, steps=0, dump_mesh=False, files=True)
            full = run(case, steps=int(case["maxSteps"]), dump_mesh=False, files=True)
            files = ["receivers"] if dim == 2 else ["receivers", "receivers_xz"]
            for f in files:
                out[f"{dim}/{name}/{f}/0"] = zero["csv:" + f]
                out[f"{dim}/{name}/{f}/n"] = {"steps": int(full["steps"]), "header": header(full["csv:" + f])}
            for f in ("vz_ieee32", "vx_ieee64" if dim == 2 else "vy_ieee64"):
                segy[f"{dim}/{name}/{f}/0"] = np.frombuffer(zero["sgy:" + f], dtype=np.uint8)
                segy[f"{dim}/{name}/{f}/n"] = np.frombuffer(full["sgy:" + f], dtype=np.uint8)
            for f in (("snapshot", "snapshot_all") if dim == 2 else ("snapshot", "snapshot_some")):
                for tag, res in (("0", zero), ("n", full)):
                    text = res["vts:" + f]
                    out[f"{dim}/{name}/{f}/{tag}"] = {"sha256": hashlib.sha256(text.encode()).hexdigest(),
                                                      "size": len(text.encode()),
                                                      "head": text[:text.index("<PointData")]}
            if dim == 2:
                out[f"2/{name}/probes/n"] = [repr(float(v)) for v in full["probes"]]
            text = zero["vts:model"]  # writeModelVts / writeModelVts3D, compute settings {1 thread, -1}
            out[f"{dim}/{name}/model"] = {"sha256": hashlib.sha256(text.encode()).hexdigest(), "size": len(text.encode()),
                                          "head": text[:text.index("<PointData")]}
            print(dim, name, "ok")
    (HERE / "receivers_csv.json").write_text(json.dumps(out, indent=0))
    np.savez_compressed(HERE / "session_segy.npz", **segy)


if __name__ == "__main__":
    main()
