"""Generate the golden fixtures from the reference's own CPU solver.

Runs oracle/_ref/ref2d and ref3d (built from the reference sources by oracle/Makefile) on the
small cases of tests/cases.py and stores, per case, the model arrays exactly as the reference
built them, the final wavefields (and CFS-PML / GSLS memories) after the case's steps, the
receiver records and the session scalars, as compressed .npz files next to this script.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE.parent))

import oracle as O  # noqa: E402
from cases import CASES_2D, CASES_3D  # noqa: E402

KEEP_SCALARS_2D = ["nx", "nz", "count", "h", "dt", "total", "steps", "fieldCount", "mechanisms", "cpmlCount",
                   "cpmlWidthX", "cpmlWidthZ", "rates", "sourceDirection", "receivers", "samples", "probeX", "probeZ",
                   "maxMetric", "minJacobian", "maxEdge", "flattenDepth", "waveDt", "dampingDt", "sourceDt",
                   "relaxationDt", "cpmlDt", "energy", "peakEnergy", "maxVelocity", "tractionRelative", "recordDt"]
KEEP_SCALARS_3D = ["nx", "ny", "nz", "count", "h", "dt", "total", "steps", "lambda", "mu", "density", "layered",
                   "receivers", "samples", "receiverIndex", "flattenDepth", "minJacobian", "maxMetricNorm",
                   "minCellLength", "maxCellEdge", "waveDt", "dampingDt", "sourceDt", "energy", "peakEnergy",
                   "maxAbsVelocity", "tractionRate"]


def save(path: Path, case: dict, res: dict, scalars):
    out = {}
    for k, v in res.items():
        if isinstance(v, np.ndarray):
            out["a_" + k] = v
    for k in scalars:
        if k in res:
            out["s_" + k] = np.atleast_1d(np.asarray(res[k], dtype=np.float64))
    for k, v in case.items():
        out["c_" + k] = np.atleast_1d(np.asarray(v, dtype=np.float64))
    np.savez_compressed(path, **out)


def main():
    for name, case in CASES_2D.items():
        res = O.run_reference_2d(case, steps=int(case["maxSteps"]))
        save(HERE / f"ref2d_{name}.npz", case, res, KEEP_SCALARS_2D)
        print("2D", name, int(res["steps"]), "steps")
    for name, case in CASES_3D.items():
        res = O.run_reference_3d(case, steps=int(case["maxSteps"]))
        for k in ("coordinates",):  # not needed by any check; keeps fixtures small
            res.pop(k, None)
        save(HERE / f"ref3d_{name}.npz", case, res, KEEP_SCALARS_3D)
        print("3D", name, int(res["steps"]), "steps")


def load(path: Path):
    """Inverse of save(): (case dict, result dict)."""
    z = np.load(path)
    case, res = {}, {}
    for k in z.files:
        v = z[k]
        if k.startswith("c_"):
            case[k[2:]] = v.tolist() if v.size > 1 else float(v[0])
        elif k.startswith("s_"):
            res[k[2:]] = v if v.size > 1 else float(v[0])
        else:
            res[k[2:]] = v
    return case, res


if __name__ == "__main__":
    main()
