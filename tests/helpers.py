"""Helpers shared by the parity tests: golden fixtures -> mesh dictionaries."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
from make_golden import load  # noqa: E402

GOLDEN = HERE / "golden"


def golden_2d():
    return sorted(p.stem[len("ref2d_"):] for p in GOLDEN.glob("ref2d_*.npz"))


def golden_3d():
    return sorted(p.stem[len("ref3d_"):] for p in GOLDEN.glob("ref3d_*.npz"))


def load_2d(name: str):
    case, res = load(GOLDEN / f"ref2d_{name}.npz")
    return case, res, mesh_2d(case, res)


def load_3d(name: str):
    case, res = load(GOLDEN / f"ref3d_{name}.npz")
    return case, res, mesh_3d(case, res)


def mesh_2d(case: dict, res: dict) -> dict:
    """Engine/oracle mesh dict from a reference 2D dump (model arrays as the reference built them)."""
    m = {k: v for k, v in res.items() if isinstance(v, np.ndarray) and v.ndim == 1 and v.size == int(res["count"]) or
         k in ("normals", "cpmlX", "cpmlZ")}
    for k in ("nx", "nz", "h", "fieldCount", "mechanisms", "cpmlCount", "cpmlWidthX", "cpmlWidthZ", "dt"):
        m[k] = res[k]
    m["rates"] = np.atleast_1d(res["rates"]).tolist()
    m["sourceDirection"] = np.atleast_1d(res["sourceDirection"]).tolist()
    kind = int(case.get("sourceKind", 0))
    amp = case.get("momentPerLength", 2e6) if kind else case.get("forcePerLength", 2e5)
    m["scale"] = amp / (float(res["h"]) ** 2)
    m["frequency"] = case.get("frequency", 30.0)
    if int(kind) == 0:
        m.pop("sourceGradientX", None)
        m.pop("sourceGradientZ", None)
    return m


def receivers_2d(res: dict) -> np.ndarray:
    nx = int(res["nx"])
    xs = np.atleast_1d(res["probeX"]).astype(np.int64)
    zs = np.atleast_1d(res["probeZ"]).astype(np.int64)
    return (xs + 3) + nx * (zs + 3)


def fields_2d(res: dict) -> np.ndarray:
    fc = int(res["fieldCount"])
    return np.stack([res[f"field{f}"] for f in range(fc)])


def records_2d(res: dict):
    R, S = int(res["receivers"]), int(res["samples"])
    return res["tracesVx"].reshape(R, S), res["tracesVz"].reshape(R, S)


def mesh_3d(case: dict, res: dict) -> dict:
    m = {k: v for k, v in res.items() if isinstance(v, np.ndarray) and k not in
         ("tracesVx", "tracesVy", "tracesVz", "receiverIndex") and not k.startswith("field")}
    for k in ("nx", "ny", "nz", "h", "lambda", "mu", "density", "dt"):
        m[k] = float(res[k])
    kind = int(case.get("sourceKind", 0))
    m["sourceAmplitude"] = case.get("sourceMoment", 2e9) if kind else case.get("sourceForce", 2e8)
    d = np.asarray(case.get("sourceDirection", (0, 0, 1)), dtype=np.float64)
    m["sourceDirection"] = (0.0, 0.0, 0.0) if kind else tuple(d / np.linalg.norm(d))
    m["frequency"] = case.get("frequency", 12.0)
    return m


def receivers_3d(res: dict) -> np.ndarray:
    return np.atleast_1d(res["receiverIndex"]).astype(np.int64)


def fields_3d(res: dict) -> np.ndarray:
    return np.stack([res[f"field{f}"] for f in range(9)])


def records_3d(res: dict):
    R, S = int(res["receivers"]), int(res["samples"])
    return [res[f"traces{c}"].reshape(R, S) for c in ("Vx", "Vy", "Vz")]
