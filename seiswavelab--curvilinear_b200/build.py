"""Build libswl_b200.so in-tree: every CUDA unit for sm_100a only (no PTX for other targets).

FP64 units are compiled with --fmad=false so the plain path reproduces the reference
arithmetic; FP32 units keep FMA contraction.  Objects are cached in _build/ by modification
time; `python build.py` or ``build()`` from Python.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "libswl_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-strict-aliasing",
          "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{SRC}"]
UNITS = {
    "runtime.cu": [],
    "engine2d_f64.cu": ["--fmad=false"],
    "engine2d_f32.cu": [],
    # the 2D stage kernels, one unit per (precision, GSLS mechanism count), built in parallel
    **{f"stages2d.cu@{r}{m}": (["--fmad=false"] if r == "f64" else []) +
       [f"-DSWL_STAGE_REAL={'double' if r == 'f64' else 'float'}", f"-DSWL_STAGE_MECH={m}"]
       for r in ("f64", "f32") for m in range(4)},
    # the persistent multi-shot 2D kernel, one unit per (precision, GSLS mechanism count)
    **{f"queue2d.cu@{r}{m}": (["--fmad=false"] if r == "f64" else []) +
       [f"-DSWL_STAGE_REAL={'double' if r == 'f64' else 'float'}", f"-DSWL_STAGE_MECH={m}", "-DSWL_STAGE_COHERENT=1"]
       for r in ("f64", "f32") for m in range(4)},
    "engine3d_f64.cu": ["--fmad=false"],
    "engine3d_f32.cu": [],
    "abi.cpp": ["-x", "cu"],
    "noalloc.cu": ["--fmad=false"],
    "geometry.cu": ["--fmad=false"],
    # C++20 host: model construction and sessions (no FMA on the host either, as in the reference)
    "host/gsls.cpp": [],
    "host/model2d.cpp": [],
    "host/model3d.cpp": [],
    "host/session.cpp": [],
    "host/server.cpp": [],
    "host/records.cpp": [],
    "host/modelio.cpp": [],
}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise FileNotFoundError("nvcc not found")


def _deps() -> float:
    """Newest modification time among headers (any header change rebuilds everything)."""
    stamps = [p.stat().st_mtime for p in list(SRC.rglob("*.cuh")) + list(SRC.rglob("*.hpp")) + list(INCLUDE.glob("*.h"))]
    return max(stamps) if stamps else 0.0


def _compile(unit: str, flags: list[str], verbose: bool, newest: float) -> Path:
    # "file@tag" compiles `file` once more under another object name (with its own flags)
    src = SRC / unit.split("@")[0]
    obj = OUT / (unit.replace("/", "_").replace("@", "_") + ".o")
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
    stamp = obj.with_suffix(".cmd")  # the command an object was built with; a change rebuilds it
    if (obj.exists() and stamp.exists() and stamp.read_text() == " ".join(cmd)
            and obj.stat().st_mtime >= max(src.stat().st_mtime, newest)):
        return obj
    if verbose:
        print(" ".join(cmd), flush=True)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{proc.stdout}\n{proc.stderr}")
    stamp.write_text(" ".join(cmd))
    if verbose and proc.stderr.strip():
        print(proc.stderr, flush=True)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    OUT.mkdir(exist_ok=True)
    newest = _deps()
    jobs = jobs or min(len(UNITS), os.cpu_count() or 4)
    with ThreadPoolExecutor(jobs) as pool:
        objs = list(pool.map(lambda kv: _compile(kv[0], kv[1], verbose, newest), UNITS.items()))
    if not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
