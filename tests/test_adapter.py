"""The reference-side adapters compile against the reference's own types (CPU only).

seiswavelab--curvilinear_b200/adapter/b200_engines.hpp is what a maintainer adds to SeisWave Lab
beside CudaEngine / CudaEngine3D.  tests/adapter_check.cpp includes the reference's real
Point::MeshT, Point::Mesh, Receiver and ReceiverTrace3D headers (read-only, from the checkout the
oracle recipe names), fills every field, and checks that the C mirrors receive each one, that
receiver nodes equal the reference's Point::index, and that an engine request without a GPU comes
back as an exception.  A field-order or type drift between the reference and the mirrors fails to
compile or fails a check.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "seiswavelab--curvilinear_b200"


def test_adapters_compile_against_the_reference_types(oracle_mod, swl, tmp_path):
    ref = oracle_mod.reference_root()
    if ref is None or shutil.which("g++") is None:
        pytest.skip("reference sources or g++ not available")
    swl.library()  # the library the adapter links
    exe = tmp_path / "adapter_check"
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror=narrowing",
           f"-I{ref / 'include'}", f"-I{ref / 'src' / 'two_d'}", f"-I{ref / 'src' / 'three_d'}", f"-I{ref / 'src' / 'common'}",
           f"-I{ROOT / 'include'}", f"-I{PKG / 'adapter'}", str(ROOT / "tests" / "adapter_check.cpp"),
           f"-L{PKG}", "-lswl_b200", f"-Wl,-rpath,{PKG}", "-o", str(exe)]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr[-4000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip().endswith("OK"), run.stdout + run.stderr
