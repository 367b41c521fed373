"""The C++ mirror of the reference's dnnsolver classes (include/
drwc_dnnsolver.hpp) compiles against the C ABI and links with the library
(run on the device in test_gpu_dnnsolver_shim.py)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "deeprwcap_b200" / "libdrwc.so"


def build_shim(out: Path) -> Path:
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "cpp" / "dnnsolver_shim.cpp"), "-L", str(LIB.parent), "-ldrwc",
           f"-Wl,-rpath,{LIB.parent}", "-pthread", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.skipif(shutil.which("g++") is None or not LIB.exists(),
                    reason="needs g++ and the built library")
def test_shim_compiles_and_links(tmp_path):
    assert build_shim(tmp_path / "shim").exists()
