"""The C++ drop-in shim (include/olap_reference_api.hpp): a caller written
against the reference's OLAPcore signatures compiles against the B200
library (CPU) and computes the same int total as a direct loop (GPU)."""
import shutil
import subprocess
from pathlib import Path

import pytest

from memory_database_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "olapcore_drop_in.cpp"


def _compile(out: Path) -> None:
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    cmd = [gxx, "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(SRC), "-o", str(out),
           str(_lib.LIB_PATH), f"-Wl,-rpath,{_lib.LIB_PATH.parent}", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_drop_in_shim_compiles(tmp_path):
    _compile(tmp_path / "drop_in")


@pytest.mark.gpu
def test_drop_in_shim_runs_on_gpu(tmp_path):
    exe = tmp_path / "drop_in"
    _compile(exe)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
