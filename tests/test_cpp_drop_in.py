"""The C++ drop-in shim (include/olap_reference_api.hpp): callers written
against the reference's signatures (the OLAP core's fused and column-wise
entry points, and the join, select, project, group, aggregation and
star-join operators) compile against the B200 library (CPU) and compute the
same results as direct loops over the same host arrays (GPU)."""
import shutil
import subprocess
from pathlib import Path

import pytest

from memory_database_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
CALLERS = {"olapcore": ROOT / "tests" / "cpp" / "olapcore_drop_in.cpp",
           "operators": ROOT / "tests" / "cpp" / "operators_drop_in.cpp"}


def _compile(src: Path, out: Path) -> None:
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(out),
           str(_lib.LIB_PATH), f"-Wl,-rpath,{_lib.LIB_PATH.parent}", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("caller", sorted(CALLERS))
def test_drop_in_shim_compiles(tmp_path, caller):
    _compile(CALLERS[caller], tmp_path / caller)


@pytest.mark.gpu
@pytest.mark.parametrize("caller", sorted(CALLERS))
def test_drop_in_shim_runs_on_gpu(tmp_path, caller):
    exe = tmp_path / caller
    _compile(CALLERS[caller], exe)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
