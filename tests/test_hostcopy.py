"""The host copies of the staged transfers (csrc/hostcopy.cpp): byte-exact
copies that count non-finite doubles, exact float-to-double widening, at
every alignment of source and destination (a C++ check compiled here)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_host_copies(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "hostcopy_check"
    src = ROOT / "stl-dev-mpi_b200" / "csrc"
    subprocess.run([cxx, "-O2", "-std=c++17", f"-I{src}", str(ROOT / "tests" / "hostcopy_check.cpp"),
                    str(src / "hostcopy.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fails 0" in r.stdout
