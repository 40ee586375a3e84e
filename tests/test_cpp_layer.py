"""The C++ operator layer (include/cup3d_b200_operators.hpp) compiles against
the C ABI, links the library, and drives a few time steps on the GPU."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "_build" / "test_operators"


def build_exe():
    EXE.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "test_operators.cpp"),
           "-L", str(ROOT / "cup3d_b200"), "-lcup3d_b200", f"-Wl,-rpath,{ROOT / 'cup3d_b200'}", "-o", str(EXE)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return EXE


def test_cpp_operator_layer_compiles_and_links():
    assert build_exe().exists()


@pytest.mark.gpu
def test_cpp_operator_layer_runs_steps():
    exe = build_exe()
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "step 3" in r.stdout
