"""The C++ drop-in class (include/nsgpu_solver.hpp) behaves like the
reference's NeoSolver on the reference's own known-answer systems: compiled
with the host C++ compiler against libnsgpu.so and run on the GPU."""
import pathlib
import shutil
import subprocess

import pytest

from neospice_b200 import _lib as L

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_gpu_solver_known_answers(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    assert cxx, "a host C++ compiler is required"
    exe = tmp_path / "gpu_solver_check"
    cuda = pathlib.Path("/usr/local/cuda")
    cmd = [cxx, "-std=c++17", "-O2", f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}",
           str(ROOT / "tests" / "cpp" / "gpu_solver_check.cpp"), "-o", str(exe),
           str(L.LIB_PATH), f"-L{cuda / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{L.LIB_PATH.parent}", f"-Wl,-rpath,{cuda / 'lib64'}"]
    subprocess.run(cmd, check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "0 failure(s)" in res.stdout
