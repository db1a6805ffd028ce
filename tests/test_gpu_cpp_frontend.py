"""The C++ front end (include/mtl4_b200/itl_gpu.hpp) used with the reference's
call syntax, compiled with g++ against libmtl4_b200.so and run."""
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT


def build_cpp_test(out: Path):
    lib = ROOT / "mtl4_b200"
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "itl_gpu_test.cpp"),
           f"-L{lib}", "-lmtl4_b200", f"-Wl,-rpath,{lib}", "-o", str(out)]
    subprocess.run(cmd, check=True)


def test_cpp_frontend_compiles(tmp_path):
    build_cpp_test(tmp_path / "itl_gpu_test")


@pytest.mark.gpu
def test_cpp_frontend_runs(tmp_path):
    exe = tmp_path / "itl_gpu_test"
    build_cpp_test(exe)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASS" in r.stdout
