"""The C++ drop-in (include/alglin_b200/BorderedCR.hh): a reference-style
program (tests/cpp/test_bcr_cpp.cc, the checks of src_tests/test7-BorderedCR.cc)
compiles against it on CPU and runs on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_bcr_cpp.cc")
EXE = os.path.join(ROOT, "tests", "cpp", "test_bcr_cpp")


def build_exe():
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", os.path.join(ROOT, "alglin_b200"), "-lalglin_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "alglin_b200"), "-o", EXE], check=True)
    return EXE


def test_cpp_dropin_compiles():
    assert os.path.exists(build_exe())


@pytest.mark.gpu
def test_cpp_dropin_runs_test7_workload():
    exe = build_exe()
    r = subprocess.run([exe, "10000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "C++ drop-in ok" in r.stdout
    assert "CyclicReduction+LU" in r.stdout
