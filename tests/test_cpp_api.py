"""The C++ drop-ins (include/alglin_b200/BorderedCR.hh, include/alglin_b200/BABD.hh):
reference-style programs (tests/cpp/test_bcr_cpp.cc, the checks of
src_tests/test7-BorderedCR.cc; tests/cpp/test_babd_cpp.cc, the BABD wrapper's
cyclic-reduction choices) compile against them on CPU and run on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_bcr_cpp.cc")
EXE = os.path.join(ROOT, "tests", "cpp", "test_bcr_cpp")


def build_exe(src=SRC, exe=EXE):
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), src,
                    "-L", os.path.join(ROOT, "alglin_b200"), "-lalglin_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "alglin_b200"), "-o", exe], check=True)
    return exe


BABD_SRC = os.path.join(ROOT, "tests", "cpp", "test_babd_cpp.cc")
BABD_EXE = os.path.join(ROOT, "tests", "cpp", "test_babd_cpp")


def test_cpp_dropin_compiles():
    assert os.path.exists(build_exe())


@pytest.mark.gpu
def test_cpp_dropin_runs_test7_workload():
    exe = build_exe()
    r = subprocess.run([exe, "10000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "C++ drop-in ok" in r.stdout
    assert "CyclicReduction+LU" in r.stdout


def test_cpp_babd_wrapper_compiles():
    assert os.path.exists(build_exe(BABD_SRC, BABD_EXE))


@pytest.mark.gpu
def test_cpp_babd_wrapper_runs():
    exe = build_exe(BABD_SRC, BABD_EXE)
    r = subprocess.run([exe, "2000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "BABD drop-in ok" in r.stdout
    for name in ("CyclicReduction+LU", "CyclicReduction+QR", "CyclicReduction+QRP"):
        assert name in r.stdout


def test_umma_layout_invariants():
    """The tcgen05 pair kernel's shared-memory layout (bcr_umma_layout.cuh) for
    every accepted shape: no overlap of regions live at the same time, 16-byte
    aligned operands, tiles inside their regions, within one CTA's limit."""
    src = os.path.join(ROOT, "tests", "cpp", "umma_layout_check.cu")
    exe = os.path.join(ROOT, "tests", "cpp", "umma_layout_check")
    subprocess.run(["nvcc", "-std=c++17", "-cudart", "shared", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "alglin_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
                    src, "-o", exe], check=True)
    try:
        r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    finally:
        os.remove(exe)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
