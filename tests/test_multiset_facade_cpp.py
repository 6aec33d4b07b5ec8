"""Multi-set MCSA through the C++ manager API (tests/cpp/multiset_facade_test.cpp):
two sets of one problem on one GPU, each driven by its own host thread and
MCSASolverManager, their Monte Carlo corrections summed by the
MultiSetLinearProblem's set reducer ("Number of Sets" = 2)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mcls_b200")
CUDA = "/usr/local/cuda"


def _build(tmp_path):
    out = str(tmp_path / "multiset_facade_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-pthread",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "multiset_facade_test.cpp"),
           "-L", LIBDIR, "-lmclsgpu", f"-Wl,-rpath,{LIBDIR}",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA}/lib64",
           "-o", out]
    subprocess.run(cmd, check=True)
    return out


def test_multiset_facade_compiles(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_two_sets_through_the_manager(tmp_path):
    p = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "multiset: 0 failure(s)" in p.stdout
