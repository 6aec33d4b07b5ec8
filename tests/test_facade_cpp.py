"""The C++ manager API (include/MCLS_*.hpp) over libmclsgpu.

tests/cpp/facade_test.cpp is compiled with g++ against the headers and the
in-tree library.  Its `cpu` mode checks parameter lists, factory names and
ParameterList typing, LinearProblem's host helpers against the reference's
tests (tpetra/test/tstTpetraLinearProblem.cpp: apply, residual update,
composite operator), and that a solve without a device throws
MCLS::Assertion; its `gpu` mode runs the reference's manager tests (signs,
fewer than 20 MCSA iterations, four successive solves, device-built Jacobi
and block-Jacobi preconditioners) through the facade on the GPU.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mcls_b200")


@pytest.fixture(scope="module")
def facade_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("facade") / "facade_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "facade_test.cpp"),
           "-L", LIBDIR, "-lmclsgpu", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    subprocess.run(cmd, check=True)
    return out


def _run(binary, mode):
    p = subprocess.run([binary, mode], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert f"{mode}: 0 failure(s)" in p.stdout


def test_facade_without_device(facade_bin):
    env_has_gpu = False
    try:
        import torch
        env_has_gpu = torch.cuda.is_available()
    except Exception:
        pass
    if env_has_gpu:
        pytest.skip("the no-device check needs a machine without a GPU")
    _run(facade_bin, "cpu")


@pytest.mark.gpu
def test_facade_solves_on_gpu(facade_bin):
    _run(facade_bin, "gpu")
