"""The Tpetra adapter (include/MCLS_TpetraAdapter.hpp) over libmclsgpu.

Trilinos is not in this image, so tests/cpp/tpetra_adapter_test.cpp compiles
the adapter against tests/cpp/tpetra_standin, a stand-in with Tpetra's names
and copy-by-view semantics for the calls the adapter makes.  `cpu` mode
checks the traits, LinearProblem's host helpers and a block solve on those
types and that the GPU managers instantiate on them; `gpu` mode runs MCSA
and a device-built point Jacobi on them, after
tpetra/test/tstTpetraMCSASolverManager.cpp:72-204.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mcls_b200")


@pytest.fixture(scope="module")
def adapter_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("tpetra") / "tpetra_adapter_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "tests", "cpp", "tpetra_standin"),
           os.path.join(ROOT, "tests", "cpp", "tpetra_adapter_test.cpp"),
           "-L", LIBDIR, "-lmclsgpu", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    subprocess.run(cmd, check=True)
    return out


def _run(binary, mode):
    p = subprocess.run([binary, mode], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert f"{mode}: 0 failure(s)" in p.stdout


def test_tpetra_adapter_without_device(adapter_bin):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("the no-device checks need a machine without a GPU")
    except ImportError:
        pass
    _run(adapter_bin, "cpu")


@pytest.mark.gpu
def test_tpetra_adapter_solves_on_gpu(adapter_bin):
    _run(adapter_bin, "gpu")
