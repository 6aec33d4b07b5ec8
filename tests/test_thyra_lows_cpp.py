"""The Thyra layer (include/Thyra_MCLSGpuLinearOpWithSolveFactory.hpp) over
libmclsgpu.

Trilinos is not in this image, so tests/cpp/thyra_lows_test.cpp compiles the
layer against tests/cpp/thyra_standin and tests/cpp/tpetra_standin,
stand-ins with Thyra's and Tpetra's names for the calls it makes.  `cpu`
mode checks the factory, solve support, apply, preconditioned ops,
uninitializeOp and the translation of solve criteria and statuses; `gpu`
mode solves blocks of right-hand sides on the device through the Thyra
interface.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mcls_b200")


@pytest.fixture(scope="module")
def thyra_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("thyra") / "thyra_lows_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "tests", "cpp", "thyra_standin"),
           "-I", os.path.join(ROOT, "tests", "cpp", "tpetra_standin"),
           os.path.join(ROOT, "tests", "cpp", "thyra_lows_test.cpp"),
           "-L", LIBDIR, "-lmclsgpu", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    subprocess.run(cmd, check=True)
    return out


def _run(binary, mode):
    p = subprocess.run([binary, mode], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert f"{mode}: 0 failure(s)" in p.stdout


def test_thyra_layer_without_device(thyra_bin):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("the no-device checks need a machine without a GPU")
    except ImportError:
        pass
    _run(thyra_bin, "cpu")


@pytest.mark.gpu
def test_thyra_layer_solves_on_gpu(thyra_bin):
    _run(thyra_bin, "gpu")
