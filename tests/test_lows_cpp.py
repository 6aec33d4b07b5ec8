"""The Stratimikos-facing solver (include/MCLS_LinearOpWithSolve.hpp) over
libmclsgpu.

tests/cpp/lows_test.cpp is compiled with g++ against the headers and the
in-tree library.  Its `cpu` mode checks the factory's parameter lists and
their validation, "Solver Type" -> manager, the preconditioner factories,
and the column loop, tolerance handling and status over a host solver behind
the SolverManager interface; its `gpu` mode solves blocks of right-hand
sides on the device through the factory ("MCSA", "Fixed Point", "Anderson",
the "Point Jacobi" preconditioner factory), after the reference's LOWS test
(thyra/test/LOWSFactoryTpetra/test_single_mcls_thyra_solver.cpp).
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mcls_b200")


@pytest.fixture(scope="module")
def lows_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("lows") / "lows_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "lows_test.cpp"),
           "-L", LIBDIR, "-lmclsgpu", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    subprocess.run(cmd, check=True)
    return out


def _run(binary, *args):
    p = subprocess.run([binary, *args], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert f"{args[0]}: 0 failure(s)" in p.stdout


def test_lows_without_device(lows_bin, tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("the no-device checks need a machine without a GPU")
    except ImportError:
        pass
    _run(lows_bin, "cpu", str(tmp_path))


@pytest.mark.gpu
def test_lows_block_solves_on_gpu(lows_bin):
    _run(lows_bin, "gpu")
