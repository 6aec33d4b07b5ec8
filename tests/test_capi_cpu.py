"""C ABI checks that need no GPU: exports, struct layouts, host-side logic."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from mcls_b200 import capi
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(mclsgpu_\w+)\s*\(", txt, re.M):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    L = capi.load()
    declared = _declared_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert set(capi.EXPORTS) <= declared


def test_abi_version_and_build_info():
    L = capi.load()
    assert L.mclsgpu_abi_version() == 1
    assert b"sm_100a" in L.mclsgpu_build_info()


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "mclsgpu.h"
#define F(T, f) printf(#T "." #f " %zu\\n", offsetof(T, f));
int main(void) {
  printf("mc %zu\\nmcsa %zu\\nprec %zu\\nstats %zu\\n", sizeof(mclsgpu_mc_params),
         sizeof(mclsgpu_mcsa_params), sizeof(mclsgpu_precond_params), sizeof(mclsgpu_stats));
  F(mclsgpu_mc_params, seed) F(mclsgpu_mc_params, rng_mode) F(mclsgpu_mc_params, precision)
  F(mclsgpu_mcsa_params, richardson_omega) F(mclsgpu_precond_params, rho_fallback)
  F(mclsgpu_stats, rho) F(mclsgpu_stats, walk_steps)
  F(mclsgpu_mcsa_params, fixed_point_type)
  printf("anderson %zu\\nwire %zu\\n", sizeof(mclsgpu_anderson_params),
         sizeof(mclsgpu_history_wire));
  F(mclsgpu_anderson_params, mixing) F(mclsgpu_anderson_params, drop_tolerance)
  F(mclsgpu_anderson_params, host_loop)
  F(mclsgpu_history_wire, state) F(mclsgpu_history_wire, step)
  F(mclsgpu_history_wire, weight) F(mclsgpu_history_wire, id)
  F(mclsgpu_history_wire, acc) F(mclsgpu_history_wire, comp)
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run(
        [str(exe)], capture_output=True, text=True, check=True).stdout.strip().splitlines())
    assert int(out["mc"]) == C.sizeof(capi.McParams)
    assert int(out["mcsa"]) == C.sizeof(capi.McsaParams)
    assert int(out["prec"]) == C.sizeof(capi.PrecondParams)
    assert int(out["stats"]) == C.sizeof(capi.Stats)
    assert int(out["mclsgpu_mc_params.seed"]) == capi.McParams.seed.offset
    assert int(out["mclsgpu_mc_params.rng_mode"]) == capi.McParams.rng_mode.offset
    assert int(out["mclsgpu_mc_params.precision"]) == capi.McParams.precision.offset
    assert int(out["mclsgpu_mcsa_params.richardson_omega"]) == capi.McsaParams.richardson_omega.offset
    assert int(out["mclsgpu_precond_params.rho_fallback"]) == capi.PrecondParams.rho_fallback.offset
    assert int(out["mclsgpu_stats.rho"]) == capi.Stats.rho.offset
    assert int(out["mclsgpu_stats.walk_steps"]) == capi.Stats.walk_steps.offset
    assert int(out["mclsgpu_mcsa_params.fixed_point_type"]) == \
        capi.McsaParams.fixed_point_type.offset
    assert int(out["anderson"]) == C.sizeof(capi.AndersonParams)
    for f in ("mixing", "drop_tolerance", "host_loop"):
        assert int(out["mclsgpu_anderson_params." + f]) == getattr(capi.AndersonParams, f).offset
    # The history record the partition driver moves between parts.
    from mcls_b200 import partition

    assert int(out["wire"]) == partition.WIRE_BYTES == capi.load().mclsgpu_history_wire_size()
    for f in ("state", "step", "weight", "id", "acc", "comp"):
        assert int(out["mclsgpu_history_wire." + f]) == partition.WIRE_DTYPE.fields[f][1]


def test_rank_seed_matches_oracle():
    # PRNG(rank) seeding with the random_device draw replaced by a master seed.
    for master in (1, 42, 2**33 + 7):
        for rank in range(4):
            assert capi.rank_seed(master, rank) == O.rank_seed(master, rank)
    assert len({capi.rank_seed(5, r) for r in range(16)}) == 16
    # test/tstPRNG.cpp:66-104: the k-th draws of different ranks differ.
    U = np.array([O.xorshift_uniforms(capi.rank_seed(5, r), 100) for r in range(8)])
    for r in range(8):
        for q in range(r + 1, 8):
            assert np.all(U[r] != U[q])


def test_null_arguments_are_rejected_without_a_device():
    L = capi.load()
    assert L.mclsgpu_context_create(0, None) == capi.ERR_INVALID_ARG
    assert L.mclsgpu_mc_solve(None, None, None, 0, None) == capi.ERR_INVALID_ARG
    assert L.mclsgpu_mcsa_solve(None, None, None, None, None) == capi.ERR_INVALID_ARG
    assert L.mclsgpu_domain_build(None, None, None, None, None, None) == capi.ERR_INVALID_ARG
    assert L.mclsgpu_context_destroy(None) == capi.OK
    assert L.mclsgpu_anderson_solve(None, None, None, None, None) == capi.ERR_INVALID_ARG
    assert L.mclsgpu_fixed_point_solve(None, None, None, None, None, None, None,
                                       None) == capi.ERR_INVALID_ARG
    assert L.mclsgpu_subdomain_build(None, 0, 0, None, 0, None, None, None, None,
                                     None) == capi.ERR_INVALID_ARG
    assert L.mclsgpu_subdomain_destroy(None) == capi.OK


def test_context_reports_missing_device():
    try:
        import torch
        has = torch.cuda.is_available()
    except Exception:
        has = False
    if has:
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert capi.load().mclsgpu_context_create(0, C.byref(h)) == capi.ERR_NO_DEVICE
