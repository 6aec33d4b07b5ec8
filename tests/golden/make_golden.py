"""Generate golden vectors from the reference's own RNG and CDF sampler.

Run with MCLS_REFERENCE_ROOT naming an MCLS source tree: it builds oracle/_ref
(src/MCLS_Xorshift.hpp, src/MCLS_RNGTraits.hpp, src/MCLS_SamplingTools.hpp,
src/MCLS_DBC.cpp compiled where they lie) and writes reference_rng.json next
to this script.  The tests compare the oracle against this file, so the GPU
box (which has no reference tree) still checks the oracle's pin.

    MCLS_REFERENCE_ROOT=<MCLS tree> python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def main():
    O.build()
    R = O.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref not built: the reference tree is required")
    out = {"generator": "oracle/_ref (reference Xorshift<>, RNGTraits, SamplingTools)"}
    streams = []
    for seed in (1, 7, 12345, 2**31 - 1, 0x9E3779B97F4A7C15):
        n = 64
        raw = np.empty(n, np.uint64)
        R.ref_xorshift_raw(seed, n, raw)
        u = np.empty(n, np.float64)
        R.ref_xorshift_uniforms(seed, n, u)
        streams.append({"seed": int(seed), "raw": [int(v) for v in raw],
                        "uniforms_hex": [float(v).hex() for v in u]})
    out["streams"] = streams
    # Sampler answers on seeded CDFs, including exact bin edges.
    rng = np.random.Generator(np.random.PCG64(2024))
    cases = []
    for size in (1, 2, 5, 9, 33):
        w = rng.uniform(0.0, 1.0, size)
        cdf = np.cumsum(w)
        cdf /= cdf[-1]
        us = list(rng.uniform(0, 1, 16)) + list(cdf) + [0.0, float(np.nextafter(1.0, 0.0))]
        ans = [int(R.ref_sample_discrete_cdf(np.ascontiguousarray(cdf), size, float(u))) for u in us]
        cases.append({"cdf_hex": [float(c).hex() for c in cdf],
                      "u_hex": [float(u).hex() for u in us], "bin": ans})
    out["sampling"] = cases
    with open(os.path.join(HERE, "reference_rng.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "reference_rng.json"))


if __name__ == "__main__":
    main()
