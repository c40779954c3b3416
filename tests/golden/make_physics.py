"""Generates tests/golden/physics.json: plaquette expectation values of the reference's own
Metropolis chain (flat-sweep.hh:64-164 with its mt19937 engines), for the statistical
device tests in tests/test_gpu_physics.py.

    python tests/golden/make_physics.py

The chain runs the su2 headers compiled behind a C ABI (oracle/ref_harness.cc ->
oracle/_ref/libsu2ref.so, ``make -C oracle ref``).  The plaquette is normalised as the
driver does (hmc.hpp:99-106): the sum of ReTr over all plaquettes / (V d(d-1)/2 Nc).  The
error is the standard error of 20 block means.

Case u1_8x4_b0.8: U(1) d=4 8^4, beta 0.8, delta 0.5, 8 hits, uniform random start,
300 thermalisation sweeps, then 3000 sweeps measured.  beta 0.8 is in the confined phase,
well away from the transition near beta 1.01, so chains from any start agree.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def blocked(x, nblocks=20):
    x = np.asarray(x)
    b = x[: len(x) // nblocks * nblocks].reshape(nblocks, -1).mean(axis=1)
    return float(x.mean()), float(b.std(ddof=1) / np.sqrt(nblocks))


def main():
    if not O.available("ref"):
        O.build("ref")
    r = O.Oracle("ref")
    L, beta, delta, n_hit, n_therm, n_meas, seed = 8, 0.8, 0.5, 8, 300, 3000, 4711
    dims = (L, L, L, L)
    U = np.random.default_rng(seed).uniform(-np.pi, np.pi, size=L ** 4 * 4)
    P = []
    for i in range(n_therm + n_meas):
        U, _ = r.sweep(1, dims, 4, beta, delta, n_hit, seed, i, U)
        if i >= n_therm:
            P.append(r.gauge_energy(1, dims, 4, U) / (L ** 4 * 6))
    m, e = blocked(P)
    out = {"u1_8x4_b0.8": {"group": "u1", "dims": list(dims), "ndims": 4, "beta": beta,
                           "delta": delta, "N_hit": n_hit, "n_therm": n_therm,
                           "n_meas": n_meas, "plaquette": m, "error": e}}
    with open(os.path.join(HERE, "physics.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
