"""Generates tests/golden/config_sizes.npz: the reference's results at the workloads' full
sizes, as digests (tests/golden/digest.py).

The values come from the su2 headers compiled behind a C ABI (oracle/ref_harness.cc ->
oracle/_ref/libsu2ref.so, ``make -C oracle ref``).  Inputs are rebuilt on any machine from
seeds: the reference's own hot start (std::mt19937, gaugeconfig.hh:277-302, restated bit for
bit in the oracle) and the device path's Philox streams (restated in the oracle), so only
the outputs are stored.

    python tests/golden/make_config_sizes.py

Cases:
  u1_256  U(1) d=2 256x256 hot start (seed 13526463, random_gauge_trafo 654321), staggered
          m = 0.05, b = the Philox complex source (seed 4242, index 0):
          D D^+ b (staggered.hpp:290-389); the CG solve of D D^+ x = b from x = 0 to
          |r| < 1e-10 |b| (CG.hpp:36-94: the reference's absolute bound, given as 1e-10 |b|);
          BiCGStab on D x = b from x = 0 to the same bound (BiCGStab.hpp:36-106).
  su2_24  SU(2) d=4 24^4 hot start (seed 4711, trafo 99): the gauge derivative at beta 2.4
          (flat-gaugemonomial.hh:105-131) and the Wilson action (flat-gaugemonomial.hh:46-54).
  su2_32  SU(2) d=4 32^4 start near the workload's plaquette: the reference's hot start with
          heat 0.13 (random_element.hh:9-25 draws rotation angles up to 0.26 pi; mean
          plaquette 0.634 against 0.630 of the thermalised beta = 2.4 field) and
          random_gauge_trafo (seed 13526463, trafo 654321): one RK3 flow step at
          eps 0.01 (flat-gradient_flow.hh:17-50) and the omf2 tau 1 n 16 trajectory at
          beta 2.4 with the Philox momenta (seed 2024, trajectory 0) injected
          (md_update.hh:18-81 with the momenta given): Delta H, the H terms, the final links.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from digest import store  # noqa: E402

from oracle import oracle as O  # noqa: E402

U1_DIMS = (256, 1, 1, 256)
SU2_24 = (24, 24, 24, 24)
SU2_32 = (32, 32, 32, 32)
SU2_32_HEAT = 0.13


def inputs(o):
    """The seeded inputs of every case, from the oracle's restatements (bit-exact)."""
    return {
        "u1_U": o.hotstart(1, U1_DIMS, 2, 13526463, 1.0, 654321),
        "u1_b": o.philox_pf_source(U1_DIMS, 4242, 0, complex_source=True),
        "su2_24_U": o.hotstart(0, SU2_24, 4, 4711, 1.0, 99),
        "su2_32_U": o.hotstart(0, SU2_32, 4, 13526463, SU2_32_HEAT, 654321),
        "su2_32_P": o.philox_momenta(0, SU2_32, 4, 2024, 0),
    }


def main():
    if not O.available("ref"):
        O.build("ref")
    if not O.available("orc"):
        O.build("oracle")
    r = O.Oracle("ref")
    x = inputs(O.Oracle("orc"))
    # the inputs must be the reference's own hot start
    assert np.array_equal(x["u1_U"], r.hotstart(1, U1_DIMS, 2, 13526463, 1.0, 654321))
    assert np.array_equal(x["su2_24_U"], r.hotstart(0, SU2_24, 4, 4711, 1.0, 99))
    assert np.array_equal(x["su2_32_U"],
                          r.hotstart(0, SU2_32, 4, 13526463, SU2_32_HEAT, 654321))
    g = {}
    t0 = time.time()

    U, b = x["u1_U"], x["u1_b"]
    store(g, "u1_DDdag_b", r.staggered_apply(U1_DIMS, 2, U, 0.05, 2, b))
    tol = 1e-10 * float(np.linalg.norm(b))
    xs, it = r.cg_ddag(U1_DIMS, 2, U, 0.05, b, np.zeros_like(b), tol)
    store(g, "u1_cg_x", xs)
    g["u1_cg_iter"] = np.array(it)
    xs, it = r.bicgstab_d(U1_DIMS, 2, U, 0.05, b, np.zeros_like(b), tol)
    store(g, "u1_bicgstab_x", xs)
    g["u1_bicgstab_iter"] = np.array(it)
    print(f"u1 256^2 done ({time.time() - t0:.0f} s)")

    U = x["su2_24_U"]
    store(g, "su2_24_force", r.gauge_derivative(0, SU2_24, 4, 2.4, U))
    g["su2_24_S"] = np.array(-2.4 / 2 * r.gauge_energy(0, SU2_24, 4, U))
    print(f"su2 24^4 done ({time.time() - t0:.0f} s)")

    U = x["su2_32_U"]
    g["su2_32_plaq"] = np.array(r.gauge_energy(0, SU2_32, 4, U) / (32 ** 4 * 6 * 2))
    store(g, "su2_32_flow", r.runge_kutta(0, SU2_32, 4, 2.4, 0.01, U))
    dH, Ut, _, H = r.md_injected(0, SU2_32, 4, 2.4, 6, 16, 1.0, U, x["su2_32_P"])
    g["su2_32_md_dH"] = np.array(dH)
    g["su2_32_md_H"] = H
    store(g, "su2_32_md_U", Ut)
    print(f"su2 32^4 done ({time.time() - t0:.0f} s)")

    out = os.path.join(HERE, "config_sizes.npz")
    np.savez_compressed(out, **g)
    print(f"wrote {out}: {os.path.getsize(out)} bytes, {len(g)} arrays")


if __name__ == "__main__":
    main()
