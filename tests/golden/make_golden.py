"""Generates tests/golden/golden.npz from the reference's own code.

The vectors come from the su2 headers compiled behind a C ABI (oracle/ref_harness.cc ->
oracle/_ref/libsu2ref.so, built by ``make -C oracle ref`` from a reference checkout), so the
fixtures pin the reference's behaviour for machines where the reference sources are absent.

    python tests/golden/make_golden.py

Cases (all FP64, small enough that the file stays a few hundred KB):
  su2_*   SU(2) d=4 4^4, hotstart(seed 13526463, delta 1) + random_gauge_trafo(654321)
          (gaugeconfig.hh:277-302, random_gauge_trafo.hh:10-33): plaquette sums, the gauge
          derivative at beta 2.4 (flat-gaugemonomial.hh:105-131), one RK3 flow step eps 0.01
          (flat-gradient_flow.hh:17-50), clover E and Q (flat-energy_density.hh:57-164),
          flow records to t = 0.05, and leapfrog (n 10) / omf2 (n 4) trajectories with
          injected momenta (md_update.hh:18-81 with the momenta given); the Polyakov loop
          (polyakov_loop.hh:48-63), the 2x3 Wilson loop (wilsonloop.hh:147-157) and spatial
          APE smearing at alpha 0.6 (smearape.hh:97-131).
  su2d3_* SU(2) d=3 4x4x1x6: plaquette sums and the gauge derivative at beta 2.0.
  u1_*    U(1) d=2 8x1x1x8 hot start: plaquette sum, gauge derivative at beta 4.0, D D^+ psi
          at m 0.05 (staggered.hpp:290-389), the CG solve of D D^+ x = psi (CG.hpp:36-94)
          and BiCGStab on D (BiCGStab.hpp:36-106) from a seeded start, tolerance 1e-10.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def main():
    if not O.available("ref"):
        O.build("ref")
    r = O.Oracle("ref")
    g = {}

    dims, nd = (4, 4, 4, 4), 4
    U = r.hotstart(0, dims, nd, 13526463, 1.0, 654321)
    g["su2_dims"] = np.array(dims)
    g["su2_U"] = U
    g["su2_plaq"] = np.array(r.gauge_energy(0, dims, nd, U))
    g["su2_plaq_ss"] = np.array(r.gauge_energy(0, dims, nd, U, spatial_only=True))
    g["su2_force"] = r.gauge_derivative(0, dims, nd, 2.4, U)
    g["su2_flow"] = r.runge_kutta(0, dims, nd, 2.4, 0.01, U)
    E, Q = r.energy_density(0, dims, nd, U)
    g["su2_E"], g["su2_Q"] = np.array(E), np.array(Q)
    g["su2_flow_rows"] = np.asarray(r.gradient_flow_rows(0, dims, nd, 2.4, U, 0.05, 0.01),
                                    dtype=np.float64)
    g["su2_polyakov"] = np.array(r.polyakov_loop(0, dims, nd, U))
    g["su2_wilson_2_3"] = np.array(r.wilson_loop(0, dims, nd, U, 2, 3))
    g["su2_ape_0.6"] = r.ape_smear(0, dims, nd, U, 0.6, True)
    P = np.random.default_rng(31).normal(size=O.Oracle.nlinks(dims, nd) * 3)
    g["su2_P"] = P
    for name, integ, n in (("leapfrog", 0, 10), ("omf2", 6, 4)):
        dH, Ut, Pt, H = r.md_injected(0, dims, nd, 2.4, integ, n, 1.0, U, P)
        g[f"su2_md_{name}_dH"] = np.array(dH)
        g[f"su2_md_{name}_U"] = Ut

    d3 = (4, 4, 1, 6)
    U3 = r.hotstart(0, d3, 3, 4711, 1.0, 99)
    g["su2d3_dims"] = np.array(d3)
    g["su2d3_U"] = U3
    g["su2d3_plaq"] = np.array(r.gauge_energy(0, d3, 3, U3))
    g["su2d3_force"] = r.gauge_derivative(0, d3, 3, 2.0, U3)

    du = (8, 1, 1, 8)
    Uu = r.hotstart(1, du, 2, 13526463, 1.0, 654321)
    V = 64
    psi = np.random.default_rng(7).normal(size=2 * V)
    g["u1_dims"] = np.array(du)
    g["u1_U"] = Uu
    g["u1_plaq"] = np.array(r.gauge_energy(1, du, 2, Uu))
    g["u1_force"] = r.gauge_derivative(1, du, 2, 4.0, Uu)
    g["u1_psi"] = psi
    g["u1_DDdag_psi"] = r.staggered_apply(du, 2, Uu, 0.05, 2, psi)
    x0 = np.random.default_rng(8).normal(size=2 * V)
    g["u1_x0"] = x0
    x, it = r.cg_ddag(du, 2, Uu, 0.05, psi, x0, 1e-10)
    g["u1_cg_x"], g["u1_cg_iter"] = x, np.array(it)
    x, it = r.bicgstab_d(du, 2, Uu, 0.05, psi, x0, 1e-10)
    g["u1_bicgstab_x"], g["u1_bicgstab_iter"] = x, np.array(it)

    out = os.path.join(HERE, "golden.npz")
    np.savez_compressed(out, **g)
    print(f"wrote {out}: {os.path.getsize(out)} bytes, {len(g)} arrays")


if __name__ == "__main__":
    main()
