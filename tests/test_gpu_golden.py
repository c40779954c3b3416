"""libsu2b (through the C ABI) against vectors produced by the reference's own code
(tests/golden/make_golden.py), with no oracle in between.

Tolerances as the parity contract: FP64 sums and fields within 1e-12 relative, Delta H within
1e-9 absolute, Krylov solutions within 1e-8 relative (both solvers stop at the same residual
and differ by rounding only).
"""
import os

import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


def lattice(gpu, dims, nd, beta, group="su2"):
    Lx, Ly, Lz, Lt = (int(v) for v in dims)
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, beta, group=group)


def test_su2_d4_gauge_path(gpu, g):
    U = g["su2_U"]
    with lattice(gpu, g["su2_dims"], 4, 2.4) as c:
        c.upload(U)
        assert c.gauge_energy() == pytest.approx(float(g["su2_plaq"]), rel=1e-12)
        assert c.gauge_energy(True) == pytest.approx(float(g["su2_plaq_ss"]), rel=1e-12)
        assert rel(c.derivative(), g["su2_force"]) < 1e-12
        E, Q = c.energy_density()
        assert E == pytest.approx(float(g["su2_E"]), rel=1e-12)
        assert Q == pytest.approx(float(g["su2_Q"]), rel=1e-10, abs=1e-13)
        c.runge_kutta(0.01)
        assert rel(c.download(), g["su2_flow"]) < 1e-12
        c.upload(U)
        rows = c.gradient_flow(0.05, 0.01)
        want = g["su2_flow_rows"]
        assert rows.shape == want.shape
        np.testing.assert_allclose(rows, want, rtol=1e-5, atol=1e-7)  # printed precision


@pytest.mark.parametrize("name,integ,n", [("leapfrog", 0, 10), ("omf2", 6, 4)])
def test_su2_trajectory_injected_momenta(gpu, g, name, integ, n):
    with lattice(gpu, g["su2_dims"], 4, 2.4) as c:
        c.upload(g["su2_U"])
        r = c.md_update(integ, n, 1.0, momenta=g["su2_P"], accept_reject=False)
        assert r.dH == pytest.approx(float(g[f"su2_md_{name}_dH"]), abs=1e-9)
        assert rel(c.download(), g[f"su2_md_{name}_U"]) < 1e-12


def test_su2_d3(gpu, g):
    with lattice(gpu, g["su2d3_dims"], 3, 2.0) as c:
        c.upload(g["su2d3_U"])
        assert c.gauge_energy() == pytest.approx(float(g["su2d3_plaq"]), rel=1e-12)
        assert rel(c.derivative(), g["su2d3_force"]) < 1e-12


def test_u1_staggered(gpu, g):
    with lattice(gpu, g["u1_dims"], 2, 4.0, group="u1") as c:
        c.upload(g["u1_U"])
        assert c.gauge_energy() == pytest.approx(float(g["u1_plaq"]), rel=1e-12)
        assert rel(c.derivative(), g["u1_force"]) < 1e-12
        assert rel(c.DDdag(0.05, g["u1_psi"]), g["u1_DDdag_psi"]) < 1e-13
        r = c.solve(g["u1_psi"], 0.05, tol=1e-10, solver="CG", x0=g["u1_x0"])
        assert r.converged
        assert rel(r.x, g["u1_cg_x"]) < 1e-8
        assert abs(r.iterations - int(g["u1_cg_iter"])) <= max(2, int(g["u1_cg_iter"]) // 10)
        r = c.solve(g["u1_psi"], 0.05, tol=1e-10, solver="BiCGStab", x0=g["u1_x0"])
        assert r.converged
        assert rel(r.x, g["u1_bicgstab_x"]) < 1e-8
