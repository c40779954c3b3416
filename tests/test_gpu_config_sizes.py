"""Parity at the workloads' full sizes, through the C ABI.

The device path is compared directly with the reference's own results at the sizes the
workloads run (tests/golden/config_sizes.npz, digests made by make_config_sizes.py from the
su2 headers), and with the oracle where the reference has no counterpart (the Philox
checkerboard Metropolis sweep):
  U(1) d=2 256x256, staggered m = 0.05: D D^+ (staggered.hpp:290-389) to 1e-12; CG on D D^+
    (CG.hpp:36-94) to |r| < 1e-10 |b| in FP64 and with FP32 inner iterations, and BiCGStab
    on D (BiCGStab.hpp:36-106): true residual, iterations, solution.
  SU(2) d=4 24^4: the action's backward against the reference's gauge derivative
    (flat-gaugemonomial.hh:105-131) to 1e-12 and against central finite differences.
  SU(2) d=4 32^4: one RK3 flow step (flat-gradient_flow.hh:17-50) to 1e-12; the omf2 tau 1
    n 16 trajectory with injected momenta (md_update.hh:18-81): Delta H to 1e-9 of the
    largest H term, the links to 1e-10; one Metropolis sweep (delta 0.15, 8 hits) against the
    oracle's replay of the device's random streams; the mixed-precision trajectory against
    the reference's FP64 one, with its error stated in the assertion bounds.
"""
import os
import sys

import numpy as np
import pytest

from helpers import rel

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from digest import check  # noqa: E402
from make_config_sizes import SU2_24, SU2_32, U1_DIMS, inputs  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(HERE, "golden", "config_sizes.npz"))


@pytest.fixture(scope="module")
def inp(orc):
    return inputs(orc)


def u1_ctx(gpu, precision="fp64"):
    Lx, Ly, Lz, Lt = U1_DIMS
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, 2, 4.0, group="u1", precision=precision)


def test_u1_256_staggered_operator(gpu, fx, inp):
    with u1_ctx(gpu) as c:
        c.upload(inp["u1_U"])
        check(c.DDdag(0.05, inp["u1_b"]), fx, "u1_DDdag_b", 1e-12)


def test_u1_256_cg(gpu, fx, inp):
    b = inp["u1_b"]
    with u1_ctx(gpu) as c:
        c.upload(inp["u1_U"])
        r = c.solve(b, 0.05, tol=1e-10, tol_mode="rel", solver="CG")
    assert r.converged and r.true_residual <= 1e-10 * np.linalg.norm(b)
    it_ref = int(fx["u1_cg_iter"])
    assert abs(r.iterations - it_ref) <= max(2, it_ref // 50)
    check(r.x, fx, "u1_cg_x", 1e-8)


def test_u1_256_mixed_cg(gpu, fx, inp):
    """FP32 inner iterations with FP64 reliable updates reach the same relative 1e-10 true
    residual and the reference's FP64 solution within the system's conditioning."""
    b = inp["u1_b"]
    with u1_ctx(gpu, "mixed") as c:
        c.upload(inp["u1_U"])
        r = c.solve(b, 0.05, tol=1e-10, tol_mode="rel", solver="CG_mixed")
    assert r.converged and r.restarts >= 1
    assert r.true_residual <= 1e-10 * np.linalg.norm(b)
    check(r.x, fx, "u1_cg_x", 1e-7)


def test_u1_256_bicgstab(gpu, fx, inp):
    b = inp["u1_b"]
    with u1_ctx(gpu) as c:
        c.upload(inp["u1_U"])
        r = c.solve(b, 0.05, tol=1e-10, tol_mode="rel", solver="BiCGStab")
    assert r.converged and r.true_residual <= 1e-10 * np.linalg.norm(b)
    it_ref = int(fx["u1_bicgstab_iter"])
    assert abs(r.iterations - it_ref) <= max(3, it_ref // 10)
    check(r.x, fx, "u1_bicgstab_x", 1e-7)


def test_su2_24_action_backward(gpu, orc, fx, inp):
    """S and dS/dU (the gauge force with fac = 1) against the reference at 24^4, against the
    oracle's force, and against central finite differences of S (eps 1e-6) on seeded links
    and directions (the bound 1e-3 covers the O(eps^2) truncation and the FP64 rounding of
    the action differences)."""
    U = inp["su2_24_U"]
    with gpu.gaugeconfig(*SU2_24, 4, 2.4) as c:
        c.upload(U)
        S, dS = c.action_backward()
        assert S == pytest.approx(float(fx["su2_24_S"]), rel=1e-12)
        check(dS, fx, "su2_24_force", 1e-12)
        assert rel(dS, orc.gauge_derivative(0, SU2_24, 4, 2.4, U)) < 1e-12
        rng = np.random.default_rng(24)
        links = rng.choice(U.size // 4, size=16, replace=False)
        comps = rng.integers(0, 3, size=16)
        eps = 1e-6
        V_ = U.copy()
        for lk, k in zip(links, comps):
            vals = []
            for sgn in (1.0, -1.0):
                x = np.zeros(3)
                x[k] = sgn * eps
                e = orc.exp_su2(x)  # exp_gauge.cc:8-18
                q = U[4 * lk:4 * lk + 4]
                a = complex(e[0], e[1]) * complex(q[0], q[1]) - \
                    complex(e[2], e[3]) * complex(q[2], -q[3])
                bb = complex(e[0], e[1]) * complex(q[2], q[3]) + \
                    complex(e[2], e[3]) * complex(q[0], -q[1])
                V_[4 * lk:4 * lk + 4] = [a.real, a.imag, bb.real, bb.imag]
                c.upload(V_)
                vals.append(c.get_S_G_hmc())
            V_[4 * lk:4 * lk + 4] = U[4 * lk:4 * lk + 4]
            fd = (vals[0] - vals[1]) / (2 * eps)
            assert abs(fd - dS[3 * lk + k]) <= 1e-3 * max(1.0, abs(dS[3 * lk + k]))


def test_su2_32_flow_step(gpu, fx, inp):
    with gpu.gaugeconfig(*SU2_32, 4, 2.4) as c:
        c.upload(inp["su2_32_U"])
        c.runge_kutta(0.01)
        check(c.download(), fx, "su2_32_flow", 1e-12)


def test_su2_32_trajectory(gpu, fx, inp):
    """The workload's trajectory (omf2, tau 1, n 16, beta 2.4) with the momenta injected,
    against the reference's md_update: Delta H to 1e-9 of the largest H term (|H| ~ 1e7
    here, so 1e-2 absolute), the H terms, the final links."""
    H = fx["su2_32_md_H"]
    hmax = float(np.max(np.abs(H)))
    with gpu.gaugeconfig(*SU2_32, 4, 2.4) as c:
        c.upload(inp["su2_32_U"])
        assert c.gauge_energy() / (32 ** 4 * 6 * 2) == pytest.approx(float(fx["su2_32_plaq"]),
                                                                       rel=1e-12)
        r = c.md_update("omf2", 16, 1.0, momenta=inp["su2_32_P"], accept_reject=False)
        assert r.accepted
        assert r.dH == pytest.approx(float(fx["su2_32_md_dH"]), abs=1e-9 * hmax)
        assert r.H_old[0] == pytest.approx(H[0], rel=1e-12)
        assert r.H_old[1] == pytest.approx(H[1], rel=1e-12)
        assert r.H_new[0] == pytest.approx(H[2], rel=1e-10)
        assert r.H_new[1] == pytest.approx(H[3], rel=1e-10)
        check(c.download(), fx, "su2_32_md_U", 1e-10)


def test_su2_32_trajectory_mixed_precision(gpu, fx, inp):
    """The same trajectory with FP32 links, momenta and forces (FP64 sums, accept and
    reunitarisation) against the reference's FP64 result.  The bounds are the stated FP32
    error of this workload: Delta H within 0.05 absolute (H_kin = 6.3e6 and S_G = -9.6e6,
    Delta H = 433 here), the links within 1e-5."""
    with gpu.gaugeconfig(*SU2_32, 4, 2.4, precision="mixed") as c:
        c.upload(inp["su2_32_U"])
        r = c.md_update("omf2", 16, 1.0, momenta=inp["su2_32_P"], accept_reject=False)
        assert r.dH == pytest.approx(float(fx["su2_32_md_dH"]), abs=5e-2)
        check(c.download(), fx, "su2_32_md_U", 1e-5)


def test_su2_32_metropolis_sweep(gpu, orc, inp):
    """One checkerboard sweep (delta 0.15, 8 hits, the workload's Metropolis) on the 32^4
    field against the oracle's replay of the device's Philox streams and order."""
    U = inp["su2_32_U"]
    with gpu.gaugeconfig(*SU2_32, 4, 2.4) as c:
        c.upload(U)
        rates = c.sweep(0.15, 8, 9, 0)
        got = c.download()
    want, rates_o = orc.metropolis_checkerboard(0, SU2_32, 4, 2.4, 0.15, 8, 9, 0, U)
    assert rel(got, want) < 1e-11
    assert np.allclose(rates, rates_o, rtol=1e-12)
