"""Parity of the U(1) staggered-fermion path of libsu2b (through the C ABI) against the oracle.

Tolerances: operator applications 1e-13 relative; Krylov solutions against the oracle's
solution of the same system within 1e-8 relative (both solves stop at the same absolute
residual, 1e-12, so they differ by rounding only); fermion force 1e-8 relative.
"""
import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu

U1_GEOMS = [((8, 1, 1, 6), 2), ((4, 4, 4, 4), 4), ((6, 4, 1, 4), 3)]
IDS = ["8x6-d2", "4^4-d4", "6x4x4-d3"]


def u1(gpu, dims, nd, beta=4.0, precision="fp64"):
    Lx, Ly, Lz, Lt = dims
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, beta, group="u1", precision=precision)


def setup(orc, dims, nd, seed=42):
    U = orc.hotstart(1, dims, nd, seed, 1.0, 654321)
    V = dims[0] * dims[1] * dims[2] * dims[3]
    rng = np.random.default_rng(seed)
    return U, rng.normal(size=2 * V), V


@pytest.mark.parametrize("dims,nd", U1_GEOMS, ids=IDS)
def test_operator(gpu, orc, dims, nd):
    U, psi, _ = setup(orc, dims, nd)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        for op, f in ((0, c.apply_D), (1, c.apply_Ddag), (2, c.DDdag)):
            assert rel(f(0.05, psi), orc.staggered_apply(dims, nd, U, 0.05, op, psi)) < 1e-13


def test_eta_known_values(orc):
    # staggered.hpp:41-48
    assert orc.eta(0, 1, 1, 0, 2) == -1.0
    assert orc.eta(1, 1, 1, 1, 3) == -1.0
    assert orc.eta(5, 0, 0, 0, 0) == 1.0


@pytest.mark.parametrize("dims,nd", U1_GEOMS, ids=IDS)
def test_cg(gpu, orc, dims, nd):
    U, b, V = setup(orc, dims, nd)
    x0 = np.random.default_rng(1).normal(size=2 * V)
    xo, it_o = orc.cg_ddag(dims, nd, U, 0.1, b, x0, 1e-12)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        r = c.solve(b, 0.1, tol=1e-12, solver="CG", x0=x0)
    assert r.converged and r.true_residual <= 1e-12
    assert rel(r.x, xo) < 1e-8
    assert abs(r.iterations - it_o) <= max(2, it_o // 20)


@pytest.mark.parametrize("dims,nd", U1_GEOMS, ids=IDS)
def test_bicgstab(gpu, orc, dims, nd):
    U, b, V = setup(orc, dims, nd)
    x0 = np.zeros(2 * V)
    xo, _ = orc.bicgstab_d(dims, nd, U, 0.1, b, x0, 1e-12)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        r = c.solve(b, 0.1, tol=1e-12, solver="BiCGStab")
    assert r.converged and r.true_residual <= 1e-12
    assert rel(r.x, xo) < 1e-8


@pytest.mark.parametrize("dims,nd", U1_GEOMS, ids=IDS)
def test_mixed_cg(gpu, orc, dims, nd):
    U, b, V = setup(orc, dims, nd)
    with u1(gpu, dims, nd, precision="mixed") as c:
        c.upload(U)
        r = c.solve(b, 0.1, tol=1e-10, tol_mode="rel", solver="CG_mixed")
        r64 = c.solve(b, 0.1, tol=1e-10, tol_mode="rel", solver="CG")
    assert r.converged and r.restarts >= 1
    assert r.true_residual <= 1e-10 * np.linalg.norm(b)
    assert rel(r.x, r64.x) < 1e-7


def test_solver_iteration_limit(gpu, orc):
    dims, nd = (8, 1, 1, 6), 2
    U, b, _ = setup(orc, dims, nd)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        r = c.solve(b, 0.01, tol=1e-14, solver="CG", max_iter=3)
    assert not r.converged and r.iterations == 3


@pytest.mark.parametrize("dims,nd", U1_GEOMS, ids=IDS)
def test_fermion_monomial(gpu, orc, dims, nd):
    U, _, V = setup(orc, dims, nd)
    phi, h = orc.fermion_heatbath(dims, nd, U, 0.1, 97234719)
    want_F = orc.fermion_derivative(dims, nd, U, 0.1, phi, 1e-12, 97234719)
    want_S = orc.fermion_accept(dims, nd, U, 0.1, phi, 1e-12, 97234719)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        F, it = c.fermion_derivative(0.1, phi, tol=1e-12, seed=97234719)
        S = c.fermion_action(0.1, phi, tol=1e-12, seed=97234719)
    assert rel(F, want_F) < 1e-8
    assert S == pytest.approx(want_S, rel=1e-10)


@pytest.mark.parametrize("dims,nd", U1_GEOMS[:2], ids=IDS[:2])
def test_fermion_hmc_trajectory(gpu, orc, dims, nd):
    U, _, V = setup(orc, dims, nd)
    P, _ = orc.initnormal(1, dims, nd, 3)
    R = orc.gaussian_spinor(dims, 0.0, 2 ** -0.5, 11)
    dH, U_want, _, H = orc.md_injected_fermion(dims, nd, 4.0, 0.1, 1e-12, 97234719, 6, 4, 0.5,
                                               U, P, R)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        r = c.md_update("omf2", 4, 0.5, momenta=P, pf_source=R, fermion_mass=0.1, cg_tol=1e-12,
                        accept_reject=False, pf_seed=97234719)
        assert rel(c.download(), U_want) < 1e-9
    assert r.H_old[2] == pytest.approx(H[2], rel=1e-12)
    assert r.H_new[2] == pytest.approx(H[5], rel=1e-9)
    assert r.dH == pytest.approx(dH, abs=1e-7)
    assert r.cg_iterations > 0


@pytest.mark.parametrize("exponent", [6, 12])
def test_fermion_trajectory_low_precision_leapfrog(gpu, orc, exponent):
    """lp_leapfrog with the det(D D^+) monomial: each momentum step rounds the summed gauge +
    fermion derivative (round_and_update_momenta, update_momenta.hh:36-58) and each gauge step
    the link angles (update_gauge.hh:20-26), against the oracle (pinned to the reference's
    own integrator with fermions).  The fermion derivative shares the scratch field of the
    gauge derivative, which this covers."""
    dims, nd = U1_GEOMS[0]
    U, _, V = setup(orc, dims, nd)
    P, _ = orc.initnormal(1, dims, nd, 3)
    R = orc.gaussian_spinor(dims, 0.0, 2 ** -0.5, 11)
    dH, U_want, _, H = orc.md_injected_fermion(dims, nd, 4.0, 0.1, 1e-12, 97234719, 1, 4, 0.5,
                                               U, P, R, exponent=exponent)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        r = c.md_update("lp_leapfrog", 4, 0.5, momenta=P, pf_source=R, fermion_mass=0.1,
                        cg_tol=1e-12, accept_reject=False, pf_seed=97234719, exponent=exponent)
        assert rel(c.download(), U_want) < 1e-9
    assert r.H_old[2] == pytest.approx(H[2], rel=1e-12)
    assert r.H_new[2] == pytest.approx(H[5], rel=1e-9)
    assert r.dH == pytest.approx(dH, abs=1e-7)


def test_pf_source_stream(orc):
    R = orc.philox_pf_source((16, 1, 1, 16), 5, 0)
    assert np.all(R[1::2] == 0.0)
    assert abs(R[0::2].var() - 0.5) < 0.1


@pytest.mark.parametrize("dims,nd", U1_GEOMS, ids=IDS)
def test_pion_correlator(gpu, orc, dims, nd):
    """C_pion (propagator.hpp:25-65) on the device against the oracle: same CG start, both
    solves stop at |r| < 1e-12, so the correlators agree to the solver tolerance."""
    U, _, _ = setup(orc, dims, nd)
    want = orc.pion_correlator(dims, nd, U, 0.1, 1e-12, 17)
    with u1(gpu, dims, nd) as c:
        c.upload(U)
        got = c.C_pion(0.1, tol=1e-12, seed=17)
    assert got[0] == 0.0
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-14)


def test_pion_correlator_rejects_su2(gpu):
    import su2_b200
    with gpu.gaugeconfig(4, 4, 4, 4, 4, 2.0) as c:
        with pytest.raises(su2_b200.Su2bError) as e:
            c.C_pion(0.1)
        assert e.value.code == 4


def test_operator_and_solve_at_1024_squared(gpu):
    """U(1) d = 2 at 1024^2 (1 M sites, 16 times the workload's volume), through properties
    that hold at any size: a shift by two sites in t and x keeps every staggered phase and
    parity, so D, D^+ and D D^+ of the shifted field and vector are the shifted results bit
    for bit, and the CG solution of the shifted system is the shifted solution (to the
    solver's tolerance: its sums add in another order)."""
    L = 1024
    rng = np.random.default_rng(77)
    U = rng.uniform(-np.pi, np.pi, size=L * L * 2)
    psi = rng.normal(size=2 * L * L)

    def shift(a, comps):
        return np.roll(a.reshape(L, L, comps), (2, 2), axis=(0, 1)).reshape(-1)

    with u1(gpu, (L, 1, 1, L), 2) as c:
        out = {}
        for key, (Ui, pi) in (("plain", (U, psi)), ("shifted", (shift(U, 2), shift(psi, 2)))):
            c.upload(Ui)
            r = c.solve(pi, 0.05, tol=1e-10, tol_mode="rel")
            assert r.converged
            out[key] = [c.apply_D(0.05, pi), c.apply_Ddag(0.05, pi), c.DDdag(0.05, pi), r.x]
        for k in range(3):
            assert np.array_equal(shift(out["plain"][k], 2), out["shifted"][k])
        assert rel(out["shifted"][3], shift(out["plain"][3], 2)) < 1e-8
