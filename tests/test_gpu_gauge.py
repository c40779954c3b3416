"""Parity of the gauge-field path of libsu2b (through the C ABI) against the oracle.

Tolerances: FP64 results within 1e-12 relative (norm-wise for fields), FP64 sums within
1e-12 relative; mixed precision (FP32 links and forces) within 1e-5 relative.
"""
import numpy as np
import pytest

from helpers import GEOM_IDS, GEOMS, group_name, rel

pytestmark = pytest.mark.gpu

SEED, TRAFO = 13526463, 654321


def make(gpu, group, dims, nd, beta=2.3, xi=1.0, precision="fp64"):
    Lx, Ly, Lz, Lt = dims
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, beta, group=group_name(group), xi=xi,
                           precision=precision)


def hot(orc, group, dims, nd, seed=SEED):
    return orc.hotstart(group, dims, nd, seed, 1.0, TRAFO)


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
def test_upload_download_roundtrip(gpu, orc, group, dims, nd):
    U = hot(orc, group, dims, nd)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        assert np.array_equal(c.download(), U)
    if group == 0:
        with make(gpu, group, dims, nd, precision="mixed") as c:
            c.upload(U)
            assert np.array_equal(c.download(), U.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
def test_plaquette_and_action(gpu, orc, group, dims, nd):
    U = hot(orc, group, dims, nd)
    for xi in (1.0, 1.3):
        with make(gpu, group, dims, nd, beta=2.3, xi=xi) as c:
            c.upload(U)
            e = orc.gauge_energy(group, dims, nd, U)
            assert c.gauge_energy() == pytest.approx(e, rel=1e-12, abs=1e-12)
            ess = orc.gauge_energy(group, dims, nd, U, spatial_only=True)
            assert c.gauge_energy(True) == pytest.approx(ess, rel=1e-12, abs=1e-12)
            w = orc.retr_sum_plaquettes(group, dims, nd, U, xi, xi != 1.0)
            assert c.retr_sum_Wplaquettes() == pytest.approx(w, rel=1e-12, abs=1e-12)
            s = orc.S_G_hmc(group, dims, nd, 2.3, U, xi, xi != 1.0)
            assert c.get_S_G_hmc() == pytest.approx(s, rel=1e-12, abs=1e-12)


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
@pytest.mark.parametrize("xi", [1.0, 0.8])
def test_gauge_force(gpu, orc, group, dims, nd, xi):
    U = hot(orc, group, dims, nd)
    ref = orc.gauge_derivative(group, dims, nd, 2.3, U, xi, 0.7)
    with make(gpu, group, dims, nd, beta=2.3, xi=xi) as c:
        c.upload(U)
        assert rel(c.derivative(0.7), ref) < 1e-12
    if group == 0:
        with make(gpu, group, dims, nd, beta=2.3, xi=xi, precision="mixed") as c:
            c.upload(U)
            assert rel(c.derivative(0.7), ref) < 1e-5


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
def test_update_and_restore(gpu, orc, group, dims, nd):
    U = hot(orc, group, dims, nd)
    P, _ = orc.initnormal(group, dims, nd, 99)
    want = orc.restore_su(group, dims, nd, orc.update_gauge(group, dims, nd, U, P, 0.137))
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        c.update_gauge(P, 0.137)
        c.restoreSU()
        assert rel(c.download(), want) < 1e-13


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
def test_energy_density(gpu, orc, group, dims, nd):
    U = hot(orc, group, dims, nd)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        for cl in (True, False):
            for ss in (False, True):
                E, Q = c.energy_density(cl, ss)
                Eo, Qo = orc.energy_density(group, dims, nd, U, cl, ss)
                assert E == pytest.approx(Eo, rel=1e-12, abs=1e-13)
                assert Q == pytest.approx(Qo, rel=1e-11, abs=1e-13)


def test_topological_charge_known_answer(gpu):
    """test.cc:81-105: a hand-built U(1) 4^4 configuration has Q = 0.0126651."""
    import math
    U = np.zeros(4 ** 4 * 4)

    def idx(t, x, y, z, mu):
        return (((t * 4 + x) * 4 + y) * 4 + z) * 4 + mu

    U[idx(1, 1, 1, 1, 0)] = 0
    U[idx(1, 1, 1, 1, 1)] = math.pi / 2
    U[idx(1, 1, 1, 1, 2)] = math.pi / 2
    U[idx(1, 1, 1, 1, 3)] = 0
    U[idx(0, 1, 1, 1, 0)] = math.pi
    U[idx(1, 0, 1, 1, 1)] = math.pi / 2
    U[idx(1, 1, 0, 0, 2)] = math.pi
    U[idx(1, 1, 1, 0, 3)] = math.pi / 2
    with gpu.gaugeconfig(4, 4, 4, 4, 4, 1.0, group="u1") as c:
        c.upload(U)
        _, Q = c.energy_density()
    assert Q == pytest.approx(0.0126651, abs=5e-8)


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
def test_flow_step(gpu, orc, group, dims, nd):
    U = hot(orc, group, dims, nd)
    want = orc.runge_kutta(group, dims, nd, 2.3, 0.01, U)
    with make(gpu, group, dims, nd, beta=2.3) as c:
        c.upload(U)
        c.runge_kutta(0.01)
        assert rel(c.download(), want) < 1e-12
    if group == 0:
        with make(gpu, group, dims, nd, beta=2.3, precision="mixed") as c:
            c.upload(U)
            c.runge_kutta(0.01)
            assert rel(c.download(), want) < 1e-5


@pytest.mark.parametrize("group,dims,nd", [GEOMS[0], GEOMS[3], GEOMS[4]],
                         ids=[GEOM_IDS[0], GEOM_IDS[3], GEOM_IDS[4]])
def test_gradient_flow_records(gpu, orc, group, dims, nd):
    U = hot(orc, group, dims, nd)
    want = orc.gradient_flow_rows(group, dims, nd, 2.3, U, 0.2, 0.01)
    with make(gpu, group, dims, nd, beta=2.3) as c:
        c.upload(U)
        got = c.gradient_flow(0.2, 0.01)
        assert np.array_equal(c.download(), U)  # the flow works on a copy
    assert got.shape == want.shape
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(got))
    np.testing.assert_allclose(got[fin], want[fin], rtol=1e-11, atol=1e-13)
    if group == 0:  # FP32 links: the step pairs between two buffers, reunitarised each step
        with make(gpu, group, dims, nd, beta=2.3, precision="mixed") as c:
            c.upload(U)
            got32 = c.gradient_flow(0.2, 0.01)
        # columns t, xi_R, P, P_ss, E_p, E_p_ss, E_c, E_c_ss, Q: FP32 link rounding only
        cols = [0, 2, 3, 4, 5, 6, 7]
        np.testing.assert_allclose(got32[:, cols], want[:, cols], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
@pytest.mark.parametrize("integ", [0, 6, 2, 4, 5])
def test_md_trajectory_injected_momenta(gpu, orc, group, dims, nd, integ):
    U = hot(orc, group, dims, nd)
    P, _ = orc.initnormal(group, dims, nd, 4242)
    dH, U_want, _, H = orc.md_injected(group, dims, nd, 2.3, integ, 6, 1.0, U, P)
    with make(gpu, group, dims, nd, beta=2.3) as c:
        c.upload(U)
        r = c.md_update(integ, 6, 1.0, momenta=P, accept_reject=False)
        assert r.accepted
        assert r.dH == pytest.approx(dH, abs=1e-9 * max(1.0, abs(H[1])))
        assert r.H_old[0] == pytest.approx(H[0], rel=1e-13)
        assert r.H_new[1] == pytest.approx(H[3], rel=1e-12)
        assert rel(c.download(), U_want) < 1e-10


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
@pytest.mark.parametrize("integ,exponent", [(1, 16), (1, 6), (3, 8)],
                         ids=["lp_leapfrog-e16", "lp_leapfrog-e6", "lp_omf4-e8"])
def test_md_trajectory_low_precision_integrators(gpu, orc, group, dims, nd, integ, exponent):
    """lp_leapfrog / lp_omf4 (integrator.hh:53-80, 158-199): the derivative rounded to
    10^-e before each momentum step and the links before each gauge step, against the
    oracle (pinned bit for bit to the reference's integrators)."""
    U = hot(orc, group, dims, nd)
    P, _ = orc.initnormal(group, dims, nd, 4242)
    dH, U_want, _, H = orc.md_injected(group, dims, nd, 2.3, integ, 6, 1.0, U, P,
                                       exponent=exponent)
    with make(gpu, group, dims, nd, beta=2.3) as c:
        c.upload(U)
        r = c.md_update(integ, 6, 1.0, momenta=P, accept_reject=False, exponent=exponent)
        assert r.accepted
        assert r.dH == pytest.approx(dH, abs=1e-9 * max(1.0, abs(H[1])))
        assert r.H_new[1] == pytest.approx(H[3], rel=1e-12)
        assert rel(c.download(), U_want) < 1e-10


def test_reference_chain_replay(gpu, orc):
    """Replaying the reference's own random stream (std::mt19937(seed+i) momenta and accept
    uniform), the device chain takes the same accept decisions with the same Delta H as the
    reference's md_update (hmc.hpp:86-101) -- config: SU(2) 8^4, beta = 2.3, omf2 tau=1."""
    group, dims, nd = 0, (8, 8, 8, 8), 4
    U0 = hot(orc, group, dims, nd)
    n = 6
    U_ref, acc, dH, plaq = orc.hmc_run(group, dims, nd, 2.3, 6, 10, 1.0, 13526463, 0, n, U0)
    with make(gpu, group, dims, nd, beta=2.3) as c:
        c.upload(U0)
        for i in range(n):
            P, u = orc.initnormal(group, dims, nd, 13526463 + i)
            r = c.md_update("omf2", 10, 1.0, momenta=P, uniform=u)
            assert r.accepted == bool(acc[i])
            assert r.dH == pytest.approx(dH[i], abs=1e-7)
            assert r.plaquette == pytest.approx(plaq[i], rel=1e-11)
        assert rel(c.download(), U_ref) < 1e-9


@pytest.mark.parametrize("group,dims,nd", [GEOMS[0], GEOMS[2], GEOMS[4]],
                         ids=[GEOM_IDS[0], GEOM_IDS[2], GEOM_IDS[4]])
def test_device_momentum_stream(gpu, orc, group, dims, nd):
    """The device's Philox momenta equal the oracle's restatement of the same stream."""
    U = hot(orc, group, dims, nd)
    P = orc.philox_momenta(group, dims, nd, 777, 5)
    na = 3 if group == 0 else 1
    assert abs(P.mean()) < 5.0 / np.sqrt(P.size) and abs(P.var() - 1) < 10.0 / np.sqrt(P.size)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        r = c.md_update("leapfrog", 1, 1e-3, seed=777, traj=5, accept_reject=False)
    assert r.H_old[0] == pytest.approx(0.5 * float(np.sum(P * P)), rel=1e-13)
    assert P.size == c.n_links * na


def test_mixed_momenta_are_the_fp64_stream(gpu, orc):
    """FP32 storage draws the same momenta as FP64 (the same two Philox draws and 53-bit
    uniforms per link, Box-Muller in FP32 arithmetic): the kinetic energy agrees to FP32
    rounding, and a trajectory from the same start and seed lands on the FP64 one within
    FP32 accuracy, so both precisions sample the same momenta trajectory by trajectory."""
    dims, nd = (8, 8, 8, 8), 4
    U = hot(orc, 0, dims, nd)
    P = orc.philox_momenta(0, dims, nd, 777, 5)
    out = {}
    for prec in ("fp64", "mixed"):
        with gpu.gaugeconfig(*dims, nd, 2.3, precision=prec) as c:
            c.upload(U)
            r = c.md_update("omf2", 4, 0.5, seed=777, traj=5, accept_reject=False)
            out[prec] = (r, c.download())
    kin = 0.5 * float(np.sum(P * P))
    assert out["fp64"][0].H_old[0] == pytest.approx(kin, rel=1e-13)
    assert out["mixed"][0].H_old[0] == pytest.approx(kin, rel=2e-7)
    assert out["mixed"][0].dH == pytest.approx(out["fp64"][0].dH, abs=5e-3)
    assert rel(out["mixed"][1], out["fp64"][1]) < 1e-5


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
def test_metropolis_checkerboard(gpu, orc, group, dims, nd):
    """The device sweep replayed by the oracle (same Philox stream and update order), for the
    isotropic and the anisotropic action (staple weights 1/xi and xi, get_staples.hh:58-79)."""
    U = hot(orc, group, dims, nd)
    for xi in (1.0, 1.3):
        U_want, r_want = orc.metropolis_checkerboard(group, dims, nd, 2.3, 0.3, 4, 99, 3, U,
                                                     xi=xi)
        with make(gpu, group, dims, nd, beta=2.3, xi=xi) as c:
            c.upload(U)
            rates = c.sweep(0.3, 4, 99, 3)
            assert rel(c.download(), U_want) < 1e-11
        np.testing.assert_array_equal(rates, r_want)


@pytest.mark.parametrize("group,dims,nd", [g for g in GEOMS if g[0] == 0],
                         ids=[i for g, i in zip(GEOMS, GEOM_IDS) if g[0] == 0])
def test_metropolis_checkerboard_mixed_precision(gpu, orc, group, dims, nd):
    """FP32 links: the staple sum and the proposals in FP32, dS, the accept test and the
    reunitarisation in FP64, on the FP64 path's random stream -- the same accept decisions
    as the oracle's FP64 replay and the links within FP32 rounding."""
    U = hot(orc, group, dims, nd)
    Us = U.astype(np.float32).astype(np.float64)
    for xi in (1.0, 1.3):
        U_want, r_want = orc.metropolis_checkerboard(group, dims, nd, 2.3, 0.3, 4, 99, 3, Us,
                                                     xi=xi)
        with make(gpu, group, dims, nd, beta=2.3, xi=xi, precision="mixed") as c:
            c.upload(U)
            rates = c.sweep(0.3, 4, 99, 3)
            assert rel(c.download(), U_want) < 1e-5
        np.testing.assert_array_equal(rates, r_want)


@pytest.mark.parametrize("group,dims,nd", [GEOMS[0], GEOMS[4]], ids=[GEOM_IDS[0], GEOM_IDS[4]])
def test_gauge_invariance(gpu, orc, group, dims, nd):
    U = hot(orc, group, dims, nd)
    V = orc.random_gauge_trafo(group, dims, nd, U, 98765)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        p0, e0 = c.gauge_energy(), c.energy_density()
        c.upload(V)
        p1, e1 = c.gauge_energy(), c.energy_density()
    assert p1 == pytest.approx(p0, rel=1e-12)
    assert e1[0] == pytest.approx(e0[0], rel=1e-12)


def test_reversibility(gpu, orc):
    """md_update's reversibility test (md_update.hh:62-74): ddH ~ 0 and U unchanged by it."""
    group, dims, nd = 0, (6, 6, 6, 6), 4
    U = hot(orc, group, dims, nd)
    with make(gpu, group, dims, nd, beta=2.3) as c:
        c.upload(U)
        a = c.md_update("omf2", 8, 1.0, seed=5, traj=0, revtest=True, accept_reject=False)
        Ua = c.download()
        c.upload(U)
        b = c.md_update("omf2", 8, 1.0, seed=5, traj=0, revtest=False, accept_reject=False)
        assert rel(c.download(), Ua) < 1e-12
    # the reversibility test runs the unfused kernel sequence, the plain trajectory the fused
    # one: the same arithmetic up to rounding
    assert a.dH == pytest.approx(b.dH, abs=1e-9)
    assert abs(a.ddH) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_plain_trajectory_matches_fused(gpu, orc, precision):
    """The plain form (start-field copy, integrator steps launched one by one, no graph) and
    the fused graph-captured trajectory are the same discrete map: the same accept decisions,
    Delta H and links up to rounding, over a chain of Philox trajectories."""
    dims, nd = (6, 6, 6, 6), 4
    U = hot(orc, 0, dims, nd)
    out = {}
    for plain in (False, True):
        with gpu.gaugeconfig(*dims, nd, 2.3, precision=precision) as c:
            c.upload(U)
            c.plain_trajectory = plain
            assert c.plain_trajectory == plain
            res = [c.md_update("omf2", 5, 1.0, seed=41, traj=k) for k in range(5)]
            out[plain] = (res, c.download())
    tol = 1e-9 if precision == "fp64" else 1e-3
    for a, b in zip(out[False][0], out[True][0]):
        assert a.accepted == b.accepted
        assert a.dH == pytest.approx(b.dH, abs=tol)
        assert a.plaquette == pytest.approx(b.plaquette, rel=1e-12 if precision == "fp64" else 1e-6)
    assert rel(out[False][1], out[True][1]) < (1e-11 if precision == "fp64" else 1e-5)


def test_error_paths(gpu):
    import su2_b200
    with pytest.raises(su2_b200.Su2bError):
        gpu.gaugeconfig(5, 4, 4, 4, 4, 2.0)  # odd extent
    with pytest.raises(su2_b200.Su2bError):
        gpu.gaugeconfig(4, 4, 2, 4, 3, 2.0)  # inactive extent != 1
    with gpu.gaugeconfig(4, 4, 4, 4, 4, 2.0) as c:
        with pytest.raises(su2_b200.Su2bError) as e:
            c.md_update("lp_leapfrog", 4, 1.0, exponent=20)  # 10^20 overflows a size_t
        assert e.value.code == 1
        with pytest.raises(su2_b200.Su2bError) as e:
            c.md_update("leapfrog", 4, 1.0, fermion_mass=0.1)  # SU(2) fermions
        assert e.value.code == 4
        with pytest.raises(su2_b200.Su2bError) as e:
            c.apply_D(0.1, np.zeros(2 * 256))
        assert e.value.code == 4
    # the decimal rounding of lp_leapfrog / lp_omf4 is defined on FP64 storage only
    with gpu.gaugeconfig(4, 4, 4, 4, 4, 2.0, precision="mixed") as c:
        with pytest.raises(su2_b200.Su2bError) as e:
            c.md_update("lp_leapfrog", 4, 1.0, exponent=6)
        assert e.value.code == 4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_size_32_4(gpu, orc, precision):
    """At 32^4: plaquette and force against the oracle, gauge invariance, and an omf2
    trajectory whose reversibility violation is at rounding level."""
    group, dims, nd = 0, (32, 32, 32, 32), 4
    U = hot(orc, group, dims, nd, seed=4711)
    tol = 1e-12 if precision == "fp64" else 1e-5
    with make(gpu, group, dims, nd, beta=2.4, precision=precision) as c:
        c.upload(U)
        # the sums are FP64 over the stored links (FP32-rounded in mixed precision); mixed
        # precision forms each plaquette's products in FP32, about 1e-7 per plaquette, which
        # add up like a random walk over the 6.3 M plaquettes (the hot start's sum itself
        # cancels to a few thousand, so the bound is on the scale of the terms)
        Us = U if precision == "fp64" else U.astype(np.float32).astype(np.float64)
        n_plaq = 6 * 32 ** 4
        want = orc.gauge_energy(group, dims, nd, Us)
        if precision == "fp64":
            assert c.gauge_energy() == pytest.approx(want, rel=1e-12)
        else:
            assert abs(c.gauge_energy() - want) < 1e-8 * n_plaq
        F = orc.gauge_derivative(group, dims, nd, 2.4, U)
        assert rel(c.derivative(), F) < tol
        r = c.md_update("omf2", 4, 0.2, seed=11, traj=1, revtest=True, accept_reject=False)
        assert abs(r.ddH) < (1e-6 if precision == "fp64" else 5e-2)
        assert np.isfinite(r.dH)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_trajectory_graph_replay(gpu, orc, precision):
    """A chain run from the captured trajectory graph equals the same chain run with direct
    launches (profiling disables the graph) bit for bit, including accept decisions and the
    rotation of the three link buffers."""
    group, dims, nd = 0, (8, 8, 8, 8), 4
    U = hot(orc, group, dims, nd)
    runs = {}
    for mode in ("graph", "direct"):
        with make(gpu, group, dims, nd, beta=2.3, precision=precision) as c:
            c.upload(U)
            if mode == "direct":
                c.profile(True)
            out = [c.md_update("omf2", 6, 1.0, seed=3, traj=k) for k in range(7)]
            runs[mode] = (out, c.download())
    for a, b in zip(runs["graph"][0], runs["direct"][0]):
        assert (a.accepted, a.dH, a.plaquette) == (b.accepted, b.dH, b.plaquette)
    assert np.array_equal(runs["graph"][1], runs["direct"][1])
    assert 0 < sum(r.accepted for r in runs["graph"][0])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_start_plaquettes_carried_over(gpu, orc, precision):
    """Consecutive trajectories take their start plaquettes from the previous trajectory's
    sums (its end field if accepted, else its start field), also after a trajectory with
    host momenta; a chain with a read-only call between trajectories (which drops that
    carry-over) evolves the same field bit for bit, with the same accept decisions and
    energies to rounding."""
    group, dims, nd = 0, (8, 8, 8, 8), 4
    U = hot(orc, group, dims, nd)
    runs = {}
    for mode in ("chain", "interleaved"):
        with make(gpu, group, dims, nd, beta=2.3, precision=precision) as c:
            c.upload(U)
            out = []
            for k in range(12):
                # uniform 1e-300 accepts; 0.999999 rejects whenever dH > 1e-6; trajectory 6
                # takes host momenta (its start sums come from the separate plaquette pass)
                u = 1e-300 if k % 3 == 0 else 0.999999
                mom = orc.initnormal(group, dims, nd, 77)[0] if k == 6 else None
                out.append(c.md_update("omf2", 3, 1.0, seed=5, traj=k, uniform=u, momenta=mom))
                if mode == "interleaved":
                    c.gauge_energy()
            runs[mode] = (out, c.download())
    chain, inter = runs["chain"][0], runs["interleaved"][0]
    for a, b in zip(chain, inter):
        assert a.accepted == b.accepted
        assert a.dH == pytest.approx(b.dH, abs=1e-9)
        assert a.plaquette == pytest.approx(b.plaquette, rel=1e-13)
    assert np.array_equal(runs["chain"][1], runs["interleaved"][1])
    acc = [r.accepted for r in chain]
    assert any(acc) and not all(acc)
    # the carried-over start energy is the previous trajectory's end or start energy exactly
    for k, (a, b) in enumerate(zip(chain, chain[1:])):
        if k + 1 == 6:  # summed afresh by the host-momenta path
            assert b.H_old[1] == pytest.approx(a.H_new[1] if a.accepted else a.H_old[1],
                                               rel=1e-13)
        else:
            assert b.H_old[1] == (a.H_new[1] if a.accepted else a.H_old[1])


def test_rejected_trajectory_keeps_start_field(gpu, orc):
    group, dims, nd = 0, (6, 6, 6, 6), 4
    U = hot(orc, group, dims, nd)
    with make(gpu, group, dims, nd, beta=2.3) as c:
        c.upload(U)
        p0 = c.gauge_energy()
        for k in range(4):
            r = c.md_update("leapfrog", 2, 2.0, seed=1, traj=k, uniform=0.999999)
            if r.dH > 1e-5:
                assert not r.accepted
                assert np.array_equal(c.download(), U)
                assert r.plaquette == pytest.approx(p0, rel=1e-14)
            else:
                assert r.accepted
                U = c.download()
                p0 = c.gauge_energy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dims", [(8, 6, 4, 8), (4, 4, 8, 4), (8, 8, 16, 6), (6, 6, 6, 6)],
                         ids=["8x6x4x8", "4x4x8x4", "8x8x16x6", "6x6x6x6"])
def test_every_force_launch_shape_is_exact(gpu, orc, precision, dims):
    """Every launch shape of the force kernel (threads per block x register cap, including
    the register-starved ones that spill) gives the oracle's force and a finite trajectory,
    on lattices whose half volume is and is not a multiple of the block's sites (6^4: 648
    sites per parity, not a multiple of 32)."""
    group, nd = 0, 4
    U = hot(orc, group, dims, nd)
    F = orc.gauge_derivative(group, dims, nd, 2.3, U)
    tol = 1e-12 if precision == "fp64" else 1e-5
    with make(gpu, group, dims, nd, beta=2.3, precision=precision) as c:
        c.upload(U)
        for v in range(gpu._abi.FORCE_VARIANTS):
            c.force_variant = v
            assert rel(c.derivative(), F) < tol, v
            r = c.md_update("omf2", 3, 0.3, momenta=orc.initnormal(group, dims, nd, 5)[0],
                            accept_reject=False)
            assert np.isfinite(r.dH)
            c.upload(U)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dims,nd", [((6, 1, 1, 4), 2), ((4, 6, 1, 4), 3), ((6, 4, 1, 6), 3)],
                         ids=["6x4-d2", "4x6x4-d3", "6x4x6-d3"])
def test_every_force_launch_shape_below_four_dims(gpu, orc, precision, dims, nd):
    """d = 2 and 3: every launch shape, including the one-thread-per-link kernel and the
    two-threads-per-site shapes (which fall back to a site shape below d = 4), gives the
    oracle's force and a finite trajectory."""
    group = 0
    U = hot(orc, group, dims, nd)
    F = orc.gauge_derivative(group, dims, nd, 2.3, U)
    tol = 1e-12 if precision == "fp64" else 1e-5
    with make(gpu, group, dims, nd, beta=2.3, precision=precision) as c:
        c.upload(U)
        for v in range(gpu._abi.FORCE_VARIANTS):
            c.force_variant = v
            assert rel(c.derivative(), F) < tol, v
            r = c.md_update("omf2", 3, 0.3, momenta=orc.initnormal(group, dims, nd, 5)[0],
                            accept_reject=False)
            assert np.isfinite(r.dH)
            c.upload(U)


def test_autotune_cache(gpu, orc, tmp_path):
    group, dims, nd = 0, (16, 16, 16, 16), 4
    U = hot(orc, group, dims, nd)
    path = str(tmp_path / "tune.txt")
    with make(gpu, group, dims, nd, beta=2.4, precision="mixed") as c:
        c.upload(U)
        t = c.autotune(path)
        assert all(v > 0 for v in t.values())
        # the first shape within 1 % of the fastest
        fastest = min(t.values())
        best = min(v for v in t if t[v] <= 1.01 * fastest)
        assert c.force_variant == best
    line = open(path).read().split()
    assert int(line[1]) == best and "/force/fp32/16x16x16x16/d4" in line[0]
    with make(gpu, group, dims, nd, beta=2.4, precision="mixed") as c:
        c.force_variant = (best + 1) % gpu._abi.FORCE_VARIANTS
        t2 = c.autotune(path)  # cached: no measurement
        assert all(v < 0 for v in t2.values()) and c.force_variant == best


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (4, 6, 8, 12), (6, 6, 6, 4), (4, 4, 6, 6)],
                         ids=["8^4", "4x6x8x12", "6^3x4", "4x4x6x6-no-pairs"])
def test_site_pairs_equal_the_link_kernel(gpu, orc, dims):
    """The trajectory on site pairs (force shape 11: the field copied into the paired layout,
    packed FP32 FFMA2 on both sites of a pair, the final field written back) gives the
    one-thread-per-link kernel's links bit for bit, and its accept decisions; the energies
    agree to the rounding of the kinetic sum's order.  With T not a multiple of 4 shape 11
    runs the one-thread-per-link kernel itself."""
    group, nd = 0, 4
    U = hot(orc, group, dims, nd)
    with make(gpu, group, dims, nd, beta=2.3, precision="mixed") as a, \
            make(gpu, group, dims, nd, beta=2.3, precision="mixed") as b:
        a.force_variant = 9
        b.force_variant = 11
        a.upload(U)
        b.upload(U)
        for k in range(6):
            kw = dict(seed=4, traj=k, accept_reject=k % 2 == 1, uniform=0.999999)
            n, tau = (3, 1.0) if k % 2 == 0 else (1, 2.0)
            ra = a.md_update("omf2", n, tau, **kw)
            rb = b.md_update("omf2", n, tau, **kw)
            assert ra.accepted == rb.accepted, k
            scale = sum(abs(h) for h in ra.H_old + ra.H_new)
            assert ra.dH == pytest.approx(rb.dH, abs=1e-13 * scale + 1e-9), k
            assert np.array_equal(a.download(), b.download()), k


def test_large_lattice_64_4(gpu):
    """At 64^4 (16.8 M sites, 2.1 GB of FP64 links per buffer), through properties that hold
    at any size: the force and one Wilson-flow step of a field shifted by one site in t and
    in z are those of the field shifted the same way, bit for bit (every site's arithmetic
    moves to a thread of the other parity and another block, across every periodic
    boundary); the plaquette sum and the clover energy density are unchanged; an omf2
    trajectory is reversible to rounding; and mixed precision follows FP64 on the same
    Philox momenta."""
    L, nd = 64, 4
    rng = np.random.default_rng(2024)
    q = rng.standard_normal((L ** 4 * nd, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    U = q.reshape(-1)
    del q
    shape = (L, L, L, L, nd)  # host order: t, x, y, z, direction

    def shift(a, comps):
        return np.roll(np.roll(a.reshape(shape + (comps,)), 1, axis=0), 1, axis=3).reshape(-1)

    Ush = shift(U, 4)
    dH = {}
    for precision in ("fp64", "mixed"):
        with make(gpu, 0, (L, L, L, L), nd, beta=2.4, precision=precision) as c:
            c.upload(U)
            d1, e1, q1 = c.derivative(), c.gauge_energy(), c.energy_density()
            c.runge_kutta(0.01)
            f1 = c.download()
            c.upload(Ush)
            d2, e2, q2 = c.derivative(), c.gauge_energy(), c.energy_density()
            c.runge_kutta(0.01)
            f2 = c.download()
            assert np.array_equal(shift(d1, 3), d2)
            assert np.array_equal(shift(f1, 4), f2)  # one Wilson-flow step
            assert e2 == pytest.approx(e1, rel=1e-12)
            assert q2[0] == pytest.approx(q1[0], rel=1e-12)  # clover energy density
            c.upload(U)
            r = c.md_update("omf2", 4, 0.2, seed=11, traj=1, revtest=True, accept_reject=False)
            assert abs(r.ddH) < (1e-6 if precision == "fp64" else 5e-2)
            dH[precision] = r.dH
    # a hot start far from equilibrium: dH of about -1.9e4, FP32 arithmetic within 1e-5 of it
    assert dH["mixed"] == pytest.approx(dH["fp64"], rel=1e-5)
