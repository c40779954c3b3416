"""Pins the C restatement (oracle/su2_oracle.c) against the reference.

- bit-for-bit (or reduction-order-level) agreement with the reference's own headers compiled
  into oracle/_ref (where the reference checkout exists);
- the known answers printed by the reference's test programs (test.cc, test/CG.cpp,
  test/BiCGStab.cpp) and the Philox4x32-10 known-answer vectors of its authors;
- the committed golden fixtures (tests/golden), generated from the reference harness.
"""
import math
import os

import numpy as np
import pytest

from helpers import GEOM_IDS, GEOMS, rel

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


# ---------------------------------------------------------------- known answers
def test_su2_product_known_answer():
    """test.cc:36-43: U1 = (0.8+0.3i, 0.1+0.4i), U2 = (0.9, 0.3+0.2i), both restoreSU'd;
    U1*U2 has det 1, ReTr 1.3264, a = (0.6632, 0.184826), b = (0.293548, 0.6632)."""
    def restore(a, b):
        r = math.sqrt(abs(a) ** 2 + abs(b) ** 2)
        return a / r, b / r

    a1, b1 = restore(0.8 + 0.3j, 0.1 + 0.4j)
    a2, b2 = restore(0.9 + 0j, 0.3 + 0.2j)
    a = a1 * a2 - b1 * b2.conjugate()
    b = a1 * b2 + b1 * a2.conjugate()
    assert abs(a * a.conjugate() + b * b.conjugate() - 1) < 1e-12
    assert 2 * a.real == pytest.approx(1.3264, abs=5e-5)
    assert (a.real, a.imag) == pytest.approx((0.6632, 0.184826), abs=5e-6)
    assert (b.real, b.imag) == pytest.approx((0.293548, 0.6632), abs=5e-6)


def _tc_config():
    U = np.zeros(4 ** 4 * 4)

    def idx(t, x, y, z, mu):
        return (((t * 4 + x) * 4 + y) * 4 + z) * 4 + mu

    for (c, mu, v) in [((1, 1, 1, 1), 0, 0), ((1, 1, 1, 1), 1, math.pi / 2),
                       ((1, 1, 1, 1), 2, math.pi / 2), ((1, 1, 1, 1), 3, 0),
                       ((0, 1, 1, 1), 0, math.pi), ((1, 0, 1, 1), 1, math.pi / 2),
                       ((1, 1, 0, 0), 2, math.pi), ((1, 1, 1, 0), 3, math.pi / 2)]:
        U[idx(*c, mu)] = v
    return U


def test_topological_charge_known_answer(orc):
    """test.cc:81-109: Q = 0.0126651 for the hand-built U(1) 4^4 field, invariant under a
    random gauge transformation."""
    U = _tc_config()
    _, Q = orc.energy_density(1, (4, 4, 4, 4), 4, U)
    assert Q == pytest.approx(0.0126651, abs=5e-8)
    V = orc.random_gauge_trafo(1, (4, 4, 4, 4), 4, U, 654321)
    _, Q2 = orc.energy_density(1, (4, 4, 4, 4), 4, V)
    assert Q2 == pytest.approx(Q, abs=1e-12)


def _dense(rows):
    A = np.array(rows, dtype=complex)
    return np.ascontiguousarray(np.stack([A.real, A.imag], -1).reshape(-1))


def _cvec(v):
    v = np.asarray(v, dtype=complex)
    return np.ascontiguousarray(np.stack([v.real, v.imag], -1).reshape(-1))


def test_cg_dense_known_answer(orc):
    """test/CG.cpp:20-39: Hermitian 3x3 system with x* = (10, 11, -1) from (5e5, -1e7, 0)."""
    i = 1j
    A = [[1, 2 + i, 1], [2 - i, 5, -6 + 6 * i], [1, -6 - 6 * i, -6]]
    xs = np.array([10, 11, -1], dtype=complex)
    b = np.array(A) @ xs
    x, _ = orc.cg_dense(_dense(A), _cvec(b), _cvec([5e5, -1e7, 0]), 1e-16)
    np.testing.assert_allclose(x, _cvec(xs), atol=1e-8)


def test_bicgstab_dense_known_answer(orc):
    """test/BiCGStab.cpp:20-35: non-Hermitian 3x3 system with x* = (10, 11, -1)."""
    i = 1j
    A = [[1, 2 + i, 1], [200, 5, -6 + 6 * i], [1, -6 - 6 * i, -6]]
    xs = np.array([10, 11, -1], dtype=complex)
    b = np.array(A) @ xs
    x, _ = orc.bicgstab_dense(_dense(A), _cvec(b), _cvec([5e5, -1e7, 0]), 1e-12)
    np.testing.assert_allclose(x, _cvec(xs), atol=1e-6)


def test_philox_known_answers(orc):
    """Philox4x32-10 known-answer vectors (Salmon et al., Random123 kat_vectors)."""
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert orc.philox([0xffffffff] * 4, [0xffffffff] * 2) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert orc.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                      [0xa4093822, 0x299f31d0]) == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_exp_zero_guard_is_a_documented_deviation(orc):
    """exp_gauge.cc:8-18 divides 0/0 at alpha = 0; the restatement keeps that (NaN), the
    device returns the identity (its limit)."""
    o = orc.exp_su2(np.zeros(3))
    assert o[0] == 1.0 and all(math.isnan(v) for v in o[1:])


# ---------------------------------------------------------------- against the reference
@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=GEOM_IDS)
def test_pin_gauge_path(orc, ref, group, dims, nd):
    U = ref.hotstart(group, dims, nd, 13526463, 1.0, 654321)
    assert np.array_equal(orc.hotstart(group, dims, nd, 13526463, 1.0, 654321), U)
    assert orc.gauge_energy(group, dims, nd, U) == pytest.approx(
        ref.gauge_energy(group, dims, nd, U), rel=1e-13, abs=1e-13)
    for xi in (1.0, 1.3):
        assert np.array_equal(orc.gauge_derivative(group, dims, nd, 2.3, U, xi, 0.7),
                              ref.gauge_derivative(group, dims, nd, 2.3, U, xi, 0.7))
        assert orc.retr_sum_plaquettes(group, dims, nd, U, xi, xi != 1) == pytest.approx(
            ref.retr_sum_plaquettes(group, dims, nd, U, xi, xi != 1), rel=1e-13, abs=1e-13)
    for cl in (0, 1):
        for ss in (0, 1):
            assert orc.energy_density(group, dims, nd, U, cl, ss) == \
                ref.energy_density(group, dims, nd, U, cl, ss)
    assert np.array_equal(orc.runge_kutta(group, dims, nd, 2.3, 0.01, U),
                          ref.runge_kutta(group, dims, nd, 2.3, 0.01, U))
    P, u = orc.initnormal(group, dims, nd, 777)
    Pr, ur = ref.initnormal(group, dims, nd, 777)
    assert np.array_equal(P, Pr) and u == ur
    for integ in (0, 6, 2, 4, 5):
        a = orc.md_injected(group, dims, nd, 2.3, integ, 5, 1.0, U, P)
        b = ref.md_injected(group, dims, nd, 2.3, integ, 5, 1.0, U, P)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
        assert a[0] == pytest.approx(b[0], abs=1e-9 * max(1, abs(b[3][1])))
    # the low-precision integrators (lp_leapfrog 1, lp_omf4 3) with rounding exponents
    for integ, e in ((1, 16), (1, 6), (3, 8), (3, 16)):
        a = orc.md_injected(group, dims, nd, 2.3, integ, 5, 1.0, U, P, exponent=e)
        b = ref.md_injected(group, dims, nd, 2.3, integ, 5, 1.0, U, P, exponent=e)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), (integ, e)
        assert a[0] == pytest.approx(b[0], abs=1e-9 * max(1, abs(b[3][1])))


@pytest.mark.parametrize("group,dims,nd", [GEOMS[0], GEOMS[3], GEOMS[4]],
                         ids=[GEOM_IDS[0], GEOM_IDS[3], GEOM_IDS[4]])
def test_pin_flow_records(orc, ref, group, dims, nd):
    U = ref.hotstart(group, dims, nd, 4711, 1.0, 654321)
    a = orc.gradient_flow_rows(group, dims, nd, 2.3, U, 0.1, 0.01)
    b = ref.gradient_flow_rows(group, dims, nd, 2.3, U, 0.1, 0.01)
    assert a.shape == b.shape
    np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-15)  # b is printed with 16 digits


def test_pin_hmc_chain(orc, ref):
    dims, nd = (4, 4, 4, 4), 4
    U = ref.hotstart(0, dims, nd, 13526463, 1.0, 654321)
    a = orc.hmc_run(0, dims, nd, 2.3, 0, 10, 1.0, 13526463, 0, 6, U)
    b = ref.hmc_run(0, dims, nd, 2.3, 0, 10, 1.0, 13526463, 0, 6, U)
    assert np.array_equal(a[1], b[1])
    np.testing.assert_allclose(a[2], b[2], atol=1e-9)
    assert rel(a[0], b[0]) < 1e-12


def test_pin_staggered(orc, ref):
    dims, nd = (8, 1, 1, 6), 2
    U = ref.hotstart(1, dims, nd, 42, 1.0, 654321)
    rng = np.random.default_rng(0)
    psi = rng.normal(size=96)
    for op in (0, 1, 2):
        assert np.array_equal(orc.staggered_apply(dims, nd, U, 0.05, op, psi),
                              ref.staggered_apply(dims, nd, U, 0.05, op, psi))
    x0 = rng.normal(size=96)
    xo, io = orc.cg_ddag(dims, nd, U, 0.05, psi, x0, 1e-10)
    xr, ir = ref.cg_ddag(dims, nd, U, 0.05, psi, x0, 1e-10)
    assert np.array_equal(xo, xr)
    assert ir == io + orc._last_solve_calls() - 1
    xo, io = orc.bicgstab_d(dims, nd, U, 0.05, psi, x0, 1e-10)
    xr, ir = ref.bicgstab_d(dims, nd, U, 0.05, psi, x0, 1e-10)
    assert np.array_equal(xo, xr)
    assert ir == io + orc._last_solve_calls() - 1
    assert np.array_equal(orc.gaussian_spinor(dims, 0, 10, 97), ref.gaussian_spinor(dims, 0, 10, 97))
    phi, h = orc.fermion_heatbath(dims, nd, U, 0.05, 97234719)
    phir, hr = ref.fermion_heatbath(dims, nd, U, 0.05, 97234719)
    assert np.array_equal(phi, phir) and h == hr
    assert orc.fermion_accept(dims, nd, U, 0.05, phi, 1e-10, 9) == \
        ref.fermion_accept(dims, nd, U, 0.05, phi, 1e-10, 9)
    assert np.array_equal(orc.fermion_derivative(dims, nd, U, 0.05, phi, 1e-10, 9),
                          ref.fermion_derivative(dims, nd, U, 0.05, phi, 1e-10, 9))
    P, _ = ref.initnormal(1, dims, nd, 5)
    R = ref.gaussian_spinor(dims, 0, 2 ** -0.5, 11)
    a = orc.md_injected_fermion(dims, nd, 4.0, 0.05, 1e-10, 97, 6, 3, 1.0, U, P, R)
    b = ref.md_injected_fermion(dims, nd, 4.0, 0.05, 1e-10, 97, 6, 3, 1.0, U, P, R)
    assert np.array_equal(a[1], b[1])
    assert a[0] == pytest.approx(b[0], abs=1e-9)
    # lp_leapfrog with fermions: the rounding applies to the summed gauge + fermion derivative
    for exponent in (6, 12):
        a = orc.md_injected_fermion(dims, nd, 4.0, 0.05, 1e-10, 97, 1, 3, 1.0, U, P, R,
                                    exponent=exponent)
        b = ref.md_injected_fermion(dims, nd, 4.0, 0.05, 1e-10, 97, 1, 3, 1.0, U, P, R,
                                    exponent=exponent)
        assert np.array_equal(a[1], b[1])
        assert a[0] == pytest.approx(b[0], abs=1e-9)


def test_metropolis_statistics_match_reference(orc, ref):
    """The device's checkerboard order with Philox streams (restated in the oracle) and the
    reference's time-slice order with mt19937 sample the same distribution: mean plaquette
    after thermalisation agrees within errors (SU(2) 4^4, beta = 2.0, delta = 0.3)."""
    dims, nd = (4, 4, 4, 4), 4
    norm = 1.0 / (256 * 6 * 2)
    U = orc.hotstart(0, dims, nd, 1, 1.0, -1)
    V = U.copy()
    a, b = [], []
    for s in range(60):
        U, _ = orc.metropolis_checkerboard(0, dims, nd, 2.0, 0.3, 4, 17, s, U)
        V, _ = ref.sweep(0, dims, nd, 2.0, 0.3, 4, 17, s, V)
        if s >= 20:
            a.append(orc.gauge_energy(0, dims, nd, U) * norm)
            b.append(ref.gauge_energy(0, dims, nd, V) * norm)
    err = 4 * math.sqrt(np.var(a) / len(a) + np.var(b) / len(b)) * 3  # autocorrelation slack
    assert abs(np.mean(a) - np.mean(b)) < err + 0.01


# ---------------------------------------------------------------- observables
@pytest.mark.parametrize("group,dims,nd", [(0, (4, 4, 4, 6), 4), (0, (4, 6, 1, 4), 3),
                                           (1, (4, 4, 4, 4), 4), (1, (8, 1, 1, 6), 2)])
def test_pin_observables(orc, ref, group, dims, nd):
    """Polyakov loop, planar Wilson loops and APE smearing against the reference's own
    polyakov_loop_spatial_average, wilsonloop and APEsmearing.  The reference sums the loops
    in OpenMP reductions, whose order moves the last bit with the thread count: 1e-13."""
    U = ref.hotstart(group, dims, nd, 321, 1.0, 654321)
    assert orc.polyakov_loop(group, dims, nd, U) == pytest.approx(
        ref.polyakov_loop(group, dims, nd, U), rel=1e-13, abs=1e-15)
    for r, t in ((1, 1), (2, 3), (3, 2)):
        assert orc.wilson_loop(group, dims, nd, U, r, t) == pytest.approx(
            ref.wilson_loop(group, dims, nd, U, r, t), rel=1e-13, abs=1e-15)
    if nd > 2:
        for spatial in (True, False):
            assert np.array_equal(orc.ape_smear(group, dims, nd, U, 0.6, spatial),
                                  ref.ape_smear(group, dims, nd, U, 0.6, spatial))


# ---------------------------------------------------------------- golden fixtures
def test_golden_fixtures(orc):
    """The restatement against vectors the reference itself produced (make_golden.py)."""
    path = os.path.join(GOLDEN, "golden.npz")
    if not os.path.exists(path):
        pytest.skip("golden fixtures not generated")
    g = np.load(path)
    U = g["su2_U"]
    dims, nd = tuple(int(v) for v in g["su2_dims"]), 4
    assert np.array_equal(orc.hotstart(0, dims, nd, 13526463, 1.0, 654321), U)
    assert orc.gauge_energy(0, dims, nd, U) == pytest.approx(float(g["su2_plaq"]), rel=1e-13)
    assert orc.gauge_energy(0, dims, nd, U, spatial_only=True) == \
        pytest.approx(float(g["su2_plaq_ss"]), rel=1e-13)
    assert np.array_equal(orc.gauge_derivative(0, dims, nd, 2.4, U), g["su2_force"])
    assert np.array_equal(orc.runge_kutta(0, dims, nd, 2.4, 0.01, U), g["su2_flow"])
    E, Q = orc.energy_density(0, dims, nd, U)
    assert (E, Q) == (float(g["su2_E"]), float(g["su2_Q"]))
    rows = orc.gradient_flow_rows(0, dims, nd, 2.4, U, 0.05, 0.01)
    want = g["su2_flow_rows"]  # written as text by the reference: compare at print precision
    assert rows.shape == want.shape
    np.testing.assert_allclose(rows, want, rtol=1e-5, atol=1e-7)
    for name, integ, n in (("leapfrog", 0, 10), ("omf2", 6, 4)):
        dH, Ut, _, _ = orc.md_injected(0, dims, nd, 2.4, integ, n, 1.0, U, g["su2_P"])
        assert dH == pytest.approx(float(g[f"su2_md_{name}_dH"]), abs=1e-10)
        assert np.array_equal(Ut, g[f"su2_md_{name}_U"])
    d3 = tuple(int(v) for v in g["su2d3_dims"])
    U3 = g["su2d3_U"]
    assert np.array_equal(orc.hotstart(0, d3, 3, 4711, 1.0, 99), U3)
    assert orc.gauge_energy(0, d3, 3, U3) == pytest.approx(float(g["su2d3_plaq"]), rel=1e-13)
    assert np.array_equal(orc.gauge_derivative(0, d3, 3, 2.0, U3), g["su2d3_force"])
    assert orc.polyakov_loop(0, dims, nd, U) == pytest.approx(float(g["su2_polyakov"]),
                                                               rel=1e-13, abs=1e-15)
    assert orc.wilson_loop(0, dims, nd, U, 2, 3) == pytest.approx(float(g["su2_wilson_2_3"]),
                                                                  rel=1e-13, abs=1e-15)
    assert np.array_equal(orc.ape_smear(0, dims, nd, U, 0.6, True), g["su2_ape_0.6"])
    Uu = g["u1_U"]
    du = tuple(int(v) for v in g["u1_dims"])
    assert np.array_equal(orc.hotstart(1, du, 2, 13526463, 1.0, 654321), Uu)
    assert orc.gauge_energy(1, du, 2, Uu) == pytest.approx(float(g["u1_plaq"]), rel=1e-13)
    assert np.array_equal(orc.gauge_derivative(1, du, 2, 4.0, Uu), g["u1_force"])
    assert np.array_equal(orc.staggered_apply(du, 2, Uu, 0.05, 2, g["u1_psi"]), g["u1_DDdag_psi"])
    x, it = orc.cg_ddag(du, 2, Uu, 0.05, g["u1_psi"], g["u1_x0"], 1e-10)
    assert np.array_equal(x, g["u1_cg_x"])
    assert int(g["u1_cg_iter"]) == it + orc._last_solve_calls() - 1
    x, it = orc.bicgstab_d(du, 2, Uu, 0.05, g["u1_psi"], g["u1_x0"], 1e-10)
    assert np.array_equal(x, g["u1_bicgstab_x"])
    assert int(g["u1_bicgstab_iter"]) == it + orc._last_solve_calls() - 1


# ---------------------------------------------------------------- configuration files
def test_reference_file_format(ref, tmp_path):
    """gaugeconfig::save writes one in-memory _su2 (size_t N_c = 2, then Re a, Im a, Re b,
    Im b) or _u1 (size_t N_c = 1, then the angle) per link in host link order
    (gaugeconfig.hh:225-230, su2.hh:11-16, u1.hh:11-15); load reads it back."""
    for group, dims, nd, nc, width in ((0, (4, 4, 4, 6), 4, 2, 4), (1, (8, 1, 1, 6), 2, 1, 1)):
        U = ref.hotstart(group, dims, nd, 99, 1.0, 654321)
        path = tmp_path / f"conf{group}"
        ref.save_gauge(group, dims, nd, U, path)
        rec = np.fromfile(path, dtype=np.dtype([("nc", "<u8"), ("v", "<f8", (width,))]))
        assert rec.size == U.size // width
        assert np.all(rec["nc"] == nc)
        assert np.array_equal(rec["v"].reshape(-1), U)
        assert np.array_equal(ref.load_gauge(group, dims, nd, path), U)


def test_pin_pion_correlator(orc, ref):
    """staggered::C_pion of the reference against the restatement, which solves once where
    the reference repeats the identical solve for every site."""
    for dims, nd in (((8, 1, 1, 6), 2), ((4, 4, 1, 4), 3)):
        U = ref.hotstart(1, dims, nd, 42, 1.0, 654321)
        assert np.array_equal(orc.pion_correlator(dims, nd, U, 0.1, 1e-12, 17),
                              ref.pion_correlator(dims, nd, U, 0.1, 1e-12, 17))


def test_oracle_at_full_sizes_against_reference_digests(orc):
    """The restatement at the workloads' full sizes against the reference's own results
    (tests/golden/config_sizes.npz): D D^+ on U(1) 256^2, the gauge derivative and action on
    SU(2) 24^4, the start plaquette and one RK3 flow step on SU(2) 32^4."""
    import os
    import sys
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    from digest import check
    from make_config_sizes import SU2_24, SU2_32, U1_DIMS, inputs
    fx = np.load(os.path.join(here, "config_sizes.npz"))
    x = inputs(orc)
    check(orc.staggered_apply(U1_DIMS, 2, x["u1_U"], 0.05, 2, x["u1_b"]), fx, "u1_DDdag_b",
          1e-13)
    check(orc.gauge_derivative(0, SU2_24, 4, 2.4, x["su2_24_U"]), fx, "su2_24_force", 1e-13)
    assert -1.2 * orc.gauge_energy(0, SU2_24, 4, x["su2_24_U"]) == \
        pytest.approx(float(fx["su2_24_S"]), rel=1e-13)
    U = x["su2_32_U"]
    assert orc.gauge_energy(0, SU2_32, 4, U) / (32 ** 4 * 12) == \
        pytest.approx(float(fx["su2_32_plaq"]), rel=1e-13)
    check(orc.runge_kutta(0, SU2_32, 4, 2.4, 0.01, U), fx, "su2_32_flow", 1e-13)
