"""Markov chains on the device against the reference's published plaquette expectation values
(doc/reference-values.txt: SU(2) 1+1d 100x100, SU(2) 3+1d 10^4), in two dimensions against
the exact result <P> = I_2(beta) / I_1(beta) of the SU(2) Wilson action, and for U(1)
against the reference code's own Metropolis chain.

P is the driver's normalised plaquette: the sum of ReTr over all plaquettes divided by
V d(d-1)/2 Nc (hmc.hpp:99-106, base_program.hpp:303-305).  The chains are the device's own
Philox streams from a fixed seed, so each run gives the same numbers; the tolerances are
four to five combined standard errors (the chain's blocked error and the published one)."""
import json
import os

import numpy as np
import pytest
from scipy.special import iv

pytestmark = pytest.mark.gpu


def haar(n_links, seed):
    q = np.random.default_rng(seed).normal(size=(n_links, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.reshape(-1)


def blocked(x, nblocks=20):
    """Mean and the standard error from nblocks block means (autocorrelation-safe when the
    blocks are longer than the autocorrelation time)."""
    x = np.asarray(x)
    b = x[: len(x) // nblocks * nblocks].reshape(nblocks, -1).mean(axis=1)
    return float(x.mean()), float(b.std(ddof=1) / np.sqrt(nblocks))


def metropolis_plaquettes(c, nplaq, delta, n_hit, n_therm, n_meas, seed):
    for k in range(n_therm):
        c.sweep(delta, n_hit, seed, k)
    out = []
    for k in range(n_meas):
        c.sweep(delta, n_hit, seed, n_therm + k)
        out.append(c.retr_sum_Wplaquettes() / nplaq)
    return out


@pytest.mark.parametrize("beta,ref,ref_err", [(1.0, 0.24018, 2e-5), (2.0, 0.43313, 2e-5)])
def test_su2_2d_metropolis_plaquette(gpu, beta, ref, ref_err):
    L = 100
    with gpu.gaugeconfig(L, 1, 1, L, 2, beta) as c:
        c.upload(haar(L * L * 2, 11))
        P = metropolis_plaquettes(c, L * L * 1 * 2, 0.5, 8, 200, 2000, 7)
    m, e = blocked(P)
    exact = iv(2, beta) / iv(1, beta)
    print(f"SU(2) 2d 100^2 beta {beta}: <P> = {m:.6f} +- {e:.6f} (published {ref}, exact "
          f"{exact:.6f})")
    assert abs(m - ref) < 5 * np.hypot(e, ref_err), (m, e, ref)
    assert abs(m - exact) < 5 * e, (m, e, exact)


def test_su2_4d_metropolis_plaquette(gpu):
    L, beta, ref, ref_err = 10, 2.0, 0.50133, 1.2e-4
    with gpu.gaugeconfig(L, L, L, L, 4, beta) as c:
        c.upload(haar(L ** 4 * 4, 12))
        P = metropolis_plaquettes(c, L ** 4 * 6 * 2, 0.3, 8, 300, 3000, 8)
    m, e = blocked(P)
    print(f"SU(2) 4d 10^4 beta {beta} Metropolis: <P> = {m:.6f} +- {e:.6f} (published {ref})")
    assert abs(m - ref) < 4 * np.hypot(e, ref_err), (m, e, ref)


def test_u1_4d_metropolis_plaquette(gpu):
    """U(1) d=4 against the reference code's own Metropolis chain (tests/golden/physics.json,
    made by tests/golden/make_physics.py), not against the published U(1) value: the
    published 0.19658(10) at beta 1.0 does not follow from the current reference code, whose
    own chain gives about 0.64 at 6^4 (the device chain about 0.585 at 10^4, beta 1.0 lying
    next to the transition near 1.01).  beta 0.8 is in the confined phase, away from it."""
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "physics.json")))
    f = g["u1_8x4_b0.8"]
    L = f["dims"][0]
    with gpu.gaugeconfig(L, L, L, L, 4, f["beta"], group="u1") as c:
        c.upload(np.random.default_rng(13).uniform(-np.pi, np.pi, size=L ** 4 * 4))
        P = metropolis_plaquettes(c, L ** 4 * 6 * 1, f["delta"], f["N_hit"], f["n_therm"],
                                  f["n_meas"], 9)
    m, e = blocked(P)
    print(f"U(1) 4d 8^4 beta {f['beta']} Metropolis: <P> = {m:.6f} +- {e:.6f} (reference chain "
          f"{f['plaquette']:.6f} +- {f['error']:.6f})")
    assert abs(m - f["plaquette"]) < 4 * np.hypot(e, f["error"]), (m, e, f["plaquette"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_su2_4d_hmc_plaquette(gpu, precision):
    """Omelyan HMC (fused trajectory path) in FP64 and in mixed precision: the same
    equilibrium plaquette as the reference's value, at a sensible acceptance."""
    L, beta, ref, ref_err = 10, 2.0, 0.50133, 1.2e-4
    nplaq = L ** 4 * 6 * 2
    with gpu.gaugeconfig(L, L, L, L, 4, beta, precision=precision) as c:
        c.upload(haar(L ** 4 * 4, 14))
        for k in range(100):  # Metropolis to equilibrium first
            c.sweep(0.3, 8, 10, k)
        P, acc = [], []
        for k in range(1200):
            r = c.md_update("omf2", 10, 1.0, seed=15, traj=k)
            if k >= 200:
                P.append(r.plaquette / nplaq)
                acc.append(r.accepted)
    m, e = blocked(P)
    print(f"SU(2) 4d 10^4 beta {beta} HMC {precision}: <P> = {m:.6f} +- {e:.6f}, acceptance "
          f"{np.mean(acc):.3f} (published {ref})")
    assert np.mean(acc) > 0.5
    assert abs(m - ref) < 4 * np.hypot(e, ref_err), (m, e, ref)


def test_mixed_precision_keeps_the_dH_distribution(gpu):
    """Mixed precision (FP32 links and forces, FP64 sums and accept/reject) against the FP64
    path on the same start: the Delta H distribution (two-sample Kolmogorov-Smirnov), its
    mean and the acceptance agree within statistical error, and both satisfy
    <exp(-Delta H)> = 1 (Creutz's equality for an area-preserving, reversible integrator).
    The two precisions draw different momenta, so they agree in distribution only."""
    from scipy.stats import ks_2samp
    L, beta = 10, 2.0
    start = haar(L ** 4 * 4, 16)
    dH, acc = {}, {}
    for precision in ("fp64", "mixed"):
        with gpu.gaugeconfig(L, L, L, L, 4, beta, precision=precision) as c:
            c.upload(start)
            for k in range(100):
                c.sweep(0.3, 8, 17, k)
            rs = [c.md_update("omf2", 8, 1.0, seed=18, traj=k) for k in range(1600)][100:]
        dH[precision] = np.array([r.dH for r in rs])
        acc[precision] = np.array([float(r.accepted) for r in rs])
    for p in dH:
        m, e = blocked(np.exp(-dH[p]))
        print(f"{p}: <dH> = {dH[p].mean():.4f}, acceptance {acc[p].mean():.3f}, "
              f"<exp(-dH)> = {m:.4f} +- {e:.4f}")
        assert abs(m - 1.0) < 5 * e + 0.02, (p, m, e)
    ks = ks_2samp(dH["fp64"], dH["mixed"])
    print(f"KS two-sample: statistic {ks.statistic:.4f}, p {ks.pvalue:.3g}")
    assert ks.pvalue > 1e-3
    m64, e64 = blocked(dH["fp64"])
    m32, e32 = blocked(dH["mixed"])
    assert abs(m64 - m32) < 5 * np.hypot(e64, e32), (m64, e64, m32, e32)
    a64, ea64 = blocked(acc["fp64"])
    a32, ea32 = blocked(acc["mixed"])
    assert abs(a64 - a32) < 5 * np.hypot(ea64, ea32), (a64, ea64, a32, ea32)
