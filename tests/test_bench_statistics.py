"""The statistics bench.py reports for mixed against FP64 at equal Delta H and plaquette,
checked on synthetic Markov chains on the CPU: blocked errors of correlated series, and the
two-sample Kolmogorov-Smirnov test with effective sample sizes."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def ar1(n, phi, seed, shift=0.0):
    """A stationary AR(1) chain of unit variance: autocorrelation phi^k, 2 tau = (1+phi)/(1-phi)."""
    r = np.random.default_rng(seed)
    e = r.normal(size=n)
    x = np.empty(n)
    x[0] = e[0]
    for i in range(1, n):
        x[i] = phi * x[i - 1] + np.sqrt(1 - phi * phi) * e[i]
    return x + shift


def test_blocked_error_sees_the_autocorrelation():
    phi = 0.8
    x = ar1(20000, phi, 3)
    m, e = bench.blocked(x)
    naive = x.std(ddof=1) / np.sqrt(len(x))
    two_tau = (1 + phi) / (1 - phi)
    assert abs(m) < 5 * e
    assert 0.6 * two_tau < (e / naive) ** 2 < 1.5 * two_tau


def test_ks_with_effective_sizes_holds_its_level_on_correlated_chains():
    """Equal distributions, correlated samples: the plain test rejects at 5 % about half the
    time; the effective-size test at most at its level."""
    from scipy import stats as st
    p_eff, p_iid = [], []
    for k in range(100):
        a, b = ar1(1000, 0.8, 2 * k), ar1(1000, 0.8, 2 * k + 1)
        p_eff.append(bench.ks_effective(a, b)[1])
        p_iid.append(st.ks_2samp(a, b).pvalue)
    assert np.mean(np.array(p_iid) < 0.05) > 0.25
    assert np.mean(np.array(p_eff) < 0.05) <= 0.08


def test_ks_with_effective_sizes_still_sees_a_shift():
    """A shift of one standard deviation is found in correlated chains of 1000 samples."""
    D, p, ra, rb = bench.ks_effective(ar1(1000, 0.8, 1), ar1(1000, 0.8, 2, shift=1.0))
    assert p < 1e-3 and ra > 2 and rb > 2


def test_ks_with_effective_sizes_on_independent_samples():
    """Independent samples: 2 tau scatters near 1 and the p-value is never below the plain
    asymptotic one (the effective sizes are at most n)."""
    from scipy import stats as st
    r = np.random.default_rng(9)
    a, b = r.normal(size=2000), r.normal(size=2000)
    D, p, ra, rb = bench.ks_effective(a, b)
    assert ra < 2 and rb < 2
    assert st.ks_2samp(a, b, method="asymp").pvalue - 1e-12 <= p <= 1.0
