"""The batched ensemble path (su2b_batch_*): every chain of a batch follows the trajectory it
follows alone in a single-lattice context with the same seed -- same accept decisions, Delta H
within 1e-10 (FP64 sums in a different order), links within 1e-13 relative in FP64 storage
and 1e-6 in FP32 storage."""
import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu

CHAINS = [dict(dims=(4, 4, 4, 4), ndims=4, beta=2.2, seed=11),
          dict(dims=(6, 4, 4, 8), ndims=4, beta=2.5, seed=12),
          dict(dims=(6, 8, 1, 4), ndims=3, beta=2.0, seed=13),
          dict(dims=(4, 4, 1, 8), ndims=3, beta=2.6, seed=14)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("integ,n", [("leapfrog", 10), ("omf2", 4)])
def test_batch_chains_equal_single_contexts(gpu, orc, precision, integ, n):
    from su2_b200.batch import chain_batch
    starts = [orc.hotstart(0, c["dims"], c["ndims"], 100 + i, 1.0, 654321)
              for i, c in enumerate(CHAINS)]
    ntraj = 4
    with chain_batch(CHAINS, precision=precision) as b:
        for i, U in enumerate(starts):
            b.upload(i, U)
        bres = [b.md_update(integ, n, 1.0, traj=t) for t in range(ntraj)]
        bU = [b.download(i) for i in range(len(CHAINS))]
        assert b.kernel_launches() > 0
    tol = 1e-13 if precision == "fp64" else 1e-6
    for i, c in enumerate(CHAINS):
        with gpu.gaugeconfig(*c["dims"], c["ndims"], c["beta"], precision=precision) as s:
            s.upload(starts[i])
            for t in range(ntraj):
                r = s.md_update(integ, n, 1.0, seed=c["seed"], traj=t)
                assert r.accepted == bres[t][i].accepted
                assert r.dH == pytest.approx(bres[t][i].dH, abs=1e-10 * max(1, abs(r.H_old[1])))
                assert r.plaquette == pytest.approx(bres[t][i].plaquette, rel=1e-12)
            assert rel(bU[i], s.download()) < tol


def test_batch_rejects_bad_chains(gpu):
    import su2_b200
    from su2_b200.batch import chain_batch
    with pytest.raises(su2_b200.Su2bError):
        chain_batch([dict(dims=(4, 1, 1, 4), ndims=2, beta=2.0, seed=1)])
    with pytest.raises(su2_b200.Su2bError):
        chain_batch([dict(dims=(5, 4, 4, 4), ndims=4, beta=2.0, seed=1)])
    with chain_batch([dict(dims=(4, 4, 4, 4), ndims=4, beta=2.0, seed=1)]) as b:
        with pytest.raises(su2_b200.Su2bError):
            b.md_update("omf4", 4, 1.0)


def test_batch_autotune_leaves_fields_and_every_shape_agrees(gpu, orc):
    """The batch tuner times every launch shape without touching the chains' fields, keeps
    the fastest, and every shape advances the ensemble identically up to the rounding of the
    per-tile partial sums (different tile sizes group the sums differently)."""
    from su2_b200.batch import chain_batch
    chains = [dict(dims=(4, 4, 4, 6), ndims=4, beta=2.3, seed=11),
              dict(dims=(8, 6, 1, 4), ndims=3, beta=2.1, seed=12)]
    starts = [orc.hotstart(0, c["dims"], c["ndims"], 100 + i, 1.0, 654321)
              for i, c in enumerate(chains)]
    runs = []
    for v in range(gpu._abi.BATCH_VARIANTS):
        with chain_batch(chains, precision="mixed") as b:
            for i, U in enumerate(starts):
                b.upload(i, U)
            if v == 0:
                t = b.autotune()
                assert all(x > 0 for x in t.values())
                fastest = min(t.values())  # the first shape within 1 % of the fastest
                assert b.variant == min(v for v in t if t[v] <= 1.01 * fastest)
                for i, U in enumerate(starts):
                    assert np.array_equal(b.download(i), U.astype(np.float32).astype(np.float64))
            b.variant = v
            res = [b.md_update("leapfrog", 5, 1.0, traj=k) for k in range(3)]
            runs.append((res, [b.download(i) for i in range(len(chains))]))
    ref_res, ref_U = runs[0]
    for res, Us in runs[1:]:
        for ra, rb in zip(ref_res, res):
            for a, b_ in zip(ra, rb):
                assert a.accepted == b_.accepted
                assert a.dH == pytest.approx(b_.dH, abs=1e-8)
        for a, b_ in zip(ref_U, Us):
            assert np.array_equal(a, b_)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_carries_start_plaquettes(gpu, orc, precision):
    """Consecutive batched trajectories take each chain's start plaquettes from the previous
    trajectory's sums (its end field if accepted, else its start field) instead of summing
    them again.  A batch that re-uploads its own fields before every trajectory (which drops
    the carry-over) evolves the same: the same accept decisions, Delta H and plaquettes bit
    for bit, the same links."""
    from su2_b200.batch import chain_batch
    starts = [orc.hotstart(0, c["dims"], c["ndims"], 200 + i, 1.0, 654321)
              for i, c in enumerate(CHAINS)]
    runs = []
    for reupload in (False, True):
        with chain_batch(CHAINS, precision=precision) as b:
            for i, U in enumerate(starts):
                b.upload(i, U)
            res = []
            for t in range(8):
                if reupload:
                    for i in range(len(CHAINS)):
                        b.upload(i, b.download(i))
                # fine and coarse trajectories: accepted and rejected ones
                n, tau = (10, 1.0) if t % 2 == 0 else (2, 2.0)
                res.append(b.md_update("leapfrog", n, tau, traj=t))
            runs.append((res, [b.download(i) for i in range(len(CHAINS))]))
    (a, Ua), (b_, Ub) = runs
    acc = [r.accepted for rs in a for r in rs]
    assert any(acc) and not all(acc)
    for ra, rb in zip(a, b_):
        for x, y in zip(ra, rb):
            assert x.accepted == y.accepted and x.dH == y.dH and x.plaquette == y.plaquette
    for u, v in zip(Ua, Ub):
        assert np.array_equal(u, v)
