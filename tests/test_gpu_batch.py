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
