"""Parity on seeded random lattice shapes, beyond the fixed geometries of the other tests:
d = 2, 3, 4, every active extent even from 2 to 10 (an extent of 2 makes the forward and
backward neighbour the same site), half volumes that are and are not multiples of a block's
sites.  For each shape, against the oracle: the plaquette sums, the gauge force through
every launch shape of the force kernel (SU(2)), an RK3 flow step, a trajectory with
injected momenta, the checkerboard Metropolis sweep, and for U(1) the staggered D D^+.

Tolerances as in the other parity tests: FP64 fields and sums within 1e-12 relative
(norm-wise), Delta H within 1e-9 max(1, |H|), mixed precision within 1e-5."""
import numpy as np
import pytest

from helpers import group_name, rel

pytestmark = pytest.mark.gpu


def random_shapes(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        nd = int(rng.integers(2, 5))
        ext = [int(2 * rng.integers(1, 6)) for _ in range(nd)]  # even, 2..10
        # active directions t, x, y, z in that order; inactive ones are 1
        Lt, rest = ext[0], ext[1:] + [1] * (4 - nd)
        dims = (rest[0], rest[1], rest[2], Lt)
        if np.prod(dims) > 4096:
            continue
        out.append((dims, nd))
    return out


SHAPES = random_shapes(10, 2024)
IDS = ["x".join(map(str, d)) + f"-d{nd}" for d, nd in SHAPES]


def make(gpu, group, dims, nd, beta=2.3, precision="fp64"):
    Lx, Ly, Lz, Lt = dims
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, beta, group=group_name(group),
                           precision=precision)


@pytest.mark.parametrize("dims,nd", SHAPES, ids=IDS)
@pytest.mark.parametrize("group", [0, 1], ids=["su2", "u1"])
def test_random_shape_parity(gpu, orc, group, dims, nd):
    U = orc.hotstart(group, dims, nd, 777, 1.0, 4321)
    F = orc.gauge_derivative(group, dims, nd, 2.3, U)
    flow = orc.runge_kutta(group, dims, nd, 2.3, 0.01, U)
    P, _ = orc.initnormal(group, dims, nd, 99)
    dH, U_md, _, H = orc.md_injected(group, dims, nd, 2.3, 6, 3, 0.5, U, P)
    U_mc, rates = orc.metropolis_checkerboard(group, dims, nd, 2.3, 0.3, 3, 5, 1, U)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        assert c.gauge_energy() == pytest.approx(orc.gauge_energy(group, dims, nd, U),
                                                 rel=1e-12)
        variants = range(gpu._abi.FORCE_VARIANTS) if group == 0 else [0]
        for v in variants:
            if group == 0:
                c.force_variant = v
            assert rel(c.derivative(), F) < 1e-12, v
        c.runge_kutta(0.01)
        assert rel(c.download(), flow) < 1e-12
        c.upload(U)
        r = c.md_update("omf2", 3, 0.5, momenta=P, accept_reject=False)
        assert r.dH == pytest.approx(dH, abs=1e-9 * max(1.0, abs(H[1])))
        assert rel(c.download(), U_md) < 1e-10
        c.upload(U)
        got = c.sweep(0.3, 3, 5, 1)
        assert rel(c.download(), U_mc) < 1e-11
        np.testing.assert_array_equal(got, rates)
    if group == 0:
        with make(gpu, group, dims, nd, precision="mixed") as c:
            c.upload(U)
            for v in range(gpu._abi.FORCE_VARIANTS):
                c.force_variant = v
                assert rel(c.derivative(), F) < 1e-5, v
    else:
        psi = np.random.default_rng(3).normal(size=2 * int(np.prod(dims)))
        want = orc.staggered_apply(dims, nd, U, 0.1, 2, psi)
        with make(gpu, group, dims, nd) as c:
            c.upload(U)
            assert rel(c.DDdag(0.1, psi), want) < 1e-13
