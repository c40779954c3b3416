"""One lattice over time slabs (su2b_slabs_*) against the single-lattice trajectory.

The slab trajectory runs the same kernels on each slab's own sites with ghost slices
refreshed after every force launch, and takes the Philox momenta of the whole lattice, so it
must give the single-lattice context's links bit for bit and its accept decisions, with the
energies equal to rounding (the sums add in another order: dH within 1e-13 of the energies'
magnitude, plaquette sums within 1e-12 relative).  Slabs here all live on one device (the exchange is a device copy); the
NCCL transport between processes shares everything but the copy.
"""
import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu

SEED, TRAFO = 13526463, 654321


def hot(orc, dims, nd):
    return orc.hotstart(0, dims, nd, SEED, 1.0, TRAFO)


def single(gpu, dims, nd, precision, beta=2.3, xi=1.0):
    Lx, Ly, Lz, Lt = dims
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, beta, group="su2", precision=precision, xi=xi)


def slabs(dims, nd, nslabs, precision, beta=2.3, **kw):
    from su2_b200.slabs import slab_lattice
    return slab_lattice(dims, nd, beta, nslabs, precision=precision, **kw)


def chain(lat, n, integrator="omf2", n_steps=4, tau=1.0, seed=11):
    """n trajectories: even ones are accepted without the test; odd ones take one coarse
    step (n = 1, tau = 2: dH large and positive) and the test with the uniform 0.999999,
    so the chain sees accepted and rejected trajectories."""
    return [lat.md_update(integrator, n_steps, tau, seed=seed, traj=k, accept_reject=False)
            if k % 2 == 0 else
            lat.md_update(integrator, 1, 2.0, seed=seed, traj=k, uniform=0.999999)
            for k in range(n)]


def same_chain(a, b):
    assert [r.accepted for r in a] == [r.accepted for r in b]
    for x, y in zip(a, b):
        # the energies are sums over the lattice added in another order
        scale = sum(abs(h) for h in x.H_old + x.H_new)
        assert x.dH == pytest.approx(y.dH, abs=1e-13 * scale + 1e-9)
        assert x.plaquette == pytest.approx(y.plaquette, rel=1e-12)
        for k in range(2):
            assert x.H_old[k] == pytest.approx(y.H_old[k], rel=1e-12)
            assert x.H_new[k] == pytest.approx(y.H_new[k], rel=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dims,nd,nslabs", [
    ((8, 8, 8, 8), 4, 1), ((8, 8, 8, 8), 4, 2), ((8, 8, 8, 8), 4, 4),
    ((4, 6, 8, 12), 4, 3), ((4, 6, 8, 12), 4, 6), ((8, 6, 1, 8), 3, 2), ((6, 1, 1, 8), 2, 4)],
    ids=["8^4/1", "8^4/2", "8^4/4", "4x6x8x12/3", "4x6x8x12/6", "8x6x8-d3/2", "6x8-d2/4"])
def test_slabs_equal_the_single_lattice(gpu, orc, precision, dims, nd, nslabs):
    U = hot(orc, dims, nd)
    with single(gpu, dims, nd, precision) as c, slabs(dims, nd, nslabs, precision) as s:
        c.upload(U)
        s.upload(U)
        assert s.gauge_energy() == pytest.approx(c.gauge_energy(), rel=1e-13)
        assert s.gauge_energy(True) == pytest.approx(c.gauge_energy(True), rel=1e-13, abs=1e-12)
        a, b = chain(c, 8), chain(s, 8)
        same_chain(a, b)
        acc = [r.accepted for r in a]
        assert any(acc) and not all(acc)
        assert np.array_equal(c.download(), s.download())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_anisotropic_slabs(gpu, orc, precision):
    """xi != 1 (the anisotropic force and sweep weights) over 2 slabs."""
    dims, nd, xi = (6, 6, 6, 8), 4, 0.8
    U = hot(orc, dims, nd)
    with single(gpu, dims, nd, precision, xi=xi) as c, \
            slabs(dims, nd, 2, precision, xi=xi) as s:
        c.upload(U)
        s.upload(U)
        same_chain(chain(c, 4), chain(s, 4))
        for k in range(2):
            assert np.array_equal(c.sweep(0.3, 4, 9, k), s.sweep(0.3, 4, 9, k))
        assert np.array_equal(c.download(), s.download())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dims,nd,nslabs", [
    ((8, 8, 8, 8), 4, 2), ((8, 8, 8, 8), 4, 4), ((4, 6, 8, 12), 4, 3), ((8, 6, 1, 8), 3, 2),
    ((6, 1, 1, 8), 2, 4)], ids=["8^4/2", "8^4/4", "4x6x8x12/3", "8x6x8-d3/2", "6x8-d2/4"])
def test_slab_metropolis_sweeps(gpu, orc, precision, dims, nd, nslabs):
    """The checkerboard sweep over slabs (local parity flipped, one piece of the faces
    exchanged after each pass) gives the single lattice's links and acceptance rates."""
    U = hot(orc, dims, nd)
    with single(gpu, dims, nd, precision) as c, slabs(dims, nd, nslabs, precision) as s:
        c.upload(U)
        s.upload(U)
        for k in range(3):
            rc, rs = c.sweep(0.25, 6, 21, k), s.sweep(0.25, 6, 21, k)
            assert np.array_equal(rc, rs), k
            assert 0.01 < rc[0] < 0.99
        assert np.array_equal(c.download(), s.download())
        assert s.gauge_energy() == pytest.approx(c.gauge_energy(), rel=1e-13)


def test_slabs_alternate_sweeps_and_trajectories(gpu, orc):
    """The workload's alternation (Metropolis sweeps between HMC trajectories) over 4 slabs
    in mixed precision: after each step the single lattice's field."""
    dims, nd = (8, 8, 8, 16), 4
    U = hot(orc, dims, nd)
    with single(gpu, dims, nd, "mixed", beta=2.4) as c, \
            slabs(dims, nd, 4, "mixed", beta=2.4) as s:
        c.upload(U)
        s.upload(U)
        for k in range(3):
            assert np.array_equal(c.sweep(0.15, 8, 5, k), s.sweep(0.15, 8, 5, k))
            same_chain([c.md_update("omf2", 6, 1.0, seed=5, traj=k)],
                       [s.md_update("omf2", 6, 1.0, seed=5, traj=k)])
            assert np.array_equal(c.download(), s.download()), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("integrator,n_steps", [("leapfrog", 5), ("omf4", 2), ("omf2", 1)])
def test_slab_integrators(gpu, orc, precision, integrator, n_steps):
    dims, nd = (6, 6, 6, 8), 4
    U = hot(orc, dims, nd)
    with single(gpu, dims, nd, precision) as c, slabs(dims, nd, 2, precision) as s:
        c.upload(U)
        s.upload(U)
        same_chain(chain(c, 4, integrator, n_steps, 0.5), chain(s, 4, integrator, n_steps, 0.5))
        assert np.array_equal(c.download(), s.download())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_force_shape_on_slabs(gpu, orc, precision):
    """Each launch shape of the force kernel, the two-threads-per-site ones and the
    one-thread-per-link one included, covers exactly a slab's own sites: the same links
    as the single lattice with that shape."""
    dims, nd = (6, 6, 6, 8), 4
    U = hot(orc, dims, nd)
    for v in range(gpu._abi.FORCE_VARIANTS):
        with single(gpu, dims, nd, precision) as c, slabs(dims, nd, 2, precision) as s:
            c.force_variant = v
            s.tune_set(v)
            assert s.tune_get() == v
            c.upload(U)
            s.upload(U)
            same_chain(chain(c, 2), chain(s, 2))
            assert np.array_equal(c.download(), s.download()), v


def test_slabs_at_the_workload_size(gpu):
    """32^4, beta 2.4, omf2 tau 1 n 16 in mixed precision over 2 and 4 slabs, with the
    launch shape the tuner picks: the single lattice's links after three trajectories."""
    dims, nd = (32, 32, 32, 32), 4
    rng = np.random.default_rng(7)
    q = rng.standard_normal((32 ** 4 * 4, 4))
    U = (q / np.linalg.norm(q, axis=1, keepdims=True)).ravel()
    with single(gpu, dims, nd, "mixed", beta=2.4) as c:
        c.upload(U)
        c.autotune()
        v = c.force_variant
        ref = chain(c, 3, "omf2", 16, 1.0, seed=3)
        Uc = c.download()
    for n in (2, 4):
        with slabs(dims, nd, n, "mixed", beta=2.4) as s:
            s.upload(U)
            s.tune_set(v)
            same_chain(ref, chain(s, 3, "omf2", 16, 1.0, seed=3))
            assert np.array_equal(Uc, s.download())


def test_part_of_the_slabs(gpu, orc):
    """A handle of one slab of two uploads its slices and ghosts from the whole field and
    downloads only its own slices; without a communicator it refuses trajectories and
    sums."""
    dims, nd = (4, 4, 4, 8), 4
    U = hot(orc, dims, nd)
    with slabs(dims, nd, 2, "fp64", first=1, count=1) as s:
        assert s.slices() == (4, 8)
        s.upload(U)
        out = np.zeros_like(U)
        s.download(out)
        row = 4 * 4 * 4 * nd * 4
        assert np.array_equal(out[4 * row:], U[4 * row:])
        assert not out[:4 * row].any()
        with pytest.raises(gpu.Su2bError) as e:
            s.md_update("omf2", 2, 1.0)
        assert e.value.code == gpu._abi.ERR_INVALID
        with pytest.raises(gpu.Su2bError):
            s.gauge_energy()
        with pytest.raises(gpu.Su2bError) as e:
            s.autotune()
        assert e.value.code == gpu._abi.ERR_INVALID


def test_slab_autotune_picks_one_shape_for_every_slab(gpu, orc):
    """The slab tuner times every force shape on the first slab, applies the single-lattice
    rule (the first shape within 1 % of the fastest) and sets it on every slab; the chain in
    that shape is the single lattice's in the same shape."""
    dims, nd = (8, 8, 8, 8), 4
    U = hot(orc, dims, nd)
    with slabs(dims, nd, 2, "mixed") as s:
        s.upload(U)
        t = s.autotune()
        assert np.all(t > 0)
        fastest = t.min()
        v = s.tune_get()
        assert v == min(k for k in range(len(t)) if t[k] <= 1.01 * fastest)
        assert np.array_equal(s.download(), U.astype(np.float32).astype(np.float64))
        got = chain(s, 2, "omf2", 4, 1.0, seed=9)
        Us = s.download()
    with single(gpu, dims, nd, "mixed") as c:
        c.upload(U)
        c.force_variant = v
        same_chain(chain(c, 2, "omf2", 4, 1.0, seed=9), got)
        assert np.array_equal(c.download(), Us)


def test_slab_errors(gpu, orc):
    from su2_b200.slabs import slab_lattice
    # Lt = 8: not a multiple of 3; one (odd) slice per slab; more slabs than slices
    for nslabs in (3, 8, 16):
        with pytest.raises(gpu.Su2bError) as e:
            slab_lattice((4, 4, 4, 8), 4, 2.3, nslabs)
        assert e.value.code == gpu._abi.ERR_INVALID
    with pytest.raises(gpu.Su2bError):
        slab_lattice((4, 4, 4, 8), 4, 2.3, 2, first=1, count=2)
    dims, nd = (4, 4, 4, 8), 4
    U = hot(orc, dims, nd)
    with slabs(dims, nd, 2, "fp64") as s:
        s.upload(U)
        for integ in ("euler", "ruth", "lp_leapfrog"):
            with pytest.raises(gpu.Su2bError) as e:
                s.md_update(integ, 2, 1.0)
            assert e.value.code == gpu._abi.ERR_UNSUPPORTED
        with pytest.raises(gpu.Su2bError) as e:
            s.md_update("omf2", 2, 1.0, momenta=orc.initnormal(0, dims, nd, 5)[0])
        assert e.value.code == gpu._abi.ERR_UNSUPPORTED
        with pytest.raises(gpu.Su2bError) as e:
            s.tune_set(gpu._abi.FORCE_VARIANTS)
        assert e.value.code == gpu._abi.ERR_INVALID
        # the handle still works after the refusals
        assert np.isfinite(s.md_update("omf2", 2, 1.0).dH)


def test_slab_graph_replay(gpu, orc):
    """A trajectory is one graph: every replay queues the same kernels, and the kernel
    count is the per-slab force launches plus the exchanges and reductions."""
    dims, nd, n = (6, 6, 6, 8), 4, 2
    U = hot(orc, dims, nd)
    with slabs(dims, nd, n, "mixed") as s:
        s.upload(U)
        counts = []
        for k in range(4):
            n0 = s.kernel_launches()
            s.md_update("omf2", 3, 1.0, seed=1, traj=k, uniform=1e-300)
            counts.append(s.kernel_launches() - n0)
        nf = 2 * 3 + 1  # omf2 force launches
        # per slab: momenta, nf forces, plaquettes, three reductions, accept; per launch
        # step one exchange; one cross-slab sum
        assert counts == [n * (nf + 6) + nf + 1] * 4
        assert rel(s.download(), U) > 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dims,nslabs", [((6, 6, 6, 16), 2), ((8, 8, 8, 16), 4),
                                         ((4, 6, 8, 12), 3), ((8, 8, 8, 8), 4)],
                         ids=["6^3x16/2", "8^3x16/4", "4x6x8x12/3", "8^4/4-no-interior"])
def test_overlapped_exchange_equals_the_single_lattice(gpu, orc, precision, dims, nslabs):
    """Boundary slices first, the exchange on a second stream while the interior slices are
    updated (the form slabs on separate GPUs run): the same links and accept decisions.
    With two slices per slab there is no interior and the step runs as without overlap."""
    nd = 4
    U = hot(orc, dims, nd)
    with single(gpu, dims, nd, precision) as c, slabs(dims, nd, nslabs, precision) as s:
        assert not s.overlap
        s.overlap = True
        assert s.overlap
        c.upload(U)
        s.upload(U)
        same_chain(chain(c, 6), chain(s, 6))
        assert np.array_equal(c.download(), s.download())
        for v in (0, 8, 9):  # a site shape, xsplit, one thread per link
            c.force_variant = v
            s.tune_set(v)
            same_chain(chain(c, 2, seed=3), chain(s, 2, seed=3))
            assert np.array_equal(c.download(), s.download()), v


def test_overlapped_exchange_launches(gpu, orc):
    """With overlap each force step is three launches per slab (two boundary slices, the
    interior) and one exchange."""
    dims, nd, n = (6, 6, 6, 16), 4, 2
    U = hot(orc, dims, nd)
    with slabs(dims, nd, n, "mixed") as s:
        s.overlap = True
        s.upload(U)
        counts = []
        for k in range(3):
            n0 = s.kernel_launches()
            s.md_update("omf2", 3, 1.0, seed=1, traj=k, uniform=1e-300)
            counts.append(s.kernel_launches() - n0)
        nf = 2 * 3 + 1
        assert counts == [n * (3 * nf + 6) + nf + 1] * 3


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dims,nd,nslabs", [((8, 8, 8, 8), 4, 2), ((4, 6, 8, 12), 4, 3),
                                            ((8, 6, 1, 8), 3, 4)],
                         ids=["8^4/2", "4x6x8x12/3", "8x6x8-d3/4"])
def test_slab_flow(gpu, orc, precision, dims, nd, nslabs):
    """The Wilson flow over slabs: RK3 steps give the single lattice's links; energy_density
    and the gradient_flow records (from a thermalised-like field, the current field left
    unchanged) agree to the rounding of the sums' order."""
    U = orc.hotstart(0, dims, nd, SEED, 0.2, TRAFO)
    with single(gpu, dims, nd, precision) as c, slabs(dims, nd, nslabs, precision) as s:
        c.upload(U)
        s.upload(U)
        for ref, got in ((c.energy_density(), s.energy_density()),
                         (c.energy_density(False, True), s.energy_density(False, True))):
            assert got[0] == pytest.approx(ref[0], rel=1e-12)
            assert got[1] == pytest.approx(ref[1], rel=1e-9, abs=1e-12)
        for _ in range(3):
            c.runge_kutta(0.02)
            s.runge_kutta(0.02)
        assert np.array_equal(c.download(), s.download())
        rc, rs = c.gradient_flow(0.3, 0.02), s.gradient_flow(0.3, 0.02)
        assert rc.shape == rs.shape and len(rc) >= 6
        assert np.array_equal(rc[:, 0], rs[:, 0])
        np.testing.assert_allclose(rs[:, 1:8], rc[:, 1:8], rtol=1e-11, atol=1e-13)
        np.testing.assert_allclose(rs[:, 8], rc[:, 8], rtol=1e-8, atol=1e-11)
        assert np.array_equal(c.download(), s.download())  # the field is unchanged


def test_slab_connect_refusals(gpu):
    """su2b_slabs_connect wants one slab per process (count 1, nranks = nslabs, rank =
    first); the NCCL id comes from the run-time NCCL and is 128 bytes.  No communicator is
    made here: one GPU holds no second rank."""
    from su2_b200.slabs import nccl_unique_id, slab_lattice
    uid = nccl_unique_id()
    assert len(uid) == 128 and any(uid)
    dims, nd = (4, 4, 4, 8), 4
    with slab_lattice(dims, nd, 2.3, 2, precision="fp64") as s:  # both slabs: no communicator
        with pytest.raises(gpu.Su2bError) as e:
            s.connect(uid, 2, 0)
        assert e.value.code == gpu._abi.ERR_INVALID
    with slab_lattice(dims, nd, 2.3, 2, precision="fp64", first=1, count=1) as s:
        for nranks, rank in ((2, 0), (3, 1), (1, 0)):  # wrong rank, wrong size
            with pytest.raises(gpu.Su2bError) as e:
                s.connect(uid, nranks, rank)
            assert e.value.code == gpu._abi.ERR_INVALID


@pytest.mark.parametrize("overlap", [False, True], ids=["plain", "overlapped"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nccl_transport_with_one_rank(gpu, orc, precision, overlap):
    """One slab holding the whole lattice, connected through NCCL to itself: each face goes
    out through the pack table, ncclSend / ncclRecv (the slabs above and below are the rank
    itself) and the unpack table, the sums through ncclAllReduce; overlapped, the boundary
    slices' exchange runs on its own stream while the interior is updated.  Trajectories,
    sweeps, flow steps, the energy density and the flow records are the single lattice's."""
    from su2_b200.slabs import nccl_unique_id
    dims, nd = (8, 8, 8, 8), 4
    U = hot(orc, dims, nd)
    with single(gpu, dims, nd, precision) as c, \
            slabs(dims, nd, 1, precision, first=0, count=1) as s:
        s.connect(nccl_unique_id(), 1, 0)
        assert s.overlap  # the overlapped exchange by default once connected
        s.overlap = overlap
        c.upload(U)
        s.upload(U)
        # the tuner's times reduced over the (one) rank; the single lattice in that shape
        t = s.autotune()
        assert np.all(t > 0) and s.tune_get() == min(
            k for k in range(len(t)) if t[k] <= 1.01 * t.min())
        c.force_variant = s.tune_get()
        same_chain(chain(c, 4), chain(s, 4))
        assert np.array_equal(c.download(), s.download())
        for k in range(2):
            assert np.array_equal(c.sweep(0.3, 4, 9, k), s.sweep(0.3, 4, 9, k))
        assert np.array_equal(c.download(), s.download())
        for _ in range(2):
            c.runge_kutta(0.02)
            s.runge_kutta(0.02)
        assert np.array_equal(c.download(), s.download())
        assert s.gauge_energy() == pytest.approx(c.gauge_energy(), rel=1e-12)
        ref, got = c.energy_density(), s.energy_density()
        assert got[0] == pytest.approx(ref[0], rel=1e-12)
        rc, rs = c.gradient_flow(0.1, 0.02), s.gradient_flow(0.1, 0.02)
        assert rc.shape == rs.shape
        np.testing.assert_allclose(rs[:, 1:8], rc[:, 1:8], rtol=1e-11, atol=1e-13)
        assert np.array_equal(c.download(), s.download())
