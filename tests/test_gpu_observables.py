"""Observables between trajectories on the device (Polyakov loop, planar Wilson loops, APE
smearing) through the C ABI, against the oracle and the golden vectors of the reference.

Tolerances: FP64 sums 1e-12 relative, smeared FP64 fields 1e-13 relative; mixed precision
(FP32 links) against the oracle on the FP32-rounded links 1e-12 for sums and 1e-6 for the
smeared field (stored back in FP32).
"""
import os

import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu

GEOMS = [(0, (4, 4, 4, 6), 4), (0, (4, 6, 1, 4), 3), (0, (6, 1, 1, 4), 2),
         (1, (4, 4, 4, 4), 4), (1, (8, 1, 1, 6), 2)]
IDS = ["su2-d4", "su2-d3", "su2-d2", "u1-d4", "u1-d2"]


def make(gpu, group, dims, nd, precision="fp64"):
    Lx, Ly, Lz, Lt = dims
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, 2.3, group="su2" if group == 0 else "u1",
                           precision=precision)


@pytest.mark.parametrize("group,dims,nd", GEOMS, ids=IDS)
def test_polyakov_and_wilson_loops(gpu, orc, group, dims, nd):
    U = orc.hotstart(group, dims, nd, 77, 1.0, 654321)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        assert c.polyakov_loop_spatial_average() == pytest.approx(
            orc.polyakov_loop(group, dims, nd, U), rel=1e-12, abs=1e-14)
        for r, t in ((1, 1), (2, 3), (3, 2), (0, 2), (4, 4)):
            assert c.wilsonloop(r, t) == pytest.approx(
                orc.wilson_loop(group, dims, nd, U, r, t), rel=1e-12, abs=1e-14)


@pytest.mark.parametrize("group,dims,nd", [g for g in GEOMS if g[2] > 2],
                         ids=[i for g, i in zip(GEOMS, IDS) if g[2] > 2])
@pytest.mark.parametrize("spatial", [True, False])
def test_ape_smearing(gpu, orc, group, dims, nd, spatial):
    U = orc.hotstart(group, dims, nd, 78, 1.0, 654321)
    want = orc.ape_smear(group, dims, nd, U, 0.55, spatial)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        c.APEsmearing(0.55, spatial)
        assert rel(c.download(), want) < 1e-13
        # the smeared field is the context's field from now on
        assert c.gauge_energy() == pytest.approx(orc.gauge_energy(group, dims, nd, want),
                                                 rel=1e-12)


def test_mixed_precision_observables(gpu, orc):
    group, dims, nd = 0, (8, 8, 8, 8), 4
    U = orc.hotstart(group, dims, nd, 79, 1.0, 654321)
    Us = U.astype(np.float32).astype(np.float64)
    with make(gpu, group, dims, nd, precision="mixed") as c:
        c.upload(U)
        assert c.polyakov_loop_spatial_average() == pytest.approx(
            orc.polyakov_loop(group, dims, nd, Us), rel=1e-12, abs=1e-14)
        assert c.wilsonloop(2, 2) == pytest.approx(orc.wilson_loop(group, dims, nd, Us, 2, 2),
                                                   rel=1e-12, abs=1e-14)
        c.APEsmearing(0.6)
        assert rel(c.download(), orc.ape_smear(group, dims, nd, Us, 0.6, True)) < 1e-6


def test_observables_golden(gpu):
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "golden.npz"))
    Lx, Ly, Lz, Lt = (int(v) for v in g["su2_dims"])
    with gpu.gaugeconfig(Lx, Ly, Lz, Lt, 4, 2.4) as c:
        c.upload(g["su2_U"])
        assert c.polyakov_loop_spatial_average() == pytest.approx(float(g["su2_polyakov"]),
                                                                  rel=1e-12, abs=1e-14)
        assert c.wilsonloop(2, 3) == pytest.approx(float(g["su2_wilson_2_3"]), rel=1e-12,
                                                   abs=1e-14)
        c.APEsmearing(0.6)
        assert rel(c.download(), g["su2_ape_0.6"]) < 1e-13


def test_observable_errors(gpu):
    import su2_b200
    with gpu.gaugeconfig(6, 1, 1, 4, 2, 2.0) as c:
        with pytest.raises(su2_b200.Su2bError):
            c.APEsmearing(0.5, spatial=True)  # no spatial plane in d = 2
        with pytest.raises(su2_b200.Su2bError):
            c.wilsonloop(-1, 2)
