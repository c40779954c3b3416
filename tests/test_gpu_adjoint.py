"""Derivatives through the C ABI: Wilson action backward, the force VJP and the adjoint of
the Wilson flow, against central finite differences (FP64) and the reference's analytic
gauge force; and gradcheck through the torch.autograd binding.

Tolerances: analytic force vs action backward 1e-12; finite differences (h = 1e-5 on the
global objective, O(h^2) truncation) within 1e-6 relative to the gradient's scale; FP32 flow
gradient within 1e-3 of the FP64 one.
"""
import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu


def su2_exp_left(U, link, k, h):
    """exp(h e_k) applied from the left to one link (reference layout)."""
    from su2_b200.autograd import _exp_links
    om = np.zeros((U.size // 4, 3))
    om[link, k] = h
    return _exp_links(U, om)


def test_action_backward_is_the_reference_force(gpu, orc):
    dims, nd = (6, 4, 4, 6), 4
    U = orc.hotstart(0, dims, nd, 7, 1.0, 654321)
    with gpu.gaugeconfig(*dims, nd, 2.4) as c:
        c.upload(U)
        S, dS = c.action_backward(1.0)
    assert S == pytest.approx(orc.S_G_hmc(0, dims, nd, 2.4, U), rel=1e-12)
    assert rel(dS, orc.gauge_derivative(0, dims, nd, 2.4, U)) < 1e-12


def test_action_backward_finite_differences(gpu, orc):
    dims, nd = (4, 4, 4, 4), 4
    U = orc.hotstart(0, dims, nd, 8, 1.0, 654321)
    with gpu.gaugeconfig(*dims, nd, 2.4) as c:
        c.upload(U)
        _, dS = c.action_backward(1.0)
    rng = np.random.default_rng(1)
    for link in rng.choice(U.size // 4, 12, replace=False):
        for k in range(3):
            h = 1e-6
            fd = (orc.S_G_hmc(0, dims, nd, 2.4, su2_exp_left(U, link, k, h)) -
                  orc.S_G_hmc(0, dims, nd, 2.4, su2_exp_left(U, link, k, -h))) / (2 * h)
            assert fd == pytest.approx(dS[3 * link + k], abs=1e-6)


def test_force_vjp_finite_differences(gpu, orc):
    dims, nd = (4, 4, 4, 4), 4
    U = orc.hotstart(0, dims, nd, 9, 1.0, 654321)
    rng = np.random.default_rng(2)
    mu = rng.normal(size=U.size // 4 * 3)
    with gpu.gaugeconfig(*dims, nd, 2.0) as c:
        c.upload(U)
        vjp = c.force_vjp(mu)

    def phi(V):  # mu . g(V), g = get_deriv(U K) = derivative at beta/Nc = 1
        return float(mu @ orc.gauge_derivative(0, dims, nd, 2.0, V, 1.0, 1.0))

    for link in rng.choice(U.size // 4, 10, replace=False):
        for k in range(3):
            h = 1e-5
            fd = (phi(su2_exp_left(U, link, k, h)) - phi(su2_exp_left(U, link, k, -h))) / (2 * h)
            assert fd == pytest.approx(vjp[3 * link + k], abs=2e-6 * max(1, abs(fd)))


@pytest.mark.parametrize("every", [0, 1, 3])
def test_flow_adjoint_finite_differences(gpu, orc, every):
    dims, nd = (4, 4, 4, 4), 4
    U = orc.hotstart(0, dims, nd, 10, 1.0, 654321)
    eps, n = 0.02, 5
    with gpu.gaugeconfig(*dims, nd, 2.4) as c:
        c.upload(U)
        O, g = c.flow_objective(eps, n, grad=True, checkpoint_every=every)
        assert np.array_equal(c.download(), U)
        rng = np.random.default_rng(3)
        for link in rng.choice(U.size // 4, 8, replace=False):
            for k in range(3):
                h = 1e-5
                c.upload(su2_exp_left(U, link, k, h))
                Op = c.flow_objective(eps, n, grad=False)
                c.upload(su2_exp_left(U, link, k, -h))
                Om = c.flow_objective(eps, n, grad=False)
                fd = (Op - Om) / (2 * h)
                assert fd == pytest.approx(g[3 * link + k], abs=1e-7 + 1e-6 * np.abs(g).max())


def test_flow_objective_matches_flow_records(gpu, orc):
    dims, nd = (4, 4, 4, 4), 4
    U = orc.hotstart(0, dims, nd, 11, 1.0, 654321)
    Vt = U.copy()
    for _ in range(4):
        Vt = orc.runge_kutta(0, dims, nd, 2.4, 0.02, Vt)
    P = orc.gauge_energy(0, dims, nd, Vt) / (256 * 2)
    want = (4 * 0.02) ** 2 * (6 - P)
    with gpu.gaugeconfig(*dims, nd, 2.4) as c:
        c.upload(U)
        assert c.flow_objective(0.02, 4, grad=False) == pytest.approx(want, rel=1e-12)


def test_flow_adjoint_fp32_against_fp64(gpu, orc):
    dims, nd = (8, 8, 8, 8), 4
    U = orc.hotstart(0, dims, nd, 12, 1.0, 654321)
    res = {}
    for prec in ("fp64", "mixed"):
        with gpu.gaugeconfig(*dims, nd, 2.4, precision=prec) as c:
            c.upload(U)
            res[prec] = c.flow_objective(0.01, 20, grad=True)
    assert res["mixed"][0] == pytest.approx(res["fp64"][0], rel=1e-5)
    assert rel(res["mixed"][1], res["fp64"][1]) < 1e-3


def test_autograd_binding_gradcheck(gpu, orc):
    import torch

    from su2_b200.autograd import FlowEnergy, WilsonAction
    dims, nd = (2, 2, 2, 4), 4
    U = orc.hotstart(0, dims, nd, 13, 1.0, 654321)
    n = U.size // 4
    with gpu.gaugeconfig(*dims, nd, 2.3) as c:
        om = (0.05 * torch.randn(n, 3, dtype=torch.float64)).requires_grad_()
        assert torch.autograd.gradcheck(lambda w: WilsonAction.apply(w, c, U), (om,), eps=1e-6,
                                        atol=1e-6, rtol=1e-5)
        assert torch.autograd.gradcheck(lambda w: FlowEnergy.apply(w, c, U, 0.05, 3, 2), (om,),
                                        eps=1e-6, atol=1e-7, rtol=1e-5)
