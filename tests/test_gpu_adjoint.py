"""Adjoint of the residual w.r.t. theta = (Gc, l, A, n) against central finite differences of the
oracle's residual (needs a B200).

Bar: 1e-6 relative (2-norm over the dofs, or over the material sets).  The return map runs with the
tight tolerance so that the finite differences resolve the viscous strain's dependence on (A, n).
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu

ADJ_TOL = 1e-6
DT = 100.0


def _tight(d):
    d["B200"]["ReturnMapTolerance"] = "tight"


def _prime(o, g, steps, dt):
    for s in steps:
        o.assemble(s, dt=dt)
        g.assemble(s, dt=dt)


def _cmp_theta(got, ref, what):
    for th in range(4):
        nr = np.linalg.norm(ref[th])
        if nr == 0.0:
            assert np.linalg.norm(got[th]) == 0.0, (what, th)
        else:
            assert rel2(got[th], ref[th]) <= ADJ_TOL, (what, th, rel2(got[th], ref[th]))


@pytest.mark.parametrize("idx,scale", [(1, 0.1), (3, 0.1)])
def test_adjoint_vectors_viscoelastic_hex(product_lib, idx, scale):
    """dR/dtheta vectors of both staggered steps (config 1: derived Gc = 2 ft^2 l / E, so dR_phase/dl
    carries dGc/dl; config 3: input Gc)."""
    mesh, d, o, g, _ = make_pair(idx, scale, overrides=_tight)
    _prime(o, g, (0, 1), DT)
    for step in (0, 1):
        f_before = g.residual(step)
        ep_before = g.get_history(abi.HIST_PLASTIC_STRAIN)
        ro, _ = o.adjoint(step, full=True, dt=DT)
        rg, _ = g.adjoint(step, full=True, dt=DT)
        _cmp_theta(rg, ro, ("step", step))
        # nothing the adjoint reads is changed by it
        assert np.array_equal(g.residual(step), f_before)
        assert np.array_equal(g.get_history(abi.HIST_PLASTIC_STRAIN), ep_before)
    # the u-step depends on (A, n) only, the phase step on (Gc, l) only
    ru, _ = g.adjoint(0, full=True, dt=DT)
    rp, _ = g.adjoint(1, full=True, dt=DT)
    assert np.linalg.norm(ru[2]) > 0 and np.linalg.norm(ru[3]) > 0
    assert not ru[0].any() and not ru[1].any() and not rp[2].any() and not rp[3].any()


@pytest.mark.parametrize("dist,lumped,irr", [("Quadratic", False, "Hist"), ("Linear", True, "Penalty"),
                                             ("CZM", True, "Hist"), ("Linear2", False, "Penalty")])
def test_adjoint_phase_options(product_lib, dist, lumped, irr):
    """Phase-step derivatives under each distribution function, lumped capacity and the penalty
    irreversibility (which scales with the input Gc even when Gc is derived)."""
    def ov(d):
        d["properties"]["PhaseField"]["DistributionFunction"] = dist
        d["Models"]["PhaseField1"]["LumpedPFCapacity"] = lumped
        d["Models"]["PhaseField1"]["Irreversible"] = irr
    mesh, d, o, g, _ = make_pair(0, 0.125, overrides=ov)
    _prime(o, g, (0, 1), 1.0)
    ro, _ = o.adjoint(1, full=True, dt=1.0)
    rg, _ = g.adjoint(1, full=True, dt=1.0)
    _cmp_theta(rg, ro, (dist, lumped, irr))


def test_adjoint_per_material_sets(product_lib):
    """lambda^T dR/dtheta per material set of the batched specimens, a random lambda and lambda = 1."""
    mesh, d, o, g, _ = make_pair(4, 0.02, overrides=_tight)
    n_mats = len(d["B200"]["Specimens"])
    _prime(o, g, (0, 1), DT)
    rng = np.random.default_rng(3)
    for step in (0, 1):
        n, _ = g.step_info(step)
        for lam in (rng.standard_normal(n), None):
            _, lo = o.adjoint(step, lam=lam, dt=DT, n_mats=n_mats)
            full, lg = g.adjoint(step, lam=lam, full=True, dt=DT, n_mats=n_mats)
            lo, lg = lo.reshape(n_mats, 4), lg.reshape(n_mats, 4)
            lv = np.ones(n) if lam is None else lam
            for th in range(4):
                if not lo[:, th].any():
                    assert not lg[:, th].any(), (step, th)
                    continue
                # lambda = 1 sums the u-step residual to (analytically) zero, so the error is measured
                # against the magnitude of the summed terms, sum_i |lambda_i dR_i/dtheta|
                scale = np.abs(lv) @ np.abs(full[th])
                err = np.abs(lg[:, th] - lo[:, th]).max()
                assert err <= ADJ_TOL * scale, (step, th, err / scale)
                # the per-set sums add up to the shared-parameter derivative
                assert abs(lg[:, th].sum() - lv @ full[th]) <= 1e-12 * scale, (step, th)


def test_adjoint_as_autograd_function(product_lib):
    """The adjoint as the backward of a torch.autograd.Function over the material parameters: the
    gradient of lambda^T R(theta) equals lambda^T dR/dtheta."""
    torch = pytest.importorskip("torch")
    mesh, d, o, g, _ = make_pair(4, 0.02, overrides=_tight)
    n_mats = len(d["B200"]["Specimens"])
    _prime(o, g, (0, 1), DT)
    step = 0
    n, _ = g.step_info(step)
    lam = np.random.default_rng(5).standard_normal(n)
    mats = [(m.gc, m.pf_l, m.creep_a, m.creep_n) for m in
            __import__("ice_fem_2025a_b200.config", fromlist=["materials"]).materials(d)]

    class Residual(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            for mi in range(n_mats):
                for k in range(4):
                    g.set_param(mi, k, float(theta[mi, k]))
            g.assemble(step, dt=DT)
            return torch.from_numpy(g.residual(step))

        @staticmethod
        def backward(ctx, grad_out):
            _, lr = g.adjoint(step, lam=grad_out.numpy(), dt=DT, n_mats=n_mats)
            return torch.from_numpy(lr.reshape(n_mats, 4))

    # re-assembling with unchanged parameters only re-converges the warm-started return map
    theta = torch.tensor(mats, dtype=torch.float64, requires_grad=True)
    r = Residual.apply(theta)
    (torch.from_numpy(lam) * r).sum().backward()
    _, lo = o.adjoint(step, lam=lam, dt=DT, n_mats=n_mats)
    full, _ = g.adjoint(step, full=True, dt=DT, n_mats=n_mats)
    got, ref = theta.grad.numpy(), lo.reshape(n_mats, 4)
    for th in range(4):
        scale = np.abs(lam) @ np.abs(full[th])
        assert np.abs(got[:, th] - ref[:, th]).max() <= ADJ_TOL * max(scale, 1e-300), th
