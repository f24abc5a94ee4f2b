"""Thermal Arrhenius coupling of the residual, dR/dT . dT (ifem_temperature_sensitivity), and the FP32 variant of
the adjoint, against central finite differences of the oracle's residual (needs a B200).

The temperature enters the displacement step through the creep factor A(T) = A0 exp(-Q/R (1/TAbs - 1/TRef)) of the
Glen return map and the phase-field step through the derived fracture energy Gc(T) = 2 ft(T)^2 l / E
(IceMaterial.cpp:49-84).  Cases: the 3D hex with the pinned temperature (a scalar derivative) and the 2D
thermomechanical slab with a temperature DOF (a nodal perturbation), with the phase step's reference-compatible
temperature read (every node at DOF 0, PhaseField.cpp:562-565) on and off.

At the melting clamp (TAbs = 273.15) the library's derivative is the one from below.

Bars: 1e-6 relative (2-norm) for the FP64 sensitivities (as the adjoint), 1e-5 for the FP32 variant.  The return map
runs with the tight tolerance so that the finite differences resolve the viscous strain's temperature dependence.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu

TOL64 = 1e-6
TOL32 = 1e-5


def _tight_ftdeg(d):
    d["B200"]["ReturnMapTolerance"] = "tight"
    d["properties"]["Ice"]["TemperatureDependent"]["ftdeg"] = 4.0e4   # Gc depends on T in the phase step


def _prime(o, g, steps, dt, du_dt=0.0):
    for s in steps:
        o.assemble(s, dt=dt, du_dt=du_dt)
        g.assemble(s, dt=dt, du_dt=du_dt)


@pytest.mark.parametrize("prec", [abi.F64, abi.F32])
def test_pinned_temperature_hex(product_lib, prec):
    mesh, d, o, g, _ = make_pair(1, 0.125, overrides=_tight_ftdeg)
    g.set_adjoint_precision(prec)
    _prime(o, g, (0, 1), 100.0)
    tol = TOL64 if prec == abi.F64 else TOL32
    for step in (0, 1):
        ro = o.temperature_sensitivity(step, None, dt=100.0)
        rg = g.temperature_sensitivity(step, None, dt=100.0)
        assert np.linalg.norm(ro) > 0, step
        assert rel2(rg, ro) <= tol, (step, rel2(rg, ro))


@pytest.mark.parametrize("ref_compat", [True, False])
def test_temperature_field_thermomechanical(product_lib, ref_compat):
    def ov(d):
        d["B200"]["ReturnMapTolerance"] = "tight"
        d["B200"]["RefCompatPhaseT"] = ref_compat
    mesh, d, o, g, state = make_pair(2, 1 / 32, overrides=ov)
    # the slab's base sits at 0 degC, the melting clamp of TAbs, where the derivative is one-sided: shift the
    # field 1 K below it so the central differences are smooth
    T = state[2][abi.STATE_CUR] - 1.0
    for c in (o, g):
        c.set_state(2, abi.STATE_CUR, T)
    _prime(o, g, (0, 1, 2), 10.0, 0.1)
    nT, _ = o.step_info(2)
    rng = np.random.default_rng(3)
    dT = 1.0 + 0.5 * np.sin(mesh.coords[:nT, 0] / 40.0) + 0.1 * rng.normal(size=nT)
    for step in (0, 1):
        ro = o.temperature_sensitivity(step, dT, dt=10.0, du_dt=0.1)
        rg = g.temperature_sensitivity(step, dT, dt=10.0, du_dt=0.1)
        assert np.linalg.norm(ro) > 0, step
        assert rel2(rg, ro) <= TOL64, (step, rel2(rg, ro))
    # the temperature step's own derivative is its tangent, not a sensitivity
    with pytest.raises(abi.IfemError):
        g.temperature_sensitivity(2, dT, dt=10.0)
    # a context with a T DOF needs the perturbation
    with pytest.raises(abi.IfemError):
        g.temperature_sensitivity(0, None, dt=10.0)


def test_fp32_adjoint_variant(product_lib):
    """The FP32 variant of dR/d(Gc, l, A, n): the full vectors on the 3D adjoint check mesh (input Gc), and
    lambda^T dR per material set on the batched specimens, whose creep factors A span several decades (the
    oracle's finite difference of a parameter shared by all sets steps every set by the same absolute amount, so
    the per-set derivatives are the comparable ones there)."""
    def tight(d):
        d["B200"]["ReturnMapTolerance"] = "tight"
    mesh, d, o, g, _ = make_pair(3, 0.1, overrides=tight)
    g.set_adjoint_precision(abi.F32)
    _prime(o, g, (0, 1), 100.0)
    for step in (0, 1):
        ro, _ = o.adjoint(step, full=True, dt=100.0)
        rg, _ = g.adjoint(step, full=True, dt=100.0)
        for th in range(4):
            if np.linalg.norm(ro[th]) == 0.0:
                assert np.linalg.norm(rg[th]) == 0.0, (step, th)
            else:
                assert rel2(rg[th], ro[th]) <= TOL32, (step, th, rel2(rg[th], ro[th]))
    mesh, d, o, g, _ = make_pair(4, 0.02, overrides=tight)
    g.set_adjoint_precision(abi.F32)
    _prime(o, g, (0, 1), 100.0)
    rng = np.random.default_rng(4)
    for step in (0, 1):
        n, _ = o.step_info(step)
        lam = rng.normal(size=n)
        _, lo = o.adjoint(step, lam=lam, dt=100.0)
        full, lg = g.adjoint(step, lam=lam, full=True, dt=100.0)
        lo, lg = lo.reshape(-1, 4), lg.reshape(-1, 4)
        for th in range(4):
            if not lo[:, th].any():
                assert not lg[:, th].any(), (step, th)
                continue
            # measured against the magnitude of the summed terms, sum_i |lambda_i dR_i/dtheta|, as the FP64 test
            scale = np.abs(lam) @ np.abs(full[th])
            err = np.abs(lg[:, th] - lo[:, th]).max()
            assert err <= TOL32 * scale, (step, th, err / scale)
