"""Lagrange-multiplier irreversibility on the GPU against the oracle (needs a B200).

LagrangeMult, AugmentedLagrangeMult and AugmentedLagrangeMult2 (PhaseFieldUtil.cpp:350-484) add the DOFs
lMult_pf (and lMult_pf2) to the phase step (PhaseField.cpp:95-101).  The step's system becomes
[phase, L(, L2)] x nodes, coupled through nodal (diagonal) blocks.  The phase, old phase and multipliers are
set so that every branch of the methods occurs, away from its switching points.

Bars: DOF numbers and CSR pattern bit-exact; residual 1e-12; FP64 tangent 1e-10, FP32 1e-5.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from tests.helpers import rel2

pytestmark = pytest.mark.gpu

METHODS = ["LagrangeMult", "AugmentedLagrangeMult", "AugmentedLagrangeMult2"]


def _pair(method, idx, prec):
    from oracle import oracle as orc
    mesh, d, st = cf.config(idx, scale=0.125)
    model = next(k for k, v in d["Models"].items() if isinstance(v, dict) and v.get("Name") == "Fracture/PhaseField")
    d["Models"][model]["Irreversible"] = method
    ph_step = d["Dofs"]["DofStep"][d["Dofs"]["DofNames"].index("phase")]
    extra = ["lMult_pf"] + (["lMult_pf2"] if method == "AugmentedLagrangeMult2" else [])
    d["Dofs"]["DofNames"] = list(d["Dofs"]["DofNames"]) + extra
    d["Dofs"]["DofStep"] = list(d["Dofs"]["DofStep"]) + [ph_step] * len(extra)
    mats, opts = cf.materials(d), cf.options_from_json(d)
    opts.tangent_precision = prec
    o = orc.context(mesh, mats, opts)
    g = abi.product_context(mesh, mats, opts)
    s = st()
    n, _ = o.step_info(1)
    nn = mesh.n_nodes
    rng = np.random.default_rng(5)
    x = np.zeros(n)
    x[:nn] = rng.uniform(0.05, 0.9, nn)
    x[nn:] = rng.uniform(-0.6, 0.6, n - nn)
    old = x.copy()
    old[:nn] = x[:nn] + np.where(rng.random(nn) < 0.5, -0.05, 0.05)
    for c in (o, g):
        cf.apply_state(c, s)
        c.set_state(1, abi.STATE_CUR, x)
        c.set_state(1, abi.STATE_OLD, old)
    return mesh, o, g


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("idx,prec", [(0, abi.PREC_FP64), (1, abi.PREC_FP64), (1, abi.PREC_FP32)])
def test_lagrange_parity(product_lib, method, idx, prec):
    mesh, o, g = _pair(method, idx, prec)
    for kind in (abi.DOF_PHASE, abi.DOF_LMULT, abi.DOF_LMULT2):
        assert np.array_equal(o.dof_numbers(kind), g.dof_numbers(kind))
    assert o.step_info(1) == g.step_info(1)
    ro, co = o.pattern(1)
    rg, cg = g.pattern(1)
    assert np.array_equal(ro, rg) and np.array_equal(co, cg)
    kdt, ktol = (abi.F64, 1e-10) if prec == abi.PREC_FP64 else (abi.F32, 1e-5)
    for rep in range(2):
        for step in (0, 1):
            o.assemble(step, dt=100.0)
            g.assemble(step, dt=100.0)
            fo, fg = o.residual(step), g.residual(step)
            assert np.all(np.isfinite(fg))
            assert rel2(fg, fo) <= 1e-12, (step, rel2(fg, fo))
            ko, kg = o.matrix_values(step), g.matrix_values(step, kdt).astype(np.float64)
            assert rel2(kg, ko) <= ktol, (step, rel2(kg, ko))
        nn = mesh.n_nodes
        assert np.linalg.norm(fo[nn:]) > 0
        for c in (o, g):
            c.commit(abi.COMMIT_TIMEDEP)


def test_lagrange_adjoint_unsupported(product_lib):
    mesh, o, g = _pair("LagrangeMult", 0, abi.PREC_FP64)
    with pytest.raises(abi.IfemError) as e:
        g.adjoint(1, dt=100.0)
    assert e.value.code == abi.ERR_UNSUPPORTED
