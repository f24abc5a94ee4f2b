"""Device constraint application (Physics::Constraint / UpdateState) and staggered Newton solves through the
C-ABI, against the CPU oracle (needs a B200).

Bars: constrained pattern bit-exact; K_con as the tangent bars (FP64 1e-10, FP32 1e-5); f_con 1e-10 (FP64
tangent) / 1e-6 (FP32 tangent, whose values enter through K C C_v); converged fields 1e-8 relative.  An
FP32-accurate tangent turns Newton's quadratic convergence into a linear one with a rate of about
cond(K) * 1e-7, so the mixed-precision solves may take more iterations: at most 2n + 1 for the FP64
tangent's n.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, newton
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu


def _pair(idx, scale, prec, overrides=None, strain=1.0e-3):
    mesh, d, o, g, _ = make_pair(idx, scale, prec=prec, overrides=overrides)
    ax = mesh.dim - 1
    H = np.ptp(mesh.coords[:, ax])
    dofs, vals = newton.box_constraints(o, mesh, strain * H)
    return mesh, o, g, dofs, vals


def _tight(d):
    d["B200"]["ReturnMapTolerance"] = "tight"


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32])
def test_constrain_matches_oracle(product_lib, prec):
    mesh, o, g, dofs, vals = _pair(0, 0.125, prec)
    f32 = prec != abi.PREC_FP64
    for ctx in (o, g):
        ctx.set_constraints(0, dofs, vals)
        ctx.set_constraints(1, [], [])
        for s in (0, 1):
            ctx.assemble(s)
            ctx.constrain(s)
    for s in (0, 1):
        assert o.constrained_info(s) == g.constrained_info(s)
        ro, co = o.constrained_pattern(s)
        rg, cg = g.constrained_pattern(s)
        assert np.array_equal(ro, rg) and np.array_equal(co, cg)
        fo, ko = o.constrained(s)
        fg, kg = g.constrained(s, abi.F32 if f32 else abi.F64)
        assert rel2(kg.astype(np.float64), ko) <= (1e-5 if f32 else 1e-10), s
        assert rel2(fg, fo) <= (1e-6 if f32 else 1e-10), (s, rel2(fg, fo))
    # no constraints: f_con = -f, K_con = K
    assert np.array_equal(g.constrained(1)[0], -g.residual(1))
    # UpdateState with the same increment
    n_free, _ = g.constrained_info(0)
    dx = np.random.default_rng(1).standard_normal(n_free) * 1e-7
    u0 = g.get_state(0, abi.STATE_CUR)
    o.set_state(0, abi.STATE_CUR, u0)
    o.assemble(0)
    o.constrain(0)
    for ctx in (o, g):
        ctx.update_state(0, dx)
    assert np.array_equal(g.get_state(0, abi.STATE_CUR), o.get_state(0, abi.STATE_CUR))


def _run(ctx, mesh, dofs, vals, n_steps, dt, strain0=1.0e-3, dstrain=2.0e-4):
    solver = newton.StaggeredNewton(ctx, {0: (dofs, vals)})
    its, fields = [], []
    for k in range(n_steps):
        logs = solver.solve_time_step(t=k * dt, dt=dt)
        assert all(lg.converged for lg in logs), [lg.errors for lg in logs]
        its.append([lg.iterations for lg in logs])
        fields.append([ctx.get_state(s, abi.STATE_CUR) for s in range(ctx.nsteps)])
        ctx.commit(2)
        H = np.ptp(mesh.coords[:, mesh.dim - 1])
        dofs, vals = newton.box_constraints(ctx, mesh, (strain0 + (k + 1) * dstrain) * H)
        solver.set_constraints({0: (dofs, vals)})
    return its, fields


def test_newton_2d_fields_and_iterations(product_lib):
    """Staggered Newton on the 2D tension specimen: FP64 and FP32-tangent GPU solves converge to the
    oracle's fields."""
    mesh, o, g64, dofs, vals = _pair(0, 0.25, abi.PREC_FP64)
    _, _, g32, _, _ = _pair(0, 0.25, abi.PREC_FP32)
    it_o, f_o = _run(o, mesh, dofs, vals, 2, 1.0)
    it_64, f_64 = _run(g64, mesh, dofs, vals, 2, 1.0)
    it_32, f_32 = _run(g32, mesh, dofs, vals, 2, 1.0)
    for k in range(2):
        for s in range(2):
            assert rel2(f_64[k][s], f_o[k][s]) <= 1e-8, (k, s, rel2(f_64[k][s], f_o[k][s]))
            assert rel2(f_32[k][s], f_o[k][s]) <= 1e-8, (k, s, rel2(f_32[k][s], f_o[k][s]))
    assert all(abs(a - b) <= 1 for ra, rb in zip(it_64, it_o) for a, b in zip(ra, rb)), (it_64, it_o)
    assert all(a <= 2 * b + 1 for ra, rb in zip(it_32, it_64) for a, b in zip(ra, rb)), (it_32, it_64)


def test_newton_hex_tc_split(product_lib):
    """The 3D damaged-viscoelastic hex under tension: the split-operand tensor-core tangent reaches the FP64
    tangent's fields.  The return map runs to the tight tolerance so that the global Newton converges
    past the local solver's error."""
    mesh, o, g64, dofs, vals = _pair(1, 0.125, abi.PREC_FP64, _tight, 1.0e-4)
    _, _, gtc, _, _ = _pair(1, 0.125, abi.PREC_TC_SPLIT, _tight, 1.0e-4)
    it_o, f_o = _run(o, mesh, dofs, vals, 2, 1.0, 1.0e-4, 2.0e-5)
    it_64, f_64 = _run(g64, mesh, dofs, vals, 2, 1.0, 1.0e-4, 2.0e-5)
    it_tc, f_tc = _run(gtc, mesh, dofs, vals, 2, 1.0, 1.0e-4, 2.0e-5)
    for k in range(2):
        for s in range(2):
            assert rel2(f_64[k][s], f_o[k][s]) <= 1e-8, (k, s, rel2(f_64[k][s], f_o[k][s]))
            assert rel2(f_tc[k][s], f_64[k][s]) <= 1e-8, (k, s, rel2(f_tc[k][s], f_64[k][s]))
    assert all(a <= 2 * b + 1 for ra, rb in zip(it_tc, it_64) for a, b in zip(ra, rb)), (it_tc, it_64)
