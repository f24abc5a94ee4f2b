"""Device solve of the constrained Newton system (ifem_solve_constrained) against a direct sparse solve of the same
system, and the staggered Newton loop with it in place of the host solve (needs a B200).

The reference solves K_con dx = f_con with PETSc (GMRESLinSolver.cpp:19-96).  The library's solve is restarted
GMRES with a node-block Jacobi preconditioner on the device.  Bars: relative residual below the requested 1e-12,
checked again on the host with the FP64 K_con; dx within 1e-6 of SuperLU's (cond(K_con) times the residual);
repeated solves bitwise equal (fixed-order reductions); Newton fields within 1e-8 of the host-solve run, with the
same iteration counts to within one.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, newton
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu


def _constrained(idx, scale, prec):
    mesh, d, o, g, _ = make_pair(idx, scale, prec=prec)
    H = np.ptp(mesh.coords[:, mesh.dim - 1])
    dofs, vals = newton.box_constraints(g, mesh, 1.0e-3 * H)
    g.set_constraints(0, dofs, vals)
    g.set_constraints(1, np.zeros(0, np.int64), np.zeros(0))
    for step in (0, 1):
        g.assemble(step, dt=1.0)
        g.constrain(step)
    return mesh, g, dofs, vals


@pytest.mark.parametrize("idx,scale,prec", [(0, 0.25, abi.PREC_FP64), (0, 0.25, abi.PREC_FP32),
                                            (1, 0.125, abi.PREC_FP64)])
def test_solve_matches_direct(product_lib, idx, scale, prec):
    import scipy.sparse.linalg as spla
    mesh, g, _, _ = _constrained(idx, scale, prec)
    for step in (0, 1):
        dx, its, rr = g.solve_constrained(step, rtol=1e-12, max_it=20000, restart=100)
        K = g.constrained_matrix(step)
        f, _ = g.constrained(step, want_matrix=False)
        assert rr <= 1e-12 and its > 0
        assert np.linalg.norm(K @ dx - f) <= 2e-12 * np.linalg.norm(f)
        ref = spla.spsolve(K.tocsc(), f)
        assert rel2(dx, ref) <= 1e-6, (step, rel2(dx, ref))
        dx2, its2, rr2 = g.solve_constrained(step, rtol=1e-12, max_it=20000, restart=100)
        assert its2 == its and np.array_equal(dx2, dx)


def test_newton_with_device_solve(product_lib):
    mesh, d, o, g_host, _ = make_pair(0, 0.25, prec=abi.PREC_FP64)
    _, _, _, g_dev, _ = make_pair(0, 0.25, prec=abi.PREC_FP64)
    H = np.ptp(mesh.coords[:, mesh.dim - 1])
    out = []
    for ctx, solve in ((g_host, newton.host_direct_solve), (g_dev, newton.device_gmres_solve)):
        dofs, vals = newton.box_constraints(ctx, mesh, 1.0e-3 * H)
        solver = newton.StaggeredNewton(ctx, {0: (dofs, vals)}, lin_solve=solve)
        its, fields = [], []
        for k in range(2):
            logs = solver.solve_time_step(t=k * 1.0, dt=1.0)
            assert all(lg.converged for lg in logs)
            its.append([lg.iterations for lg in logs])
            fields.append([ctx.get_state(s, abi.STATE_CUR) for s in range(ctx.nsteps)])
            ctx.commit(2)
            dofs, vals = newton.box_constraints(ctx, mesh, (1.0e-3 + (k + 1) * 2.0e-4) * H)
            solver.set_constraints({0: (dofs, vals)})
        out.append((its, fields))
    (it_h, f_h), (it_d, f_d) = out
    for k in range(2):
        for s in range(2):
            assert rel2(f_d[k][s], f_h[k][s]) <= 1e-8, (k, s, rel2(f_d[k][s], f_h[k][s]))
    assert all(abs(a - b) <= 1 for ra, rb in zip(it_d, it_h) for a, b in zip(ra, rb)), (it_d, it_h)


def test_solve_errors(product_lib):
    mesh, d, o, g, _ = make_pair(0, 0.25, prec=abi.PREC_FP64)
    H = np.ptp(mesh.coords[:, mesh.dim - 1])
    dofs, vals = newton.box_constraints(g, mesh, 1.0e-3 * H)
    g.set_constraints(0, dofs, vals)
    g.assemble(0, dt=1.0)
    with pytest.raises(abi.IfemError) as e:          # no constrained system yet
        g.solve_constrained(0)
    assert e.value.code == abi.ERR_STATE
    g.constrain(0)
    with pytest.raises(abi.IfemError) as e:          # tolerance out of reach in 3 iterations
        g.solve_constrained(0, rtol=1e-14, max_it=3, restart=10)
    assert e.value.code == abi.ERR_NUMERIC
