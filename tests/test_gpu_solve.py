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

from ice_fem_2025a_b200 import abi, config as cf, newton
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


@pytest.mark.parametrize("idx,scale", [(0, 0.5), (1, 0.5), (2, 0.5)])
def test_amg_matches_direct(product_lib, idx, scale):
    """Smoothed-aggregation multigrid: the u-step solve reaches 1e-10 in a small fraction of the block-Jacobi
    iterations and gives SuperLU's dx; the phase step (constants as the near-null space) converges too."""
    import scipy.sparse.linalg as spla
    mesh, g, _, _ = _constrained(idx, scale, abi.PREC_FP64)
    for step in (0, 1):
        K = g.constrained_matrix(step)
        f, _ = g.constrained(step, want_matrix=False)
        ref = spla.spsolve(K.tocsc(), f)
        g.set_preconditioner(step, abi.PC_BLOCK_JACOBI)
        try:
            _, its_bj, _ = g.solve_constrained(step, rtol=1e-10, max_it=4000, restart=100)
        except abi.IfemError:
            its_bj = 4000
        g.set_preconditioner(step, abi.PC_AMG)
        dx, its, rr = g.solve_constrained(step, rtol=1e-10, max_it=2000, restart=100)
        sizes, ms = g.preconditioner_info(step)
        assert rr <= 1e-10 and np.linalg.norm(K @ dx - f) <= 2e-10 * np.linalg.norm(f)
        assert rel2(dx, ref) <= 1e-6, (step, rel2(dx, ref))
        assert sizes[0] == K.shape[0] and ms > 0
        if step == 0 and K.shape[0] > 20000:
            assert len(sizes) >= 2 and its * 4 <= its_bj, (sizes, its, its_bj)
        dx2, its2, _ = g.solve_constrained(step, rtol=1e-10, max_it=2000, restart=100)
        assert its2 == its and np.array_equal(dx2, dx)   # deterministic set-up and V-cycle


def test_amg_reuse_across_newton(product_lib):
    """PC_AMG_REUSE keeps the hierarchy of the first solve; the staggered Newton loop reaches the host-solve
    fields with it."""
    mesh, d, o, g_host, _ = make_pair(0, 0.25, prec=abi.PREC_FP64)
    _, _, _, g_dev, _ = make_pair(0, 0.25, prec=abi.PREC_FP64)
    H = np.ptp(mesh.coords[:, mesh.dim - 1])
    g_dev.set_preconditioner(0, abi.PC_AMG_REUSE)
    out = []
    for ctx, solve in ((g_host, newton.host_direct_solve), (g_dev, newton.device_gmres_solve)):
        dofs, vals = newton.box_constraints(ctx, mesh, 1.0e-3 * H)
        solver = newton.StaggeredNewton(ctx, {0: (dofs, vals)}, lin_solve=solve)
        logs = solver.solve_time_step(t=0.0, dt=1.0)
        assert all(lg.converged for lg in logs)
        out.append([ctx.get_state(s, abi.STATE_CUR) for s in range(ctx.nsteps)])
    for s in range(2):
        assert rel2(out[1][s], out[0][s]) <= 1e-8, (s, rel2(out[1][s], out[0][s]))
    assert g_dev.preconditioner_info(0)[0]


def test_amg_cosserat_rotations(product_lib):
    """The Cosserat u-step (ux, uy, uz, ox, oy, oz): the near-null space carries the micro-rotations with the
    rigid rotations; the solve gives SuperLU's dx."""
    import scipy.sparse.linalg as spla
    mesh, d, st = cf.cosserat_config(3, scale=0.25, rheology="LinearElastic", split="None")
    g = abi.product_context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(g, st())
    H = np.ptp(mesh.coords[:, 2])
    bot = np.where(mesh.coords[:, 2] <= mesh.coords[:, 2].min() + 1e-9 * H)[0]
    top = np.where(mesh.coords[:, 2] >= mesh.coords[:, 2].max() - 1e-9 * H)[0]
    dofs, vals = [], []
    for kind, nodes, v in ((abi.DOF_UX, bot, 0.0), (abi.DOF_UY, bot, 0.0), (abi.DOF_UZ, bot, 0.0),
                           (abi.DOF_UZ, top, -1e-3 * H)):
        num = g.dof_numbers(kind)[nodes]
        dofs.append(num); vals.append(np.full(num.size, v))
    dofs, vals = np.concatenate(dofs), np.concatenate(vals)
    o = np.argsort(dofs)
    g.set_constraints(0, dofs[o], vals[o])
    g.assemble(0, t=1.0, dt=0.1)
    g.constrain(0)
    K = g.constrained_matrix(0)
    f, _ = g.constrained(0, want_matrix=False)
    g.set_preconditioner(0, abi.PC_AMG)
    dx, its, rr = g.solve_constrained(0, rtol=1e-10, max_it=2000, restart=100)
    assert rel2(dx, spla.spsolve(K.tocsc(), f)) <= 1e-6
    g.close()


def test_amg_fp32_matrix_and_refusals(product_lib):
    """The multigrid set-up reads an FP32 K_con as well; a step with Lagrange-multiplier DOFs is refused."""
    import scipy.sparse.linalg as spla
    mesh, g, _, _ = _constrained(0, 0.5, abi.PREC_FP32)
    K = g.constrained_matrix(0)
    f, _ = g.constrained(0, want_matrix=False)
    g.set_preconditioner(0, abi.PC_AMG)
    dx, its, rr = g.solve_constrained(0, rtol=1e-10, max_it=2000, restart=100)
    assert its < 100 and rel2(dx, spla.spsolve(K.tocsc(), f)) <= 1e-6
    with pytest.raises(abi.IfemError) as e:
        g.set_preconditioner(0, 7)
    assert e.value.code == abi.ERR_INVALID
    # a strength threshold and three sweeps: a deeper hierarchy, still SuperLU's dx
    g.set_multigrid(0, 0.05, 3)
    dx3, its3, _ = g.solve_constrained(0, rtol=1e-10, max_it=2000, restart=100)
    assert its3 <= its and rel2(dx3, spla.spsolve(K.tocsc(), f)) <= 1e-6
    for bad in ((-0.1, 2), (1.0, 2), (0.0, 0), (0.0, 9)):
        with pytest.raises(abi.IfemError) as e:
            g.set_multigrid(0, *bad)
        assert e.value.code == abi.ERR_INVALID
    mesh, d, st = cf.config(0, scale=0.125)
    model = next(k for k, v in d["Models"].items() if isinstance(v, dict) and v.get("Name") == "Fracture/PhaseField")
    d["Models"][model]["Irreversible"] = "LagrangeMult"
    ph_step = d["Dofs"]["DofStep"][d["Dofs"]["DofNames"].index("phase")]
    d["Dofs"]["DofNames"] = list(d["Dofs"]["DofNames"]) + ["lMult_pf"]
    d["Dofs"]["DofStep"] = list(d["Dofs"]["DofStep"]) + [ph_step]
    h = abi.product_context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(h, st())
    h.set_constraints(1, np.zeros(0, np.int64), np.zeros(0))
    h.assemble(1, dt=1.0)
    h.constrain(1)
    h.set_preconditioner(1, abi.PC_AMG)
    with pytest.raises(abi.IfemError) as e:
        h.solve_constrained(1, rtol=1e-8, max_it=50)
    assert e.value.code == abi.ERR_UNSUPPORTED
    h.close()
