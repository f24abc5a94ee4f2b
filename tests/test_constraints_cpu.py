"""Constraint application and the staggered Newton harness on the CPU oracle.

The oracle's Physics::Constraint restatement is checked against the same algebra done with scipy on the full
system (K_con = K[free, free], f_con = -(f - K[:, con] C_v)[free]); the harness must converge and leave the
constrained dofs at their values.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, newton
from tests.helpers import make_pair, rel2


def _setup(scale=0.125):
    mesh, d, o, _, _ = make_pair(0, scale, gpu=False)
    H = np.ptp(mesh.coords[:, 1])
    dofs, vals = newton.box_constraints(o, mesh, 1.0e-3 * H)
    return mesh, o, dofs, vals


def test_oracle_constraint_algebra(oracle_lib):
    mesh, o, dofs, vals = _setup()
    step = 0
    o.set_constraints(step, dofs, vals)
    o.assemble(step)
    o.constrain(step)
    K = o.matrix(step).tocsr()
    f = o.residual(step)
    u = o.get_state(step, abi.STATE_CUR)
    n = f.size
    con = np.unique(dofs)
    free = np.setdiff1d(np.arange(n), con)
    cv_map = dict(zip(dofs.tolist(), vals.tolist()))
    cv = np.array([cv_map[c] for c in con]) - u[con]
    f_ref = -(f - K[:, con] @ cv)[free]
    K_ref = K[free][:, free].tocsr()
    K_ref.sort_indices()
    rp, ci = o.constrained_pattern(step)
    assert np.array_equal(rp, K_ref.indptr) and np.array_equal(ci, K_ref.indices)
    fc, vc = o.constrained(step)
    assert np.array_equal(vc, K_ref.data)
    assert rel2(fc, f_ref) <= 1e-14
    assert o.constrained_info(step) == (free.size, K_ref.nnz)
    # UpdateState: free dofs += dx, constrained dofs += C_v
    dx = np.random.default_rng(0).standard_normal(free.size) * 1e-6
    o.update_state(step, dx)
    u2 = o.get_state(step, abi.STATE_CUR)
    assert np.array_equal(u2[free], u[free] + dx)
    assert np.array_equal(u2[con], u[con] + cv)


def test_oracle_constraint_errors(oracle_lib):
    mesh, o, dofs, vals = _setup()
    with pytest.raises(abi.IfemError):
        o.set_constraints(0, [dofs[0], dofs[0]], [0.0, 1.0])      # doubly constrained, different values
    with pytest.raises(abi.IfemError):
        o.set_constraints(0, [10 ** 9], [0.0])                   # out of range
    o.set_constraints(0, [dofs[0], dofs[0]], [0.5, 0.5])          # equal duplicates merge
    n, _ = o.step_info(0)
    assert o.constrained_info(0)[0] == n - 1


def test_newton_harness_oracle(oracle_lib):
    mesh, o, dofs, vals = _setup()
    solver = newton.StaggeredNewton(o, {0: (dofs, vals)})
    # one u-step solve: equilibrium of the free dofs, constrained dofs at their values
    solver.err0, solver.errit0 = [None, None], [None, None]
    log = newton.StepLog()
    assert solver.solve_step_standard(0, (0.0, 1.0, 0.0, 0.0), log)
    u = o.get_state(0, abi.STATE_CUR)
    cmap = dict(zip(dofs.tolist(), vals.tolist()))
    assert np.abs(u[list(cmap)] - np.array(list(cmap.values()))).max() <= 1e-18
    f_free, _ = o.constrained(0, want_matrix=False)
    assert np.abs(f_free).max() <= 1e-9 * np.abs(o.residual(0)).max()
    # staggered time steps (one sweep per step, as the reference's max_outer_it = 1)
    for k in range(2):
        logs = solver.solve_time_step(t=float(k), dt=1.0)
        assert all(lg.converged for lg in logs), [lg.errors for lg in logs]
        assert 1 <= logs[0].iterations <= 8 and logs[1].iterations <= 4
        o.commit(2)
