"""GPU vs CPU-oracle parity through the C-ABI (needs a B200).

Bars: index maps bit-exact; FP64 residual <= 1e-12 relative (2-norm);
FP32 tangent <= 1e-5 relative (Frobenius); FP64 tangent and history <= 1e-10 relative.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu

RES_TOL = 1e-12
K64_TOL = 1e-10
K32_TOL = 1e-5


def _check_step(o, g, step, dt=1.0, du_dt=0.0, ddu_dt=0.0, ktol=K64_TOL, f32=False):
    o.assemble(step, dt=dt, du_dt=du_dt, ddu_dt=ddu_dt)
    g.assemble(step, dt=dt, du_dt=du_dt, ddu_dt=ddu_dt)
    fo, fg = o.residual(step), g.residual(step)
    assert np.all(np.isfinite(fg))
    assert rel2(fg, fo) <= RES_TOL, (step, rel2(fg, fo))
    _, nnz = o.step_info(step)
    if nnz:
        ko = o.matrix_values(step)
        kg = g.matrix_values(step, abi.F32 if f32 else abi.F64).astype(np.float64)
        assert rel2(kg, ko) <= ktol, (step, rel2(kg, ko))
    return fo, fg


@pytest.mark.parametrize("idx,scale", [(0, 0.125), (1, 0.125), (2, 1 / 32), (4, 0.02)])
def test_dofs_and_pattern_bit_exact(product_lib, idx, scale):
    mesh, d, o, g, _ = make_pair(idx, scale)
    for kind in range(5):
        assert np.array_equal(o.dof_numbers(kind), g.dof_numbers(kind))
    for s in range(o.nsteps):
        assert o.step_info(s) == g.step_info(s)
        ro, co = o.pattern(s)
        rg, cg = g.pattern(s)
        assert np.array_equal(ro, rg) and np.array_equal(co, cg)


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32])
def test_config0_le_at2(product_lib, prec):
    mesh, d, o, g, _ = make_pair(0, 0.125, prec=prec)
    f32 = prec != abi.PREC_FP64
    for _ in range(2):
        _check_step(o, g, 0, ktol=K32_TOL if f32 else K64_TOL, f32=f32)
        _check_step(o, g, 1, ktol=K32_TOL if f32 else K64_TOL, f32=f32)
    assert abs(g.stats(1).crack_length - o.stats(1).crack_length) <= 1e-12 * abs(o.stats(1).crack_length)
    for field in (abi.HIST_ENERGY, abi.HIST_PLASTIC_STRAIN):
        assert rel2(g.get_history(field), o.get_history(field)) <= 1e-12


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32, abi.PREC_TC_SPLIT])
def test_config1_viscoelastic_hex(product_lib, prec):
    mesh, d, o, g, _ = make_pair(1, 0.125, prec=prec)
    f32 = prec != abi.PREC_FP64
    for it in range(3):          # stateful: each assembly warm-starts the return map
        _check_step(o, g, 0, dt=100.0, ktol=K32_TOL if f32 else K64_TOL, f32=f32)
        for field in (abi.HIST_PLASTIC_STRAIN, abi.HIST_MAT, abi.HIST_VISC_DISS):
            assert rel2(g.get_history(field), o.get_history(field)) <= 1e-10, (it, field)
        _check_step(o, g, 1, dt=100.0, ktol=K32_TOL if f32 else K64_TOL, f32=f32)
    so, sg = o.stats(0), g.stats(0)
    assert sg.rm_iterations > 0 and abs(sg.rm_iterations - so.rm_iterations) <= 0.01 * so.rm_iterations


def test_config2_thermomechanical(product_lib):
    mesh, d, o, g, _ = make_pair(2, 1 / 32)
    for step in (0, 1, 2):
        _check_step(o, g, step, dt=10.0, du_dt=0.1)


def test_config4_batched_materials(product_lib):
    mesh, d, o, g, _ = make_pair(4, 0.02)
    for step in (0, 1):
        _check_step(o, g, step, dt=100.0)


def test_full_extraction_operators(product_lib):
    """elem_data input: factorisable operators (kron path) and a non-factorisable perturbation
    (full-operator path) both match the oracle."""
    mesh, d, o, g, _ = make_pair(1, 0.125, use_kron=False)
    _check_step(o, g, 0, dt=100.0)
    from ice_fem_2025a_b200 import config as cf
    from oracle import oracle as orc
    mesh2, d2, st = cf.config(0, scale=0.125)
    full = mesh2.elem_data().copy()
    full[:, 0, 1] += 1e-3     # breaks the Kronecker structure -> full-operator kernels
    mesh2.full_data = full
    m = mesh2
    mats, opts = cf.materials(d2), cf.options_from_json(d2)
    o2 = orc.context(m, mats, opts, use_kron=False)
    g2 = abi.product_context(m, mats, opts, use_kron=False)
    s = st()
    cf.apply_state(o2, s)
    cf.apply_state(g2, s)
    _check_step(o2, g2, 0)
    _check_step(o2, g2, 1)


@pytest.mark.parametrize("prec", [abi.PREC_FP32, abi.PREC_TC_SPLIT])
def test_deterministic_bitwise(product_lib, prec):
    mesh, d, o, g, _ = make_pair(1, 0.125, prec=prec, gpu=True)
    g.assemble(0, dt=100.0)
    g.reset_step()
    g.assemble(0, dt=100.0)
    f1, k1 = g.residual(0), g.matrix_values(0, abi.F32)
    g.reset_step()
    g.assemble(0, dt=100.0)
    g.reset_step()
    g.assemble(0, dt=100.0)
    f2, k2 = g.residual(0), g.matrix_values(0, abi.F32)
    assert np.array_equal(f1.view(np.uint64), f2.view(np.uint64))
    assert np.array_equal(k1.view(np.uint32), k2.view(np.uint32))


def test_commit_reset_history(product_lib):
    mesh, d, o, g, state = make_pair(1, 0.125)
    for c in (o, g):
        c.assemble(0, dt=100.0)
        c.commit()
        U = c.get_state(0, abi.STATE_CUR)
        c.set_state(0, abi.STATE_CUR, U * 1.5)
        c.assemble(0, dt=100.0)
        c.reset_step()
    for field in range(5):
        assert rel2(g.get_history(field), o.get_history(field)) <= 1e-10
        assert rel2(g.get_history(field, old=1), o.get_history(field, old=1)) <= 1e-10


def test_nonfinite_state_reports_numeric_error(product_lib):
    mesh, d, o, g, state = make_pair(0, 0.125)
    U = g.get_state(0, abi.STATE_CUR)
    U[3] = np.nan
    g.set_state(0, abi.STATE_CUR, U)
    with pytest.raises(abi.IfemError) as ei:
        g.assemble(0)
    assert ei.value.code == abi.ERR_NUMERIC


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_TC_SPLIT])
def test_consistent_tangent_hex(product_lib, prec):
    """The consistent tangent (exact Jacobian of the converged return map) against the oracle's, whose
    consistency is pinned by central finite differences of its residual on the CPU."""
    def tight(d):
        d["B200"]["ReturnMapTolerance"] = "tight"
    mesh, d, o, g, _ = make_pair(1, 0.125, prec=prec, tangent=abi.TANGENT_CONSISTENT, overrides=tight)
    f32 = prec != abi.PREC_FP64
    for _ in range(2):
        _check_step(o, g, 0, dt=100.0, ktol=K32_TOL if f32 else 1e-9, f32=f32)
    # the consistent and the reference tangent differ where the return map is active
    g.set_tangent(abi.TANGENT_REFERENCE, prec)
    g.assemble(0, dt=100.0)
    k_ref = g.matrix_values(0, abi.F32 if f32 else abi.F64).astype(np.float64)
    g.set_tangent(abi.TANGENT_CONSISTENT, prec)
    g.assemble(0, dt=100.0)
    k_con = g.matrix_values(0, abi.F32 if f32 else abi.F64).astype(np.float64)
    assert rel2(k_con, k_ref) > 1e-6
