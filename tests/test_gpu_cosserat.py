"""GPU vs oracle parity of the Cosserat model (Fracture/CossPhaseField, CossPhaseField.cpp:337-800) in 2D: the
u-step with micro-rotations (ux, uy, oz), the phase step driven by the Cosserat split and the T step's viscous
heating (needs a B200).

Cases: linear-elastic ice with each split the Cosserat material defines (None, SpecStress, DruckerPrager,
StarConvex, with energy-consistent stresses), and the damaged viscoelastic-plastic ice of the reference's
TriAxial2D input (SpecStress without consistent stresses, HO_Linear2, augmented Lagrange irreversibility,
inertia, damping, viscous heating), plus viscoelastic-plastic ice with the history irreversibility; FP64 and
FP32 tangents; the initialisation period (t < 0) and two assemblies in a row (warm-started return map).

Bars: residual <= 1e-12 relative (2-norm), tangent <= 1e-10 (FP64) / 1e-5 (FP32), history <= 1e-10.  The return
map runs to round-off ("tight"), so that both sides stop at the same converged state; with the reference's loose
stopping test (e/e0 < 1e-5) the two sides may stop one iteration apart at some ips.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from tests.helpers import rel2

pytestmark = pytest.mark.gpu

CASES = {
    "le_none": dict(rheology="LinearElastic", split="None", consistent=True),
    "le_specstress": dict(rheology="LinearElastic", split="SpecStress", consistent=True),
    "le_druckerprager": dict(rheology="LinearElastic", split="DruckerPrager", consistent=True),
    "le_starconvex": dict(rheology="LinearElastic", split="StarConvex", consistent=True),
    "dvep_triaxial2d": dict(rheology="DamViscoElasticPlastic", split="SpecStress", consistent=False),
    "vep_hist": dict(rheology="ViscoElasticPlastic", split="SpecStress", consistent=False, distribution="Quadratic",
                     irreversible="Hist"),
}


def _pair(case, prec, tight=True, scale=0.125):
    from oracle import oracle as orc
    kw = dict(CASES[case])
    consistent = kw.pop("consistent")
    mesh, d, st = cf.cosserat_config(2, scale=scale, **kw)
    d["properties"]["PhaseField"]["ConsistentEnergy"] = consistent
    if kw["split"] == "DruckerPrager":
        d["properties"]["Ice"]["FractureProperties"]["B_DP"] = 0.3
    if kw["split"] == "StarConvex":
        d["properties"]["Ice"]["FractureProperties"]["StarConvexGamma"] = 0.5
    if tight:
        d["B200"]["ReturnMapTolerance"] = "tight"
    mats, opts = cf.materials(d), cf.options_from_json(d)
    opts.tangent_precision = prec
    o = orc.context(mesh, mats, opts)
    g = abi.product_context(mesh, mats, opts)
    state = st()
    for c in (o, g):
        cf.apply_state(c, state)
    return mesh, d, o, g, state


def _compare(o, g, step, f32):
    fo, fg = o.residual(step), g.residual(step)
    assert np.all(np.isfinite(fg)), step
    assert rel2(fg, fo) <= 1e-12, (step, rel2(fg, fo))
    ko = o.matrix_values(step)
    kg = g.matrix_values(step, abi.F32 if f32 and step == 0 else abi.F64).astype(np.float64)
    assert rel2(kg, ko) <= (1e-5 if f32 else 1e-10), (step, rel2(kg, ko))


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32])
@pytest.mark.parametrize("case", sorted(CASES))
def test_cosserat_parity(product_lib, case, prec):
    mesh, d, o, g, state = _pair(case, prec)
    f32 = prec != abi.PREC_FP64
    kw = dict(dt=0.05, du_dt=20.0, ddu_dt=400.0)
    assert g.dof_numbers(abi.DOF_OZ).tolist() == o.dof_numbers(abi.DOF_OZ).tolist()
    for it, t in enumerate((-1.0, 1.0, 1.0)):
        if it == 2:   # a second assembly warm-starts the return map; move the displacement a little
            U = state[0][abi.STATE_CUR] * 1.02
            for c in (o, g):
                c.set_state(0, abi.STATE_CUR, U)
        for step in range(o.nsteps):
            for c in (o, g):
                c.assemble(step, t=t, **kw)
            _compare(o, g, step, f32)
        for field in (abi.HIST_ENERGY, abi.HIST_PLASTIC_STRAIN, abi.HIST_VISC_DISS, abi.HIST_DAM_VISC_DISS,
                      abi.HIST_MAT):
            ho, hg = o.get_history(field), g.get_history(field)
            assert rel2(hg, ho) <= 1e-10, (case, it, field, rel2(hg, ho))
    assert abs(g.stats(1).crack_length - o.stats(1).crack_length) <= 1e-12 * abs(o.stats(1).crack_length)
    for c in (o, g):
        c.commit()
    o.close()
    g.close()


def test_cosserat_reference_tolerance(product_lib):
    """The reference's own return-map tolerance on the TriAxial2D material: residual parity holds where both
    sides take the same iterations; the overall bar is the return map's own accuracy."""
    mesh, d, o, g, state = _pair("dvep_triaxial2d", abi.PREC_FP64, tight=False)
    for c in (o, g):
        c.assemble(0, t=1.0, dt=0.05, du_dt=20.0, ddu_dt=400.0)
    assert rel2(g.residual(0), o.residual(0)) <= 1e-6
    assert g.stats(0).rm_iterations > 0
    o.close()
    g.close()


def test_cosserat_unsupported_paths(product_lib):
    mesh, d, o, g, state = _pair("le_none", abi.PREC_FP64)
    with pytest.raises(abi.IfemError):
        g.adjoint(0, full=True, dt=0.1)
    o.close()
    g.close()
    mesh, d, st = cf.cosserat_config(2, scale=0.125, rheology="DamViscoElastic", split="SpecStress")
    with pytest.raises(abi.IfemError):
        abi.product_context(mesh, cf.materials(d), cf.options_from_json(d))
