"""GPU vs oracle parity of the phase-field model options that change the assembled physics.

Each case switches one reference input on (or to another value) and assembles the displacement step and the
phase-field step twice in a row, on the 2D B2_2 mesh (general kernels) and on the 3D hex (sum-factorised
kernels, and the tensor-core tangent where the u-step tangent changes):

  Intertia with velocities / accelerations, SolidProperties/Damping   PhaseField.cpp:436-466
  DamFunction (all twelve), PhaseField/p for Porder                   PhaseFieldUtil.cpp:24-25, 77-183
  DensityDamage with inertia, gravity and ConsistentDegradation       PhaseField.cpp:241-255, 466-472, 666-676
  ViscoDriving / ViscoDrivingFactor                                   PhaseField.cpp:258-268, 657-664
  LumpedDriving, LumpedPFCapacity                                     PhaseField.cpp:644-656, 692-706
  DistributionFunction (residual and tangent of all ten, the second-gradient ones included)
                                                                      PhaseFieldUtil.cpp:185-348
  FractureProperties/Viscosity and ViscousStab                        PhaseField.cpp:708-710

Bars as in the other parity tests: residual <= 1e-12 relative (2-norm), FP64 tangent <= 1e-10, FP32-accurate
tangent <= 1e-5 (Frobenius).
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu

RES_TOL = 1e-12
K64_TOL = 1e-10
K32_TOL = 1e-5

# time-scheme scalars and rate magnitudes chosen so the inertia and damping terms are a visible fraction of the
# elastic terms on both meshes
DU_DT, DDU_DT = 1.0e3, 1.0e9


def _pf(d):
    return d["properties"]["PhaseField"]


def _model(d):
    return d["Models"]["PhaseField1"]


def _ice(d):
    return d["properties"]["Ice"]


def _set(path_fn, key, value):
    def f(d):
        path_fn(d)[key] = value
    return f


def _all(*fns):
    def f(d):
        for fn in fns:
            fn(d)
    return f


def _vep(d):
    S = _ice(d)["SolidProperties"]
    S["Rheology"] = "ViscoElasticPlastic"
    S.setdefault("A", 2.4e-24)
    S.setdefault("n", 3.0)
    S["sy"], S["F_deg"], S["hardening"], S["pl_visc"] = 2.0e5, 0.0, 0.0, 0.0
    _ice(d)["TemperatureDependent"]["sydeg"] = 0.0


INERTIA = _all(_set(_model, "Intertia", True), _set(_pf, "DensityDamage", "Quadratic"))
CASES = {
    "inertia": INERTIA,
    "damping": _all(lambda d: _ice(d)["SolidProperties"].__setitem__("Damping", 1.0e9)),
    "inertia_gravity_consistent_degradation": _all(INERTIA, _set(_model, "Gravity", True),
                                                    _set(_pf, "ConsistentDegradation", True)),
    "lumped_driving": _set(_model, "LumpedDriving", True),
    "lumped_capacity": _set(_model, "LumpedPFCapacity", True),
    "pf_viscosity_and_stabilisation": _all(lambda d: _ice(d)["FractureProperties"].__setitem__("Viscosity", 1.0e4),
                                           _set(_model, "ViscousStab", 1.0e-3)),
    # the plastic dissipation that drives the phase field comes from the viscoelastic-plastic return map
    # (DamDissRate, SolidMaterial.cpp:303-445); the other rheologies leave it zero
    "visco_driving": _all(_vep, _set(_pf, "ViscoDriving", "Quadratic"), _set(_pf, "ViscoDrivingFactor", 0.7)),
}
for _name in abi.DAM:
    CASES[f"dam_{_name}"] = _set(_pf, "DamFunction", _name)
for _p in (1.0, 2.5, 3.5):
    CASES[f"porder_p{_p}"] = _all(_set(_pf, "DamFunction", "Porder"), _set(_pf, "p", _p))
for _name in ("Linear", "Cubic", "CZM", "Porder"):
    CASES[f"density_damage_{_name}"] = _all(INERTIA, _set(_pf, "DensityDamage", _name), _set(_model, "Gravity", True),
                                            _set(_pf, "ConsistentDegradation", True), _set(_pf, "p", 2.5))
_COEFS = _set(_pf, "Coefs", [2.0, 0.5, 1.0, 0.5, 0.1])   # the Custom distribution's coefficients
for _name in abi.DIST:
    CASES[f"dist_{_name}"] = _all(_set(_pf, "DistributionFunction", _name), _COEFS)
    CASES[f"dist_{_name}_lumped"] = _all(_set(_pf, "DistributionFunction", _name), _COEFS,
                                         _set(_model, "LumpedPFCapacity", True))

# cases whose u-step tangent differs from the default one: also run through the tensor-core tangent in 3D
U_TANGENT_CASES = {"inertia", "damping", "inertia_gravity_consistent_degradation", "dam_Cubic", "dam_CZM",
                   "porder_p2.5", "density_damage_Cubic"}


def _rates(g, o, mesh, seed):
    """Nonzero velocities and accelerations of the displacement step (dStateVectors, ddStateVectors)."""
    rng = np.random.default_rng(seed + 7)
    n, _ = o.step_info(0)
    du = rng.normal(0.0, 1.0, n)
    ddu = rng.normal(0.0, 1.0e4, n)
    for c in (o, g):
        c.set_state(0, abi.STATE_D, du)
        c.set_state(0, abi.STATE_DD, ddu)


def _run(case, idx, prec):
    mesh, d, o, g, _ = make_pair(idx, 0.125, overrides=CASES[case], prec=prec)
    _rates(g, o, mesh, 0)
    dt = 100.0 if idx == 1 else 1.0
    f32 = prec != abi.PREC_FP64
    for it in range(2):
        for step in (0, 1):
            for c in (o, g):
                c.assemble(step, dt=dt, du_dt=DU_DT, ddu_dt=DDU_DT)
            fo, fg = o.residual(step), g.residual(step)
            assert np.all(np.isfinite(fg)), (case, step)
            assert rel2(fg, fo) <= RES_TOL, (case, it, step, rel2(fg, fo))
            ko = o.matrix_values(step)
            kg = g.matrix_values(step, abi.F32 if f32 and step == 0 else abi.F64).astype(np.float64)
            tol = K32_TOL if f32 else K64_TOL
            assert rel2(kg, ko) <= tol, (case, it, step, rel2(kg, ko))
        for field in (abi.HIST_ENERGY, abi.HIST_PLASTIC_STRAIN, abi.HIST_DAM_VISC_DISS):
            assert rel2(g.get_history(field), o.get_history(field)) <= 1e-10, (case, it, field)
    assert abs(g.stats(1).crack_length - o.stats(1).crack_length) <= 1e-12 * abs(o.stats(1).crack_length)
    o.close()
    g.close()


@pytest.mark.parametrize("case", sorted(CASES))
def test_option_2d(product_lib, case):
    _run(case, 0, abi.PREC_FP64)


@pytest.mark.parametrize("case", sorted(CASES))
def test_option_3d_hex(product_lib, case):
    _run(case, 1, abi.PREC_FP64)


@pytest.mark.parametrize("case", sorted(U_TANGENT_CASES))
def test_option_3d_hex_tensor_core_tangent(product_lib, case):
    _run(case, 1, abi.PREC_TC_SPLIT)


def test_ref_compat_phase_t_off(product_lib):
    """Thermomechanical slab with the phase step reading each node's own temperature (RefCompatPhaseT off)."""
    def off(d):
        d["B200"]["RefCompatPhaseT"] = False
    mesh, d, o, g, _ = make_pair(2, 1 / 32, overrides=off)
    assert o.opts.ref_compat_phase_t == 0
    for step in (0, 1, 2):
        for c in (o, g):
            c.assemble(step, dt=10.0, du_dt=0.1)
        assert rel2(g.residual(step), o.residual(step)) <= RES_TOL, step
        assert rel2(g.matrix_values(step), o.matrix_values(step)) <= K64_TOL, step
    # the switch changes the phase step where the temperature varies
    on = lambda d: None
    _, _, o2, _, _ = make_pair(2, 1 / 32, overrides=on, gpu=False)
    for step in (0, 1):
        o2.assemble(step, dt=10.0, du_dt=0.1)
    assert rel2(o2.residual(1), o.residual(1)) > 1e-8
