"""Viscoelastic-plastic (VEP) rheology on the GPU against the oracle (needs a B200).

The ice of the 2D and 3D workloads is made viscoelastic-plastic (SolidMaterial.cpp:303-521) with a yield
stress below the seeded stresses, so most integration points flow plastically and creep.  Two u-step
assemblies are checked, with a commit and a 5% larger displacement between them.  The second starts from the
committed hardening and the first one's multipliers.  Without the change of strain, the second trial stress
would be the first converged stress, which lies on the yield surface.  Round-off would then decide the
return map's elastic/plastic branch (SolidMaterial.cpp:395-403) differently on the two sides.  A context that
asks for the tensor-core tangent uses the FP32 CUDA-core tangent: the tensor-core path takes its inputs from the
sum-factorised points kernel, which has no VEP branch.

Bars as the parity tests: residual 1e-12; FP64 tangent 1e-10, FP32 1e-5; history 1e-10 relative.  The
multipliers converge linearly under the reference's stopping test, so the history differs from the oracle's by
about 1e-12 relative, not by round-off alone.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu


def _vep(sy=2.0e5, F=0.0, hard=0.0, plv=0.0):
    def ov(d):
        S = d["properties"]["Ice"]["SolidProperties"]
        S["Rheology"] = "ViscoElasticPlastic"
        S.setdefault("A", 2.4e-24)
        S.setdefault("n", 3.0)
        S["sy"], S["F_deg"], S["hardening"], S["pl_visc"] = sy, F, hard, plv
        d["properties"]["Ice"]["TemperatureDependent"]["sydeg"] = 0.0
    return ov


HIST_FIELDS = (abi.HIST_MAT, abi.HIST_PLASTIC_STRAIN, abi.HIST_VISC_DISS, abi.HIST_DAM_VISC_DISS)


def _next_step(o, g, state):
    for c in (o, g):
        c.commit(abi.COMMIT_TIMEDEP)
        c.set_state(0, abi.STATE_CUR, state[0][abi.STATE_CUR] * 1.05)


def _check(o, g, ktol, kdt):
    o.assemble(0, dt=100.0)
    g.assemble(0, dt=100.0)
    fo, fg = o.residual(0), g.residual(0)
    assert np.all(np.isfinite(fg))
    assert rel2(fg, fo) <= 1e-12, rel2(fg, fo)
    ko, kg = o.matrix_values(0), g.matrix_values(0, kdt).astype(np.float64)
    assert rel2(kg, ko) <= ktol, rel2(kg, ko)
    for fld in HIST_FIELDS:
        ho, hg = o.get_history(fld), g.get_history(fld)
        assert hg.shape == ho.shape
        assert rel2(hg, ho) <= 1e-10, (fld, rel2(hg, ho))
    return o.get_history(abi.HIST_MAT)


@pytest.mark.parametrize("idx,prec", [(1, abi.PREC_FP64), (1, abi.PREC_FP32), (1, abi.PREC_TC_SPLIT),
                                      (0, abi.PREC_FP64)])
def test_vep_parity(product_lib, idx, prec):
    mesh, d, o, g, state = make_pair(idx, 0.125, overrides=_vep(), prec=prec)
    kdt = abi.F64 if prec == abi.PREC_FP64 else abi.F32
    ktol = 1e-10 if prec == abi.PREC_FP64 else 1e-5
    mh = _check(o, g, ktol, kdt)
    nip = 27 if mesh.dim == 3 else 9
    mh = mh.reshape(mesh.n_elems * nip, 4)
    assert np.mean(mh[:, 2] != 0.0) > 0.5      # most ips flow plastically
    _next_step(o, g, state)
    _check(o, g, ktol, kdt)


def test_vep_hardening_friction_viscosity(product_lib):
    mesh, d, o, g, state = make_pair(1, 0.125, overrides=_vep(sy=2.0e5, F=20.0, hard=1e8, plv=1e6))
    mh = _check(o, g, 1e-10, abi.F64).reshape(-1, 4)
    assert np.any(mh[:, 0] > 0.0)                # hardening recorded
    _next_step(o, g, state)
    _check(o, g, 1e-10, abi.F64)


def test_vep_unsupported_paths(product_lib):
    mesh, d, o, g, _ = make_pair(1, 0.125, overrides=_vep())
    with pytest.raises(abi.IfemError) as e:
        g.adjoint(0, dt=100.0)
    assert e.value.code == abi.ERR_UNSUPPORTED
    # DamViscoElasticPlastic has no return map in the reference (SolidMaterial.cpp:185-188)
    from ice_fem_2025a_b200 import config as cf
    mesh, d, _ = cf.config(1, scale=0.125)
    _vep()(d)
    d["properties"]["Ice"]["SolidProperties"]["Rheology"] = "DamViscoElasticPlastic"
    with pytest.raises(abi.IfemError) as e:
        abi.product_context(mesh, cf.materials(d), cf.options_from_json(d))
    assert e.value.code == abi.ERR_UNSUPPORTED
