"""Every built energy split on the GPU against the oracle, in both steps (needs a B200).

PhaseFieldMaterial::EnergySplit (PhaseFieldMaterial.cpp:47-94) feeds the u-step's stresses and tangent, and
the phase step's driving energy through the history H = max(H_old, psi+).  Each split runs on the 2D and the
3D workload, with the energy-consistent stresses and without them (ConsistentEnergy false: stresses D eps).
SpecStress exists only without them; the reference throws otherwise.  Its psi+ comes from a 3x3 symmetric
eigen-decomposition.  SpecStrains and DruckerPrager (B_DP of both signs, which reach different regimes) have
full 6x6 split tangents and run on the general kernels; a tensor-core request there gets the FP32 tangent.

Bars as the parity tests: residuals 1e-12, FP64 tangents 1e-10, energy history 1e-12 relative.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu

CASES = [("None", True), ("None", False), ("VolStrains", True), ("VolStrains", False), ("VolStress", True),
         ("VolStress", False), ("StarConvex", True), ("ICE", True), ("ICE", False), ("SpecStress", False),
         ("SpecStrains", True), ("SpecStrains", False), ("DruckerPrager", True), ("DruckerPrager", False),
         ("DruckerPragerNeg", True)]


def _split(split, ce):
    def ov(d):
        F = d["properties"]["Ice"]["FractureProperties"]
        F["Split"] = "DruckerPrager" if split.startswith("DruckerPrager") else split
        F["B_DP"] = -0.3 if split == "DruckerPragerNeg" else 0.3
        F["StarConvexGamma"] = 0.5
        F["eRef"], F["cReduce"] = 1.0e-4, 0.5
        T = d["properties"]["Ice"]["TemperatureDependent"]
        T.setdefault("Ice_cReduceFact", 0.01)
        T.setdefault("Ice_eReduceFact", 1.0e-5)
        d["properties"]["PhaseField"]["ConsistentEnergy"] = ce
    return ov


@pytest.mark.parametrize("idx", [0, 1])
@pytest.mark.parametrize("split,ce", CASES)
def test_split_parity(product_lib, idx, split, ce):
    mesh, d, o, g, _ = make_pair(idx, 0.125, overrides=_split(split, ce))
    for step in (0, 1):
        o.assemble(step, dt=100.0)
        g.assemble(step, dt=100.0)
        fo, fg = o.residual(step), g.residual(step)
        assert np.all(np.isfinite(fg))
        assert rel2(fg, fo) <= 1e-12, (step, rel2(fg, fo))
        ko, kg = o.matrix_values(step), g.matrix_values(step, abi.F64)
        assert rel2(kg, ko) <= 1e-10, (step, rel2(kg, ko))
    eo, eg = o.get_history(abi.HIST_ENERGY), g.get_history(abi.HIST_ENERGY)
    assert rel2(eg, eo) <= 1e-12, rel2(eg, eo)


def test_specstress_needs_inconsistent_energy(product_lib):
    from ice_fem_2025a_b200 import config as cf
    mesh, d, _ = cf.config(1, scale=0.125)
    _split("SpecStress", True)(d)
    with pytest.raises(abi.IfemError) as e:
        abi.product_context(mesh, cf.materials(d), cf.options_from_json(d))
    assert e.value.code == abi.ERR_UNSUPPORTED


def test_full_split_with_tensor_core_request(product_lib):
    mesh, d, o, g, _ = make_pair(1, 0.125, overrides=_split("DruckerPrager", True), prec=abi.PREC_TC_SPLIT)
    o.assemble(0, dt=100.0)
    g.assemble(0, dt=100.0)
    assert rel2(g.residual(0), o.residual(0)) <= 1e-12
    assert rel2(g.matrix_values(0, abi.F32).astype(np.float64), o.matrix_values(0)) <= 1e-5
