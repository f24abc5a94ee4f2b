"""The tensor-core tangent's per-element operand scaling over many orders of magnitude (needs a B200).

The split-operand tangent forms its FP16 hi/lo pairs after scaling the material tangents C_q and the shape
gradients G of each element by powers of two chosen from bounds of their largest magnitudes.  These cases
move both far from the benchmark's:
- the mesh size by 1e-3 and 1e+3 on the damaged viscoelastic ice: G scales with its inverse and the ip
  weights in C_q with its cube, so max |C_q| moves by 1e-9 and 1e+9;
- the stiffness by 1e-6 and 1e+6 on the same ice made linear elastic: C_q scales with it.  A viscous
  return map at a million times the stiffness does not converge, in the oracle either; elastic ice keeps
  the comparison on the tangent.
Bars as the parity tests: tangent 1e-5 relative (Frobenius) against the FP64 oracle, residual 1e-12.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from tests.helpers import rel2

pytestmark = pytest.mark.gpu


def _contexts(young_factor, length_factor):
    from oracle import oracle as orc
    mesh, d, st = cf.config(1, scale=0.125)
    if young_factor != 1.0:
        d["properties"]["Ice"]["SolidProperties"]["Young"] *= young_factor
        d["properties"]["Ice"]["SolidProperties"]["Rheology"] = "LinearElastic"
    mesh.coords = mesh.coords * length_factor
    mats = cf.materials(d)
    opts = cf.options_from_json(d)
    opts.tangent_precision = abi.PREC_TC_SPLIT
    o = orc.context(mesh, mats, opts)
    g = abi.product_context(mesh, mats, opts)
    state = st()
    cf.apply_state(o, state)
    cf.apply_state(g, state)
    return o, g


@pytest.mark.parametrize("young_factor,length_factor", [(1e-6, 1.0), (1e6, 1.0), (1.0, 1e-3), (1.0, 1e3)])
def test_tangent_scaling(product_lib, young_factor, length_factor):
    o, g = _contexts(young_factor, length_factor)
    o.assemble(0, dt=100.0)
    g.assemble(0, dt=100.0)
    fo, fg = o.residual(0), g.residual(0)
    assert np.all(np.isfinite(fg))
    assert rel2(fg, fo) <= 1e-12, rel2(fg, fo)
    ko = o.matrix_values(0)
    kg = g.matrix_values(0, abi.F32).astype(np.float64)
    assert np.all(np.isfinite(kg))
    assert rel2(kg, ko) <= 1e-5, rel2(kg, ko)
