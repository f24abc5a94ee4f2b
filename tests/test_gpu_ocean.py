"""OceanBC's u-step term on the GPU against the oracle (needs a B200).

OceanBCModel::Assemble_U (OceanBC.cpp:96-150) adds the water pressure rho g (hw - y) of each node on its ux row,
weighted by the phase-field lumped integral, after the phase-field model.  The water level is set inside the
domain (nodes above it get nothing) or above it, on the 2D workloads (configs 0 and 2) with their seeded phase
fields.  Bars: residual 1e-12 relative, tangent 1e-10 (the term has none); the slab-pipelined u-step equals one
pass bit for bit.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from tests.helpers import rel2
from tests.test_oracle_kat import _ocean

pytestmark = pytest.mark.gpu


def _pair(idx, hw_frac, prec=abi.PREC_FP64):
    from oracle import oracle as orc
    mesh, d, st = cf.config(idx, scale=0.125)
    y = mesh.coords[:, 1]
    _ocean(d, y.min() + hw_frac * (y.max() - y.min()))
    mats, opts = cf.materials(d), cf.options_from_json(d)
    opts.tangent_precision = prec
    o = orc.context(mesh, mats, opts)
    g = abi.product_context(mesh, mats, opts)
    s = st()
    cf.apply_state(o, s)
    cf.apply_state(g, s)
    return o, g


@pytest.mark.parametrize("idx,hw_frac", [(0, 0.6), (0, 1.5), (2, 0.4)])
def test_ocean_parity(product_lib, idx, hw_frac):
    o, g = _pair(idx, hw_frac)
    o.assemble(0, dt=100.0)
    g.assemble(0, dt=100.0)
    fo, fg = o.residual(0), g.residual(0)
    assert rel2(fg, fo) <= 1e-12, rel2(fg, fo)
    assert rel2(g.matrix_values(0), o.matrix_values(0)) <= 1e-10


def test_ocean_with_slabs_bit_identical(product_lib):
    _, one = _pair(0, 0.6, abi.PREC_FP32)
    _, sl = _pair(0, 0.6, abi.PREC_FP32)
    sl.set_readback_slabs(5)
    one.assemble(0, dt=100.0)
    sl.assemble(0, dt=100.0)
    assert np.array_equal(one.residual(0), sl.residual(0))
    assert np.array_equal(one.matrix_values(0, abi.F32), sl.matrix_values(0, abi.F32))


def test_ocean_3d_rejected(product_lib):
    mesh, d, st = cf.config(1, scale=0.125)
    _ocean(d, 0.3)
    with pytest.raises(abi.IfemError) as e:
        abi.product_context(mesh, cf.materials(d), cf.options_from_json(d))
    assert e.value.code == abi.ERR_UNSUPPORTED
