"""Parity at the benchmark size: the 3D quadratic hex 32x32x64 mesh (65,536 elements, 27 ips), damaged Glen
viscoelastic ice, against the multi-threaded oracle on the same mesh and state.

At this size every persistent CTA of the tensor-core tangent processes about 443 elements, so the double-buffered
TMEM operand, the triple-buffered table and operand rings and the mbarrier parity wrap all run many times, as in
the benchmark.  The displacement alternates between two nearby fields, so each assembly warm-starts the return map
from the previous one (SolidMaterial.cpp:209-210), as consecutive Newton iterations do.

Bars: residual <= 1e-12 relative (2-norm); tangent <= 1e-5 (FP32-accurate tensor-core split) and <= 1e-10 (FP64)
relative in the Frobenius norm; history <= 1e-10; crack length <= 1e-12.
"""
import os

import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu

DT = 100.0


def _compare(o, g, step, ktol, f32):
    fo, fg = o.residual(step), g.residual(step)
    assert np.all(np.isfinite(fg))
    rf = rel2(fg, fo)
    ko = o.matrix_values(step)
    kg = g.matrix_values(step, abi.F32 if f32 else abi.F64).astype(np.float64)
    rk = rel2(kg, ko)
    assert rf <= 1e-12, (step, rf)
    assert rk <= ktol, (step, rk)
    return rf, rk


def test_config1_full_size_tensor_core_and_fp64(product_lib):
    mesh, d, o, g, state = make_pair(1, 1.0, prec=abi.PREC_TC_SPLIT)
    assert mesh.n_elems == 65536
    nthreads = os.cpu_count() or 1
    U0 = state[0][abi.STATE_CUR]
    U1 = U0 * (1.0 + 1e-3)
    # tensor-core split tangent twice (two warm starts), then the plain FP64 tangent
    for it, prec in enumerate((abi.PREC_TC_SPLIT, abi.PREC_TC_SPLIT, abi.PREC_FP64)):
        g.set_tangent(abi.TANGENT_REFERENCE, prec)
        U = U1 if it % 2 else U0
        for c in (o, g):
            c.set_state(0, abi.STATE_CUR, U)
        o.assemble_mt(0, nthreads, dt=DT)
        g.assemble(0, dt=DT)
        f32 = prec != abi.PREC_FP64
        _compare(o, g, 0, 1e-5 if f32 else 1e-10, f32)
        for field in (abi.HIST_PLASTIC_STRAIN, abi.HIST_MAT, abi.HIST_VISC_DISS, abi.HIST_DAM_VISC_DISS):
            assert rel2(g.get_history(field), o.get_history(field)) <= 1e-10, (it, field)
        o.assemble_mt(1, nthreads, dt=DT)
        g.assemble(1, dt=DT)
        _compare(o, g, 1, 1e-5 if f32 else 1e-10, f32)
        assert rel2(g.get_history(abi.HIST_ENERGY), o.get_history(abi.HIST_ENERGY)) <= 1e-10
        lo, lg = o.stats(1).crack_length, g.stats(1).crack_length
        assert abs(lg - lo) <= 1e-12 * abs(lo), (lg, lo)
    o.close()
    g.close()
