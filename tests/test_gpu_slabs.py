"""Slab-pipelined displacement assembly (needs a B200).

`ifem_set_readback_slabs(n)` splits the u-step into n element slabs.  After each slab it gathers the rows whose
incident elements are all done, and `ifem_get_matrix` / `ifem_get_residual` copy those rows while later slabs
still compute.  Every launch sees the same inputs and the gather adds a row's element blocks in the same
ascending element order, so the residual and the CSR values equal the one-pass assembly bit for bit.  The
cases cover a structured box (rows complete slab by slab), a 2D mesh, a shuffled element order (most rows
complete only in the last slab), a slab count that does not divide the element count, both matrix precisions,
the converting read-back (which waits for the whole step) and the asynchronous two-step sequence of a
staggered solver.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf

pytestmark = pytest.mark.gpu


def _ctx(idx, scale, prec, slabs, shuffle_seed=None):
    mesh, d, st = cf.config(idx, scale=scale)
    if shuffle_seed is not None:
        perm = np.random.default_rng(shuffle_seed).permutation(mesh.elems.shape[0])
        mesh.elems = np.ascontiguousarray(mesh.elems[perm])
        mesh.elem_kron = np.ascontiguousarray(mesh.elem_kron[perm])
        if mesh.elem_mat is not None:
            mesh.elem_mat = np.ascontiguousarray(mesh.elem_mat[perm])
        if mesh.full_data is not None:
            mesh.full_data = np.ascontiguousarray(mesh.full_data[perm])
    opts = cf.options_from_json(d)
    opts.tangent_precision = prec
    g = abi.product_context(mesh, cf.materials(d), opts)
    cf.apply_state(g, st())
    if slabs != 1:
        g.set_readback_slabs(slabs)
    return g


def _outputs(g, step, kdtype):
    g.assemble(step, dt=100.0)
    return g.residual(step), g.matrix_values(step, kdtype), g.stats(step)


@pytest.mark.parametrize("idx,scale,prec,slabs,shuffle", [
    (1, 0.25, abi.PREC_TC_SPLIT, 4, None),
    (1, 0.25, abi.PREC_TC_SPLIT, 7, None),
    (1, 0.125, abi.PREC_FP64, 4, None),
    (1, 0.125, abi.PREC_FP32, 16, None),
    (1, 0.125, abi.PREC_TC_SPLIT, 4, 3),
    (0, 0.125, abi.PREC_FP64, 3, None),
])
def test_slabs_bit_identical(product_lib, idx, scale, prec, slabs, shuffle):
    kdt = abi.F64 if prec == abi.PREC_FP64 else abi.F32
    one = _ctx(idx, scale, prec, 1, shuffle)
    sl = _ctx(idx, scale, prec, slabs, shuffle)
    f1, k1, s1 = _outputs(one, 0, kdt)
    fs, ks, ss = _outputs(sl, 0, kdt)
    assert np.all(np.isfinite(fs)) and np.all(np.isfinite(ks))
    assert np.array_equal(f1, fs)
    assert np.array_equal(k1, ks)
    assert s1.rm_iterations == ss.rm_iterations
    # converting read-back of the slabbed step (waits for the whole step)
    other = abi.F32 if kdt == abi.F64 else abi.F64
    assert np.array_equal(one.matrix_values(0, other), sl.matrix_values(0, other))
    # the phase step is not slabbed and follows as before
    p1, q1, _ = _outputs(one, 1, kdt)
    ps, qs, _ = _outputs(sl, 1, kdt)
    assert np.array_equal(p1, ps) and np.array_equal(q1, qs)


def test_slabs_async_staggered_sequence(product_lib):
    one = _ctx(1, 0.25, abi.PREC_TC_SPLIT, 1)
    sl = _ctx(1, 0.25, abi.PREC_TC_SPLIT, 4)
    out = []
    for g in (one, sl):
        nu, zu = g.step_info(0)
        npp, zp = g.step_info(1)
        fu, ku = np.empty(nu), np.empty(zu, np.float32)
        fp, kp = np.empty(npp), np.empty(zp, np.float32)
        for _ in range(2):
            g.assemble_async(0, dt=100.0)
            g.assemble_async(1, dt=100.0)
            g.matrix_into(0, ku)
            g.residual_into(0, fu)
            g.matrix_into(1, kp)
            g.residual_into(1, fp)
            g.sync(0)
            g.sync(1)
        out.append((fu, ku, fp, kp))
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_slabs_argument_checks(product_lib):
    g = _ctx(1, 0.125, abi.PREC_TC_SPLIT, 1)
    for bad in (0, 17, -1):
        with pytest.raises(abi.IfemError):
            g.set_readback_slabs(bad)
    g.set_readback_slabs(16)
    g.set_readback_slabs(1)
