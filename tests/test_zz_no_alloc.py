"""The allocation-free crack-length entry point (ifem_crack_length_noalloc).

Callers whose device memory is owned by a host framework's pool, or that monitor the crack between
time steps and cannot afford cudaMalloc's device-wide synchronisation, use it with their own
buffers.  It must give the crack length that the phase-step assembly reports, call after call.
This file is collected last so that a run that stops at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the crack-length tolerance of the phase-step parity tests


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("idx,scale", [(0, 0.125), (1, 0.125)])
def test_noalloc_crack_length_matches_phase_assembly(idx, scale):
    import torch
    lib = abi.load_product()
    fn = lib.ifem_crack_length_noalloc
    fn.argtypes = [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.c_double, C.c_int32, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    mesh, d, st = cf.config(idx, scale=scale)
    mats, opts = cf.materials(d), cf.options_from_json(d)
    g = abi.product_context(mesh, mats, opts)
    state = st()
    cf.apply_state(g, state)
    g.assemble(0, dt=100.0)
    g.assemble(1, dt=100.0)
    expected = g.stats(1).crack_length          # the existing entry point's value
    # ... which is itself the oracle's crack length of the same state (PhaseField.cpp:540,650)
    from oracle import oracle as orc
    o = orc.context(mesh, mats, opts)
    cf.apply_state(o, state)
    o.assemble(0, dt=100.0)
    o.assemble(1, dt=100.0)
    assert abs(expected - o.stats(1).crack_length) <= TOL * abs(o.stats(1).crack_length)
    o.close()
    dev = torch.device("cuda", 0)
    coords = torch.tensor(mesh.coords, dtype=torch.float64, device=dev).contiguous()
    weights = torch.tensor(mesh.weights if mesh.weights is not None else np.ones(mesh.n_nodes),
                           dtype=torch.float64, device=dev)
    elems = torch.tensor(mesh.elems.astype(np.int32), device=dev).contiguous()
    kron = torch.tensor(mesh.elem_kron, dtype=torch.float64, device=dev).contiguous()
    phase = torch.tensor(state[1][abi.STATE_CUR], dtype=torch.float64, device=dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    for call in range(2):                        # two calls in a row share the library's scratch array
        out.fill_(-1.0)
        rc = fn(mesh.dim, mesh.n_elems, _ptr(coords), _ptr(weights), _ptr(elems), _ptr(kron), _ptr(phase),
                mats[0].pf_l, opts.distribution, _ptr(out), None)
        assert rc == abi.OK
        torch.cuda.synchronize(dev)
        got = float(out.item())
        assert abs(got - expected) <= TOL * abs(expected), (call, got, expected)
    g.close()


def test_noalloc_rejects_oversized_mesh():
    """A mesh above the 2^21-element limit is refused before any work, with the output left untouched."""
    import torch
    lib = abi.load_product()
    fn = lib.ifem_crack_length_noalloc
    fn.argtypes = [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.c_double, C.c_int32, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    dev = torch.device("cuda", 0)
    # real (small) device buffers, so no argument is a fabricated address
    coords = torch.zeros(3 * 8, dtype=torch.float64, device=dev)
    weights = torch.ones(8, dtype=torch.float64, device=dev)
    elems = torch.zeros(27, dtype=torch.int32, device=dev)
    kron = torch.zeros(27, dtype=torch.float64, device=dev)
    phase = torch.zeros(8, dtype=torch.float64, device=dev)
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    rc = fn(3, (1 << 21) + 1, _ptr(coords), _ptr(weights), _ptr(elems), _ptr(kron), _ptr(phase), 1e-3, 3,
            _ptr(out), None)
    assert rc == abi.ERR_CAPACITY
    torch.cuda.synchronize(dev)
    assert float(out.item()) == -1.0
