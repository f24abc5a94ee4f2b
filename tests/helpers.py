"""Shared helpers of the parity tests: build the same workload in the oracle and on the GPU."""
import numpy as np

from ice_fem_2025a_b200 import abi, config as cf


def make_pair(idx, scale, seed=0, overrides=None, prec=abi.PREC_FP64, tangent=abi.TANGENT_REFERENCE,
              use_kron=True, gpu=True):
    from oracle import oracle as orc
    mesh, d, st = cf.config(idx, scale=scale, seed=seed)
    if overrides:
        overrides(d)
    mats = cf.materials(d)
    opts = cf.options_from_json(d)
    opts.tangent_precision = prec
    opts.tangent_mode = tangent
    o = orc.context(mesh, mats, opts, use_kron=use_kron)
    g = abi.product_context(mesh, mats, opts, use_kron=use_kron) if gpu else None
    state = st()
    cf.apply_state(o, state)
    if g is not None:
        cf.apply_state(g, state)
    return mesh, d, o, g, state


def rel2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)
