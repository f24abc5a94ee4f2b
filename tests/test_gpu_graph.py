"""Batched calibration sweep under a CUDA graph (needs a B200): the replayed graph of the u-step, the phase
step and their adjoints over all specimens equals the same calls made one by one, bit for bit, and picks up
parameter changes made between replays."""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi
from tests.helpers import make_pair, rel2

pytestmark = pytest.mark.gpu

DT = 100.0


def _outputs(g, n_mats):
    out = []
    for s in (0, 1):
        full, sets = g.adjoint_results(s, n_mats)
        out += [g.residual(s), g.matrix_values(s, abi.F32), full, sets]
    return out


def test_graph_replay_matches_direct_calls(product_lib):
    mesh, d, o, g, state = make_pair(4, 0.02, prec=abi.PREC_FP32)
    _, _, _, g2, _ = make_pair(4, 0.02, prec=abi.PREC_FP32, gpu=True)
    n_mats = len(d["B200"]["Specimens"])
    # direct calls on g2
    for s in (0, 1):
        g2.assemble(s, dt=DT)
        g2.adjoint(s, full=True, dt=DT, n_mats=n_mats)
    ref = _outputs(g2, n_mats)
    # one graph replay on g
    g.graph_capture([0, 1], with_adjoint=True, dt=DT)
    g.graph_launch()
    g.sync(0)
    g.sync(1)
    got = _outputs(g, n_mats)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    # the same replay against the oracle (residual and tangent bars)
    for s in (0, 1):
        o.assemble(s, dt=DT)
        assert rel2(g.residual(s), o.residual(s)) <= 1e-12
        assert rel2(g.matrix_values(s, abi.F32).astype(np.float64), o.matrix_values(s)) <= 1e-5


def test_graph_replay_sees_parameter_changes(product_lib):
    mesh, d, o, g, state = make_pair(4, 0.02, prec=abi.PREC_FP32)
    n_mats = len(d["B200"]["Specimens"])
    g.graph_capture([1], with_adjoint=True, dt=DT)
    g.graph_launch()
    g.sync(1)
    f0 = g.residual(1)
    gc0 = d["B200"]["Specimens"][0]["gc"]
    for c in (g, o):
        c.set_param(0, 0, 2.0 * gc0)
    g.graph_launch()
    g.sync(1)
    o.assemble(1, dt=DT)
    f1 = g.residual(1)
    assert not np.array_equal(f0, f1)
    assert rel2(f1, o.residual(1)) <= 1e-12
