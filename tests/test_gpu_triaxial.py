"""GPU vs oracle parity of the TriAxial boundary loads (TriAxialModel, TriAxial.cpp:124-276) on the displacement
step, 2D (B1_2 lines) and 3D (NURBS3_Plane2 faces), after the phase-field terms (needs a B200).

Cases: the confining phase (t + dt < 0: pressures on the side and top groups) and the displacement-controlled
phase (t + dt >= 0: the top penalty, with u0 from a commit at negative time), the side pressure degraded by the
phase field; FP64, FP32 and (3D) tensor-core tangents; the model's sums and failure detection against the
oracle's; a CUDA-graph replay; invalid groups.

Bars: residual <= 1e-12 relative (2-norm), tangent <= 1e-10 (FP64) / 1e-5 (FP32-accurate), sums <= 1e-12.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from tests.helpers import rel2

pytestmark = pytest.mark.gpu


def _pair(dim, prec=abi.PREC_FP64, scale=0.25, **prm):
    from oracle import oracle as orc
    mesh, d, st = cf.triaxial_config(dim, scale=scale)
    d["Models"]["Tri"].update(prm)
    mats, opts = cf.materials(d), cf.options_from_json(d)
    opts.tangent_precision = prec
    o = orc.context(mesh, mats, opts)
    g = abi.product_context(mesh, mats, opts)
    state = st()
    for c in (o, g):
        cf.apply_state(c, state)
        cf.attach_triaxial(c, mesh, d)
    return mesh, d, o, g


def _check(o, g, f32, t, dt=1.0):
    for c in (o, g):
        c.assemble(0, t=t, dt=dt)
    fo, fg = o.residual(0), g.residual(0)
    assert rel2(fg, fo) <= 1e-12, rel2(fg, fo)
    ko = o.matrix_values(0)
    kg = g.matrix_values(0, abi.F32 if f32 else abi.F64).astype(np.float64)
    assert rel2(kg, ko) <= (1e-5 if f32 else 1e-10), rel2(kg, ko)
    so, sg = o.triaxial_state(), g.triaxial_state()
    for k in ("area", "f_ext", "uz_sum"):
        assert abs(sg[k] - so[k]) <= 1e-12 * max(abs(so[k]), 1e-300), (k, sg[k], so[k])


@pytest.mark.parametrize("dim,prec", [(2, abi.PREC_FP64), (2, abi.PREC_FP32), (3, abi.PREC_FP64),
                                      (3, abi.PREC_FP32), (3, abi.PREC_TC_SPLIT)])
def test_triaxial_parity(product_lib, dim, prec):
    mesh, d, o, g = _pair(dim, prec)
    f32 = prec != abi.PREC_FP64
    dt = 0.5
    # confining phase, then a commit at negative time sets u0, then displacement control
    _check(o, g, f32, t=-2.0, dt=dt)
    for c in (o, g):
        c.triaxial_commit(-1.0)
    assert g.triaxial_state()["u0"] == pytest.approx(o.triaxial_state()["u0"], rel=1e-12)
    _check(o, g, f32, t=0.0, dt=dt)
    _check(o, g, f32, t=3.0, dt=dt)
    # the phase step is unchanged by the model
    for c in (o, g):
        c.assemble(1, dt=dt)
    assert rel2(g.residual(1), o.residual(1)) <= 1e-12
    o.close()
    g.close()


def test_triaxial_failure_detection_and_graph(product_lib):
    mesh, d, o, g = _pair(3, abi.PREC_FP64, p0=-1.0e5, dU=-1.0e-4)
    for c in (o, g):
        c.assemble(0, t=-2.0, dt=1.0)
    mts = [c.triaxial_commit(-1.0, max_time=50.0) for c in (o, g)]
    assert mts[0] == mts[1] == 50.0
    assert g.triaxial_state() == pytest.approx(o.triaxial_state(), rel=1e-12)
    # the same load history on both sides: a 2 MPa peak, then a drop below 5 %
    for time, f in ((1.0, -4.0e6), (2.0, -1.0e4)):
        res = []
        for c in (o, g):
            st = c.triaxial_state()
            st.update(area=2.0, f_ext=f)
            c.set_triaxial_state(st)
            res.append((c.triaxial_commit(time, max_time=50.0), c.triaxial_state()))
        assert res[0][0] == res[1][0]
        assert res[1][1] == pytest.approx(res[0][1], rel=1e-15)
    assert g.triaxial_state()["t_break"] == 2.0
    # after failure: side pressure 0, the top under displacement control; also replayed from a CUDA graph (each
    # assembly warm-starts the return map from the last one, so both start from the committed history)
    for c in (o, g):
        c.reset_step()
    _check(o, g, False, t=3.0)
    assert g.triaxial_state()["p0"] == 0.0
    f_direct = g.residual(0)
    g.reset_step()
    g.graph_capture([0], t=3.0, dt=1.0)
    g.graph_launch()
    assert np.array_equal(g.residual(0), f_direct)
    assert g.triaxial_state()["f_ext"] == pytest.approx(o.triaxial_state()["f_ext"], rel=1e-12)
    o.close()
    g.close()


def test_triaxial_invalid_groups(product_lib):
    mesh, d, o, g = _pair(3, abi.PREC_FP64)
    groups = cf.box_face_groups(mesh)
    side, top = groups["side"], groups["top"]
    bad = top[0].copy()
    bad[0, 0] = mesh.n_nodes + 5                      # not a mesh node
    with pytest.raises(abi.IfemError):
        g.set_triaxial(side, (bad, top[1]))
    far = top[0].copy()
    far[0, :] = top[0][-1, :]                         # pairs across faces that share no element
    far[0, 0] = top[0][0, 0]
    with pytest.raises(abi.IfemError):
        g.set_triaxial(side, (far, top[1]))
    with pytest.raises(abi.IfemError):
        g.set_triaxial((side[0][:0], side[1][:0]), top)   # empty side group
    o.close()
    g.close()
