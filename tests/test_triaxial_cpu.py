"""Known-answer tests of the oracle's TriAxial model (TriAxial.cpp:13-276) and its boundary element groups
(B1_2 lines in 2D, NURBS3_Plane2 faces in 3D), on the CPU.

The groups are those of the reference's generator (GenerateMesh.m:298-367) on a box centred on the vertical axis:
- the face weights integrate to the side and top areas, the shape values form a partition of unity, and the
  normals of getNormals point outward;
- a uniform confining pressure has zero resultant on the closed side surface, and the top pressure's resultant is
  p0 times the top area; the displacement penalty of a uniform top displacement gives k (u - u_target) per area;
- the side pressure is degraded by (1 - phi)^2 when DamagedForces is on;
- the failure detection of TriAxialModel::Commit: u0 while time < 0, the minimum load, the load drop, t_postFail.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from oracle import oracle as orc


def _ctx(dim, scale=0.25, tri=True, **prm):
    mesh, d, st = cf.triaxial_config(dim, scale=scale)
    d["Models"]["Tri"].update(prm)
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o, st())
    groups = cf.attach_triaxial(o, mesh, d) if tri else cf.box_face_groups(mesh)
    return mesh, d, o, groups


@pytest.mark.parametrize("dim", [2, 3])
def test_face_areas_partition_and_outward_normals(dim):
    mesh, d, o, groups = _ctx(dim)
    lo, hi = mesh.coords.min(axis=0), mesh.coords.max(axis=0)
    L = hi - lo
    side_area = 2.0 * L[1] if dim == 2 else 2.0 * (L[0] + L[1]) * L[2]
    top_area = L[0] if dim == 2 else L[0] * L[1]
    for grp, name, area in ((0, "side", side_area), (1, "top", top_area)):
        faces, _ = groups[name]
        tot = 0.0
        for f in range(faces.shape[0]):
            N, w, n = o.face_shapes(grp, f)
            assert np.allclose(N.sum(axis=1), 1.0, atol=1e-14)
            tot += w.sum()
            P = N @ mesh.coords[faces[f]]
            assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-14)
            if name == "side":   # outward: away from the vertical axis, horizontal
                lat = P[:, :dim - 1]
                assert np.all(np.einsum('qd,qd->q', n[:, :dim - 1], lat) > 0)
                assert np.allclose(n[:, dim - 1], 0.0, atol=1e-14)
        assert abs(tot - area) <= 1e-12 * area, (name, tot, area)


def _tri_residual(o, mesh, d, t, dt=1.0, **prm):
    """Residual of the TriAxial model alone: the u-step with the model minus the u-step without it."""
    o.assemble(0, t=t, dt=dt)
    f1 = o.residual(0)
    o2 = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    for kind in (abi.STATE_CUR, abi.STATE_OLD):
        for s in (0, 1):
            o2.set_state(s, kind, o.get_state(s, kind))
    o2.assemble(0, t=t, dt=dt)
    f0 = o2.residual(0)
    o2.close()
    return f1 - f0


@pytest.mark.parametrize("dim", [2, 3])
def test_uniform_pressure_resultants(dim):
    p0 = -2.0e6
    mesh, d, o, groups = _ctx(dim, p0=p0, DamagedForces=False)
    r = _tri_residual(o, mesh, d, t=-10.0)
    nn = mesh.n_nodes
    L = mesh.coords.max(axis=0) - mesh.coords.min(axis=0)
    top_area = L[0] if dim == 2 else L[0] * L[1]
    for c in range(dim - 1):   # the side pressure cancels over the closed lateral surface
        assert abs(r[c * nn:(c + 1) * nn].sum()) <= 1e-9 * abs(p0) * L[dim - 1]
    # t + dt < 0: the top carries p0 along +e_top
    assert abs(r[(dim - 1) * nn:].sum() - p0 * top_area) <= 1e-12 * abs(p0 * top_area)
    st = o.triaxial_state()
    assert abs(st["area"] - top_area) <= 1e-12 * top_area
    assert abs(st["f_ext"] + p0 * top_area) <= 1e-12 * abs(p0 * top_area)
    # the side load on the x = max faces alone is p0 times their area, along +x
    faces, _ = groups["side"]
    xmax = mesh.coords[:, 0].max()
    on_right = np.unique(faces[np.all(np.isclose(mesh.coords[faces, 0], xmax), axis=1)])
    interior = np.setdiff1d(on_right, np.unique(faces[~np.all(np.isclose(mesh.coords[faces, 0], xmax), axis=1)]))
    right_area = L[1] if dim == 2 else L[1] * L[2]
    assert interior.size > 0
    assert abs(r[:nn][on_right].sum() - p0 * right_area) <= 0.5 * abs(p0) * right_area   # edges are shared


@pytest.mark.parametrize("dim", [2, 3])
def test_top_displacement_penalty(dim):
    k, du = 1.0e11, -1.0e-4
    mesh, d, o, groups = _ctx(dim, p0=0.0, dummy=k, dU=du, DamagedForces=False)
    nn = mesh.n_nodes
    U = o.get_state(0, abi.STATE_CUR)
    U[(dim - 1) * nn:] = -3.0e-6            # uniform vertical displacement
    o.set_state(0, abi.STATE_CUR, U)
    u0 = 1.0e-6
    st = o.triaxial_state(); st["u0"] = u0
    o.set_triaxial_state(st)
    t, dt = 2.0, 0.5
    r = _tri_residual(o, mesh, d, t=t, dt=dt)
    L = mesh.coords.max(axis=0) - mesh.coords.min(axis=0)
    top_area = L[0] if dim == 2 else L[0] * L[1]
    target = u0 + (t + dt) * du
    expect = k * (-3.0e-6 - target) * top_area
    assert abs(r[(dim - 1) * nn:].sum() - expect) <= 1e-10 * abs(expect)
    st = o.triaxial_state()
    assert abs(st["uz_sum"] / st["area"] + 3.0e-6) <= 1e-12 * 3.0e-6
    # the penalty block sums to k times the top area
    K = o.matrix(0)
    top_nodes = np.unique(groups["top"][0])
    rows = (dim - 1) * nn + top_nodes
    blk = K[rows][:, rows].sum()
    o2 = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o2, {0: {abi.STATE_CUR: U}})
    o2.set_state(1, abi.STATE_CUR, o.get_state(1, abi.STATE_CUR))
    o2.assemble(0, t=t, dt=dt)
    blk0 = o2.matrix(0)[rows][:, rows].sum()
    assert abs((blk - blk0) - k * top_area) <= 1e-9 * k * top_area


def test_damaged_side_pressure():
    """DamagedForces scales the side pressure by (1 - phi)^2 (QuadraticNoRes): a uniform phi = 0.3 gives 0.49."""
    p0 = 1.5e6
    res = []
    for dam in (False, True):
        mesh, d, o, _ = _ctx(3, p0=p0, DamagedForces=dam)
        o.set_state(1, abi.STATE_CUR, np.full(o.step_info(1)[0], 0.3))
        res.append(_tri_residual(o, mesh, d, t=-1.0))
    nn = mesh.n_nodes
    side = slice(0, 2 * nn)
    assert np.allclose(res[1][side], 0.49 * res[0][side], rtol=1e-12, atol=1e-12 * np.abs(res[0]).max())


def test_commit_failure_detection():
    """TriAxialModel::Commit (TriAxial.cpp:75-122), loaded downwards (dU < 0), with injected assembly sums."""
    mesh, d, o, _ = _ctx(2, p0=-1.0e5, dU=-1e-4, t_postFail=0.5)
    def commit(time, f_ext, uz_sum=0.0, area=2.0):
        st = o.triaxial_state()
        st.update(area=area, f_ext=f_ext, uz_sum=uz_sum)
        o.set_triaxial_state(st)
        return o.triaxial_commit(time, max_time=100.0), o.triaxial_state()
    mt, st = commit(-1.0, 0.0, uz_sum=-4.0e-6)
    assert st["u0"] == -2.0e-6 and mt == 100.0 and not st["min_load_passed"]
    mt, st = commit(1.0, 2.0 * 5.0e5)          # F/A * sign = -5e5 < max(1e3, |p0|): not yet
    assert not st["min_load_passed"]
    mt, st = commit(2.0, -2.0 * 2.0e6)         # 2 MPa in compression: passed
    assert st["min_load_passed"] and st["max_load"] == 2.0e6 and st["t_break"] == 0.0
    mt, st = commit(3.0, -2.0 * 1.5e5)         # 0.15 MPa > 5% of 2 MPa: intact
    assert st["t_break"] == 0.0 and mt == 100.0
    mt, st = commit(4.0, -2.0 * 0.5e5)         # 0.05 MPa < 0.1 MPa: broken at t = 4
    assert st["t_break"] == 4.0 and mt == 4.5
    mt, st = commit(5.0, 0.0)                  # detected once
    assert st["t_break"] == 4.0 and mt == 100.0
    assert st["u0"] == -2.0e-6                 # u0 only changes while time < 0
    # after failure the side pressure is removed at the next assembly
    o.assemble(0, t=5.0, dt=1.0)
    assert o.triaxial_state()["p0"] == 0.0
