"""Known-answer tests of the oracle's Cosserat model (Fracture/CossPhaseField, CosseratMaterial.cpp) on the CPU.

The reference ships no fixtures for it, so the restatement is pinned by:
- a rigid rotation with the matching micro-rotation (u = w times x, oz = w_z in 2D; ox, oy, oz = w_x, -w_y, w_z in
  3D, where the reference's B couples oy with the opposite sign) leaves every strain and curvature zero, so the
  linear-elastic residual vanishes;
- a uniform macro strain (linear u, oz the macro rotation) gives constant stresses, whose divergence vanishes at
  interior nodes;
- the u-step tangent equals the central finite difference of the residual for linear-elastic ice with the
  splits whose stresses derive from their energy (None, DruckerPrager and StarConvex with energy-consistent
  stresses, SpecStress without them, where the stresses are D_coss e);
- the driving energy is zero before t = 0 (the initialisation period) and the history maximum holds after it;
- the damaged viscoelastic-plastic return map leaves the plastic strain unchanged below the yield stress with no
  creep, and moves it once the stress exceeds the yield stress.
"""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from oracle import oracle as orc


def _ctx(rheology="LinearElastic", split="None", consistent=True, inertia=False, damping=0.0, scale=0.125, dim=2, **kw):
    mesh, d, st = cf.cosserat_config(dim, scale=scale, rheology=rheology, split=split, **kw)
    d["properties"]["PhaseField"]["ConsistentEnergy"] = consistent
    d["Models"]["PhaseField1"]["Intertia"] = inertia
    d["properties"]["Ice"]["SolidProperties"]["Damping"] = damping
    if split == "DruckerPrager":
        d["properties"]["Ice"]["FractureProperties"]["B_DP"] = 0.3
    if split == "StarConvex":
        d["properties"]["Ice"]["FractureProperties"]["StarConvexGamma"] = 0.5
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o, st())
    return mesh, d, o


def _set_u(o, mesh, ux, uy, oz):
    o.set_state(0, abi.STATE_CUR, np.concatenate([ux, uy, oz]))


def test_rigid_rotation_is_stress_free():
    mesh, d, o = _ctx()
    x, y = mesh.coords[:, 0], mesh.coords[:, 1]
    th = 1.0e-3
    _set_u(o, mesh, -th * y + 2e-4, th * x - 1e-4, np.full(mesh.n_nodes, th))
    o.assemble(0, t=1.0, dt=0.1)
    f = o.residual(0)
    E = 5.0e9
    assert np.abs(f).max() <= 1e-9 * E * th * 0.05   # relative to a stress of E theta over the box size
    # 3D: u = w x x with the micro-rotations (ox, oy, oz) = (w_x, -w_y, w_z): ConstructBMatCoss couples oy with
    # the xz / zx strains with the opposite sign of ox and oz (CossPhaseField.cpp:1205-1207)
    mesh, d, o = _ctx(dim=3, scale=0.25)
    X = mesh.coords
    wv = np.array([4e-4, -7e-4, 1e-3])
    u = np.cross(np.broadcast_to(wv, X.shape), X)
    n = mesh.n_nodes
    om = wv * np.array([1.0, -1.0, 1.0])
    o.set_state(0, abi.STATE_CUR, np.concatenate([u[:, 0], u[:, 1], u[:, 2]] + [np.full(n, v) for v in om]))
    o.assemble(0, t=1.0, dt=0.1)
    assert np.abs(o.residual(0)).max() <= 1e-9 * E * 1e-3 * 0.05


def test_uniform_strain_patch():
    mesh, d, o = _ctx(scale=0.25)
    x, y = mesh.coords[:, 0], mesh.coords[:, 1]
    # micro-rotation = macro rotation (d_x u_y - d_y u_x) / 2: the couple vanishes and the oz rows balance too
    _set_u(o, mesh, 1e-4 * x + 3e-5 * y, -2e-5 * x - 5e-5 * y, np.full(mesh.n_nodes, 0.5 * (-2e-5 - 3e-5)))
    o.set_state(1, abi.STATE_CUR, np.zeros(o.step_info(1)[0]))   # undamaged: uniform stress
    o.assemble(0, t=1.0, dt=0.1)
    f = o.residual(0)
    n = mesh.n_nodes
    lo, hi = mesh.coords.min(axis=0), mesh.coords.max(axis=0)
    h = (hi - lo) / np.array(mesh.shape)
    inner = np.all((mesh.coords > lo + 1.5 * h) & (mesh.coords < hi - 1.5 * h), axis=1)
    assert inner.sum() > 0
    scale = np.abs(f).max()
    for c in range(3):
        assert np.abs(f[c * n:(c + 1) * n][inner]).max() <= 1e-9 * scale, c


@pytest.mark.parametrize("dim,split,consistent", [(2, "None", True), (2, "SpecStress", False), (2, "SpecStress", True),
                                                  (2, "DruckerPrager", True), (2, "StarConvex", True),
                                                  (3, "None", True), (3, "StarConvex", True)])
def test_u_tangent_matches_finite_differences(dim, split, consistent):
    mesh, d, o = _ctx(split=split, consistent=consistent, dim=dim, scale=0.25 if dim == 3 else 0.125)
    U = o.get_state(0, abi.STATE_CUR)
    o.assemble(0, t=1.0, dt=0.1)
    K = o.matrix(0).toarray()
    rng = np.random.default_rng(2)
    cols = rng.choice(U.size, 6, replace=False)
    for j in cols:
        h = 1e-7 * max(1e-6, np.abs(U).max())
        fs = []
        for sgn in (1, -1):
            V = U.copy(); V[j] += sgn * h
            o.set_state(0, abi.STATE_CUR, V)
            o.assemble(0, t=1.0, dt=0.1)
            fs.append(o.residual(0))
        fd = (fs[0] - fs[1]) / (2 * h)
        if split == "SpecStress" and consistent:
            # the reference's projector is not the derivative of its stresses; only check it is finite
            assert np.all(np.isfinite(K[:, j]))
            continue
        assert np.linalg.norm(fd - K[:, j]) <= 1e-5 * np.linalg.norm(K[:, j]), (split, j)
    o.set_state(0, abi.STATE_CUR, U)


def test_energy_initialisation_period_and_history():
    mesh, d, o = _ctx(irreversible="Hist")
    o.assemble(0, t=-1.0, dt=0.1)
    o.assemble(1, t=-1.0, dt=0.1)
    assert not o.get_history(abi.HIST_ENERGY).any()
    o.assemble(1, t=1.0, dt=0.1)
    E1 = o.get_history(abi.HIST_ENERGY)
    assert E1.max() > 0
    o.commit()
    U = o.get_state(0, abi.STATE_CUR)
    o.set_state(0, abi.STATE_CUR, 0.5 * U)
    o.assemble(1, t=2.0, dt=0.1)
    assert np.array_equal(o.get_history(abi.HIST_ENERGY), E1)   # smaller strains: the history holds


def test_viscoplastic_return_map_yield():
    mesh, d, o = _ctx(rheology="DamViscoElasticPlastic", split="SpecStress", consistent=False)
    d["properties"]["Ice"]["SolidProperties"]["A"] = 0.0
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    st = cf.state_cosserat(mesh, 0)
    cf.apply_state(o, st)
    o.set_state(1, abi.STATE_CUR, np.zeros(o.step_info(1)[0]))   # undamaged
    U = st[0][abi.STATE_CUR]
    o.set_state(0, abi.STATE_CUR, 1e-3 * U)                        # far below the 9.5 MPa yield stress
    o.assemble(0, t=1.0, dt=0.1)
    assert np.abs(o.get_history(abi.HIST_PLASTIC_STRAIN)).max() <= 1e-12
    o.set_state(0, abi.STATE_CUR, 40.0 * U)                        # well above it
    o.assemble(0, t=1.0, dt=0.1)
    ep = o.get_history(abi.HIST_PLASTIC_STRAIN)
    assert np.abs(ep).max() > 1e-6
    assert o.stats(0).rm_iterations > 0
    assert np.all(np.isfinite(o.residual(0)))


def test_viscoplastic_roundoff_sensitivity():
    """The Cosserat return map's 20x20 system (rows scaled by 1e3 and -1e-6) amplifies round-off: a relative
    change of 1e-15 in the displacements moves the converged residual by far more than 1e-15.  This sets the
    GPU parity bar of the viscoelastic-plastic cases."""
    res = []
    for pert in (0.0, 1e-15):
        mesh, d, st = cf.cosserat_config(2, scale=0.125, rheology="DamViscoElasticPlastic", split="SpecStress")
        d["properties"]["PhaseField"]["ConsistentEnergy"] = False
        d["B200"]["ReturnMapTolerance"] = "tight"
        o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
        s = st()
        cf.apply_state(o, s)
        o.set_state(0, abi.STATE_CUR, s[0][abi.STATE_CUR] * (1.0 + pert))
        o.assemble(0, t=-1.0, dt=0.05, du_dt=20.0, ddu_dt=400.0)
        res.append(o.residual(0))
    sens = np.linalg.norm(res[1] - res[0]) / np.linalg.norm(res[0])
    assert 1e-13 < sens < 1e-8, sens
