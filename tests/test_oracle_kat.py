"""Known-answer tests of the CPU oracle (the reference ships no fixtures or golden vectors, so the
restatement is pinned by closed forms, invariants and finite differences)."""
import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from ice_fem_2025a_b200.meshgen import box_mesh
from oracle import oracle as orc


def _ctx(idx, scale, **kw):
    mesh, d, st = cf.config(idx, scale=scale)
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d), **kw)
    return mesh, d, o, st


@pytest.mark.parametrize("idx,scale", [(0, 0.125), (1, 0.125)])
def test_shape_functions_partition_of_unity_and_volume(idx, scale):
    """Mesh::Check integrates the weights to the group volume (mesh.cpp:306-339)."""
    mesh, d, o, _ = _ctx(idx, scale)
    vol = 0.0
    for el in range(mesh.n_elems):
        N, G, w = o.shape(el)
        assert np.allclose(N.sum(axis=1), 1.0, atol=1e-14)
        assert np.allclose(G.sum(axis=2), 0.0, atol=1e-9)
        vol += w.sum()
    box = np.prod(mesh.coords.max(axis=0) - mesh.coords.min(axis=0))
    assert abs(vol - box) <= 1e-12 * box


def test_linear_field_gradient_exact():
    """Patch test at the shape-function level: a linear field is reproduced exactly."""
    mesh, d, o, _ = _ctx(1, 0.125)
    a = np.array([0.3, -1.2, 2.5])
    f = mesh.coords @ a
    for el in (0, mesh.n_elems // 2, mesh.n_elems - 1):
        N, G, w = o.shape(el)
        fe = f[mesh.elems[el]]
        assert np.allclose(G @ fe, a[None, :], atol=1e-10)


def test_le_tangent_symmetric_and_rigid_modes():
    mesh, d, o, st = _ctx(0, 0.125)
    cf.apply_state(o, st())
    o.assemble(0)
    K = o.matrix(0)
    n = mesh.n_nodes
    assert abs(K - K.T).max() <= 1e-12 * abs(K).max()
    for t in (np.r_[np.ones(n), np.zeros(n)], np.r_[np.zeros(n), np.ones(n)]):
        assert np.abs(K @ t).max() <= 1e-12 * abs(K).max()
    # rotation about z is a null mode of the linear-elastic stiffness
    X = mesh.coords
    r = np.r_[-X[:, 1], X[:, 0]]
    assert np.abs(K @ r).max() <= 1e-9 * abs(K).max() * np.abs(r).max()


def test_le_patch_test_uniform_strain():
    """Uniform strain field: residual equals the boundary traction integral; interior nodes are
    free of force (constant stress patch test)."""
    mesh, d, st = cf.config(0, scale=0.125)
    d["properties"]["Ice"]["FractureProperties"]["Split"] = "None"
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    X = mesh.coords
    eps = np.array([1e-4, -2e-4, 0.5e-4])        # exx, eyy, gamma_xy
    ux = eps[0] * X[:, 0] + 0.5 * eps[2] * X[:, 1]
    uy = eps[1] * X[:, 1] + 0.5 * eps[2] * X[:, 0]
    o.set_state(0, abi.STATE_CUR, np.r_[ux, uy])
    o.assemble(0)
    f = o.residual(0)
    lo, hi = X.min(axis=0), X.max(axis=0)
    interior = np.all((X > lo + 1e-12) & (X < hi - 1e-12), axis=1)
    n = mesh.n_nodes
    fmax = np.abs(f).max()
    assert np.abs(f[:n][interior]).max() <= 1e-9 * fmax
    assert np.abs(f[n:][interior]).max() <= 1e-9 * fmax
    assert abs(f[:n].sum()) <= 1e-9 * fmax and abs(f[n:].sum()) <= 1e-9 * fmax


def test_dof_numbering_formula():
    """DofSpace::SyncDofs serial numbering: dof = base(kind) + rank(node) (DofSpace.cpp:486-513)."""
    mesh, d, o, _ = _ctx(2, 1 / 32)
    n = mesh.n_nodes
    assert np.array_equal(o.dof_numbers(abi.DOF_UX), np.arange(n))
    assert np.array_equal(o.dof_numbers(abi.DOF_UY), n + np.arange(n))
    assert np.array_equal(o.dof_numbers(abi.DOF_PHASE), np.arange(n))
    assert np.array_equal(o.dof_numbers(abi.DOF_T), np.arange(n))
    assert (o.dof_numbers(abi.DOF_UZ) == -1).all()


def test_pattern_is_union_of_element_pairs():
    mesh, d, o, _ = _ctx(0, 0.125)
    rp, ci = o.pattern(0)
    n = mesh.n_nodes
    pairs = set()
    for e in mesh.elems:
        dofs = np.r_[e, e + n]
        for r in dofs:
            for c in dofs:
                pairs.add((r, c))
    assert rp[-1] == len(pairs)
    got = set()
    for r in range(rp.size - 1):
        cols = ci[rp[r]:rp[r + 1]]
        assert np.all(np.diff(cols) > 0)
        got.update((r, c) for c in cols)
    assert got == pairs


def test_return_map_closed_form_uniaxial():
    """Glen return map at a converged point satisfies f(6) = A dt F^n - dlambda = 0 and
    strain split eps = eps_e + eps_p (SolidMaterial.cpp:291-297)."""
    mesh, d, st = cf.config(1, scale=0.125)
    m = cf.materials(d)[0]
    T = 263.15
    eps = np.array([-1e-4, 0.3e-4, 0.3e-4, 0.2e-4, 0.0, 0.0])
    epl, h, D, it, diss = orc.return_map(m, T, eps, np.zeros(6), np.zeros(6), 0.0, 1.0, 1000.0, tol_mode=1)
    E, nu = m.young, m.poisson
    G = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    ee = eps - epl
    S = lam * ee[:3].sum() * np.r_[1, 1, 1, 0, 0, 0] + np.r_[2 * G * ee[:3], G * ee[3:]]
    s = S / 1e6
    dev = s.copy(); dev[:3] -= s[:3].mean()
    J2 = 0.5 * (dev[:3] @ dev[:3] + 2 * (s[3:] @ s[3:]))
    F = 1e6 * np.sqrt(2 * J2)
    A = m.creep_a * np.exp(-m.q_creep / 8.31446261815324 * (1 / T - 1 / m.t_ref))
    assert abs(A * 1000.0 * F ** 3 - h) <= 1e-10 * abs(h)
    assert it >= 2 and h > 0


def test_consistent_tangent_matches_finite_difference_at_point():
    mesh, d, st = cf.config(1, scale=0.125)
    m = cf.materials(d)[0]
    eps = np.array([-1e-4, 0.3e-4, 0.2e-4, 0.2e-4, -0.1e-4, 0.05e-4])
    _, _, Dc, _, _ = orc.return_map(m, 263.15, eps, np.zeros(6), np.zeros(6), 0.0, 1.0, 1000.0, tol_mode=1, tangent_mode=1)
    h = 1e-10
    fd = np.zeros((6, 6))
    for j in range(6):
        ep, em = eps.copy(), eps.copy()
        ep[j] += h; em[j] -= h
        a, *_ = orc.return_map(m, 263.15, ep, np.zeros(6), np.zeros(6), 0.0, 1.0, 1000.0, tol_mode=1)
        b, *_ = orc.return_map(m, 263.15, em, np.zeros(6), np.zeros(6), 0.0, 1.0, 1000.0, tol_mode=1)
        fd[:, j] = ((ep - a) - (em - b)) / (2 * h)    # d eps_e / d eps
    assert np.abs(fd - Dc).max() <= 1e-5 * np.abs(Dc).max()


def test_volstrain_split_energy_closed_form():
    mesh, d, st = cf.config(0, scale=0.125)
    m = cf.materials(d)[0]
    E, nu = m.young, m.poisson
    G = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu)); K = lam + 2 / 3 * G
    e = np.array([1e-4, -3e-4, 0.0, 2e-4, 0.0, 0.0])     # compressive volumetric part
    Dd, Du, Sd, Su, en = orc.energy_split(m, 273.15, e)
    p = e[:3].sum()
    dev = np.r_[e[:3] - p / 3, 0.5 * e[3:]]
    ed = G * (dev[:3] @ dev[:3] + 2 * dev[3:] @ dev[3:])
    assert p < 0 and abs(en - ed) <= 1e-12 * en
    S = Sd + Su
    Sfull = lam * p * np.r_[1, 1, 1, 0, 0, 0] + np.r_[2 * G * e[:3], G * e[3:]]
    assert np.allclose(S, Sfull, rtol=1e-12, atol=1e-12 * np.abs(Sfull).max())
    assert np.allclose(Dd + Du, (Dd + Du).T)


def test_phase_tangent_finite_difference():
    """Phase-step tangent is the exact derivative of its residual (Hist irreversibility)."""
    mesh, d, o, st = _ctx(0, 0.125)
    s = st()
    cf.apply_state(o, s)
    o.assemble(0)
    phi0 = o.get_state(1, abi.STATE_CUR)
    o.assemble_nohist(1)
    K = o.matrix(1).toarray()
    rng = np.random.default_rng(1)
    v = rng.normal(size=phi0.size)
    h = 1e-6
    o.set_state(1, abi.STATE_CUR, phi0 + h * v); o.assemble_nohist(1); fp = o.residual(1)
    o.set_state(1, abi.STATE_CUR, phi0 - h * v); o.assemble_nohist(1); fm = o.residual(1)
    fd = (fp - fm) / (2 * h)
    assert np.linalg.norm(fd - K @ v) <= 1e-7 * np.linalg.norm(K @ v)


def test_u_consistent_tangent_finite_difference_viscous():
    """Consistent U tangent (dVE, tight return map) vs central FD of the oracle residual."""
    mesh, d, st = cf.config(1, scale=0.125)
    d["B200"]["Tangent"] = "consistent"
    d["B200"]["ReturnMapTolerance"] = "tight"
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o, st())
    o.assemble_nohist(0, dt=100.0)
    K = o.matrix(0)
    U0 = o.get_state(0, abi.STATE_CUR)
    rng = np.random.default_rng(2)
    v = rng.normal(size=U0.size) * np.abs(U0).max()
    h = 1e-7
    o.set_state(0, abi.STATE_CUR, U0 + h * v); o.assemble_nohist(0, dt=100.0); fp = o.residual(0)
    o.set_state(0, abi.STATE_CUR, U0 - h * v); o.assemble_nohist(0, dt=100.0); fm = o.residual(0)
    fd = (fp - fm) / (2 * h)
    assert np.linalg.norm(fd - K @ v) <= 1e-6 * np.linalg.norm(K @ v)


def test_reference_tangent_differs_from_consistent_for_glen():
    """The reference's return-map Jacobian zeroes d2F (SolidMaterial.cpp:289): its tangent is not
    the derivative of its residual, which is why both variants exist."""
    mesh, d, st = cf.config(1, scale=0.125)
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o, st())
    o.assemble_nohist(0, dt=100.0)
    Kr = o.matrix_values(0)
    o.set_tangent(abi.TANGENT_CONSISTENT, abi.PREC_FP64)
    o.assemble_nohist(0, dt=100.0)
    Kc = o.matrix_values(0)
    assert np.linalg.norm(Kr - Kc) > 1e-6 * np.linalg.norm(Kc)


def test_commit_and_reset_semantics():
    mesh, d, o, st = _ctx(1, 0.125)
    cf.apply_state(o, st())
    o.assemble(0, dt=100.0)
    ep1 = o.get_history(abi.HIST_PLASTIC_STRAIN)
    o.commit()
    assert np.array_equal(o.get_history(abi.HIST_PLASTIC_STRAIN, old=1), ep1)
    U = o.get_state(0, abi.STATE_CUR)
    o.set_state(0, abi.STATE_CUR, 2 * U)
    o.assemble(0, dt=100.0)
    assert not np.array_equal(o.get_history(abi.HIST_PLASTIC_STRAIN), ep1)
    o.reset_step()
    assert np.array_equal(o.get_history(abi.HIST_PLASTIC_STRAIN), ep1)


def test_history_max_irreversibility():
    mesh, d, o, st = _ctx(0, 0.125)
    s = st()
    cf.apply_state(o, s)
    o.assemble(1)
    h1 = o.get_history(abi.HIST_ENERGY)
    o.commit()
    o.set_state(0, abi.STATE_CUR, 0.5 * s[0][abi.STATE_CUR])
    o.assemble(1)
    h2 = o.get_history(abi.HIST_ENERGY)
    assert np.all(h2 >= h1) and np.array_equal(h2, h1)


def _specstress_material():
    _, d, _ = cf.config(1, scale=0.125)
    d["properties"]["Ice"]["FractureProperties"]["Split"] = "SpecStress"
    d["properties"]["PhaseField"]["ConsistentEnergy"] = False
    return d, cf.materials(d)[0]


@pytest.mark.parametrize("seed", range(6))
def test_specstress_energy_matches_numpy_eigh(seed):
    """SpecStress (PhaseFieldMaterial.cpp:118-151): psi+ = 1/2 sigma+ : eps, sigma+ the positive principal part of
    sigma = D eps (the oracle's Jacobi eigen-solver against LAPACK); stresses and tangent are D eps / D."""
    d, m = _specstress_material()
    E, nu = m.young, m.poisson
    G = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6)); D[:3, :3] = lam; D += np.diag([2 * G] * 3 + [G] * 3)
    rng = np.random.default_rng(seed)
    e = rng.normal(scale=1e-4, size=6)
    if seed == 4:
        e[:3] = -np.abs(e[:3]); e[3:] = 0          # all principal stresses compressive: psi+ = 0
    if seed == 5:
        e = np.array([2e-4, 2e-4, 2e-4, 0, 0, 0])  # repeated eigenvalue, all tensile: psi+ = full energy
    Dd, Du, Sd, Su, en = orc.energy_split(m, 273.15, e)
    S = D @ e
    Sn = S.copy()
    for i in range(4):                             # the reference's perturbation of near-zero components
        if Sn[i] ** 2 < 1e-9:
            Sn[i] = (i + 1) * 1e-9
    M = np.array([[Sn[0], Sn[3], Sn[5]], [Sn[3], Sn[1], Sn[4]], [Sn[5], Sn[4], Sn[2]]])
    lv, V = np.linalg.eigh(M)
    P = (V * np.maximum(lv, 0)) @ V.T
    ref = 0.5 * (np.r_[P[0, 0], P[1, 1], P[2, 2], P[0, 1], P[1, 2], P[0, 2]] @ e)
    assert abs(en - ref) <= 1e-12 * max(abs(ref), 0.5 * S @ e), (en, ref)
    if seed == 4:
        assert en == 0.0
    if seed == 5:
        assert en == pytest.approx(0.5 * S @ e, rel=1e-13)
    assert np.allclose(Sd, S, rtol=1e-14, atol=0) and np.all(Su == 0)
    assert np.allclose(Dd, D, rtol=1e-14, atol=0) and np.all(Du == 0)


def test_specstress_with_consistent_energy_refused():
    """SpecStress with a consistent energy split throws in the reference (PhaseFieldMaterial.cpp:148-150): the
    context is refused at creation."""
    mesh, d, _ = cf.config(1, scale=0.125)
    d["properties"]["Ice"]["FractureProperties"]["Split"] = "SpecStress"
    d["properties"]["PhaseField"]["ConsistentEnergy"] = True
    with pytest.raises(abi.IfemError) as e:
        orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    assert e.value.code == abi.ERR_UNSUPPORTED


def _split_material(split, b_dp=0.3):
    _, d, _ = cf.config(1, scale=0.125)
    d["properties"]["Ice"]["FractureProperties"]["Split"] = split
    d["properties"]["Ice"]["FractureProperties"]["B_DP"] = b_dp
    d["properties"]["PhaseField"]["ConsistentEnergy"] = True
    return cf.materials(d)[0]


def _fd_split(m, e, h=1e-9):
    """Central differences of the energy (-> damaged stress) and of both stresses (-> tangents)."""
    I = np.eye(6)
    ev = lambda x: orc.energy_split(m, 273.15, x)
    dE = np.array([(ev(e + h * I[i])[4] - ev(e - h * I[i])[4]) / (2 * h) for i in range(6)])
    dSd = np.array([(ev(e + h * I[i])[2] - ev(e - h * I[i])[2]) / (2 * h) for i in range(6)]).T
    dSu = np.array([(ev(e + h * I[i])[3] - ev(e - h * I[i])[3]) / (2 * h) for i in range(6)]).T
    return dE, dSd, dSu


@pytest.mark.parametrize("e,b_dp,regime", [([1e-4, 1e-4, 1e-4, 0, 0, 0], 0.3, "damageable"),
                                           ([-1e-4, -1e-4, -1e-4, 1e-5, 0, 0], 0.3, "mixed"),
                                           ([-2e-4, 1e-4, 5e-5, 3e-4, 1e-4, -2e-4], 0.3, "damageable"),
                                           ([-3e-4, -3e-4, -3e-4, 2e-5, 0, 0], -0.3, "undamageable")])
def test_drucker_prager_split_derivatives(e, b_dp, regime):
    """DruckerPragerSplit (PhaseFieldMaterial.cpp:292-343): in each regime the damaged stress is the energy's
    gradient, the tangents are the stresses' Jacobians, and the two stresses add up to D eps.  The
    undamageable regime, 2 G sqrt(J2) < 3 B K I1 after I1 <= -6 B sqrt(J2), needs B < 0."""
    m = _split_material("DruckerPrager", b_dp)
    e = np.array(e)
    Dd, Du, Sd, Su, en = orc.energy_split(m, 273.15, e)
    dE, dSd, dSu = _fd_split(m, e)
    E, nu = m.young, m.poisson
    G = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6)); D[:3, :3] = lam; D += np.diag([2 * G] * 3 + [G] * 3)
    sc = np.abs(D @ e).max()
    assert np.abs(dE - Sd).max() <= 1e-8 * sc
    assert np.abs(dSd - Dd).max() <= 1e-6 * np.abs(D).max()
    assert np.abs(dSu - Du).max() <= 1e-6 * np.abs(D).max()
    assert np.abs(Sd + Su - D @ e).max() <= 1e-12 * sc
    if regime == "undamageable":
        assert en == 0.0 and not Sd.any() and not Dd.any()
    elif regime == "damageable":
        assert not Su.any() and en == pytest.approx(0.5 * (D @ e) @ e, rel=1e-13)
    else:
        assert Sd.any() and Su.any()


@pytest.mark.parametrize("e", [[-2e-4, 1e-4, 0, 3e-4, 0, 0], [3e-4, 1e-4, 0, -2e-4, 0, 0],
                               [-3e-4, -1e-4, 0, 1e-4, 0, 0]])
def test_spec_strain_split_derivatives_plane_strain(e):
    """SpecStrainSplit (PhaseFieldMaterial.cpp:239-290) on plane-strain states with distinct principal strains:
    the damaged stress is the energy's gradient and the tangents are the stresses' Jacobians."""
    m = _split_material("SpecStrains")
    e = np.array(e, dtype=float)
    Dd, Du, Sd, Su, en = orc.energy_split(m, 273.15, e)
    dE, dSd, dSu = _fd_split(m, e)
    sc = np.abs(Sd + Su).max()
    # finite differences in e_zz cross the kink at e_zz = 0 (s_0 = e_zz switches sides): compare off it
    assert np.abs(np.delete(dE - Sd, 2)).max() <= 1e-7 * sc
    mask = np.ones((6, 6), bool); mask[:, 2] = False
    assert np.abs((dSd - Dd)[mask]).max() <= 1e-6 * np.abs(Dd + Du).max()
    assert np.abs((dSu - Du)[mask]).max() <= 1e-6 * np.abs(Dd + Du).max()


def _lagrange_ctx(method, idx=0, seed=3):
    """Phase-field context with Lagrange-multiplier irreversibility: lMult_pf (and lMult_pf2) DOFs in the
    phase step; phase, old phase and multipliers set away from the methods' switching points."""
    mesh, d, st = cf.config(idx, scale=0.125)
    model = next(k for k, v in d["Models"].items() if isinstance(v, dict) and v.get("Name") == "Fracture/PhaseField")
    d["Models"][model]["Irreversible"] = method
    ph_step = d["Dofs"]["DofStep"][d["Dofs"]["DofNames"].index("phase")]
    extra = ["lMult_pf"] + (["lMult_pf2"] if method == "AugmentedLagrangeMult2" else [])
    d["Dofs"]["DofNames"] = list(d["Dofs"]["DofNames"]) + extra
    d["Dofs"]["DofStep"] = list(d["Dofs"]["DofStep"]) + [ph_step] * len(extra)
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    s = st()
    cf.apply_state(o, s)
    n, _ = o.step_info(1)
    nn = mesh.n_nodes
    rng = np.random.default_rng(seed)
    ph = o.get_state(1, abi.STATE_CUR)
    ph[:nn] = rng.uniform(0.05, 0.9, nn)
    ph[nn:] = rng.uniform(-0.6, 0.6, n - nn)                                   # multipliers
    old = ph.copy()
    old[:nn] = ph[:nn] + np.where(rng.random(nn) < 0.5, -0.05, 0.05)           # both sides of phi = phi_old
    o.set_state(1, abi.STATE_CUR, ph)
    o.set_state(1, abi.STATE_OLD, old)
    return mesh, d, o, s


@pytest.mark.parametrize("method", ["LagrangeMult", "AugmentedLagrangeMult", "AugmentedLagrangeMult2"])
def test_lagrange_irreversibility_tangent_finite_difference(method):
    """EnforceIrreversible with multipliers (PhaseFieldUtil.cpp:350-484): the [phase, L(, L2)] step's tangent is
    the derivative of its residual, and the multiplier DOFs follow the phase DOFs in the step's numbering."""
    mesh, d, o, s = _lagrange_ctx(method)
    nn = mesh.n_nodes
    nl = 2 if method == "AugmentedLagrangeMult2" else 1
    n, _ = o.step_info(1)
    assert n == (1 + nl) * nn
    assert np.array_equal(o.dof_numbers(abi.DOF_LMULT)[:nn], np.arange(nn, 2 * nn))
    o.assemble(0, dt=100.0)
    x0 = o.get_state(1, abi.STATE_CUR)
    o.assemble_nohist(1, dt=100.0)
    K = o.matrix(1).toarray()
    f0 = o.residual(1)
    assert np.linalg.norm(f0[nn:]) > 0 and np.linalg.norm(K[nn:, :nn]) + np.linalg.norm(K[nn:, nn:]) > 0
    v = np.random.default_rng(4).normal(size=x0.size)
    h = 1e-7
    o.set_state(1, abi.STATE_CUR, x0 + h * v); o.assemble_nohist(1, dt=100.0); fp = o.residual(1)
    o.set_state(1, abi.STATE_CUR, x0 - h * v); o.assemble_nohist(1, dt=100.0); fm = o.residual(1)
    fd = (fp - fm) / (2 * h)
    assert np.linalg.norm(fd - K @ v) <= 1e-6 * np.linalg.norm(K @ v)


def test_lagrange_dofs_must_match_the_method():
    mesh, d, st = cf.config(0, scale=0.125)
    d["Dofs"]["DofNames"] = list(d["Dofs"]["DofNames"]) + ["lMult_pf"]
    d["Dofs"]["DofStep"] = list(d["Dofs"]["DofStep"]) + [1]
    with pytest.raises(abi.IfemError):   # multipliers without a Lagrange method
        orc.context(mesh, cf.materials(d), cf.options_from_json(d))


def _ocean(d, hw, rho=1025.0):
    d["Models"]["Ocean"] = {"Name": "OceanBC", "hw": hw, "Fluid": "Water", "ElementGroup_u": "internal",
                            "ElementGroup_phase": "internal", "pwAboveWater": 0.0}
    d["properties"]["Water"] = {"SolidProperties": {"Density": rho}, "FluidProperties": {"Viscosity": 1e-3}}


def test_ocean_bc_total_load_closed_form():
    """OceanBCModel::Assemble_U (OceanBC.cpp:96-150) with the phase at 1 and the water above the 0.05 x 0.1 m box:
    the ux loads add up to rho g A (hw - y_centroid), since quadratic B-splines on Greville control points
    reproduce y, and the uy rows are untouched.  With the water level inside the box, the nodes above it get
    nothing."""
    mesh, d, st = cf.config(0, scale=0.125)
    o0 = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    hw, rho = 0.3, 1025.0
    _ocean(d, hw, rho)
    o1 = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    _ocean(d, 0.04, rho)
    o2 = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    s = st()
    n1, _ = o0.step_info(1)
    for o in (o0, o1, o2):
        cf.apply_state(o, s)
        o.set_state(1, abi.STATE_CUR, np.ones(n1))
        o.assemble(0, dt=100.0)
    df = o1.residual(0) - o0.residual(0)
    ux, uy = o1.dof_numbers(abi.DOF_UX), o1.dof_numbers(abi.DOF_UY)
    area, yc = 0.05 * 0.1, 0.05
    assert df[ux].sum() == pytest.approx(rho * 9.81 * area * (hw - yc), rel=1e-10)
    assert np.all(df[uy] == 0.0) and np.all(df[ux] > 0)
    df2 = o2.residual(0) - o0.residual(0)
    y = mesh.coords[:, 1]
    assert np.all(df2[ux][y > 0.04] == 0.0) and np.all(df2[ux][y < 0.04] > 0.0)


def test_ocean_bc_is_2d_only():
    mesh, d, st = cf.config(1, scale=0.125)
    _ocean(d, 0.3)
    with pytest.raises(abi.IfemError) as e:
        orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    assert e.value.code == abi.ERR_UNSUPPORTED


@pytest.mark.parametrize("idx", [0, 1])
def test_second_gradients_exact_for_quadratic_fields(idx):
    """getShapeGrads2 (B2_2.cpp:90-125, NURBS3_Cube2.cpp:117-216): on elements that do not touch the boundary the
    uniform quadratic B-spline with control values f(control point) represents f = x^T A x / 2 + b x up
    to a constant, so the second gradients are A at every ip (xx, yy(, zz), xy(, yz, xz)) and the first gradients
    A x + b.  (At the boundary the open knot vector's control values would need the polar form instead.)"""
    mesh, d, o, _ = _ctx(idx, 0.125)
    dim = mesh.dim
    rng = np.random.default_rng(5)
    A = rng.normal(size=(dim, dim)); A = A + A.T
    b = rng.normal(size=dim)
    X = mesh.coords
    f = 0.5 * np.einsum("ni,ij,nj->n", X, A, X) + X @ b
    pairs = [(0, 0), (1, 1), (0, 1)] if dim == 2 else [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    want = np.array([A[i, j] for i, j in pairs])
    sh = mesh.shape[:dim]
    inner = [(2, 2, 2), tuple(n // 2 for n in sh) + (0,) * (3 - dim), tuple(n - 3 for n in sh) + (0,) * (3 - dim)]
    for ijk in inner:
        el = ijk[0] + sh[0] * (ijk[1] + (sh[1] * ijk[2] if dim == 3 else 0))
        N, G, G2, w = o.shape2(el)
        fe = f[mesh.elems[el]]
        xq = N @ X[mesh.elems[el]]
        assert np.allclose(G2 @ fe, want[None, :], atol=1e-6 * np.abs(A).max())
        assert np.allclose(G @ fe, xq @ A + b, atol=1e-8 * (np.abs(A).max() + np.abs(b).max()))
        N1, G1, w1 = o.shape(el)
        assert np.allclose(N, N1, atol=1e-15) and np.allclose(w, w1, rtol=1e-13)


@pytest.mark.parametrize("dist", ["HO_Quadratic", "HO_CZM", "HO_Linear", "HO_Linear2", "Custom"])
@pytest.mark.parametrize("idx", [0, 1])
def test_second_gradient_distribution_tangent_finite_difference(idx, dist):
    """The phase-step tangent of the second-gradient crack densities (PhaseFieldUtil.cpp:223-280) is the exact
    derivative of their residual, with the lumped capacity (PhaseFieldUtil.cpp:282-348) on."""
    mesh, d, st = cf.config(idx, scale=0.125)
    d["properties"]["PhaseField"]["DistributionFunction"] = dist
    d["properties"]["PhaseField"]["Coefs"] = [2.0, 0.5, 1.0, 0.5, 0.1]
    d["Models"]["PhaseField1"]["LumpedPFCapacity"] = True
    d["Models"]["PhaseField1"]["Irreversible"] = "None"
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o, st())
    dt = 100.0 if idx == 1 else 1.0
    o.assemble(0, dt=dt)
    phi0 = o.get_state(1, abi.STATE_CUR)
    o.assemble_nohist(1, dt=dt)
    K = o.matrix(1).toarray()
    rng = np.random.default_rng(2)
    v = rng.normal(size=phi0.size)
    h = 1e-6
    o.set_state(1, abi.STATE_CUR, phi0 + h * v); o.assemble_nohist(1, dt=dt); fp = o.residual(1)
    o.set_state(1, abi.STATE_CUR, phi0 - h * v); o.assemble_nohist(1, dt=dt); fm = o.residual(1)
    fd = (fp - fm) / (2 * h)
    assert np.linalg.norm(fd - K @ v) <= 1e-7 * np.linalg.norm(K @ v)
