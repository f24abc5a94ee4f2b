"""Reference-style input dictionaries -> ABI structs, and the workload presets.

``from_json`` reads the same keys the reference's constructors read:
  properties/<Mat>/SolidProperties     SolidMaterial.cpp:5-67, BaseMaterial.cpp:9
  properties/<Mat>/FractureProperties  PhaseFieldMaterial.cpp:5-32, PhaseFieldUtil.cpp:5-6
  properties/<Mat>/TemperatureDependent IceMaterial.cpp:8-32
  properties/<Mat>/ThermalProperties   ThermalMaterial.cpp:5-10
  properties/PhaseField                PhaseField.cpp:198-267, PhaseFieldUtil.cpp:7-25, PhaseFieldMaterial.cpp:20-21
  Models/<PhaseField model>            PhaseField.cpp:193-228, PhaseFieldUtil.cpp:33-39
  Dofs/DofNames, Dofs/DofStep          DofSpace.cpp:14-21
Keys under "B200" have no reference counterpart (pinned temperature, Gc mode, tangent options).
"""
from __future__ import annotations

import copy
import math
import numpy as np

from . import abi
from .meshgen import box_face_groups, box_mesh, concat_meshes

DOF_NAME = {"ux": abi.DOF_UX, "uy": abi.DOF_UY, "uz": abi.DOF_UZ, "phase": abi.DOF_PHASE, "T": abi.DOF_T,
            "lMult_pf": abi.DOF_LMULT, "lMult_pf2": abi.DOF_LMULT2, "ox": abi.DOF_OX, "oy": abi.DOF_OY,
            "oz": abi.DOF_OZ}
PHASE_MODELS = ("Fracture/PhaseField", "Fracture/CossPhaseField")


def _get(d, path, default=None, required=False):
    cur = d
    for k in path:
        if not isinstance(cur, dict) or k not in cur:
            if required:
                raise KeyError("/".join(path))
            return default
        cur = cur[k]
    return cur


def material_from_json(d, mat_name) -> abi.Material:
    m = abi.Material()
    P = ("properties", mat_name)
    m.young = _get(d, P + ("SolidProperties", "Young"), required=True)
    m.poisson = _get(d, P + ("SolidProperties", "Poisson"), required=True)
    m.density = _get(d, P + ("SolidProperties", "Density"), required=True)
    m.damping = _get(d, P + ("SolidProperties", "Damping"), 0.0)
    rheo = _get(d, P + ("SolidProperties", "Rheology"), "LinearElastic")
    if rheo not in abi.RHEO:
        raise ValueError(f"Solid material model type {rheo} not supported")
    m.rheology = abi.RHEO[rheo]
    m.creep_a = _get(d, P + ("SolidProperties", "A"), 0.0, required=rheo != "LinearElastic")
    m.creep_n = _get(d, P + ("SolidProperties", "n"), 1.0, required=rheo != "LinearElastic")
    m.phi_visc_lim = _get(d, P + ("SolidProperties", "PhiViscLim"), 1.0e3)
    m.pf_l = _get(d, P + ("FractureProperties", "l"), required=True)
    m.gc = _get(d, P + ("FractureProperties", "Gc"), required=True)
    m.pf_visc = _get(d, P + ("FractureProperties", "Viscosity"), 0.0)
    split = _get(d, P + ("FractureProperties", "Split"), required=True)
    if split not in abi.SPLIT:
        raise ValueError(f"Stress split function type {split} not supported")
    m.split = abi.SPLIT[split]
    m.star_convex_gamma = _get(d, P + ("FractureProperties", "StarConvexGamma"), 0.0)
    m.ice_eref = _get(d, P + ("FractureProperties", "eRef"), 0.0)
    m.ice_creduce = _get(d, P + ("FractureProperties", "cReduce"), 0.0)
    m.b_dp = _get(d, P + ("FractureProperties", "B_DP"), 0.0, required=split == "DruckerPrager")
    T = P + ("TemperatureDependent",)
    m.t_ref = _get(d, T + ("TRef",), required=True)
    m.t_offset = _get(d, T + ("TOffset",), 0.0)
    m.q_creep = _get(d, T + ("QCreep",), required=True)
    m.ft0 = _get(d, T + ("ft0",), required=True)
    m.ftdeg = _get(d, T + ("ftdeg",), required=True)
    m.ice_creduce_fact = _get(d, T + ("Ice_cReduceFact",), 0.0)
    m.ice_ereduce_fact = _get(d, T + ("Ice_eReduceFact",), 0.0)
    m.k_thermal = _get(d, P + ("ThermalProperties", "ThermalConductivity"), 0.0)
    m.cp = _get(d, P + ("ThermalProperties", "HeatCapacity"), 0.0)
    m.consistent_energy = 1 if _get(d, ("properties", "PhaseField", "ConsistentEnergy"), True) else 0
    m.gc_mode = 1 if _get(d, ("B200", "GcMode"), "derived") == "input" else 0
    if rheo in ("ViscoElasticPlastic", "DamViscoElasticPlastic"):
        # SolidMaterial.cpp:50-65 and IceMaterial.cpp:36-37 (sydeg is read for every ice material there)
        m.vep_sy = _get(d, P + ("SolidProperties", "sy"), required=True)
        m.vep_sydeg = _get(d, T + ("sydeg",), required=True)
        m.vep_f_deg = _get(d, P + ("SolidProperties", "F_deg"), 0.0)
        m.vep_g_deg = _get(d, P + ("SolidProperties", "G_deg"), m.vep_f_deg)
        m.vep_hardening = _get(d, P + ("SolidProperties", "hardening"), 0.0)
        m.vep_pl_visc = _get(d, P + ("SolidProperties", "pl_visc"), 0.0)
    # CosseratMaterial.cpp:3-10 (the reference's ice always reads l_coss and G_coss; the phase-field model
    # does not use them)
    m.l_coss = _get(d, P + ("SolidProperties", "l_coss"), 0.0)
    m.g_coss = _get(d, P + ("SolidProperties", "G_coss"), 0.0)
    m.hard_e_ref = _get(d, P + ("SolidProperties", "hard_eRef"), 0.0)
    return m


def options_from_json(d, model_name=None) -> abi.Options:
    o = abi.Options()
    names = _get(d, ("Dofs", "DofNames"), required=True)
    steps = _get(d, ("Dofs", "DofStep"), required=True)
    if len(names) != len(steps):
        raise ValueError("Please specify dof steps for all dofs")
    o.n_dofs = len(names)
    for i, (n, s) in enumerate(zip(names, steps)):
        if n not in DOF_NAME:
            raise ValueError(f"DOF {n} not supported by this path")
        o.dof_kind[i] = DOF_NAME[n]
        o.dof_step[i] = s
    models = _get(d, ("Models",), {})
    if model_name is None:
        model_name = next(k for k, v in models.items() if isinstance(v, dict) and v.get("Name") in PHASE_MODELS)
    M = ("Models", model_name)
    PF = ("properties", "PhaseField")
    o.cosserat = 1 if _get(d, M + ("Name",)) == "Fracture/CossPhaseField" else 0
    # CossPhaseField.cpp:267-273 reads GravityDamage; PhaseField.cpp:249-250 uses DensityDamage for gravity
    o.gravity_dam_function = abi.DAM[_get(d, PF + ("GravityDamage" if o.cosserat else "DensityDamage",),
                                          required=True)]
    o.dam_function = abi.DAM[_get(d, PF + ("DamFunction",), required=True)]
    o.density_dam_function = abi.DAM[_get(d, PF + ("DensityDamage",), required=True)]
    o.visco_driving_factor = _get(d, PF + ("ViscoDrivingFactor",), 0.0)
    o.visco_dam_function = abi.DAM[_get(d, PF + ("ViscoDriving",), "None")]
    o.distribution = abi.DIST[_get(d, PF + ("DistributionFunction",), "Quadratic")]
    if o.distribution == abi.DIST["Custom"]:
        coefs = _get(d, PF + ("Coefs",), required=True)
        if len(coefs) != 5:
            raise ValueError("properties/PhaseField/Coefs needs 5 values")
        for i, v in enumerate(coefs):
            o.dist_coefs[i] = float(v)
    o.irreversible = abi.IRR[_get(d, M + ("Irreversible",), "Hist")]
    o.k0 = _get(d, PF + ("k0",), required=True)
    o.porder_p = _get(d, PF + ("p",), 2.0)
    o.consistent_degradation = 1 if _get(d, PF + ("ConsistentDegradation",), False) else 0
    o.visc_num = _get(d, M + ("ViscousStab",), required=True)
    o.inertia = 1 if _get(d, M + ("Intertia",), False) else 0
    o.gravity = 1 if _get(d, M + ("Gravity",), False) else 0
    o.lumped_cap = 1 if _get(d, M + ("LumpedPFCapacity",), False) else 0
    o.lumped_drive = 1 if _get(d, M + ("LumpedDriving",), False) else 0
    o.viscous_heating = 1 if _get(d, M + ("ViscousHeating",), False) else 0
    o.thermal_model = 1 if any(isinstance(v, dict) and v.get("Name") == "Thermal/ThermalModel"
                               for v in models.values()) else 0
    B = ("B200",)
    o.ref_compat_phase_t = 1 if _get(d, B + ("RefCompatPhaseT",), True) else 0
    o.pinned_temperature = _get(d, B + ("PinnedTemperature",), 273.15)
    o.tangent_mode = {"reference": 0, "consistent": 1}[_get(d, B + ("Tangent",), "reference")]
    o.tangent_precision = {"fp64": 0, "fp32": 1, "tc_split": 2, "tf32x3": 2}[_get(d, B + ("TangentPrecision",), "fp64")]
    o.rm_tol_mode = {"reference": 0, "tight": 1}[_get(d, B + ("ReturnMapTolerance",), "reference")]
    o.rm_max_it = _get(d, B + ("ReturnMapMaxIt",), 250)
    o.penalty_factor = 1.0e6
    o.lag_fact = 1.0
    # OceanBC (OceanBC.cpp:40-80): water level and the fluid material's density
    ocean = next((k for k, v in models.items() if isinstance(v, dict) and v.get("Name") == "OceanBC"), None)
    if ocean is not None:
        o.ocean_bc = 1
        o.ocean_hw = _get(d, ("Models", ocean, "hw"), required=True)
        fluid = _get(d, ("Models", ocean, "Fluid"), required=True)
        o.ocean_density = _get(d, ("properties", fluid, "SolidProperties", "Density"), required=True)
    return o


# --------------------------------------------------------------------------------------------
# Workload presets (the five configurations the benchmarks and parity tests use)
# --------------------------------------------------------------------------------------------
def _ice(young=9.5e9, poisson=0.35, density=917.0, rheology="LinearElastic", A=0.0, n=3.0,
         l=2.0e-3, gc=1.0, split="VolStrains", t_ref=273.15, t_offset=0.0, q=0.0, ft0=None, ftdeg=0.0,
         visc=0.0, k=2.0, cp=2.1e3, damping=0.0):
    if ft0 is None:                       # Gc = 2 ft0^2 l / E  (IceMaterial.cpp:71-72) -> ft0 for the requested Gc
        ft0 = math.sqrt(gc * young / (2.0 * l))
    return {
        "SolidProperties": {"Density": density, "Young": young, "Poisson": poisson, "Damping": damping,
                            "Rheology": rheology, "A": A, "n": n},
        "FractureProperties": {"Split": split, "l": l, "Gc": gc, "Viscosity": visc},
        "TemperatureDependent": {"TemperatureDependent": True, "TRef": t_ref, "TOffset": t_offset,
                                 "QCreep": q, "ft0": ft0, "ftdeg": ftdeg, "sydeg": 0.0},
        "ThermalProperties": {"ThermalConductivity": k, "HeatCapacity": cp},
    }


def _base_json(dim, names, steps, ice, *, gravity=False, viscous_heating=False, thermal=False,
               b200=None):
    d = {
        "mesh": {"dim": dim, "ipcount1D": 3},
        "properties": {
            "PhaseField": {"DamFunction": "Quadratic", "DensityDamage": "None", "DistributionFunction": "Quadratic",
                           "k0": 1.0e-12, "ConsistentEnergy": True, "ConsistentDegradation": False},
            "Ice": ice,
        },
        "Dofs": {"DofNames": names, "DofStep": steps},
        "Models": {"Names": ["PhaseField1"] + (["Thermal"] if thermal else []),
                   "PhaseField1": {"Name": "Fracture/PhaseField", "ElementGroup_u": "internal",
                                   "ElementGroup_phase": "internal", "ElementGroup_T": "internal",
                                   "Material": "Ice", "ViscousStab": 0.0, "Irreversible": "Hist",
                                   "Gravity": gravity, "ViscousHeating": viscous_heating}},
        "B200": dict(b200 or {}),
    }
    if thermal:
        d["Models"]["Thermal"] = {"Name": "Thermal/ThermalModel", "ElementGroup_T": "internal", "Material": "Ice"}
    return d


GLEN_A0 = 2.4e-24      # Pa^-3 s^-1 at 0 degC
GLEN_Q = 115.0e3       # J/mol


def config(idx: int, scale: float = 1.0, seed: int = 0):
    """Return (mesh, json_dict, state_fn) of workload `idx` (0..4).  `scale` shrinks the mesh
    (element counts per direction multiplied by scale, at least 2) for parity tests."""
    def sz(n):
        return max(2, int(round(n * scale)))
    if idx == 0:
        mesh = box_mesh((sz(64), sz(128)), (0.05, 0.1))
        d = _base_json(2, ["ux", "uy", "phase"], [0, 0, 1], _ice(), b200={"PinnedTemperature": 273.15})
        return mesh, d, lambda ctx=None, s=1.0: state_config0(mesh, seed, s)
    if idx in (1, 3):
        n = (32, 32, 64) if idx == 1 else (48, 48, 48)
        L = (0.05, 0.05, 0.1) if idx == 1 else (0.05, 0.05, 0.05)
        mesh = box_mesh(tuple(sz(v) for v in n), L)
        ice = _ice(rheology="DamViscoElastic", A=GLEN_A0, n=3.0, q=GLEN_Q)
        b = {"PinnedTemperature": 263.15}
        if idx == 3:
            b["GcMode"] = "input"
        d = _base_json(3, ["ux", "uy", "uz", "phase"], [0, 0, 0, 1], ice, b200=b)
        phi_max = 0.5 if idx == 1 else 0.9
        return mesh, d, lambda ctx=None, s=1.0: state_smooth(mesh, seed, phi_max=phi_max, uniform_phi=(idx == 3))
    if idx == 2:
        mesh = box_mesh((sz(512), sz(256)), (400.0, 200.0))
        ice = _ice(rheology="DamViscoElastic", A=1.0e-24, n=3.0, q=150.0e3, l=2.5, gc=4.0,
                   t_offset=273.15, ftdeg=4.0e4)
        d = _base_json(2, ["ux", "uy", "phase", "T"], [0, 0, 1, 2], ice, gravity=True,
                       viscous_heating=True, thermal=True, b200={"RefCompatPhaseT": True})
        return mesh, d, lambda ctx=None, s=1.0: state_config2(mesh, seed)
    if idx == 4:
        return batch_config(specimen_draws(scale, seed), seed)
    raise ValueError(idx)


def triaxial_config(dim: int, scale: float = 1.0, seed: int = 0):
    """A triaxial compression specimen (TestCases/TriAxialCompression/TriAxial.json, TriAxial2D.json): a box
    centred on the vertical axis, as the reference's cylinder is, the damaged Glen ice of the 3D workload
    (linear-elastic ice in 2D), and a TriAxial model "Tri" with a confining pressure on the side group and a
    displacement-controlled top group.  Returns (mesh, json_dict, state_fn)."""
    def sz(n):
        return max(2, int(round(n * scale)))
    if dim == 3:
        mesh = box_mesh((sz(16), sz(16), sz(32)), (0.05, 0.05, 0.1), origin=(-0.025, -0.025, 0.0))
        ice = _ice(rheology="DamViscoElastic", A=GLEN_A0, n=3.0, q=GLEN_Q)
        d = _base_json(3, ["ux", "uy", "uz", "phase"], [0, 0, 0, 1], ice, b200={"PinnedTemperature": 263.15})
    else:
        mesh = box_mesh((sz(32), sz(64)), (0.05, 0.1), origin=(-0.025, 0.0))
        d = _base_json(2, ["ux", "uy", "phase"], [0, 0, 1], _ice(), b200={"PinnedTemperature": 263.15})
    d["Models"]["Names"].append("Tri")
    d["Models"]["Tri"] = {"Name": "TriAxial", "SideGroup": "side", "TopGroup": "top", "p0": -1.0e6, "dU": -1.0e-4,
                          "DamagedForces": True, "dummy": 1.0e11, "Material": "Ice", "t_postFail": 0.5}
    return mesh, d, lambda ctx=None, s=1.0: state_smooth(mesh, seed, phi_max=0.5)


def cosserat_config(dim: int, scale: float = 1.0, seed: int = 0, rheology: str = "DamViscoElasticPlastic",
                    split: str = "SpecStress", distribution: str = "HO_Linear2",
                    irreversible: str = "AugmentedLagrangeMult", thermal: bool = True):
    """A Cosserat phase-field specimen with the inputs of TestCases/TriAxialCompression/TriAxial2D.json and
    TriAxial.json (Fracture/CossPhaseField, damaged viscoelastic-plastic ice with micro-rotations, spectral
    stress split, HO_Linear2 crack density, augmented Lagrange irreversibility, inertia, damping and viscous
    heating), on a box centred on the vertical axis.  Returns (mesh, json_dict, state_fn)."""
    def sz(n):
        return max(2, int(round(n * scale)))
    if dim == 3:
        mesh = box_mesh((sz(8), sz(8), sz(16)), (0.05, 0.05, 0.1), origin=(-0.025, -0.025, 0.0))
        names, steps = ["ux", "uy", "uz", "ox", "oy", "oz", "phase"], [0, 0, 0, 0, 0, 0, 1]
    else:
        mesh = box_mesh((sz(32), sz(64)), (0.05, 0.1), origin=(-0.025, 0.0))
        names, steps = ["ux", "uy", "oz", "phase"], [0, 0, 0, 1]
    if irreversible in ("LagrangeMult", "AugmentedLagrangeMult", "AugmentedLagrangeMult2"):
        names.append("lMult_pf"); steps.append(1)
    if irreversible == "AugmentedLagrangeMult2":
        names.append("lMult_pf2"); steps.append(1)
    if thermal:
        names.append("T"); steps.append(2)
    ice = _ice(young=5.0e9, poisson=0.35, density=910.0, rheology=rheology, A=1.0e-24, n=3.0, l=1.5e-3, gc=4.0,
               split=split, t_ref=273.15, t_offset=273.15, q=150.0e3, ft0=0.2e6, ftdeg=4.0e4, visc=0.1,
               damping=1.0e6)
    ice["SolidProperties"].update({"G_coss": 1.8e9, "l_coss": 2.5e-3, "PhiViscLim": 0.2, "sy": 9.5e6,
                                   "hardening": -0.9, "hard_eRef": 2.0e-4, "pl_visc": 1.0e3})
    ice["TemperatureDependent"]["sydeg"] = 0.5e6
    d = _base_json(dim, names, steps, ice, thermal=thermal, viscous_heating=thermal,
                   b200={"PinnedTemperature": -11.0})
    d["properties"]["PhaseField"].update({"DensityDamage": "Step2", "GravityDamage": "Step2",
                                          "DistributionFunction": distribution, "ConsistentEnergy": False})
    mdl = d["Models"]["PhaseField1"]
    mdl.update({"Name": "Fracture/CossPhaseField", "Irreversible": irreversible, "Intertia": True,
                "LumpedPFCapacity": False})
    return mesh, d, lambda ctx=None, s=1.0: state_cosserat(mesh, seed, thermal)


def state_cosserat(mesh, seed=0, thermal=True):
    """Smooth displacements (axial compression 1e-4 plus a random field), micro-rotations of the order of the
    strains, a smooth phase field in [0, 0.5], velocities and accelerations, and a temperature near -11 degC."""
    rng = np.random.default_rng(seed)
    X = mesh.coords
    dim = mesh.dim
    h = (X.max(axis=0) - X.min(axis=0)) / np.array(mesh.shape[:dim])
    length = 5.0 * h.mean()
    base = np.array([3.0e-5, 3.0e-5, -1.0e-4])[3 - dim:] if dim == 2 else np.array([3.0e-5, 3.0e-5, -1.0e-4])
    comps = [base[c] * X[:, c] + _smooth_field(X, rng, 6, length) * 1.0e-4 * length / (2 * np.pi) for c in range(dim)]
    rots = [_smooth_field(X, rng, 4, length) * 5.0e-5 for _ in range(1 if dim == 2 else 3)]
    U = np.concatenate(comps + rots)
    phi = 0.5 * 0.5 * (1.0 + np.tanh(_smooth_field(X, rng, 4, 3 * length)))
    st = {0: {abi.STATE_CUR: U, abi.STATE_OLD: U * 0.98, abi.STATE_D: rng.normal(0, 1e-4, U.size),
              abi.STATE_DD: rng.normal(0, 1e-2, U.size)},
          1: {abi.STATE_CUR: phi, abi.STATE_OLD: phi * 0.95}}
    if thermal:
        T = -11.0 + 2.0 * _smooth_field(X, rng, 3, 3 * length)
        st[2] = {abi.STATE_CUR: T, abi.STATE_OLD: T}
    return st


def triaxial_params(d, model: str = "Tri") -> dict:
    """Models/<model> inputs of a TriAxial model (TriAxial.cpp:53-60) as keyword arguments of set_triaxial."""
    m = _get(d, ("Models", model), required=True)
    return {"p0": float(m["p0"]), "du": float(m["dU"]), "penalty": float(m["dummy"]),
            "t_post_fail": float(m["t_postFail"]), "damaged_forces": bool(m["DamagedForces"])}


def attach_triaxial(ctx, mesh, d, model: str = "Tri"):
    """Attach the TriAxial model of `d` to a context, on the box mesh's "side" and "top" face groups."""
    m = _get(d, ("Models", model), required=True)
    groups = box_face_groups(mesh)
    ctx.set_triaxial(groups[m["SideGroup"]], groups[m["TopGroup"]], **triaxial_params(d, model))
    return groups


def specimen_draws(scale: float = 1.0, seed: int = 0):
    """Sizes and (Gc, l, A, n) of the batched calibration specimens, drawn from the seed: 256 specimens of
    nx x 2nx elements with nx in [16, 96] at full scale (2..4 when scale < 1), parameters log-uniform around the
    2D tension specimen's values.  Each entry carries its global index, so any subset rebuilds identically.

    A is drawn log-uniform (factor e^{+-1}) around the n = 3 Glen factor at the reference stress of 1 MPa:
    A = A0 e^u (1 MPa)^(3 - n), so every specimen creeps at 1 MPa within e^{+-1} of the n = 3 rate.  The unscaled
    A0 e^u with n up to 3.5 makes the creep at the specimens' 10-30 MPa peak stresses so stiff that the
    reference's viscous return map (SolidMaterial.cpp:200-269) stops at its 250-iteration cap, unconverged, at
    74 of the 18.4 M integration points, where its answer depends on the round-off of the iteration path."""
    rng = np.random.default_rng(seed)
    n_spec = max(2, int(round(256 * scale)))
    out = []
    for i in range(n_spec):
        nx = int(rng.integers(16, 97)) if scale >= 1.0 else int(rng.integers(2, 5))
        out.append(dict(index=i, nx=nx,
                        gc=float(np.exp(rng.uniform(np.log(0.5), np.log(2.0)))),
                        l=float(np.exp(rng.uniform(np.log(1e-3), np.log(4e-3)))),
                        A=float(GLEN_A0 * np.exp(rng.uniform(-1.0, 1.0))),
                        n=float(np.exp(rng.uniform(np.log(2.5), np.log(3.5))))))
        out[-1]["A"] *= 1.0e6 ** (3.0 - out[-1]["n"])
    return out


def batch_config(specs, seed: int = 0):
    """(mesh, json_dict, state_fn) of a set of specimens (all of specimen_draws, or one rank's share)."""
    meshes = [box_mesh((sp["nx"], 2 * sp["nx"]), (0.05, 0.1)) for sp in specs]
    mesh = concat_meshes(meshes)
    ice = _ice(rheology="DamViscoElastic", A=GLEN_A0, n=3.0, q=GLEN_Q)
    d = _base_json(2, ["ux", "uy", "phase"], [0, 0, 1], ice,
                   b200={"PinnedTemperature": 263.15, "GcMode": "input"})
    d["B200"]["Specimens"] = [dict(gc=sp["gc"], l=sp["l"], A=sp["A"], n=sp["n"]) for sp in specs]
    offsets = [sp["index"] for sp in specs]
    return mesh, d, lambda ctx=None, s=1.0: state_batch(mesh, meshes, seed, offsets)


def materials(d, mat_name="Ice"):
    """All material sets of a dictionary (one, or one per specimen for the batched sweep)."""
    base = material_from_json(d, mat_name)
    specs = _get(d, ("B200", "Specimens"))
    if not specs:
        return [base]
    out = []
    for s in specs:
        m = copy.copy(base)
        m.gc, m.pf_l, m.creep_a, m.creep_n = s["gc"], s["l"], s["A"], s["n"]
        out.append(m)
    return out


# --------------------------------------------------------------------------------------------
# Synthetic states (seeded); each returns {step: {kind: vector}} in DOF numbering order
# --------------------------------------------------------------------------------------------
def _node_fields(mesh):
    return mesh.coords


def _gaussians(X, centers, sigma, peak):
    phi = np.zeros(X.shape[0])
    for c in centers:
        r2 = ((X - c) ** 2).sum(axis=1)
        phi += peak * np.exp(-0.5 * r2 / sigma ** 2)
    return np.minimum(phi, 1.0)


def state_config0(mesh, seed=0, load_frac=1.0):
    """Bottom fixed, top pulled to strain 1e-3*load_frac (linear field) + 1e-6 m nodal noise;
    phase = 3 seeded Gaussian flaws (sigma 1 mm, peak 0.5)."""
    rng = np.random.default_rng(seed)
    X = mesh.coords
    eps = 1.0e-3 * load_frac
    ux = rng.normal(0.0, 1e-6, mesh.n_nodes)
    uy = eps * X[:, 1] + rng.normal(0.0, 1e-6, mesh.n_nodes)
    lo, hi = X.min(axis=0), X.max(axis=0)
    centers = lo + rng.uniform(0.2, 0.8, size=(3, 2)) * (hi - lo)
    phi = _gaussians(X, centers, 1.0e-3, 0.5)
    U = np.concatenate([ux, uy])
    return {0: {abi.STATE_CUR: U, abi.STATE_OLD: U * 0.95},
            1: {abi.STATE_CUR: phi, abi.STATE_OLD: phi * 0.9}}


def _smooth_field(X, rng, n_modes, length):
    f = np.zeros(X.shape[0])
    for _ in range(n_modes):
        k = rng.normal(size=X.shape[1])
        k *= 2 * np.pi / length / np.linalg.norm(k)
        f += rng.normal() * np.sin(X @ k + rng.uniform(0, 2 * np.pi))
    return f / np.sqrt(n_modes)


def state_smooth(mesh, seed=0, phi_max=0.5, uniform_phi=False):
    """Confined compression (1 MPa-like) plus a smooth random strain field of amplitude 1e-4
    with a length scale of 5 elements; phase smooth in [0, phi_max] (or uniform per node)."""
    rng = np.random.default_rng(seed)
    X = mesh.coords
    dim = mesh.dim
    h = (X.max(axis=0) - X.min(axis=0)) / np.array(mesh.shape[:dim])
    length = 5.0 * h.mean()
    base = np.array([-3.0e-5, -3.0e-5, -1.0e-4])[:dim]
    comps = []
    for c in range(dim):
        pert = _smooth_field(X, rng, 6, length) * 1.0e-4 * length / (2 * np.pi)
        comps.append(base[c] * X[:, c] + pert)
    U = np.concatenate(comps)
    if uniform_phi:
        phi = rng.uniform(0.0, phi_max, mesh.n_nodes)
    else:
        phi = phi_max * 0.5 * (1.0 + np.tanh(_smooth_field(X, rng, 4, 3 * length)))
    UO = U * 0.98
    return {0: {abi.STATE_CUR: U, abi.STATE_OLD: UO},
            1: {abi.STATE_CUR: phi, abi.STATE_OLD: phi * 0.95}}


def state_config2(mesh, seed=0):
    rng = np.random.default_rng(seed)
    X = mesh.coords
    H = X[:, 1].max()
    ux = 1e-4 * X[:, 0] * (X[:, 1] / H) + rng.normal(0, 1e-5, mesh.n_nodes)
    uy = -2e-4 * X[:, 1] + rng.normal(0, 1e-5, mesh.n_nodes)
    phi = _gaussians(X, X.min(axis=0) + rng.uniform(0.3, 0.7, size=(3, 2)) * (X.max(axis=0) - X.min(axis=0)), 5.0, 0.6)
    T = -20.0 * (X[:, 1] / H)            # degC: -20 at the surface (top), 0 at the base
    U = np.concatenate([ux, uy])
    return {0: {abi.STATE_CUR: U, abi.STATE_OLD: U * 0.98},
            1: {abi.STATE_CUR: phi, abi.STATE_OLD: phi * 0.95},
            2: {abi.STATE_CUR: T, abi.STATE_OLD: T, abi.STATE_D: rng.normal(0, 1e-4, mesh.n_nodes)}}


def state_batch(mesh, meshes, seed=0, indices=None):
    parts_u, parts_v, parts_p = [], [], []
    for i, m in enumerate(meshes):
        st = state_config0(m, seed + (indices[i] if indices is not None else i), 1.0)
        U = st[0][abi.STATE_CUR]
        n = m.n_nodes
        parts_u.append(U[:n]); parts_v.append(U[n:]); parts_p.append(st[1][abi.STATE_CUR])
    U = np.concatenate(parts_u + parts_v)
    phi = np.concatenate(parts_p)
    return {0: {abi.STATE_CUR: U, abi.STATE_OLD: U * 0.95},
            1: {abi.STATE_CUR: phi, abi.STATE_OLD: phi * 0.9}}


def apply_state(ctx, state):
    """Copy a synthetic state into a context (node-ordered fields map 1:1 onto DOF numbers
    because every node of the group carries every DOF, numbered type-major in node order)."""
    for step, kinds in state.items():
        if step >= ctx.nsteps:
            continue
        n, _ = ctx.step_info(step)
        for kind, v in kinds.items():
            ctx.set_state(step, kind, v[:n] if v.size >= n else np.pad(v, (0, n - v.size)))
