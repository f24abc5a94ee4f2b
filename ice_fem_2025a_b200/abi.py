"""ctypes view of include/icefem_b200.h and a thin Python handle over the C-ABI.

The native library ``ice_fem_2025a_b200/_lib/libicefem_b200.so`` is the product; this module only
marshals arguments.  ``Context`` works for any library exporting the ifem_* functions under a
prefix (the CPU oracle under ``tests`` uses the prefix ``oracle_``).
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

# ---- constants (icefem_b200.h) ----
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_NUMERIC, ERR_UNSUPPORTED, ERR_CAPACITY = range(8)
ELEM_B2_2, ELEM_NURBS3_CUBE2 = 1, 2
DOF_UX, DOF_UY, DOF_UZ, DOF_PHASE, DOF_T, DOF_LMULT, DOF_LMULT2, DOF_OX, DOF_OY, DOF_OZ = range(10)
RHEO = {"LinearElastic": 0, "ViscoElastic": 1, "DamViscoElastic": 2, "ViscoElasticExpl": 3,
        "DamViscoElasticExpl": 4, "ViscoElasticPlastic": 5, "DamViscoElasticPlastic": 6}
RHEO_VEP, RHEO_DVEP = 5, 6
SPLIT = {"None": 0, "VolStrains": 1, "SpecStrains": 2, "VolStress": 3, "SpecStress": 4, "DruckerPrager": 5, "ICE": 6,
         "StarConvex": 7}
DAM = {"None": 0, "Step2": 1, "Step5": 2, "Step8": 3, "Linear": 4, "Quadratic": 5, "Cubic": 6,
       "LinearNoRes": 7, "QuadraticNoRes": 8, "CubicNoRes": 9, "CZM": 10, "Porder": 11}
DIST = {"Linear": 0, "CZM": 1, "Linear2": 2, "Quadratic": 3, "HO_Linear": 4, "HO_Linear2": 5, "HO_CZM": 6,
        "HO_Quadratic": 7, "Local": 8, "Custom": 9}
DIST_SECOND_GRADIENT = (4, 5, 6, 7, 9)   # the distributions that integrate second gradients of the phase field
IRR = {"None": 0, "Hist": 1, "Penalty": 2, "LagrangeMult": 3, "AugmentedLagrangeMult": 4, "AugmentedLagrangeMult2": 5}
TANGENT_REFERENCE, TANGENT_CONSISTENT = 0, 1
PREC_FP64, PREC_FP32, PREC_TC_SPLIT = 0, 1, 2
PREC_TF32X3 = PREC_TC_SPLIT   # former name of PREC_TC_SPLIT
RM_REFERENCE, RM_TIGHT = 0, 1
PC_BLOCK_JACOBI, PC_AMG, PC_AMG_REUSE = 0, 1, 2
COMMIT_TIMEDEP, COMMIT_PATHDEP = 1, 2
HIST_ENERGY, HIST_PLASTIC_STRAIN, HIST_VISC_DISS, HIST_DAM_VISC_DISS, HIST_MAT = range(5)
STATE_CUR, STATE_OLD, STATE_D, STATE_DD = range(4)
F64, F32 = 0, 1

_dp = C.POINTER(C.c_double)


class MeshDesc(C.Structure):
    _fields_ = [("dim", C.c_int32), ("elem_type", C.c_int32), ("ipcount1d", C.c_int32),
                ("reserved0", C.c_int32), ("n_nodes", C.c_int64), ("n_elems", C.c_int64),
                ("coords", _dp), ("node_weights", _dp), ("elems", C.POINTER(C.c_int64)),
                ("elem_data", _dp), ("elem_kron", _dp), ("elem_mat", C.POINTER(C.c_int32))]


class Material(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "young", "poisson", "density", "damping", "creep_a", "creep_n", "phi_visc_lim",
        "pf_l", "gc", "pf_visc", "star_convex_gamma", "ice_eref", "ice_creduce",
        "t_ref", "t_offset", "q_creep", "ft0", "ftdeg", "ice_creduce_fact", "ice_ereduce_fact",
        "k_thermal", "cp")] + [(n, C.c_int32) for n in ("rheology", "split", "consistent_energy", "gc_mode")] + \
        [(n, C.c_double) for n in ("vep_sy", "vep_sydeg", "vep_f_deg", "vep_g_deg", "vep_hardening", "vep_pl_visc",
                                   "b_dp", "l_coss", "g_coss", "hard_e_ref")]


class Options(C.Structure):
    _fields_ = ([("n_dofs", C.c_int32), ("dof_kind", C.c_int32 * 10), ("dof_step", C.c_int32 * 10)] +
                [(n, C.c_int32) for n in (
                    "dam_function", "density_dam_function", "visco_dam_function", "distribution",
                    "irreversible", "inertia", "gravity", "lumped_cap", "lumped_drive", "viscous_heating",
                    "consistent_degradation", "thermal_model", "ref_compat_phase_t", "tangent_mode",
                    "tangent_precision", "rm_tol_mode", "rm_max_it", "ocean_bc")] +
                [(n, C.c_double) for n in ("k0", "visc_num", "visco_driving_factor", "pinned_temperature",
                                           "penalty_factor", "lag_fact", "ocean_hw", "ocean_density", "porder_p")] +
                [("dist_coefs", C.c_double * 5), ("cosserat", C.c_int32), ("gravity_dam_function", C.c_int32)])


class Time(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("du_dt", C.c_double), ("ddu_dt", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_element", C.c_double), ("ms_scatter", C.c_double),
                ("rm_iterations", C.c_int64), ("rm_capped", C.c_int64), ("nonfinite", C.c_int64),
                ("crack_length", C.c_double), ("ms_points", C.c_double), ("ms_tangent", C.c_double)]


class FaceGroup(C.Structure):
    _fields_ = [("n_faces", C.c_int64), ("faces", C.POINTER(C.c_int64)), ("face_data", _dp)]


class TriAxialParams(C.Structure):
    _fields_ = [("p0", C.c_double), ("du", C.c_double), ("penalty", C.c_double), ("t_post_fail", C.c_double),
                ("damaged_forces", C.c_int32), ("reserved", C.c_int32)]


class TriAxialState(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("area", "f_ext", "uz_sum", "u0", "t_break", "max_load", "p0")] + \
        [("min_load_passed", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


# exported symbols of include/icefem_b200.h (tests check the library exports all of them)
ABI_FUNCTIONS = (
    "abi_version", "ctx_create", "ctx_destroy", "last_error", "step_info", "get_dof_numbers",
    "build_pattern", "set_state", "get_state", "assemble", "get_residual", "get_matrix",
    "device_outputs", "commit", "reset_step", "get_history", "set_history", "set_tangent",
    "get_stats", "adjoint", "set_param", "assemble_async", "sync", "get_stream")


class IfemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ifem error {code}: {msg}")
        self.code = code


def multigrid_plan(A, node_of_row, modes, threshold=0.0, lib=None, max_levels=16):
    """Rows and nonzeros per level of the multigrid hierarchy for the CSR matrix A (scipy), planned on the host
    (ifem_multigrid_plan; no GPU needed)."""
    import scipy.sparse as sp
    A = sp.csr_matrix(A)
    lib = lib or load_product()
    rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(A.indices, dtype=np.int32)
    v = np.ascontiguousarray(A.data, dtype=np.float64)
    nd = np.ascontiguousarray(node_of_row, dtype=np.int32)
    B = np.ascontiguousarray(np.asarray(modes, dtype=np.float64).reshape(A.shape[0], -1))
    nl = C.c_int32()
    rows = np.zeros(max_levels, np.int64)
    nnz = np.zeros(max_levels, np.int64)
    rc = lib.ifem_multigrid_plan(C.c_int64(A.shape[0]), _ptr(rp, C.c_int64), _ptr(ci, C.c_int32), _ptr(v, C.c_double),
                                 _ptr(nd, C.c_int32), C.c_int64(int(nd.max()) + 1 if nd.size else 0),
                                 C.c_int32(B.shape[1]), _ptr(B, C.c_double), C.c_double(threshold),
                                 C.c_int32(max_levels), C.byref(nl), _ptr(rows, C.c_int64), _ptr(nnz, C.c_int64))
    if rc != OK:
        raise IfemError(rc, "ifem_multigrid_plan")
    k = min(nl.value, max_levels)
    return rows[:k].tolist(), nnz[:k].tolist()


def _here():
    return os.path.dirname(os.path.abspath(__file__))


def product_library_path() -> str:
    return os.path.join(_here(), "_lib", "libicefem_b200.so")


_product = None


def load_product():
    """Load the CUDA library; raises (never falls back) when it is missing."""
    global _product
    if _product is None:
        path = product_library_path()
        if not os.path.exists(path):
            raise RuntimeError(f"CUDA library missing: {path} (run ice_fem_2025a_b200.build.build())")
        _product = C.CDLL(path, mode=C.RTLD_GLOBAL)
    return _product


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


class Context:
    """Handle over one ifem context (product library or oracle, chosen by `lib`/`prefix`)."""

    def __init__(self, lib, prefix, mesh, mats, opts, device=0, use_kron=True):
        self.lib, self.prefix = lib, prefix
        self.mesh = mesh
        self.mats = list(mats)
        self._keep = []
        d = MeshDesc()
        d.dim, d.elem_type, d.ipcount1d = mesh.dim, mesh.elem_type, 3
        d.n_nodes, d.n_elems = mesh.n_nodes, mesh.n_elems
        coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
        elems = np.ascontiguousarray(mesh.elems, dtype=np.int64)
        self._keep += [coords, elems]
        d.coords, d.elems = _ptr(coords, C.c_double), _ptr(elems, C.c_int64)
        if mesh.weights is not None:
            w = np.ascontiguousarray(mesh.weights, dtype=np.float64)
            self._keep.append(w)
            d.node_weights = _ptr(w, C.c_double)
        if use_kron:
            k = np.ascontiguousarray(mesh.elem_kron, dtype=np.float64)
            self._keep.append(k)
            d.elem_kron = _ptr(k, C.c_double)
        else:
            full = np.ascontiguousarray(mesh.elem_data(), dtype=np.float64)
            self._keep.append(full)
            d.elem_data = _ptr(full, C.c_double)
        if mesh.elem_mat is not None:
            em = np.ascontiguousarray(mesh.elem_mat, dtype=np.int32)
            self._keep.append(em)
            d.elem_mat = _ptr(em, C.c_int32)
        mats = list(mats) if isinstance(mats, (list, tuple)) else [mats]
        marr = (Material * len(mats))(*mats)
        self._mats = marr
        self.opts = opts
        h = C.c_void_p()
        fn = self._fn("ctx_create")
        rc = fn(C.byref(d), marr, len(mats), C.byref(opts), device, C.byref(h))
        if rc != OK:
            buf = C.create_string_buffer(512)
            self._fn("last_error")(None, buf, 512)
            raise IfemError(rc, buf.value.decode())
        self.h = h
        self.nsteps = max(opts.dof_step[i] for i in range(opts.n_dofs)) + 1

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _check(self, rc):
        if rc != OK:
            buf = C.create_string_buffer(512)
            self._fn("last_error")(self.h, buf, 512)
            raise IfemError(rc, buf.value.decode())

    def close(self):
        if getattr(self, "h", None):
            self._fn("ctx_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- queries ----
    def step_info(self, step):
        n, z = C.c_int64(), C.c_int64()
        self._check(self._fn("step_info")(self.h, step, C.byref(n), C.byref(z)))
        return n.value, z.value

    def dof_numbers(self, kind):
        out = np.empty(self.mesh.n_nodes, dtype=np.int64)
        self._check(self._fn("get_dof_numbers")(self.h, kind, _ptr(out, C.c_int64)))
        return out

    def pattern(self, step):
        n, z = self.step_info(step)
        rp = np.empty(n + 1, dtype=np.int32)
        ci = np.empty(z, dtype=np.int32)
        self._check(self._fn("build_pattern")(self.h, step, _ptr(rp, C.c_int32), _ptr(ci, C.c_int32)))
        return rp, ci

    # ---- state ----
    def set_state(self, step, kind, vec):
        v = np.ascontiguousarray(vec, dtype=np.float64)
        self._check(self._fn("set_state")(self.h, step, kind, _ptr(v, C.c_double), v.size))

    def get_state(self, step, kind):
        n, _ = self.step_info(step)
        out = np.empty(n)
        self._check(self._fn("get_state")(self.h, step, kind, _ptr(out, C.c_double), n))
        return out

    def assemble(self, step, t=0.0, dt=1.0, du_dt=0.0, ddu_dt=0.0):
        tm = Time(t, dt, du_dt, ddu_dt)
        self._check(self._fn("assemble")(self.h, step, C.byref(tm)))

    def assemble_async(self, step, t=0.0, dt=1.0, du_dt=0.0, ddu_dt=0.0):
        tm = Time(t, dt, du_dt, ddu_dt)
        self._check(self._fn("assemble_async")(self.h, step, C.byref(tm)))

    def sync(self, step):
        self._check(self._fn("sync")(self.h, step))

    def stream(self):
        p = C.c_void_p()
        self._check(self._fn("get_stream")(self.h, C.byref(p)))
        return p.value

    def residual_into(self, step, out):
        """Copy f[step] into a preallocated (e.g. pinned) float64 array."""
        self._check(self._fn("get_residual")(self.h, step, out.ctypes.data_as(C.POINTER(C.c_double)), out.size))

    def matrix_into(self, step, out):
        dt = F64 if out.dtype == np.float64 else F32
        self._check(self._fn("get_matrix")(self.h, step, out.ctypes.data_as(C.c_void_p), out.size, dt))

    def residual(self, step):
        n, _ = self.step_info(step)
        out = np.empty(n)
        self._check(self._fn("get_residual")(self.h, step, _ptr(out, C.c_double), n))
        return out

    def matrix_values(self, step, dtype=F64):
        _, z = self.step_info(step)
        out = np.empty(z, dtype=np.float64 if dtype == F64 else np.float32)
        self._check(self._fn("get_matrix")(self.h, step, out.ctypes.data_as(C.c_void_p), z, dtype))
        return out

    def matrix(self, step, dtype=F64):
        import scipy.sparse as sp
        rp, ci = self.pattern(step)
        v = self.matrix_values(step, dtype)
        n = rp.size - 1
        return sp.csr_matrix((v, ci, rp), shape=(n, n))

    def commit(self, kind=COMMIT_TIMEDEP):
        self._check(self._fn("commit")(self.h, kind))

    def reset_step(self):
        self._check(self._fn("reset_step")(self.h))

    def hist_size(self, field):
        n = self.mesh.n_elems * (9 if self.mesh.dim == 2 else 27)
        coss = bool(self.opts.cosserat)
        if field == HIST_PLASTIC_STRAIN:
            return n * (18 if coss else 6)   # the Cosserat model keeps 18 strain components
        if field == HIST_MAT and (any(m.rheology == RHEO_VEP for m in self.mats) or
                                  (coss and any(m.rheology != RHEO["LinearElastic"] for m in self.mats))):
            return n * 4   # [hardening, dLambda_v, dLambda_p, unused / creep path] per ip
        return n

    def get_history(self, field, old=0):
        out = np.empty(self.hist_size(field))
        self._check(self._fn("get_history")(self.h, field, old, _ptr(out, C.c_double), out.size))
        return out

    def set_history(self, field, vec, old=0):
        v = np.ascontiguousarray(vec, dtype=np.float64)
        self._check(self._fn("set_history")(self.h, field, old, _ptr(v, C.c_double), v.size))

    def set_tangent(self, mode, prec):
        self._check(self._fn("set_tangent")(self.h, mode, prec))

    def set_readback_slabs(self, n_slabs):
        """Assemble the displacement step in `n_slabs` element slabs; the read-back copies each slab's rows
        while later slabs compute (product library only)."""
        self._check(self._fn("set_readback_slabs")(self.h, int(n_slabs)))

    def stats(self, step):
        s = Stats()
        self._check(self._fn("get_stats")(self.h, step, C.byref(s)))
        return s

    # ---- constraints (Constrainer / Physics::Constraint / Physics::UpdateState) ----
    def set_constraints(self, step, dofs, values):
        d = np.ascontiguousarray(dofs, dtype=np.int64)
        v = np.ascontiguousarray(np.broadcast_to(values, d.shape), dtype=np.float64)
        self._check(self._fn("set_constraints")(self.h, step, C.c_int64(d.size), _ptr(d, C.c_int64),
                                                 _ptr(v, C.c_double)))

    def constrained_info(self, step):
        n, z = C.c_int64(), C.c_int64()
        self._check(self._fn("constrained_info")(self.h, step, C.byref(n), C.byref(z)))
        return n.value, z.value

    def constrained_pattern(self, step):
        n, z = self.constrained_info(step)
        rp = np.empty(n + 1, dtype=np.int32)
        ci = np.empty(z, dtype=np.int32)
        self._check(self._fn("build_constrained_pattern")(self.h, step, _ptr(rp, C.c_int32), _ptr(ci, C.c_int32)))
        return rp, ci

    def constrain(self, step, want_matrix=True):
        self._check(self._fn("constrain")(self.h, step, 1 if want_matrix else 0))

    def constrained(self, step, dtype=F64, want_matrix=True):
        """(f_con, K_con values) of the last constrain() call."""
        n, z = self.constrained_info(step)
        f = np.empty(n)
        vals = np.empty(z, dtype=np.float64 if dtype == F64 else np.float32) if want_matrix else None
        self._check(self._fn("get_constrained")(self.h, step, _ptr(f, C.c_double),
                                                 None if vals is None else vals.ctypes.data_as(C.c_void_p),
                                                 C.c_int64(z), dtype))
        return f, vals

    def constrained_matrix(self, step, dtype=F64):
        import scipy.sparse as sp
        rp, ci = self.constrained_pattern(step)
        _, vals = self.constrained(step, dtype)
        n = rp.size - 1
        return sp.csr_matrix((vals.astype(np.float64), ci, rp), shape=(n, n))

    def solve_constrained(self, step, rtol=1e-10, max_it=2000, restart=50):
        """Device GMRES solve of K_con dx = f_con (after constrain(step)); returns (dx, iterations, relative
        residual).  Raises IfemError (ERR_NUMERIC) when rtol is not reached."""
        n, _ = self.constrained_info(step)
        dx = np.empty(n)
        its, rr = C.c_int32(), C.c_double()
        self._check(self._fn("solve_constrained")(self.h, step, C.c_double(rtol), int(max_it), int(restart),
                                                  _ptr(dx, C.c_double), C.byref(its), C.byref(rr)))
        return dx, its.value, rr.value

    def set_preconditioner(self, step, kind):
        """PC_BLOCK_JACOBI, PC_AMG (smoothed-aggregation multigrid set up at each solve) or PC_AMG_REUSE (set up
        once and reused)."""
        self._check(self._fn("set_preconditioner")(self.h, step, int(kind)))

    def set_multigrid(self, step, threshold=0.0, sweeps=2):
        """Strength threshold of the aggregation graph and Jacobi sweeps of the multigrid (ifem_set_multigrid)."""
        self._check(self._fn("set_multigrid")(self.h, step, C.c_double(threshold), int(sweeps)))

    def preconditioner_info(self, step):
        """(rows per multigrid level, finest first; set-up time in ms) of the last solve."""
        nl, sizes, ms = C.c_int32(), (C.c_int64 * 8)(), C.c_double()
        self._check(self._fn("preconditioner_info")(self.h, step, C.byref(nl), sizes, C.byref(ms)))
        return [sizes[i] for i in range(min(nl.value, 8))], ms.value

    def update_state(self, step, dx):
        v = np.ascontiguousarray(dx, dtype=np.float64)
        self._check(self._fn("update_state")(self.h, step, _ptr(v, C.c_double)))

    # ---- TriAxial boundary loads (TriAxialModel) ----
    def set_triaxial(self, side, top, p0=0.0, du=-1e-4, penalty=1e14, t_post_fail=0.5, damaged_forces=True):
        """side, top: (faces [n, nfn] node ids, face_data [n, nfn, nfn] extraction operators)."""
        groups = []
        for faces, data in (side, top):
            f = np.ascontiguousarray(faces, dtype=np.int64)
            d = np.ascontiguousarray(data, dtype=np.float64)
            self._keep += [f, d]
            groups.append(FaceGroup(f.shape[0], _ptr(f, C.c_int64), _ptr(d, C.c_double)))
        prm = TriAxialParams(float(p0), float(du), float(penalty), float(t_post_fail), 1 if damaged_forces else 0, 0)
        self._check(self._fn("set_triaxial")(self.h, C.byref(groups[0]), C.byref(groups[1]), C.byref(prm)))

    def triaxial_commit(self, time, max_time=np.inf, kind=COMMIT_TIMEDEP):
        """TriAxialModel::Commit at simulation time `time`; returns physics->MaxTime after it."""
        mt = C.c_double(max_time)
        self._check(self._fn("triaxial_commit")(self.h, kind, C.c_double(time), C.byref(mt)))
        return mt.value

    def triaxial_state(self):
        st = TriAxialState()
        self._check(self._fn("triaxial_get_state")(self.h, C.byref(st)))
        return st.as_dict()

    def set_triaxial_state(self, d):
        st = TriAxialState()
        for k, v in d.items():
            setattr(st, k, v)
        self._check(self._fn("triaxial_set_state")(self.h, C.byref(st)))

    # ---- batched sweeps: CUDA graph of assemblies (+ adjoints) ----
    def graph_capture(self, steps, with_adjoint=False, t=0.0, dt=1.0, du_dt=0.0, ddu_dt=0.0):
        st = np.ascontiguousarray(steps, dtype=np.int32)
        tm = Time(t, dt, du_dt, ddu_dt)
        self._check(self._fn("graph_capture")(self.h, st.size, _ptr(st, C.c_int32), C.byref(tm),
                                               1 if with_adjoint else 0))

    def graph_launch(self):
        self._check(self._fn("graph_launch")(self.h))

    def adjoint_results(self, step, n_mats=None):
        n, _ = self.step_info(step)
        drd = np.zeros(4 * n)
        lr = np.zeros(4 * self._n_mats(n_mats))
        self._check(self._fn("adjoint_results")(self.h, step, _ptr(drd, C.c_double), _ptr(lr, C.c_double)))
        return drd.reshape(4, n), lr

    def set_param(self, mat, theta, value):
        self._check(self._fn("set_param")(self.h, mat, theta, C.c_double(float(value))))

    def set_adjoint_precision(self, dtype):
        self._check(self._fn("set_adjoint_precision")(self.h, int(dtype)))

    def temperature_sensitivity(self, step, dT=None, t=0.0, dt=1.0, du_dt=0.0, ddu_dt=0.0):
        """dR_step/dT . dT (dT: perturbation of the T step's state, or None for the pinned temperature)."""
        n, _ = self.step_info(step)
        tm = Time(t, dt, du_dt, ddu_dt)
        out = np.zeros(n)
        dTv = None if dT is None else np.ascontiguousarray(dT, dtype=np.float64)
        self._check(self._fn("temperature_sensitivity")(self.h, step, C.byref(tm), _ptr(dTv, C.c_double),
                                                        _ptr(out, C.c_double)))
        return out

    def _n_mats(self, n_mats):
        """Material sets of the context: the per-set outputs hold 4 values for each of them."""
        if n_mats is not None and n_mats != len(self.mats):
            raise ValueError(f"the context has {len(self.mats)} material sets, not {n_mats}")
        return len(self.mats)

    def adjoint(self, step, lam=None, full=False, t=0.0, dt=1.0, du_dt=0.0, ddu_dt=0.0, n_mats=None):
        n, _ = self.step_info(step)
        tm = Time(t, dt, du_dt, ddu_dt)
        drd = np.zeros(4 * n) if full else None
        lr = np.zeros(4 * self._n_mats(n_mats))
        lamv = None if lam is None else np.ascontiguousarray(lam, dtype=np.float64)
        self._check(self._fn("adjoint")(self.h, step, C.byref(tm), _ptr(lamv, C.c_double),
                                        _ptr(drd, C.c_double), _ptr(lr, C.c_double)))
        return (drd.reshape(4, n) if full else None), lr


def product_context(mesh, mats, opts, device=0, use_kron=True) -> Context:
    return Context(load_product(), "ifem_", mesh, mats, opts, device=device, use_kron=use_kron)
