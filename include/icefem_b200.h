/*
 * icefem_b200.h — C-ABI of the B200 element-assembly library for IceFEM's
 * phase-field / viscoplastic / thermal models.
 *
 * The reference plugs physics into its Newton loop through
 *   class BaseModel { virtual void Assemble(Mat& K, Vec& f, Constrainer*, size_t step); ... }
 * (Models/BaseModel/BaseModel.h:32-116), implemented for this path by
 *   PhaseFieldDamage (Models/Fracture/PhaseField/PhaseField.h:53-128, PhaseField.cpp:291-768)
 *   ThermalModel     (Models/Thermal/ThermalModel.cpp:72-135).
 * Every entry point below replaces one piece of that interface (cited per function) and uses only
 * plain C types: pointers, sizes and status codes.  Nothing throws or traps; every call returns an
 * ifem_status and ifem_last_error() gives a message.  A context owns its device buffers (state,
 * per-integration-point history, the device CSR matrix and residual of each staggered step).
 *
 * Pointers passed to set/get functions may be host or device pointers (copies use
 * cudaMemcpyDefault).  One context is not thread-safe; distinct contexts are independent.
 */
#ifndef ICEFEM_B200_H
#define ICEFEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IFEM_ABI_VERSION 1

/* ---- status codes (the reference throws std::invalid_argument / std::runtime_error) ---- */
typedef enum {
  IFEM_OK = 0,
  IFEM_ERR_INVALID = 1,     /* bad argument or configuration (reference: std::invalid_argument) */
  IFEM_ERR_CUDA = 2,        /* CUDA runtime error */
  IFEM_ERR_NOMEM = 3,       /* allocation failed */
  IFEM_ERR_STATE = 4,       /* call out of order (e.g. assemble before set_state) */
  IFEM_ERR_NUMERIC = 5,     /* NaN / Inf produced by the kernels (reference: NonLinSolver.cpp:250-269) */
  IFEM_ERR_UNSUPPORTED = 6, /* option the reference has but this library does not implement */
  IFEM_ERR_CAPACITY = 7     /* size beyond a fixed limit */
} ifem_status;

/* ---- element types (mesh/ElementTypes/TypeRegister.cpp) ---- */
enum { IFEM_ELEM_B2_2 = 1,          /* 2D quadratic Bezier quad, 9 nodes (B2_2.cpp:4-88) */
       IFEM_ELEM_NURBS3_CUBE2 = 2   /* 3D quadratic rational Bezier hex, 27 nodes (NURBS3_Cube2.cpp:4-115) */ };

/* ---- DOF kinds; the order of ifem_options.dof_kind mirrors "Dofs/DofNames" ---- */
enum { IFEM_DOF_UX = 0, IFEM_DOF_UY = 1, IFEM_DOF_UZ = 2, IFEM_DOF_PHASE = 3, IFEM_DOF_T = 4,
       IFEM_DOF_LMULT = 5,   /* "lMult_pf": Lagrange multipliers of the irreversibility (PhaseField.h:57, :95-101) */
       IFEM_DOF_LMULT2 = 6,  /* "lMult_pf2": second multipliers of AugmentedLagrangeMult2 (PhaseField.h:59) */
       IFEM_DOF_OX = 7, IFEM_DOF_OY = 8, IFEM_DOF_OZ = 9   /* Cosserat micro-rotations "ox", "oy", "oz"
                                (CossPhaseField.h:15, CossPhaseField.cpp:170-180): oz in 2D, all three in 3D */ };
#define IFEM_N_DOF_KINDS 10

/* ---- rheologies (SolidMaterial.h:13-22) ----
 * VEP: viscoelastic-plastic return map (SolidMaterial.cpp:303-445), history size 4.  DVEP
 * ("DamViscoElasticPlastic") is rejected with IFEM_ERR_UNSUPPORTED by the phase-field model, as the reference's
 * UpdatePlasticStrains has no case for it and throws (SolidMaterial.cpp:185-188); the Cosserat model has LE, VEP
 * and DVEP only (CosseratMaterial.cpp:450-500). */
enum { IFEM_RHEO_LE = 0, IFEM_RHEO_VE = 1, IFEM_RHEO_DVE = 2, IFEM_RHEO_VE_EXPL = 3, IFEM_RHEO_DVE_EXPL = 4,
       IFEM_RHEO_VEP = 5, IFEM_RHEO_DVEP = 6 };

/* ---- energy splits (PhaseFieldMaterial.h:41-51, same numeric values) ----
 * SPECSTRESS needs consistent_energy = 0: the reference throws otherwise (PhaseFieldMaterial.cpp:148-150).
 * SPECSTRAINS follows the reference's plane-strain principal strains (xx, yy, xy and zz) in 2D and 3D. */
enum { IFEM_SPLIT_NONE = 0, IFEM_SPLIT_VOLSTRAINS = 1, IFEM_SPLIT_SPECSTRAINS = 2, IFEM_SPLIT_VOLSTRESS = 3,
       IFEM_SPLIT_SPECSTRESS = 4, IFEM_SPLIT_DRUCKERPRAGER = 5, IFEM_SPLIT_ICE = 6, IFEM_SPLIT_STARCONVEX = 7 };

/* ---- degradation functions (PhaseFieldUtil.h:12-26, same numeric values) ---- */
enum { IFEM_DAM_NONE = 0, IFEM_DAM_STEP2 = 1, IFEM_DAM_STEP5 = 2, IFEM_DAM_STEP8 = 3,
       IFEM_DAM_LINEAR = 4, IFEM_DAM_QUADRATIC = 5, IFEM_DAM_CUBIC = 6, IFEM_DAM_LINEAR_NR = 7,
       IFEM_DAM_QUADRATIC_NR = 8, IFEM_DAM_CUBIC_NR = 9, IFEM_DAM_CZM = 10, IFEM_DAM_PORDER = 11 };

/* ---- crack-density (distribution) functions (PhaseFieldUtil.h:29-41, same numeric values) ----
 * The HO_* variants and CUSTOM also integrate second gradients of the phase field (PhaseFieldUtil.cpp:223-280,
 * getShapeGrads2 of B2_2.cpp:90-125 / NURBS3_Cube2.cpp:117-216); CUSTOM takes ifem_options.dist_coefs. */
enum { IFEM_DIST_LINEAR = 0, IFEM_DIST_CZM = 1, IFEM_DIST_LINEAR2 = 2, IFEM_DIST_QUADRATIC = 3,
       IFEM_DIST_HO_LINEAR = 4, IFEM_DIST_HO_LINEAR2 = 5, IFEM_DIST_HO_CZM = 6, IFEM_DIST_HO_QUADRATIC = 7,
       IFEM_DIST_LOCAL = 8, IFEM_DIST_CUSTOM = 9 };

/* ---- irreversibility (PhaseFieldUtil.h:51-60) ---- */
enum { IFEM_IRR_NONE = 0, IFEM_IRR_HIST = 1, IFEM_IRR_PENALTY = 2,
       IFEM_IRR_LAGRANGE = 3,  /* LagrangeMult: needs IFEM_DOF_LMULT in the phase step (PhaseFieldUtil.cpp:383-399) */
       IFEM_IRR_AUGLAG = 4,    /* AugmentedLagrangeMult: IFEM_DOF_LMULT (:401-441) */
       IFEM_IRR_AUGLAG2 = 5    /* AugmentedLagrangeMult2: IFEM_DOF_LMULT and IFEM_DOF_LMULT2 (:444-484) */ };

/* ---- tangent formula ---- */
enum { IFEM_TANGENT_REFERENCE = 0,  /* the reference's own K: ddF zeroed, Damage in K(6,:) (SolidMaterial.cpp:289-299) */
       IFEM_TANGENT_CONSISTENT = 1  /* exact derivative of the residual kernel (for Newton / FD checks) */ };

/* ---- tangent arithmetic ---- */
enum { IFEM_PREC_FP64 = 0,   /* plain FP64 tangent */
       IFEM_PREC_FP32 = 1,   /* FP32 CUDA-core tangent (FP64 residual) */
       IFEM_PREC_TC_SPLIT = 2, /* 3D hex: tcgen05 tensor cores, FP16 hi/lo operand pairs under a per-element
                                  power-of-two scale (three products), FP32 accumulate: FP32-accurate */
       IFEM_PREC_TF32X3 = IFEM_PREC_TC_SPLIT /* former name of IFEM_PREC_TC_SPLIT */ };

/* ---- return-map tolerance ---- */
enum { IFEM_RM_REFERENCE = 0,  /* e<1e-16 || e/e0<1e-9, cap 250 (SolidMaterial.cpp:243-250) */
       IFEM_RM_TIGHT = 1       /* iterate to round-off (finite-difference checks) */ };

/* ---- commit types (BaseModel.h:15-18) ---- */
enum { IFEM_COMMIT_TIMEDEP = 1, IFEM_COMMIT_PATHDEP = 2 };

/* ---- history fields (PhaseField.h:117-120) ---- */
enum { IFEM_HIST_ENERGY = 0,        /* Energy_Hist        [nel*nip]     */
       IFEM_HIST_PLASTIC_STRAIN = 1,/* Plastic_Strain     [nel*nip*6], [nel*nip*18] for the Cosserat model */
       IFEM_HIST_VISC_DISS = 2,     /* ViscDiss           [nel*nip]     */
       IFEM_HIST_DAM_VISC_DISS = 3, /* DamViscDiss        [nel*nip]     */
       IFEM_HIST_MAT = 4            /* MatHist [nel*nip*hs], ip-major: hs = 1 (dLambda) for the VE family,
                                       hs = 4 (hardening, dLambda_v, dLambda_p, unused) when a material
                                       set is VEP (SolidMaterial.cpp:50-51, 424-432) */ };

/* ---- state-vector kinds (physics.h: StateVectors / StateVectorsOld / dStateVectors / ddStateVectors) ---- */
enum { IFEM_STATE_CUR = 0, IFEM_STATE_OLD = 1, IFEM_STATE_D = 2, IFEM_STATE_DD = 3 };

/* ---- CSR value arithmetic for ifem_get_matrix ---- */
enum { IFEM_F64 = 0, IFEM_F32 = 1 };

/* Mesh of one element group ("internal"), as Mesh::LoadFromFile holds it (mesh.cpp:53-303).
 * elem_data is the per-element Bezier extraction operator C with N = C * N_bernstein, stored
 * row-major C[j][k] (ElemData(j,k), elementgroup.cpp:59-63).  For tensor-product meshes the
 * caller may pass elem_kron instead: dim 3x3 row-major 1-D factors per element, ordered x,y(,z),
 * with C = kron(Cz, kron(Cy, Cx)) as bezierExtraction3D.m builds it; the library checks and uses
 * the factored form when elem_data factors exactly.  Node-local order is x fastest. */
typedef struct {
  int32_t dim;             /* 2 or 3 */
  int32_t elem_type;       /* IFEM_ELEM_* */
  int32_t ipcount1d;       /* Gauss points per direction; 3 (the only count used by the configs) */
  int32_t reserved0;
  int64_t n_nodes;
  int64_t n_elems;
  const double* coords;        /* [n_nodes*dim] node-major x,y(,z) */
  const double* node_weights;  /* [n_nodes] NURBS weights ("W" node data) or NULL => 1 */
  const int64_t* elems;        /* [n_elems*nen] global node ids */
  const double* elem_data;     /* [n_elems*nen*nen] or NULL */
  const double* elem_kron;     /* [n_elems*dim*9] or NULL */
  const int32_t* elem_mat;     /* [n_elems] material-set index or NULL (all 0) */
} ifem_mesh_desc;

/* One material set: "properties/<Material>" (SolidMaterial.cpp:5-107, PhaseFieldMaterial.cpp:3-33,
 * IceMaterial.cpp:5-43, ThermalMaterial.cpp:5-10).  Temperatures in the units of the T DOF;
 * TAbs = min(T + t_offset, 273.15) (IceMaterial.cpp:51-54). */
typedef struct {
  double young, poisson, density, damping;        /* SolidProperties */
  double creep_a, creep_n, phi_visc_lim;          /* A (at TRef), n, PhiViscLim (default 1e3) */
  double pf_l, gc, pf_visc;                       /* FractureProperties l, Gc, Viscosity */
  double star_convex_gamma, ice_eref, ice_creduce;
  double t_ref, t_offset, q_creep, ft0, ftdeg;    /* TemperatureDependent */
  double ice_creduce_fact, ice_ereduce_fact;
  double k_thermal, cp;                           /* ThermalProperties */
  int32_t rheology;                               /* IFEM_RHEO_* */
  int32_t split;                                  /* IFEM_SPLIT_* */
  int32_t consistent_energy;                      /* properties/PhaseField/ConsistentEnergy (default 1) */
  int32_t gc_mode;                                /* 0: Gc = 2 ft^2 l / E (IceMaterial.cpp:71-72); 1: Gc = gc */
  /* VEP only (SolidMaterial.cpp:50-65, IceMaterial.cpp:36-37,81-82): yield stress at TRef and its
   * temperature slope (sy = sy0 - sydeg (TAbs - TRef)), friction / dilatancy angles in degrees ("F_deg",
   * "G_deg"; G_deg defaults to F_deg), hardening modulus, plastic viscosity "pl_visc" */
  double vep_sy, vep_sydeg, vep_f_deg, vep_g_deg, vep_hardening, vep_pl_visc;
  double b_dp;   /* DruckerPrager split only: FractureProperties "B_DP" (PhaseFieldMaterial.cpp:23-25) */
  /* Cosserat model only (CosseratMaterial.cpp:3-10): SolidProperties "l_coss", "G_coss" and "hard_eRef" */
  double l_coss, g_coss, hard_e_ref;
} ifem_material;

/* Model options: "Models/<PhaseField>", "properties/PhaseField", "Dofs" keys. */
typedef struct {
  int32_t n_dofs;                 /* entries in dof_kind/dof_step ("Dofs/DofNames", "Dofs/DofStep") */
  int32_t dof_kind[IFEM_N_DOF_KINDS]; /* IFEM_DOF_* in DofNames order */
  int32_t dof_step[IFEM_N_DOF_KINDS];
  int32_t dam_function;           /* DamFunction */
  int32_t density_dam_function;   /* DensityDamage (inertia and gravity, PhaseField.cpp:241-255) */
  int32_t visco_dam_function;     /* ViscoDriving */
  int32_t distribution;           /* DistributionFunction (default Quadratic) */
  int32_t irreversible;           /* Irreversible (default Hist) */
  int32_t inertia;                /* "Intertia" */
  int32_t gravity;                /* "Gravity" */
  int32_t lumped_cap;             /* LumpedPFCapacity */
  int32_t lumped_drive;           /* LumpedDriving */
  int32_t viscous_heating;        /* ViscousHeating */
  int32_t consistent_degradation; /* ConsistentDegradation */
  int32_t thermal_model;          /* a Thermal/ThermalModel on the same group assembles after the phase-field model */
  int32_t ref_compat_phase_t;     /* 1: replicate Assemble_Phase's unfilled dofsT (PhaseField.cpp:562-565) */
  int32_t tangent_mode;           /* IFEM_TANGENT_* */
  int32_t tangent_precision;      /* IFEM_PREC_* */
  int32_t rm_tol_mode;            /* IFEM_RM_* */
  int32_t rm_max_it;              /* return-map cap (reference: 250) */
  int32_t ocean_bc;               /* 1: an OceanBC model acts on the u-step after the phase-field model
                                     (OceanBC.cpp:96-150, 2D only): F_ux(n) += W(n) rho_w g max(0, hw - y_n) */
  double k0;                      /* k0 */
  double visc_num;                /* ViscousStab */
  double visco_driving_factor;    /* ViscoDrivingFactor */
  double pinned_temperature;      /* T value used at every ip when no T DOF exists */
  double penalty_factor;          /* PenaltyFactor (1e6) */
  double lag_fact;                /* LagFact of the augmented Lagrange methods (1.0, PhaseFieldUtil.h:74) */
  double ocean_hw;                /* OceanBC "hw": water level (y coordinate) */
  double ocean_density;           /* OceanBC fluid density: properties/<Fluid>/SolidProperties/Density */
  double porder_p;                /* properties/PhaseField/p: exponent of PorderDamage (PhaseFieldUtil.cpp:24-25,
                                     122-130); the reference's default is 2, and 0 here also means 2 */
  double dist_coefs[5];           /* properties/PhaseField/Coefs of the Custom distribution (PhaseFieldUtil.cpp:27-30) */
  int32_t cosserat;               /* 1: the model is Fracture/CossPhaseField (CossPhaseField.cpp:337-800): micro-
                                     rotation dofs in the u-step (oz in 2D, ox oy oz in 3D), 18-component strains,
                                     LinearElastic, ViscoElasticPlastic or DamViscoElasticPlastic ice, the None,
                                     SpecStress, DruckerPrager or StarConvex split; no lumped driving or capacity */
  int32_t gravity_dam_function;   /* Cosserat model: properties/PhaseField/GravityDamage (the phase-field model uses
                                     DensityDamage for gravity) */
} ifem_options;

/* Time-scheme scalars (TimeSchemes.cpp:65-76) and the time. */
typedef struct { double t, dt, du_dt, ddu_dt; } ifem_time;

/* Per-step timing/diagnostics of the last assembly (physics.cpp:266-282 prints the same per model). */
typedef struct {
  double ms_total, ms_element, ms_scatter;   /* device time of the last assembly; element = points + tangent */
  int64_t rm_iterations;     /* return-map Newton iterations summed over ips */
  int64_t rm_capped;         /* ips that hit the iteration cap */
  int64_t nonfinite;         /* non-finite values seen in element residuals */
  double crack_length;       /* LCrack of the last phase assembly (PhaseField.cpp:540,650) */
  double ms_points, ms_tangent;  /* U step: integration-point kernel / element-tangent kernel */
} ifem_stats;

typedef struct ifem_ctx ifem_ctx;

/* Library/ABI version (no reference counterpart). */
int ifem_abi_version(void);

/* PhaseFieldDamage::PhaseFieldDamage + init + Setup + DofSpace::SyncDofs (PhaseField.cpp:24-102,
 * 167-284; DofSpace.cpp:177-754; physics.cpp:15-45).  Copies the mesh to the device, numbers the
 * DOFs, builds every step's CSR pattern and element->nonzero maps, allocates state and history.
 * mats: n_mats material sets (elem_mat indexes them).  device: CUDA ordinal. */
int ifem_ctx_create(const ifem_mesh_desc* mesh, const ifem_material* mats, int32_t n_mats,
                    const ifem_options* opts, int32_t device, ifem_ctx** out);

/* PhaseFieldDamage::~PhaseFieldDamage + Physics teardown. */
int ifem_ctx_destroy(ifem_ctx* ctx);

/* Last error message of this context (or of the last failed create when ctx is NULL). */
int ifem_last_error(const ifem_ctx* ctx, char* buf, size_t len);

/* DofSpace::LocalDofNumRange / TotalDofRange for a step (DofSpace.cpp:486-513), nnz of its matrix. */
int ifem_step_info(const ifem_ctx* ctx, int32_t step, int64_t* n_dofs, int64_t* nnz);

/* The DOF number of (node, dof kind): DofSpace::getDofForNodes (DofSpace.cpp:826-842). -1 if absent. */
int ifem_get_dof_numbers(const ifem_ctx* ctx, int32_t kind, int64_t* dofs_out /* [n_nodes] */);

/* The AIJ pattern that MatSetValues(ADD_VALUES) builds in Physics::K[step] (physics.cpp:228-251,
 * math.cpp:301-304): union of element DOF pairs, columns ascending.  32-bit like PetscInt. */
int ifem_build_pattern(const ifem_ctx* ctx, int32_t step, int32_t* row_ptr_out /* [n_dofs+1] */,
                       int32_t* col_idx_out /* [nnz] */);

/* Physics::StateVectors/StateVectorsOld/dStateVectors/ddStateVectors[step] := src (n = n_dofs). */
int ifem_set_state(ifem_ctx* ctx, int32_t step, int32_t kind, const double* src, int64_t n);
int ifem_get_state(const ifem_ctx* ctx, int32_t step, int32_t kind, double* dst, int64_t n);

/* Physics::Assemble(step) for the models of this context: zero K,f then
 * PhaseFieldDamage::Assemble (PhaseField.cpp:291-309) and, when thermal_model is set,
 * ThermalModel::Assemble (ThermalModel.cpp:72-135), scattered deterministically into the
 * device CSR and residual.  Updates history exactly as the reference does on every call. */
int ifem_assemble(ifem_ctx* ctx, int32_t step, const ifem_time* tm);

/* ifem_assemble without the final wait: enqueues the kernels on the context's stream and returns.
 * ifem_sync waits for them, reads the diagnostics and reports errors (no reference counterpart;
 * used to overlap assemblies with other work and to capture them in CUDA graphs). */
int ifem_assemble_async(ifem_ctx* ctx, int32_t step, const ifem_time* tm);
int ifem_sync(ifem_ctx* ctx, int32_t step);

/* The cudaStream_t the context launches on (for event timing and graph capture). */
int ifem_get_stream(const ifem_ctx* ctx, void** stream);

/* Copy the assembled residual f[step] (n_dofs doubles) / CSR values (nnz, IFEM_F64 or IFEM_F32); blocking.
   The copy waits for the last assembly of `step` only, on a copy stream of its own, so the read-back of one
   step runs while an assembly of another step queued after it (ifem_assemble_async) computes. */
int ifem_get_residual(const ifem_ctx* ctx, int32_t step, double* dst, int64_t n);
int ifem_get_matrix(const ifem_ctx* ctx, int32_t step, void* dst, int64_t nnz, int32_t dtype);

/* Device pointers of the assembled residual / CSR values (dtype written to *dtype_out), for a
 * device solver that consumes them in place.  Valid until the next assemble or destroy. */
int ifem_device_outputs(const ifem_ctx* ctx, int32_t step, const double** f_dev,
                        const void** vals_dev, int32_t* dtype_out);

/* PhaseFieldDamage::Commit (PhaseField.cpp:123-145) / ResetStep (PhaseField.cpp:147-163). */
int ifem_commit(ifem_ctx* ctx, int32_t commit_type);
int ifem_reset_step(ifem_ctx* ctx);

/* PhaseFieldDamage::load/save of history (PhaseField.cpp:107-119), extended to all fields so a
 * viscoplastic restart is exact.  old = 0 current, 1 committed ("...Old") copy. */
int ifem_get_history(const ifem_ctx* ctx, int32_t field, int32_t old, double* dst, int64_t n);
int ifem_set_history(ifem_ctx* ctx, int32_t field, int32_t old, const double* src, int64_t n);

/* Change tangent formula / precision between assemblies (no reference counterpart: the
 * reference tangent is always FP64 Eigen). */
int ifem_set_tangent(ifem_ctx* ctx, int32_t tangent_mode, int32_t tangent_precision);

/* Pipeline the displacement step's assembly with its read-back (no reference counterpart: the reference
 * assembles into host PETSc objects).  With n_slabs > 1 the elements are split into n_slabs contiguous
 * ranges; after each range the rows whose incident elements are all done are gathered, and
 * ifem_get_matrix / ifem_get_residual copy those rows while later ranges still compute.  Results are
 * identical to n_slabs = 1 (the default).  Mesh orders that number nodes and elements along the same
 * direction (structured boxes, slab-sorted meshes) complete rows early; other orders stay correct and
 * complete most rows in the last slab.  1 <= n_slabs <= 16; graph captures always run one pass. */
int ifem_set_readback_slabs(ifem_ctx* ctx, int32_t n_slabs);

/* PhaseFieldDamage::GetTimeData (crack length) plus kernel diagnostics of the last assembly. */
int ifem_get_stats(const ifem_ctx* ctx, int32_t step, ifem_stats* out);

/* Adjoint of the residual kernel w.r.t. the material parameters theta = (Gc, l, A, n)
 * (no reference counterpart; the reference has no sensitivities).  Evaluates at the stored state
 * and start-of-assembly history without changing either.
 * dr_dtheta: [4*n_dofs] dR/dtheta_k for a parameter shared by all material sets (may be NULL);
 * lambda: [n_dofs] adjoint vector (NULL = all ones);
 * lam_dr: [4*n_mats] lambda^T dR/dtheta_k of each material set, set-major (may be NULL). */
int ifem_adjoint(ifem_ctx* ctx, int32_t step, const ifem_time* tm, const double* lambda,
                 double* dr_dtheta, double* lam_dr);

/* Set one parameter of one material set (theta index 0..3 = Gc, l, A, n) — used by calibration
 * sweeps and finite-difference checks. */
int ifem_set_param(ifem_ctx* ctx, int32_t mat, int32_t theta, double value);

/* Arithmetic of the adjoint's sensitivity stresses and their contraction with the shape gradients (no reference
 * counterpart): IFEM_F64 (default) or IFEM_F32.  The return map and its 7x7 sensitivity solve stay FP64 either
 * way; the element sums are gathered in FP64.  Applies to ifem_adjoint, graph replays captured afterwards and
 * ifem_temperature_sensitivity. */
int ifem_set_adjoint_precision(ifem_ctx* ctx, int32_t dtype);

/* Thermal Arrhenius coupling of the residual (no reference counterpart; the reference's staggered scheme never
 * forms it): the directional derivative dR_step/dT . dT of the u-step residual through A(T) and of the phase-step
 * residual through Gc(T) = 2 ft(T)^2 l / E (IceMaterial.cpp:49-84), at the stored state and start-of-assembly
 * history, like ifem_adjoint.  With a temperature DOF, dT [n_T] is a perturbation of the T step's state (host or
 * device memory); without one, dT must be NULL and the derivative is with respect to the pinned temperature.
 * At and above the melting clamp TAbs = min(T + TOffset, 273.15) the derivative is the one from below at the
 * clamp and zero above it.
 * dr_out: [n_dofs of step].  The T step itself, the VEP return map, the ICE split, SpecStrains / DruckerPrager
 * and Lagrange multipliers give IFEM_ERR_INVALID / IFEM_ERR_UNSUPPORTED. */
int ifem_temperature_sensitivity(ifem_ctx* ctx, int32_t step, const ifem_time* tm, const double* dT, double* dr_out);

/* Results of the last adjoint of a step (ifem_adjoint or a graph replay with adjoints): dr_dtheta
 * [4*n_dofs] and lam_dr [4*n_mats] as in ifem_adjoint (a graph replay uses lambda = 1); either may be NULL. */
int ifem_adjoint_results(const ifem_ctx* ctx, int32_t step, double* dr_dtheta, double* lam_dr);

/* Batched calibration sweeps (no reference counterpart): record the assemblies of n_steps staggered steps,
 * in the given order and each optionally followed by its adjoint, as one CUDA graph owned by the context.
 * Device buffers are bound at capture; their contents (state, history, material parameters changed by
 * ifem_set_param) are read at each replay.  The time data tm is fixed at capture.  A new capture replaces the
 * previous graph. */
int ifem_graph_capture(ifem_ctx* ctx, int32_t n_steps, const int32_t* steps, const ifem_time* tm,
                       int32_t with_adjoint);

/* Replay the captured graph on the context's stream; asynchronous like ifem_assemble_async (ifem_sync(ctx,
 * step) completes a step, ifem_adjoint_results reads its adjoint). */
int ifem_graph_launch(ifem_ctx* ctx);

/* ---- Constraints on the device CSR: Constrainer (Physics/Constrainer.cpp:38-126), Physics::Constraint /
 *      ConstraintFOnly (Physics/physics.cpp:314-362) and Physics::UpdateState (physics.cpp:408-419) ----
 * U selects the free dofs (ascending dof order), C the constrained ones (ascending dof order, the order of
 * the reference's std::map).  C_v = value - state is taken when ifem_constrain runs. */

/* Constrainer::SetZero + AddConstraint for one staggered step: n constrained dofs (step numbering) and their
 * values.  A dof given twice with the same value counts once; with different values the call fails with
 * IFEM_ERR_INVALID (the reference throws, Constrainer.cpp:46-52).  A new set of dofs rebuilds the reduced
 * pattern (the reference's dofsChanged / dofVersion); n = 0 removes all constraints. */
int ifem_set_constraints(ifem_ctx* ctx, int32_t step, int64_t n, const int64_t* dofs, const double* values);

/* ConstrainedSizeLocal and the nnz of K_con = U^T K U. */
int ifem_constrained_info(const ifem_ctx* ctx, int32_t step, int64_t* n_free, int64_t* nnz);

/* Pattern of K_con (the PtAP product's): free rows and columns renumbered, columns ascending. */
int ifem_build_constrained_pattern(const ifem_ctx* ctx, int32_t step, int32_t* row_ptr_out /* [n_free+1] */,
                                   int32_t* col_idx_out /* [nnz] */);

/* Constrainer::Assemble (C_v = value - state) followed by Physics::Constraint (want_matrix != 0) or
 * ConstraintFOnly (want_matrix == 0), on the device, after an assembly of the step:
 *   K_con = U^T K U                     (values in the precision of the assembled matrix)
 *   f_con = -(U^T (f - K C C_v))        (FP64; the products K C C_v are added row by row in column order) */
int ifem_constrain(ifem_ctx* ctx, int32_t step, int32_t want_matrix);

/* Copy f_con [n_free] and the K_con values [nnz] (dtype IFEM_F64 or IFEM_F32); either destination may be NULL. */
int ifem_get_constrained(const ifem_ctx* ctx, int32_t step, double* f_con, void* vals, int64_t nnz, int32_t dtype);

/* Device pointers of f_con and of the K_con values (valid until the next ifem_constrain or
 * ifem_set_constraints of the step), for a device solver. */
int ifem_device_constrained(const ifem_ctx* ctx, int32_t step, const double** f_con, const void** vals,
                            int32_t* dtype_out);

/* Device solve of K_con dx = f_con from the last ifem_constrain(want_matrix = 1), in place of the reference's
 * PETSc linear solve (GMRESLinSolver.cpp:19-96: GMRES with ASM/MUMPS preconditioning): restarted GMRES(restart)
 * preconditioned by the inverses of the node blocks (a node's displacement components) or the multigrid of
 * ifem_set_preconditioner, all vectors on the
 * device.  Stops when ||f_con - K_con dx|| <= rtol ||f_con||
 * or after max_it iterations; dx [n_free] is host or device memory.  IFEM_ERR_NUMERIC when the tolerance was
 * not reached (dx then holds the last iterate).  This block-Jacobi preconditioner suits the phase step and modest
 * u-step systems; stiff elasticity needs many iterations. */
int ifem_solve_constrained(ifem_ctx* ctx, int32_t step, double rtol, int32_t max_it, int32_t restart, double* dx,
                           int32_t* iterations, double* rel_residual);

/* Preconditioner of ifem_solve_constrained for a step, in place of the reference's PCASM / MUMPS choice
 * (GMRESLinSolver.cpp:33-60):
 *   IFEM_PC_BLOCK_JACOBI  inverses of the node blocks (default);
 *   IFEM_PC_AMG           smoothed-aggregation multigrid (Vanek, Mandel, Brezina 1996), one V-cycle per
 *                         application, set up from K_con at every solve;
 *   IFEM_PC_AMG_REUSE     the same, set up at the first solve and reused (a modified-Newton preconditioner) until
 *                         the preconditioner or the constraints are set again.
 * The multigrid's near-null space is the rigid-body modes of the displacement step (translations, rotations; the
 * Cosserat micro-rotations follow the rotation) and one constant per component of the other steps.  A step with
 * Lagrange-multiplier DOFs (IFEM_DOF_LMULT, IFEM_DOF_LMULT2: an indefinite saddle-point system) gets
 * IFEM_ERR_UNSUPPORTED from the solve. */
#define IFEM_PC_BLOCK_JACOBI 0
#define IFEM_PC_AMG 1
#define IFEM_PC_AMG_REUSE 2
int ifem_set_preconditioner(ifem_ctx* ctx, int32_t step, int32_t kind);

/* Multigrid parameters of a step, as PETSc's GAMG options (-pc_gamg_threshold, the smoother's sweeps): couplings
 * |a_ij| < strength_threshold sqrt(|a_ii a_jj|) are left out of the aggregation graph at the finest level (the
 * threshold halves on each coarser level; 0, the default, keeps every coupling), and sweeps (1..8, default 2)
 * damped-Jacobi sweeps run before and after the coarse correction.  Drops the step's hierarchy. */
int ifem_set_multigrid(ifem_ctx* ctx, int32_t step, double strength_threshold, int32_t sweeps);

/* The multigrid hierarchy the set-up would build for a matrix, planned on the host only (no context, no device
 * memory): CSR row_ptr [n+1], col_idx / vals [nnz], node_of_row [n] (each row's mesh node, 0 .. n_nodes-1), the
 * near-null space modes [n][n_modes] row-major, the strength threshold of ifem_set_multigrid.  levels gets the
 * number of levels (the last one is inverted densely), rows_out / nnz_out (either may be NULL) the first
 * max_levels levels' sizes. */
int ifem_multigrid_plan(int64_t n, const int64_t* row_ptr, const int32_t* col_idx, const double* vals,
                        const int32_t* node_of_row, int64_t n_nodes, int32_t n_modes, const double* modes,
                        double strength_threshold, int32_t max_levels, int32_t* levels, int64_t* rows_out,
                        int64_t* nnz_out);

/* The multigrid hierarchy of the last solve: number of levels, rows per level (sizes [8], the finest first; the
 * last level is solved by a dense inverse) and the set-up's wall time in ms; levels = 0 without one. */
int ifem_preconditioner_info(const ifem_ctx* ctx, int32_t step, int32_t* levels, int64_t* sizes /* [8] */,
                             double* setup_ms);

/* Physics::UpdateState: state_cur += U dx + C C_v, with dx [n_free] (host or device) and the C_v of the last
 * ifem_constrain.  Velocities and accelerations (UpdateVelAcc) stay as set by ifem_set_state. */
int ifem_update_state(ifem_ctx* ctx, int32_t step, const double* dx);

/* ---- TriAxial boundary loads: TriAxialModel (Models/ExternalForce/TriAxial.cpp:13-215) ----
 * A boundary element group of the mesh file ("elementgroups/<name>" with its "BE" operators): quadratic Bezier
 * lines B1_2 in 2D (mesh/ElementTypes/Bezier/B1_2.cpp) or quadratic NURBS faces NURBS3_Plane2 in 3D
 * (mesh/ElementTypes/NURBS/NURBS3_Plane2.cpp, rational with the mesh's node weights), nfn = 3 or 9 nodes per
 * face, node-local order as in the mesh file.  The faces use the mesh's ipcount1d Gauss points per direction. */
typedef struct {
  int64_t n_faces;
  const int64_t* faces;       /* [n_faces*nfn] global node ids */
  const double* face_data;    /* [n_faces*nfn*nfn] ElemData(j,k) row-major (elementgroup.cpp:40-67) */
} ifem_face_group;

/* Models/<name> inputs of a TriAxial model (TriAxial.cpp:34-71). */
typedef struct {
  double p0;              /* "p0": pressure on the side group along its normals (and on the top before t = 0) */
  double du;              /* "dU": rate of the top displacement target u0 + t dU */
  double penalty;         /* "dummy": penalty stiffness of the top displacement target */
  double t_post_fail;     /* "t_postFail": time simulated after failure is detected */
  int32_t damaged_forces; /* "DamagedForces": side pressure scaled by (1 - phi)^2 (QuadraticNoRes) */
  int32_t reserved;
} ifem_triaxial;

/* The model's running state (TriAxial.h:44-56): the last u-step assembly's sums over the top group and the
 * failure detection of TriAxialModel::Commit.  A new model starts with area 1, u0 = -1e8, max_load = -1e9. */
typedef struct {
  double area, f_ext, uz_sum;     /* sum w, sum -w p_ext and sum w u_top over the top group's ips */
  double u0;                      /* top displacement at t = 0 (set by commits while time < 0) */
  double t_break;                 /* time failure was detected (0: not yet); the side pressure is 0 after it */
  double max_load;                /* largest committed F_ext / area * sign(dU) */
  double p0;                      /* the side pressure in use (p0, or 0 after failure) */
  int32_t min_load_passed;
  int32_t reserved;
} ifem_triaxial_state;

/* TriAxialModel::init / Setup: attach a TriAxial model with a side and a top group to the displacement step.
 * Its loads are added after the phase-field model's terms (the order of the reference's Models list), the side
 * group's before the top group's, each group's faces in order (TriAxial.cpp:124-276):
 *   side:  f += D(phi) w N n p0, with n the outward normal of getNormals (the face normal t1 x t2, or (t_y, -t_x)
 *          in 2D, flipped when a step along it moves the point toward the origin)
 *   top, t + dt < 0:  f += w N e_top p0
 *   top, t + dt >= 0: f += w N e_top k (u_top - u0 - (t + dt) dU),  K += w k N N^T on the u_top block
 * with t = ifem_time.t the time at the start of the step and e_top the last coordinate direction.  Both groups
 * must be non-empty; the face nodes must be mesh nodes with displacement dofs.  Replaces an earlier model.
 * While a TriAxial model is attached the displacement step is assembled in one pass (no read-back slabs);
 * the call drops a captured graph (capture again afterwards). */
int ifem_set_triaxial(ifem_ctx* ctx, const ifem_face_group* side, const ifem_face_group* top, const ifem_triaxial* prm);

/* TriAxialModel::Commit (TriAxial.cpp:75-122) for the commit type (IFEM_COMMIT_*) at the simulation time `time`
 * (physics->time): updates the failure detection from the last displacement-step assembly.  When failure is
 * detected, *max_time (physics->MaxTime, in/out, may be NULL) becomes t_break + t_postFail. */
int ifem_triaxial_commit(ifem_ctx* ctx, int32_t commit_type, double time, double* max_time);

/* The model's state (after a synchronising read of the last assembly's sums), and TriAxialModel::GetTimeData:
 * p_Ext = f_ext / area and U_Ext = uz_sum / area. */
int ifem_triaxial_get_state(const ifem_ctx* ctx, ifem_triaxial_state* out);
int ifem_triaxial_set_state(ifem_ctx* ctx, const ifem_triaxial_state* in);

/* Crack length sum_e sum_ip gamma * w of a phase field (the quantity the phase-step assembly
 * accumulates as LCrack, PhaseField.cpp:540,650, with the crack density of PhaseFieldUtil.cpp:185-221),
 * for callers that cannot let the library allocate device memory: code whose device memory is
 * owned by a host framework's pool, or a per-time-step monitor that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree.  This entry point has no counterpart in the reference.
 *
 * Every pointer is a device pointer supplied by the caller: coords [n_nodes*dim], node_weights
 * [n_nodes] (3D, may be NULL), elems int32 [n_elems*nen], elem_kron [n_elems*dim*9] (factored
 * extraction operators), phase [n_nodes] indexed by node, length_out [1].  Enqueued on `stream`
 * (a cudaStream_t, NULL = default stream); the result is valid once the stream has reached it.
 * Scratch: a fixed device array of 2^21 doubles (16 MiB) inside the library, held on every GPU
 * that loads it until the process exits; meshes with more than 2^21 elements are rejected with
 * IFEM_ERR_CAPACITY.  The first call on a device is its set-up: it looks the array's address up with
 * that device current, so make it before any stream capture (a call under capture with no earlier
 * call on the device returns IFEM_ERR_STATE).  Later calls outside a capture look the address up
 * again, so a cudaDeviceReset between calls is safe.  One array serves every call on a device and
 * keeps the last call's contents (every call overwrites the slots it uses): calls that overlap on the
 * GPU race, so callers on several streams must serialise their calls.
 * Allocates nothing: no cudaMalloc, cudaFree or allocating library routine. */
int ifem_crack_length_noalloc(int32_t dim, int64_t n_elems, const double* coords, const double* node_weights,
                              const int32_t* elems, const double* elem_kron, const double* phase,
                              double length_scale, int32_t distribution, double* length_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ICEFEM_B200_H */
