// Internal data structures shared by the host code (host.cu) and the kernels.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/icefem_b200.h"

namespace ifem {

// error raised by the host code and turned into a status code at the C-ABI
struct Err {
  int code;
  std::string msg;
};

constexpr double kR = 8.31446261815324;  // BaseMaterial.h:26
constexpr int kStatWords = 8;     // per-step device counters

// Per-element blocks written by the points kernel for the tensor-core tangent, element-major so that one bulk
// copy moves each (sizes in elements; every block is a multiple of 16 bytes):
constexpr int kTcCq = 36 * 27;    // C_q, float [36][27]
constexpr int kTcGeo = 13 * 27 + 1;  // per-ip geometry, float [13][27] + padding: Jinv (9), 1/wFun, dW/wFun^2 (3)
constexpr int kTcNx = 84;         // 1-D basis tables float [2][3][3][3], nodal NURBS weights [27], max |C_q|,
                                  // a bound of max |G|, padding
constexpr int kTcKd = 28;         // lumped diagonal terms, double [27] + padding

// Element matrices are stored as [element][local node a1][row block], the row block holding
// (comp b1, comp b2, node a2) padded to a multiple of 4 entries so it can be read with 16-byte loads.
__host__ __device__ constexpr int ke_block(int nc, int nen) { return ((nc * nc * nen + 3) / 4) * 4; }

// Material set, temperature-independent part precomputed on the host with the expressions of
// SolidMaterial.cpp:9-11 and IceMaterial.cpp:49-84.
struct MatDev {
  double E, nu, G, lame, K;
  double A0, n, q_creep, t_ref, t_offset, ft0, ftdeg;
  double l, gc_input, visc, phi_visc_lim;
  double star_gamma, ice_eref, ice_creduce, ice_creduce_fact, ice_ereduce_fact;
  double density, damping, k_thermal, cp;
  // values at the pinned temperature (used when there is no T DOF), computed on the host
  double A_pin, Gc_pin, eref_pin, cred_pin;
  // viscoelastic-plastic (VEP): yield stress at TRef and its slope, friction factors of the yield surface and
  // the potential, hardening modulus, plastic viscosity; yield stress at the pinned temperature
  double sy0, sydeg, yield_alpha, pot_alpha, hardening, pl_visc, sy_pin;
  double b_dp;        // DruckerPrager split
  double g_coss, l_coss, hard_e_ref;   // Cosserat model (CosseratMaterial.cpp:3-10)
  int rheology, split, consistent_energy, gc_mode;
};

struct Geo {
  int dim, nen, nip, kron;  // kron = 1: per-element 1-D extraction factors, 0: full operators
  int64_t nel, nn;
  const double* X;        // [nn*dim]
  const double* W;        // [nn] or nullptr
  const int32_t* conn;    // [nel*nen]
  const double* ext;      // kron: [nel*dim*9], full: [nel*nen*nen]
  const int32_t* emat;    // [nel] or nullptr
  const MatDev* mats;     // material sets (device)
  int64_t el0, el1;       // elements [el0, el1) processed by a u-step launch (layouts keep the nel stride)
};

// Gauss rule and Bernstein values at the Gauss points (computed on the host with the
// reference's formulas, IPScheme.cpp:62-109, BaseElemType.cpp:197-213).
struct Rule {
  double w1[3];       // 1-D weights (already /2)
  double B[3][3];     // B[point][function]
  double dB[3][3];
  double d2B[3][3];   // second derivatives (BaseElemType.cpp:209-211), for the second-gradient distributions
  double wip[27];     // tensor-product weights in ip order (x fastest)
};

struct Hist {
  double *EP, *EPo;   // [6][nh]
  double *EH, *EHo, *VD, *VDo, *DVD, *DVDo;  // [nh]
  double *MH, *MHo;   // [mh][nh]: mh = 1 (dLambda) or, with a VEP material set, 4 (hardening, dLambda_v, dLambda_p, -)
};

struct DofMap {
  const int32_t* node_rank;  // [nn] rank of the node in the group's sorted unique nodes (-1: absent)
  int32_t base[IFEM_N_DOF_KINDS];  // dof offset of each kind inside its step (-1: absent)
  int32_t step[IFEM_N_DOF_KINDS];
};

struct ModelOpts {
  int dam_f, dens_f, visc_f, dist, irr, inertia, gravity, lumped_cap, lumped_drive;
  int consistent_deg, tangent_mode, rm_tol_mode, rm_max_it, hasT, ref_compat_T;
  double k0, visc_num, visco_fact, pinned_T, penalty;
  double g[3];
  double lag_fact;   // LagFact of the augmented Lagrange irreversibility methods
  double dist_coefs[5];   // Coefs of the Custom distribution
  double porder_p;   // exponent of PorderDamage (properties/PhaseField/p, default 2)
  int grav_f;        // degradation of the gravity terms: DensityDamage, or GravityDamage in the Cosserat model
};

struct StepState { const double *cur, *old, *d, *dd; };

// Stats words: 0 rm iterations, 1 rm capped, 2 nonfinite, 3 tensor-core pipeline time-out,
// 4 gather bulk-copy time-out
struct UParams {
  Geo geo; Rule rule; DofMap dm; ModelOpts mo; Hist h;
  StepState su, sp, sT;
  double dt, du_dt, ddu_dt;
  double* Fe;          // [nel][dim*nen]
  double* WLe;         // [nel][nen]
  void* Cq;            // [36][nh] float or double, already scaled by the ip weight; [nel][kTcCq] float when
                       // the tensor-core tangent follows (geoq set)
  int cq_f32;
  float* geoq;         // 3D tensor-core tangent: per-ip geometry [nel][kTcGeo]; or nullptr
  double* Kd;          // tensor-core tangent: lumped diagonal terms [nel][kTcKd] (inertia, damping); or nullptr
  float* nxq;          // tensor-core tangent: 1-D basis tables and nodal weights [nel][kTcNx]; or nullptr
  unsigned long long* stats;
  int vep;             // a material set is viscoelastic-plastic or has a DruckerPrager / SpecStrains split: the
                       // general points kernel in its full-tangent variant
  int spec;            // every material set has the VolStrains split and n = 3, and the degradation is Quadratic:
                       // the sum-factorised kernels' instance with these fixed at compile time
};

struct TParams {       // U-step tangent
  Geo geo; Rule rule; ModelOpts mo;
  const void* Cq; int64_t nh;
  const double* WLe; const double* phase_cur; DofMap dm;
  double du_dt, ddu_dt;
  void* Ke;            // [nel][nen][dim][dim][nen]
  const float* geoq;   // per-ip geometry written by the points kernel (tensor-core path)
  const double* Kd;    // lumped diagonal terms written by the points kernel (tensor-core path)
  const float* nxq;    // 1-D basis tables written by the points kernel (tensor-core path)
};

struct PParams {       // phase step
  Geo geo; Rule rule; DofMap dm; ModelOpts mo; Hist h;
  StepState su, sp, sT;
  double dt;
  double* Fe;          // [nel][nen]
  void* Ke;            // [nel][nen][nen]
  int ke_f32;
  int write_hist;
  double* lcrack_el;   // [nel]
  unsigned long long* stats;
  int general;         // a SpecStrains / DruckerPrager split or Lagrange multipliers: the general phase kernel
  double* wl_out;      // [nel][nen] lumped weights sum_q w N (Lagrange multipliers), or nullptr
  int spec;            // as UParams::spec
  // Cosserat model: the driving energy per ip (split, zero before t = 0, history applied) and |N_uu dU|^2 with
  // the micro-rotation rates, from k_coss_energy; nullptr for the phase-field model
  const double* e_in;
  const double* v2_in;
};

// Lagrange-multiplier irreversibility: the phase element (Ke1, Fe1 of the phase DOFs) grown to the
// [phase, L(, L2)] system with the nodal multiplier terms
struct LagParams {
  Geo geo; DofMap dm; ModelOpts mo;
  const double* phase_cur; const double* phase_old;   // phase-step state vectors
  int nlag;                                           // 1 or 2 multiplier kinds
  const void* Ke1; const double* Fe1; const double* WL;
  void* Ke; double* Fe;                               // [nel][nen][nc][nc][nen] (padded rows), [nel][nc][nen]
  int ke_f32;
};

struct ThParams {      // T step: viscous heating residual and/or thermal model
  Geo geo; Rule rule; DofMap dm; Hist h;
  StepState sT;
  double dt, du_dt;
  int visc_heat, thermal;
  double* Fvh;         // [nel][nen]
  double* Fth;         // [nel][nen]
  void* Ke;            // [nel][nen][nen]
  int ke_f32;
  unsigned long long* stats;
};

struct GParams {       // node-row gather into CSR + residual
  int nc, nen;
  int64_t n_nodes;             // nodes of the step (rank order); rows [node0, n_nodes) are gathered
  int64_t node0;
  const int32_t* rank_node;    // [n_nodes] rank -> node id (unused by the kernel; kept for checks)
  const int32_t* nbr_ptr;      // [n_nodes+1] CSR of sorted neighbour ranks
  const int32_t* inc_ptr;      // [n_nodes+1]
  const int32_t* inc_el;       // [n_inc] incident elements (ascending)
  const uint8_t* inc_loc;      // [n_inc] local index of the node in the element
  const void* emap;            // [nel][nen][nen] position of node a2 in the sorted neighbours of node a1
  int emap16;                  // 0: uint8, 1: uint16
  const void* Ke; int ke_f32;  // [nel][nen][nc][nc][nen]  (nullptr: residual only)
  const double* Fe1;           // [nel][nc*nen] first residual source (element order)
  const double* Fe2;           // second residual source, summed after the first over all elements
  const int64_t* rowptr;       // [ndofs+1]
  int32_t row_base[6];         // dof offset of component b (row = row_base[b] + rank)
  int32_t blk_pos[6];          // column block of component b inside a row
  double* f;                   // [ndofs]
  void* vals; int vals_f32;    // [nnz]
  int acc_stride;              // doubles of shared accumulator per warp
  const void* inc_em;          // [n_inc][32] emap rows in incidence order (uint8 / uint16 as emap16)
  int max_inc;                 // largest number of elements incident to one node
  int max_deg;                 // largest number of neighbours of one node
  unsigned long long* err;     // set when a bulk-copy wait times out
};

struct ConsParams {    // constraint application on one step's CSR
  int64_t n_free;
  const int32_t* row_src;      // [n_free] free index -> dof (row of K)
  const int32_t* fmap;         // [ndofs] free index, or -1 - constrained index
  const int64_t* rowptr; const int32_t* colidx;
  const void* vals; int vals_f32;   // K values (nullptr: the step has no matrix)
  const double* f;             // residual [ndofs]
  const double* cv;            // C_v [n_cons]
  const int64_t* rowptr_con;   // [n_free+1]
  void* vals_con; int want_matrix;
  double* f_con;               // [n_free]
};

// kernel launchers (kernels_*.cu)
void launch_u_points(const UParams& p, cudaStream_t s);
bool launch_u_points_hex(const UParams& p, cudaStream_t s);   // kernels_points.cu (3D, factored extraction)
void launch_u_tangent(const TParams& p, int f32, cudaStream_t s);
void launch_phase(const PParams& p, cudaStream_t s);
void launch_phase_ho(const PParams& p, cudaStream_t s);      // kernels_ho.cu (second-gradient distributions)
__host__ __device__ constexpr bool dist_second_gradient(int d) { return (d >= 4 && d <= 7) || d == 9; }
bool launch_phase_hex(const PParams& p, cudaStream_t s);      // kernels_points.cu (3D, factored extraction)
void launch_thermal(const ThParams& p, cudaStream_t s);
void launch_gather(const GParams& p, cudaStream_t s);
bool launch_gather_bulk(const GParams& p, cudaStream_t s);   // kernels_gather.cu
bool launch_gather_direct1(const GParams& p, cudaStream_t s);   // kernels_gather1.cu (one-component rows)
void launch_reduce_sum(const double* x, int64_t n, double* out, cudaStream_t s);
void launch_phase_lagrange(const LagParams& p, cudaStream_t s);

// device Krylov solve of the constrained system (kernels_solve.cu)
void launch_spmv(int64_t n, const int64_t* rp, const int32_t* ci, const void* v, int f32, const double* x, double* y,
                 cudaStream_t s);
void launch_diag_inv(int64_t n, const int64_t* rp, const int32_t* ci, const void* v, int f32, double* dinv,
                     cudaStream_t s);
void launch_dots(int64_t n, const double* V, int64_t ld, int k, const double* w, double* out, cudaStream_t s,
                 bool with_norm = false);
void launch_comb(int64_t n, const double* V, int64_t ld, const double* c, int k, double a, double* w, cudaStream_t s);
void launch_scale(int64_t n, double a, const double* x, const double* d, double* y, cudaStream_t s);
void launch_sub(int64_t n, const double* b, const double* y, double* r, cudaStream_t s);
// smoothed-aggregation multigrid preconditioner of the device GMRES (amg.cu)
struct AmgHierarchy;
struct AmgOptions {
  double theta = 0.0;   // strength threshold of the aggregation graph at the finest level (halved per level)
  int sweeps = 2;       // damped-Jacobi sweeps before and after the coarse correction
};
AmgHierarchy* amg_build(int64_t n, const std::vector<int64_t>& rp, const std::vector<int32_t>& ci,
                        const std::vector<double>& v, const std::vector<int32_t>& node_of_row, int64_t nnodes, int nm,
                        const std::vector<double>& B, const AmgOptions& opt);
void amg_apply(AmgHierarchy* h, const double* in, double* out, cudaStream_t s);
void amg_free(AmgHierarchy* h);
int amg_levels(const AmgHierarchy* h, int64_t* sizes, int max_levels);
double amg_setup_ms(const AmgHierarchy* h);
void launch_block_setup(int64_t nfree, const int32_t* row_src, int64_t nu, int nc, int32_t* tbl, const int64_t* rp,
                        const int32_t* ci, const void* v, int f32, double* Binv, cudaStream_t s);
void launch_block_apply(int64_t nu, int nc, const int32_t* tbl, const double* Binv, const double* x, double* y,
                        cudaStream_t s);

// OceanBC u-step term (2D): residual-only element contributions [nel][2][nen]
// Cosserat model (kernels_coss.cu): the u-step ips (return map, split, w sigma and w C per ip), the element
// residual and tangent from them, and the phase step's driving energy
struct CossParams {
  Geo geo; Rule rule; DofMap dm; ModelOpts mo; Hist h;
  StepState su, sp, sT;
  double t, dt, du_dt, ddu_dt;
  double* Sc;          // [nh][18] w (Dam sigma_d + sigma_u)
  double* Cc;          // [nh][324] w (Dam D_d + D_u) DPlast
  double* Fe;          // [nel][nc * nen]
  void* Ke; int ke_f32;   // [nel][nen][ke_block(nc, nen)]
  double* Ec;          // phase step: driving energy per ip
  double* V2c;         // phase step: |N_uu dU|^2 per ip
  int mh;              // MatHist values per ip
  unsigned long long* stats;
};
void launch_coss_u(const CossParams& p, cudaStream_t s);
// gather of steps with more than 3 components per node (the 3D Cosserat u-step): one warp per (node, component)
void launch_gather_rows(const GParams& p, cudaStream_t s);
void launch_coss_energy(const CossParams& p, cudaStream_t s);

struct OceanParams {
  Geo geo; Rule rule; DofMap dm;
  const double* phase_cur;
  double hw, density;
  double* Fo;
};
void launch_ocean_u(const OceanParams& p, cudaStream_t s);
// TriAxial boundary loads (kernels_face.cu): faces [0, nside) form the side group, [nside, nside + ntop) the top
// group; each face has nfn = 3 (2D lines) or 9 (3D faces) nodes
struct FaceParams {
  int dim, nfn;
  int64_t nside, ntop;
  Rule rule;
  const double* X;           // mesh coordinates [nn][dim]
  const double* W;           // node weights [nn] (3D faces) or nullptr
  const int32_t* faces;      // [nf][nfn]
  const double* C;           // [nf][nfn][nfn] extraction operators
  DofMap dm;
  const double* ucur;        // displacement state (u-step numbering)
  const double* phase;       // phase state, or nullptr when the side pressure is not degraded
  double p0, t, du, u0, penalty;
  double* F;                 // [nf][dim][nfn] face residuals
  double* K;                 // [ntop][nfn][nfn] top-face matrices (the u_top block)
  double* sums;              // [3][ntop]: area, f_ext, uz_sum per top face
  // gather: unique face nodes, their incidences (face * nfn + a, ascending face) and the CSR positions
  int64_t nnodes;
  const int32_t* node;
  const int32_t* inc_ptr;
  const int32_t* inc;
  const int64_t* kpos;       // [ntop][nfn][nfn]
  const int64_t* rowptr;
  const int32_t* colidx;
  double* f;
  void* vals;
  int vals_f32;
  unsigned long long* err;   // set when a face pair is outside the pattern
};
void launch_face_kpos(const FaceParams& p, int64_t* kpos, cudaStream_t s);
void launch_face_loads(const FaceParams& p, cudaStream_t s);
void launch_face_gather(const FaceParams& p, cudaStream_t s);
void launch_u_tangent_tc(const TParams& p, unsigned long long* err, int n_sm, cudaStream_t s);
size_t tc_smem_bytes();
// constraints (kernels_cons.cu)
void launch_cons_cv(const int64_t* con_dof, const double* con_val, int64_t n, const double* u, double* cv,
                    cudaStream_t s);
void launch_constrain(const ConsParams& p, cudaStream_t s);
void launch_update_state(const int32_t* fmap, int64_t n, const double* dx, const double* cv, double* u,
                         cudaStream_t s);
// adjoint (kernels_adjoint.cu): dF[theta][el][comp*nen + node], theta = (Gc, l, A, n)
// dT, dFT: temperature perturbation (T-step numbering, or nullptr for the pinned temperature) and the element
// vectors of dR/dT . dT (nullptr: not computed); dF may be nullptr.  f32: the FP32 adjoint variant.
void launch_adjoint_u(const UParams& p, double* dF, const double* dT, double* dFT, int f32, cudaStream_t s);
void launch_adjoint_phase(const PParams& p, double* dF, const double* dT, double* dFT, int f32, cudaStream_t s);
void launch_adjoint_lambda(const double* dF, int64_t nel, int nc, int nen, const int32_t* conn, const DofMap& dm,
                           int kind0, const double* lambda, double* per_el, const int32_t* mat_ptr,
                           const int32_t* mat_el, int n_mats, double* out, cudaStream_t s);
void build_rule(int ip1d, int dim, Rule& R);   // Gauss rule + Bernstein values (throws on ip1d != 3)

}  // namespace ifem
