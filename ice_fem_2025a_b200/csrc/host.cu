// Host side of the C-ABI (include/icefem_b200.h): context set-up (DOF numbering, CSR pattern,
// element -> nonzero maps), assembly orchestration and state/history management.
//
// Set-up follows the reference's serial path:
//   DofSpace::AddDofs/SyncDofs  (DofSpace.cpp:105-154, 486-513): per step, DOF types in DofNames
//     order, each over the group's unique nodes in ascending node id -> dof = base(kind) + rank(node)
//   MatSetValues pattern       (math.cpp:301-304, physics.cpp:241-244): union of the element DOF
//     pairs, columns ascending, zeros kept
//   getDofForNodes             (DofSpace.cpp:974-1008): element DOF vectors component-major.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <map>
#include <vector>

#include "icefem_internal.h"

namespace ifem {

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) throw Err{IFEM_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

template <class T>
T* dalloc(size_t n) {
  if (n == 0) n = 1;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) throw Err{IFEM_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  return static_cast<T*>(p);
}

template <class T>
T* dupload(const std::vector<T>& v) {
  T* p = dalloc<T>(v.size());
  if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return p;
}

struct StepDev {
  int kind = -1;          // 0 U, 1 phase, 2 T
  int nc = 0;
  int64_t ndofs = 0, nnz = 0;
  int comp_kind[6] = {-1, -1, -1, -1, -1, -1};
  int32_t row_base[6] = {0, 0, 0, 0, 0, 0};
  int32_t blk_pos[6] = {0, 0, 0, 0, 0, 0};
  double* state[4] = {nullptr, nullptr, nullptr, nullptr};
  double* f = nullptr;
  void* vals = nullptr;
  int vals_f32 = 0;
  int64_t* rowptr = nullptr;
  int32_t* colidx = nullptr;
  unsigned long long* stats_d = nullptr;
  double* lcrack_d = nullptr;
  ifem_stats stats{};
  bool assembled = false;
  bool slabbed = false;   // the last assembly ran in slabs, each with its completion event
  // constraints (Constrainer): host copies of the set, device maps and the reduced system
  int64_t n_cons = 0, n_free = 0, nnz_con = 0;
  bool cons_set = false, cons_built = false;
  int32_t* fmap = nullptr;        // [ndofs] free index or -1 - constrained index
  int32_t* row_src = nullptr;     // [n_free]
  int64_t* con_dof = nullptr;     // [n_cons] ascending
  double* con_val = nullptr;      // [n_cons]
  double* cv = nullptr;           // [n_cons] C_v of the last ifem_constrain
  int64_t* rowptr_con = nullptr;  // [n_free+1]
  int32_t* colidx_con = nullptr;  // [nnz_con]
  void* vals_con = nullptr;       // [nnz_con] (allocated as doubles)
  int vals_con_f32 = 0;
  double* f_con = nullptr;        // [n_free]
  double* dx = nullptr;           // [n_free] staging for ifem_update_state
  bool kcon_ready = false;        // vals_con holds K_con of the last ifem_constrain(want_matrix = 1)
  double* kw = nullptr;           // Krylov workspace of ifem_solve_constrained
  size_t kw_len = 0;
  double* kbinv = nullptr;        // node-block preconditioner: inverse blocks [n_unique][3][3]
  int pc_kind = 0;                // IFEM_PC_*
  AmgHierarchy* amg = nullptr;    // multigrid hierarchy of the last set-up
  AmgOptions amg_opt{};
  int32_t* ktbl = nullptr;        // free row of (node, component) or -1
};

}  // namespace ifem

using namespace ifem;

constexpr int kMaxSteps = 8;   // staggered solver steps per context
constexpr int kMaxSlabs = 16;  // element slabs of a pipelined u-step

struct ifem_ctx {
  int device = 0;
  int n_sm = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  // copy-out stream: the residual and matrix of a step are read back once that step's last assembly is done
  // (its event), so the read-back of one step overlaps the assembly of the next one queued behind it
  cudaStream_t cstream = nullptr;
  cudaEvent_t done_ev[kMaxSteps] = {};
  // slab-pipelined u-step: slab k assembles elements [slab_el[k], slab_el[k+1]) and then gathers the node rows
  // [slab_node[k], slab_node[k+1]) whose incident elements are all done; its event lets the read-back copy
  // those rows while later slabs compute.  node_last[r] = largest element incident to node ranks 0..r.
  int slabs = 1;
  std::vector<int64_t> slab_el, slab_node, slab_off;   // slab_off[k*3+b]: CSR offset of row_base[b]+slab_node[k]
  std::vector<int32_t> node_last;
  cudaEvent_t slab_ev[kMaxSlabs] = {};
  std::string err;
  int dim = 0, nen = 0, nip = 0, kron = 1;
  int64_t nel = 0, nn = 0, nh = 0, n_unique = 0;
  double *X = nullptr, *W = nullptr, *ext = nullptr;
  int32_t *conn = nullptr, *emat = nullptr;
  std::vector<int32_t> emat_h;
  MatDev* mats_d = nullptr;
  std::vector<MatDev> mats_h;
  std::vector<ifem_material> mats_in;
  ifem_options opt{};
  ModelOpts mo{};
  Rule rule{};
  int nsteps = 0, step_u = -1, step_ph = -1, step_T = -1;
  int mh = 1;                      // MatHist values per ip: 4 when a material set is viscoelastic-plastic
  bool general = false;            // u-step: VEP or a SpecStrains / DruckerPrager split: general kernel only
  bool ph_general = false;         // phase step: SpecStrains / DruckerPrager or Lagrange multipliers: general kernel
  bool hasT = false;
  bool coss = false;               // Fracture/CossPhaseField
  int ncs = 6;                     // strain components per ip in the plastic-strain history (18: Cosserat)
  double *Sc = nullptr, *Cc = nullptr;   // Cosserat u-step: w sigma [nh][18], w (g D+ + D-) DPlast [nh][324]
  double *Ec = nullptr, *V2c = nullptr;  // Cosserat phase step: driving energy, |N_uu dU|^2 per ip
  bool spec = false;               // VolStrains split and n = 3 in every material set, Quadratic degradation: the
                                   // specialised instances of the sum-factorised kernels
  int32_t* node_rank = nullptr;
  int32_t kind_base[IFEM_N_DOF_KINDS] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
  int32_t kind_step[IFEM_N_DOF_KINDS] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
  int nlag = 0;                    // Lagrange multipliers per phase node (irreversibility methods 3-5)
  double* WLp = nullptr;           // [nel][nen] lumped weights of the phase step (Lagrange multipliers)
  void* Ke2 = nullptr;             // [nel][nen][nc][nc][nen] phase element systems with multipliers
  double* Fl = nullptr;            // [nel][nc][nen] their residuals
  double* Fo = nullptr;            // [nel][2][nen] OceanBC element residuals
  // TriAxial model (ifem_set_triaxial): face groups (side faces first), face terms, gather lists, state
  bool tri_on = false, tri_assembled = false;
  ifem_triaxial tri_prm{};
  ifem_triaxial_state tri_st{};
  int64_t tri_nside = 0, tri_ntop = 0, tri_nnodes = 0;
  int32_t *tri_faces = nullptr, *tri_node = nullptr, *tri_inc_ptr = nullptr, *tri_inc = nullptr;
  double *tri_C = nullptr, *tri_F = nullptr, *tri_K = nullptr, *tri_sums = nullptr, *tri_tot = nullptr;
  int64_t* tri_kpos = nullptr;
  size_t Ke2_bytes = 0;
  std::vector<int64_t> kind_dof_node;  // unused placeholder for clarity
  int32_t *nbr_ptr = nullptr, *inc_ptr = nullptr, *inc_el = nullptr;
  uint8_t* inc_loc = nullptr;
  void* emap = nullptr;
  void* inc_em = nullptr;          // emap rows in incidence order, 32 entries each
  int max_inc = 0;
  int emap16 = 0, max_deg = 0;
  Hist h{};
  double *Fe = nullptr, *Fe2 = nullptr, *WLe = nullptr, *lc_el = nullptr;
  void *Cq = nullptr, *Ke = nullptr;
  float* geoq = nullptr;
  double* Kd = nullptr;              // lumped diagonal terms for the tensor-core tangent
  float* nxq = nullptr;              // per-element 1-D basis tables for the tensor-core tangent
  size_t Cq_bytes = 0, Ke_bytes = 0;
  std::vector<StepDev> steps;
  // adjoint buffers, allocated on the first adjoint: element derivatives and per-element sums are shared
  // (stream-ordered), the results (dR/dtheta [4][ndofs], lambda^T dR [n_mats][4]) are kept per step
  double *adj_dF = nullptr, *adj_lam = nullptr, *adj_el = nullptr;
  int32_t *adj_mat_ptr = nullptr, *adj_mat_el = nullptr;
  std::vector<double*> adj_f, adj_out;
  int adj_f32 = 0;                   // FP32 variant of the adjoint contraction (ifem_set_adjoint_precision)
  // temperature sensitivity: perturbation [n_T], element vectors [nel][nc][nen], result [ndofs of the step]
  double *sens_dT = nullptr, *sens_dF = nullptr, *sens_f = nullptr;
  int64_t sens_f_len = 0;
  // captured CUDA graph of assemblies (+ adjoints)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool capturing = false;
  std::vector<int> graph_steps;
};

namespace ifem {

static thread_local std::string g_create_err;

// ------------------------------------------------------------------------------------------
// set-up helpers
// ------------------------------------------------------------------------------------------
static int fact(int n) { return (n == 0) || (n == 1) ? 1 : n * fact(n - 1); }

static void make_rule(int ip1d, Rule& R) {
  if (ip1d != 3) throw Err{IFEM_ERR_UNSUPPORTED, "ipcount1D must be 3"};
  const double c[3] = {-std::sqrt(3.0 / 5.0), 0, std::sqrt(3.0 / 5.0)};
  const double w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  double cc[3];
  for (int i = 0; i < 3; ++i) { cc[i] = (c[i] + 1) / 2; R.w1[i] = w[i] / 2; }
  const int p = 2;
  for (int pt = 0; pt < 3; ++pt) {
    const double x = cc[pt];
    for (int i = 0; i < p + 1; ++i) {  // BezierBasis (BaseElemType.cpp:197-213)
      const double pre = fact(p) / fact(p - i) / fact(i);
      R.B[pt][i] = pre * std::pow(1.0 - x, std::max(0, p - i)) * std::pow(x, std::max(0, i));
      R.dB[pt][i] = pre * ((i - p) * std::pow(1.0 - x, std::max(0, p - i - 1)) * std::pow(x, std::max(0, i)) +
                           i * std::pow(1.0 - x, p - i) * std::pow(x, std::max(0, i - 1)));
      R.d2B[pt][i] = pre * (2 * i * std::pow(x, std::max(0, i - 1)) * (i - p) * std::pow(1.0 - x, std::max(0, p - i - 1)) +
                            i * std::pow(x, std::max(0, i - 2)) * (i - 1) * std::pow(1.0 - x, std::max(0, p - i)) +
                            (i - p + 1) * std::pow(x, std::max(0, i)) * (i - p) * std::pow(1.0 - x, std::max(0, p - i - 2)));
    }
  }
}

static void make_wip(int dim, Rule& R) {
  int cnt = 0;
  if (dim == 2) {
    for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) R.wip[cnt++] = R.w1[i] * R.w1[j];
  } else {
    for (int k = 0; k < 3; ++k) for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) R.wip[cnt++] = R.w1[i] * R.w1[j] * R.w1[k];
  }
}

void build_rule(int ip1d, int dim, Rule& R) {
  make_rule(ip1d, R);
  make_wip(dim, R);
}

static MatDev make_mat(const ifem_material& m, const ifem_options& o) {
  MatDev d{};
  d.E = m.young * (1 - 0.0);
  d.nu = m.poisson;
  d.G = d.E / (2.0 * (1 + d.nu));
  d.lame = d.E * d.nu / ((1.0 + d.nu) * (1.0 - 2.0 * d.nu));
  d.K = d.lame + 2.0 / 3.0 * d.G;
  d.A0 = m.creep_a; d.n = m.creep_n; d.q_creep = m.q_creep; d.t_ref = m.t_ref; d.t_offset = m.t_offset;
  d.ft0 = m.ft0; d.ftdeg = m.ftdeg; d.l = m.pf_l; d.gc_input = m.gc; d.visc = m.pf_visc;
  d.phi_visc_lim = m.phi_visc_lim;
  d.star_gamma = m.star_convex_gamma; d.ice_eref = m.ice_eref; d.ice_creduce = m.ice_creduce;
  d.ice_creduce_fact = m.ice_creduce_fact; d.ice_ereduce_fact = m.ice_ereduce_fact;
  d.density = m.density; d.damping = m.damping; d.k_thermal = m.k_thermal; d.cp = m.cp;
  d.rheology = m.rheology; d.split = m.split; d.consistent_energy = m.consistent_energy; d.gc_mode = m.gc_mode;
  // pinned-temperature values (IceMaterial.cpp:49-84)
  double TAbs = o.pinned_temperature + m.t_offset;
  if (TAbs > 273.15) TAbs = 273.15;
  const double ExpTerm = -m.q_creep / kR * (1 / TAbs - 1 / m.t_ref);
  d.A_pin = m.creep_a * std::exp(ExpTerm);
  const double ft = 1.0 * (m.ft0 - m.ftdeg * (TAbs - m.t_ref));
  d.Gc_pin = (m.gc_mode == 1) ? m.gc : 2.0 * ft * ft / d.E * m.pf_l;
  d.eref_pin = m.ice_eref; d.cred_pin = m.ice_creduce;
  if (m.split == IFEM_SPLIT_ICE) {
    d.eref_pin = m.ice_eref + m.ice_ereduce_fact * std::sqrt(std::max(1e-3, -(TAbs - m.t_ref)));
    d.cred_pin = m.ice_creduce - (TAbs - m.t_ref) * m.ice_creduce_fact;
  }
  // viscoelastic-plastic parameters (SolidMaterial.cpp:50-65; sy at temperature: IceMaterial.cpp:81-82)
  auto dp_alpha = [](double deg) {
    const double a = 3.14159265358979323846 / 180.0 * deg;
    return 6.0 * std::sin(a) / (3.0 - std::sin(a));
  };
  d.sy0 = m.vep_sy; d.sydeg = m.vep_sydeg;
  d.yield_alpha = dp_alpha(m.vep_f_deg); d.pot_alpha = dp_alpha(m.vep_g_deg);
  d.hardening = m.vep_hardening; d.pl_visc = m.vep_pl_visc;
  d.sy_pin = m.vep_sy - m.vep_sydeg * (TAbs - m.t_ref);
  d.b_dp = m.b_dp;
  d.g_coss = m.g_coss; d.l_coss = m.l_coss; d.hard_e_ref = m.hard_e_ref;
  if (o.cosserat) {   // CosseratMaterial.cpp:107-154, 450-514
    if (m.rheology != IFEM_RHEO_LE && m.rheology != IFEM_RHEO_VEP && m.rheology != IFEM_RHEO_DVEP)
      throw Err{IFEM_ERR_UNSUPPORTED, "Rheology type not defined in CosseratMaterial.cpp"};
    if (m.split != IFEM_SPLIT_NONE && m.split != IFEM_SPLIT_SPECSTRESS && m.split != IFEM_SPLIT_DRUCKERPRAGER &&
        m.split != IFEM_SPLIT_STARCONVEX)
      throw Err{IFEM_ERR_UNSUPPORTED, "Stress split function type not defined for a Cosserat Material"};
    if (m.rheology != IFEM_RHEO_LE && !(m.hard_e_ref != 0.0))
      throw Err{IFEM_ERR_INVALID, "the Cosserat return map needs hard_eRef != 0"};
    return d;
  }
  if (m.rheology == IFEM_RHEO_DVEP)
    throw Err{IFEM_ERR_UNSUPPORTED, "Rheology type not defined: DamViscoElasticPlastic has no return map"};
  if (m.rheology < 0 || m.rheology > IFEM_RHEO_VEP) throw Err{IFEM_ERR_UNSUPPORTED, "rheology"};
  if (m.split < IFEM_SPLIT_NONE || m.split > IFEM_SPLIT_STARCONVEX) throw Err{IFEM_ERR_UNSUPPORTED, "energy split"};
  if (m.split == IFEM_SPLIT_SPECSTRESS && m.consistent_energy)   // PhaseFieldMaterial.cpp:148-150
    throw Err{IFEM_ERR_UNSUPPORTED, "Spectral Stress split not implemented when using a consistent split for energy/stress damage"};
  return d;
}

// C = kron(Cz, kron(Cy, Cx)) -> factors, exact up to a few ulps, or false
static bool factor_kron(int dim, const double* C, double* k) {
  const int nen = dim == 2 ? 9 : 27;
  int j0 = 0, k0 = 0;
  double best = 0;
  for (int j = 0; j < nen; ++j) for (int c = 0; c < nen; ++c)
    if (std::fabs(C[j * nen + c]) > best) { best = std::fabs(C[j * nen + c]); j0 = j; k0 = c; }
  if (best == 0) return false;
  const int ix0 = j0 % 3, iy0 = (j0 / 3) % 3, iz0 = j0 / 9, jx0 = k0 % 3, jy0 = (k0 / 3) % 3, jz0 = k0 / 9;
  auto at = [&](int ix, int iy, int iz, int jx, int jy, int jz) { return C[(ix + 3 * iy + 9 * iz) * nen + jx + 3 * jy + 9 * jz]; };
  const double c0 = at(ix0, iy0, iz0, jx0, jy0, jz0);
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
    k[a * 3 + b] = at(a, iy0, iz0, b, jy0, jz0);
    k[9 + a * 3 + b] = at(ix0, a, iz0, jx0, b, jz0) / c0;
    if (dim == 3) k[18 + a * 3 + b] = at(ix0, iy0, a, jx0, jy0, b) / c0;
  }
  double maxdiff = 0;
  for (int j = 0; j < nen; ++j) for (int c = 0; c < nen; ++c) {
    const int ix = j % 3, iy = (j / 3) % 3, iz = j / 9, jx = c % 3, jy = (c / 3) % 3, jz = c / 9;
    double v = k[9 + iy * 3 + jy] * k[ix * 3 + jx];
    if (dim == 3) v = k[18 + iz * 3 + jz] * v;
    maxdiff = std::max(maxdiff, std::fabs(v - C[j * nen + c]));
  }
  return maxdiff <= 8.0 * 2.220446049250313e-16 * best;
}

static void destroy(ifem_ctx* c) {
  if (!c) return;
  auto F = [](void* p) { if (p) cudaFree(p); };
  F(c->X); F(c->W); F(c->ext); F(c->conn); F(c->emat); F(c->mats_d); F(c->node_rank);
  F(c->nbr_ptr); F(c->inc_ptr); F(c->inc_el); F(c->inc_loc); F(c->emap); F(c->inc_em);
  F(c->h.EP); F(c->h.EPo); F(c->h.EH); F(c->h.EHo); F(c->h.VD); F(c->h.VDo); F(c->h.DVD); F(c->h.DVDo);
  F(c->h.MH); F(c->h.MHo);
  F(c->Fe); F(c->Fe2); F(c->WLe); F(c->lc_el); F(c->Cq); F(c->Ke); F(c->geoq); F(c->Kd); F(c->nxq);
  F(c->WLp); F(c->Ke2); F(c->Fl); F(c->Fo);
  F(c->Sc); F(c->Cc); F(c->Ec); F(c->V2c);
  F(c->tri_faces); F(c->tri_node); F(c->tri_inc_ptr); F(c->tri_inc); F(c->tri_C); F(c->tri_F); F(c->tri_K);
  F(c->tri_sums); F(c->tri_tot); F(c->tri_kpos);
  F(c->adj_dF); F(c->adj_lam); F(c->adj_el); F(c->adj_mat_ptr); F(c->adj_mat_el);
  for (double* q : c->adj_f) F(q);
  for (double* q : c->adj_out) F(q);
  F(c->sens_dT); F(c->sens_dF); F(c->sens_f);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  for (auto& s : c->steps) {
    for (int k = 0; k < 4; ++k) F(s.state[k]);
    F(s.f); F(s.vals); F(s.rowptr); F(s.colidx); F(s.stats_d); F(s.lcrack_d);
    F(s.fmap); F(s.row_src); F(s.con_dof); F(s.con_val); F(s.cv); F(s.rowptr_con); F(s.colidx_con);
    F(s.vals_con); F(s.f_con); F(s.dx);
    amg_free(s.amg); s.amg = nullptr;
  }
  for (int i = 0; i < 5; ++i) if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  for (auto& e : c->done_ev) if (e) cudaEventDestroy(e);
  for (auto& e : c->slab_ev) if (e) cudaEventDestroy(e);
  if (c->cstream) cudaStreamDestroy(c->cstream);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

// the specialised kernel instances apply when every material set has the VolStrains split and, where a return
// map runs, n = 3, and the degradation function is Quadratic
static void set_spec(ifem_ctx* c) {
  c->spec = c->opt.dam_function == IFEM_DAM_QUADRATIC;
  for (const ifem_material& m : c->mats_in)
    c->spec = c->spec && m.split == IFEM_SPLIT_VOLSTRAINS && (m.rheology == IFEM_RHEO_LE || m.creep_n == 3.0);
}

static void create(ifem_ctx* c, const ifem_mesh_desc* mesh, const ifem_material* mats, int n_mats,
                   const ifem_options* opts, int device) {
  if (!mesh || !mats || !opts || n_mats < 1) throw Err{IFEM_ERR_INVALID, "null argument"};
  c->device = device;
  CK(cudaSetDevice(device));
  CK(cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, device));
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  for (int i = 0; i < 5; ++i) CK(cudaEventCreate(&c->ev[i]));
  CK(cudaStreamCreateWithFlags(&c->cstream, cudaStreamNonBlocking));
  for (auto& e : c->done_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto& e : c->slab_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  c->dim = mesh->dim;
  if (mesh->elem_type == IFEM_ELEM_B2_2 && mesh->dim == 2) c->nen = 9;
  else if (mesh->elem_type == IFEM_ELEM_NURBS3_CUBE2 && mesh->dim == 3) c->nen = 27;
  else throw Err{IFEM_ERR_UNSUPPORTED, "element type / dim"};
  c->nip = c->nen;
  make_rule(mesh->ipcount1d, c->rule);
  make_wip(c->dim, c->rule);
  c->nel = mesh->n_elems; c->nn = mesh->n_nodes;
  if (c->nel < 0 || c->nn < 0 || c->nn > INT32_MAX) throw Err{IFEM_ERR_INVALID, "mesh sizes"};
  if (c->nel > 0 && (!mesh->coords || !mesh->elems)) throw Err{IFEM_ERR_INVALID, "mesh arrays"};
  c->nh = c->nel * c->nip;
  const int nen = c->nen, dim = c->dim;
  // connectivity
  std::vector<int32_t> conn((size_t)c->nel * nen);
  for (size_t i = 0; i < conn.size(); ++i) {
    const int64_t v = mesh->elems[i];
    if (v < 0 || v >= c->nn) throw Err{IFEM_ERR_INVALID, "element node out of range"};
    conn[i] = (int32_t)v;
  }
  for (int64_t e = 0; e < c->nel; ++e)
    for (int a = 0; a < nen; ++a) for (int b = a + 1; b < nen; ++b)
      if (conn[e * nen + a] == conn[e * nen + b]) throw Err{IFEM_ERR_INVALID, "repeated node in element"};
  // extraction operators
  std::vector<double> ext;
  if (mesh->elem_kron) {
    c->kron = 1;
    ext.assign(mesh->elem_kron, mesh->elem_kron + (size_t)c->nel * dim * 9);
  } else if (mesh->elem_data) {
    ext.resize((size_t)c->nel * dim * 9);
    bool ok = true;
    for (int64_t e = 0; e < c->nel && ok; ++e) ok = factor_kron(dim, mesh->elem_data + (size_t)e * nen * nen, &ext[e * dim * 9]);
    if (ok) c->kron = 1;
    else { c->kron = 0; ext.assign(mesh->elem_data, mesh->elem_data + (size_t)c->nel * nen * nen); }
  } else throw Err{IFEM_ERR_INVALID, "mesh needs elem_data or elem_kron"};
  // materials
  c->opt = *opts;
  if (c->opt.rm_max_it <= 0) c->opt.rm_max_it = 250;
  c->mats_in.assign(mats, mats + n_mats);
  for (int i = 0; i < n_mats; ++i) c->mats_h.push_back(make_mat(mats[i], c->opt));
  for (int i = 0; i < n_mats; ++i) if (mats[i].rheology == IFEM_RHEO_VEP) c->mh = 4;   // HistSize 4 (SolidMaterial.cpp:50-51)
  c->general = c->mh == 4;
  for (int i = 0; i < n_mats; ++i)
    if (mats[i].split == IFEM_SPLIT_SPECSTRAINS || mats[i].split == IFEM_SPLIT_DRUCKERPRAGER) c->general = c->ph_general = true;
  c->coss = opts->cosserat != 0;
  if (c->coss) {   // Cosserat model: its own u-step kernels, the general phase kernel with the Cosserat energy
    c->ncs = 18;
    c->mh = 1;
    for (int i = 0; i < n_mats; ++i) if (mats[i].rheology != IFEM_RHEO_LE) c->mh = 4;
    c->general = false;
    c->ph_general = true;
  }
  if (mesh->elem_mat) {
    c->emat_h.assign(mesh->elem_mat, mesh->elem_mat + c->nel);
    for (int32_t v : c->emat_h) if (v < 0 || v >= n_mats) throw Err{IFEM_ERR_INVALID, "elem_mat out of range"};
  }
  // DOF kinds and steps
  bool has[IFEM_N_DOF_KINDS] = {};
  int maxstep = -1;
  if (opts->n_dofs < 1 || opts->n_dofs > IFEM_N_DOF_KINDS) throw Err{IFEM_ERR_INVALID, "n_dofs"};
  for (int i = 0; i < opts->n_dofs; ++i) {
    const int k = opts->dof_kind[i];
    if (k < 0 || k >= IFEM_N_DOF_KINDS || has[k]) throw Err{IFEM_ERR_INVALID, "dof kinds"};
    if (opts->dof_step[i] < 0 || opts->dof_step[i] > 7) throw Err{IFEM_ERR_INVALID, "dof step"};
    has[k] = true;
    c->kind_step[k] = opts->dof_step[i];
    maxstep = std::max(maxstep, opts->dof_step[i]);
  }
  if (!has[IFEM_DOF_UX] || !has[IFEM_DOF_UY] || (dim == 3 && !has[IFEM_DOF_UZ]) || !has[IFEM_DOF_PHASE])
    throw Err{IFEM_ERR_INVALID, "Dof of type ux/uy(/uz)/phase is not defined"};
  if (c->kind_step[IFEM_DOF_UX] != c->kind_step[IFEM_DOF_UY] || (dim == 3 && c->kind_step[IFEM_DOF_UZ] != c->kind_step[IFEM_DOF_UX]))
    throw Err{IFEM_ERR_INVALID, "displacements must share a solver step"};
  c->step_u = c->kind_step[IFEM_DOF_UX];
  c->step_ph = c->kind_step[IFEM_DOF_PHASE];
  // micro-rotations: oz in 2D, ox oy oz in 3D, in the displacement step (CossPhaseField.cpp:170-219)
  if (opts->cosserat) {
    const bool ok = has[IFEM_DOF_OZ] && c->kind_step[IFEM_DOF_OZ] == c->step_u &&
                    (dim == 3 ? (has[IFEM_DOF_OX] && has[IFEM_DOF_OY] && c->kind_step[IFEM_DOF_OX] == c->step_u &&
                                 c->kind_step[IFEM_DOF_OY] == c->step_u)
                              : (!has[IFEM_DOF_OX] && !has[IFEM_DOF_OY]));
    if (!ok) throw Err{IFEM_ERR_INVALID, "the Cosserat model needs oz (2D) or ox, oy, oz (3D) in the displacement step"};
  } else if (has[IFEM_DOF_OX] || has[IFEM_DOF_OY] || has[IFEM_DOF_OZ]) {
    throw Err{IFEM_ERR_INVALID, "micro-rotation dofs need the Cosserat model"};
  }
  c->hasT = has[IFEM_DOF_T];
  c->step_T = c->hasT ? c->kind_step[IFEM_DOF_T] : -1;
  if (c->step_u == c->step_ph || (c->hasT && (c->step_T == c->step_u || c->step_T == c->step_ph)))
    throw Err{IFEM_ERR_UNSUPPORTED, "u, phase and T must be solved in distinct staggered steps"};
  if (opts->ocean_bc && dim != 2) throw Err{IFEM_ERR_UNSUPPORTED, "OceanBC is a 2D model"};
  if (c->opt.irreversible < IFEM_IRR_NONE || c->opt.irreversible > IFEM_IRR_AUGLAG2)
    throw Err{IFEM_ERR_UNSUPPORTED, "irreversibility method"};
  // Lagrange-multiplier irreversibility: the multipliers are DOFs of the phase step (PhaseField.cpp:95-101,
  // 270-280); other methods have none
  c->nlag = c->opt.irreversible == IFEM_IRR_AUGLAG2 ? 2
          : (c->opt.irreversible == IFEM_IRR_LAGRANGE || c->opt.irreversible == IFEM_IRR_AUGLAG) ? 1 : 0;
  if (has[IFEM_DOF_LMULT] != (c->nlag >= 1) || has[IFEM_DOF_LMULT2] != (c->nlag == 2))
    throw Err{IFEM_ERR_INVALID, "lMult_pf / lMult_pf2 DOFs must match the irreversibility method"};
  if ((c->nlag >= 1 && c->kind_step[IFEM_DOF_LMULT] != c->step_ph) ||
      (c->nlag == 2 && c->kind_step[IFEM_DOF_LMULT2] != c->step_ph))
    throw Err{IFEM_ERR_INVALID, "the Lagrange multipliers must be in the phase-field solver step"};
  if (c->nlag) c->ph_general = true;
  set_spec(c);
  c->nsteps = maxstep + 1;
  if (c->nsteps > kMaxSteps) throw Err{IFEM_ERR_UNSUPPORTED, "more than 8 solver steps"};
  // model options
  ModelOpts& mo = c->mo;
  mo.dam_f = opts->dam_function; mo.dens_f = opts->density_dam_function; mo.visc_f = opts->visco_dam_function;
  mo.dist = opts->distribution; mo.irr = opts->irreversible; mo.inertia = opts->inertia; mo.gravity = opts->gravity;
  mo.lumped_cap = opts->lumped_cap; mo.lumped_drive = opts->lumped_drive; mo.consistent_deg = opts->consistent_degradation;
  mo.tangent_mode = opts->tangent_mode; mo.rm_tol_mode = opts->rm_tol_mode; mo.rm_max_it = c->opt.rm_max_it;
  mo.hasT = c->hasT ? 1 : 0; mo.ref_compat_T = opts->ref_compat_phase_t;
  mo.k0 = opts->k0; mo.visc_num = opts->visc_num; mo.visco_fact = opts->visco_driving_factor;
  mo.pinned_T = opts->pinned_temperature; mo.penalty = opts->penalty_factor > 0 ? opts->penalty_factor : 1.0e6;
  mo.lag_fact = opts->lag_fact > 0 ? opts->lag_fact : 1.0;
  mo.porder_p = opts->porder_p != 0.0 ? opts->porder_p : 2.0;
  mo.grav_f = opts->cosserat ? opts->gravity_dam_function : opts->density_dam_function;
  if (opts->cosserat) { mo.lumped_cap = 0; mo.lumped_drive = 0; }   // the Cosserat phase step has neither
  mo.g[0] = 0; mo.g[1] = 0; mo.g[2] = 0;
  if (opts->gravity) { if (dim == 3) mo.g[2] = -9.81; else mo.g[1] = -9.81; }  // PhaseField.h:95, PhaseField.cpp:168-171
  if (mo.dist < 0 || mo.dist > 9) throw Err{IFEM_ERR_UNSUPPORTED, "distribution function"};
  for (int i = 0; i < 5; ++i) mo.dist_coefs[i] = opts->dist_coefs[i];
  if (mo.dist == IFEM_DIST_CUSTOM && !(opts->dist_coefs[0] != 0.0))
    throw Err{IFEM_ERR_INVALID, "the Custom distribution needs Coefs[0] != 0"};
  // unique nodes and ranks
  std::vector<int32_t> rank(c->nn, -1);
  for (int32_t v : conn) rank[v] = 1;
  int64_t cnt = 0;
  std::vector<int32_t> rank_node;
  for (int64_t n = 0; n < c->nn; ++n) if (rank[n] >= 0) { rank[n] = (int32_t)cnt++; rank_node.push_back((int32_t)n); }
  c->n_unique = cnt;
  // DOF numbering per step (kinds in DofNames order)
  for (int s = 0; s < c->nsteps; ++s) {
    int64_t counter = 0;
    for (int i = 0; i < opts->n_dofs; ++i) {
      if (opts->dof_step[i] != s) continue;
      const int k = opts->dof_kind[i];
      if (k == IFEM_DOF_UZ && dim != 3) continue;
      c->kind_base[k] = (int32_t)counter;
      counter += cnt;
    }
    if (counter > INT32_MAX) throw Err{IFEM_ERR_CAPACITY, "more than 2^31 DOFs in a step"};
    StepDev sd;
    sd.ndofs = counter;
    c->steps.push_back(sd);
  }
  // incidence (elements ascending) and neighbour lists in rank space
  std::vector<int32_t> inc_ptr(cnt + 1, 0);
  for (int32_t v : conn) inc_ptr[rank[v] + 1]++;
  for (int64_t r = 0; r < cnt; ++r) inc_ptr[r + 1] += inc_ptr[r];
  std::vector<int32_t> inc_el(inc_ptr[cnt]);
  std::vector<uint8_t> inc_loc(inc_ptr[cnt]);
  {
    std::vector<int32_t> fill(inc_ptr.begin(), inc_ptr.end() - 1);
    for (int64_t e = 0; e < c->nel; ++e)
      for (int a = 0; a < nen; ++a) {
        const int r = rank[conn[e * nen + a]];
        inc_el[fill[r]] = (int32_t)e;
        inc_loc[fill[r]] = (uint8_t)a;
        fill[r]++;
      }
  }
  c->node_last.assign(cnt, -1);
  for (int64_t r = 0; r < cnt; ++r) {
    const int32_t last = inc_ptr[r + 1] > inc_ptr[r] ? inc_el[inc_ptr[r + 1] - 1] : -1;
    c->node_last[r] = std::max(last, r > 0 ? c->node_last[r - 1] : -1);
  }
  std::vector<int32_t> nbr_ptr(cnt + 1, 0);
  std::vector<int32_t> nbr;
  nbr.reserve((size_t)cnt * (dim == 3 ? 125 : 25));
  {
    std::vector<int64_t> mark(cnt, -1);
    std::vector<int32_t> tmp;
    for (int64_t r = 0; r < cnt; ++r) {
      tmp.clear();
      for (int k = inc_ptr[r]; k < inc_ptr[r + 1]; ++k) {
        const int64_t e = inc_el[k];
        for (int a = 0; a < nen; ++a) {
          const int32_t rk = rank[conn[e * nen + a]];
          if (mark[rk] != r) { mark[rk] = r; tmp.push_back(rk); }
        }
      }
      std::sort(tmp.begin(), tmp.end());
      nbr.insert(nbr.end(), tmp.begin(), tmp.end());
      nbr_ptr[r + 1] = (int32_t)nbr.size();
      c->max_deg = std::max<int>(c->max_deg, (int)tmp.size());
    }
  }
  c->emap16 = c->max_deg > 255 ? 1 : 0;
  if (c->max_deg > 65535) throw Err{IFEM_ERR_CAPACITY, "node degree above 65535"};
  // element -> position maps
  {
    const size_t ne = (size_t)c->nel * nen * nen;
    std::vector<uint8_t> em8;
    std::vector<uint16_t> em16;
    if (c->emap16) em16.resize(ne); else em8.resize(ne);
    for (int64_t e = 0; e < c->nel; ++e)
      for (int a1 = 0; a1 < nen; ++a1) {
        const int32_t r1 = rank[conn[e * nen + a1]];
        const int32_t* b = nbr.data() + nbr_ptr[r1];
        const int32_t* en = nbr.data() + nbr_ptr[r1 + 1];
        for (int a2 = 0; a2 < nen; ++a2) {
          const int32_t r2 = rank[conn[e * nen + a2]];
          const int pos = (int)(std::lower_bound(b, en, r2) - b);
          const size_t i = ((size_t)e * nen + a1) * nen + a2;
          if (c->emap16) em16[i] = (uint16_t)pos; else em8[i] = (uint8_t)pos;
        }
      }
    c->emap = c->emap16 ? (void*)dupload(em16) : (void*)dupload(em8);
    // the same rows in incidence order (node by node, ascending element), padded to 32 entries, for the
    // gather's bulk copies
    const size_t ninc = inc_el.size();
    std::vector<uint8_t> ie8;
    std::vector<uint16_t> ie16;
    if (c->emap16) ie16.assign(ninc * 32, 0); else ie8.assign(ninc * 32, 0);
    for (size_t k = 0; k < ninc; ++k)
      for (int a2 = 0; a2 < nen; ++a2) {
        const size_t i = ((size_t)inc_el[k] * nen + inc_loc[k]) * nen + a2;
        if (c->emap16) ie16[k * 32 + a2] = em16[i]; else ie8[k * 32 + a2] = em8[i];
      }
    c->inc_em = c->emap16 ? (void*)dupload(ie16) : (void*)dupload(ie8);
    for (int64_t r = 0; r < cnt; ++r) c->max_inc = std::max<int>(c->max_inc, inc_ptr[r + 1] - inc_ptr[r]);
  }
  // per-step CSR pattern
  for (int s = 0; s < c->nsteps; ++s) {
    StepDev& sd = c->steps[s];
    std::vector<int> comps;
    if (s == c->step_u) {
      sd.kind = 0; comps = {IFEM_DOF_UX, IFEM_DOF_UY};
      if (dim == 3) comps.push_back(IFEM_DOF_UZ);
      if (c->coss && dim == 3) { comps.push_back(IFEM_DOF_OX); comps.push_back(IFEM_DOF_OY); }
      if (c->coss) comps.push_back(IFEM_DOF_OZ);   // ux, uy, oz (2D); ux, uy, uz, ox, oy, oz (3D)
    }
    else if (s == c->step_ph) {
      sd.kind = 1;
      comps = {IFEM_DOF_PHASE};
      if (c->nlag >= 1) comps.push_back(IFEM_DOF_LMULT);
      if (c->nlag == 2) comps.push_back(IFEM_DOF_LMULT2);
    }
    else if (c->hasT && s == c->step_T) { sd.kind = 2; comps = {IFEM_DOF_T}; }
    sd.nc = (int)comps.size();
    for (int b = 0; b < sd.nc; ++b) { sd.comp_kind[b] = comps[b]; sd.row_base[b] = c->kind_base[comps[b]]; }
    for (int b = 0; b < sd.nc; ++b) {
      int pos = 0;
      for (int b2 = 0; b2 < sd.nc; ++b2) if (sd.row_base[b2] < sd.row_base[b]) ++pos;
      sd.blk_pos[b] = pos;
    }
    const bool hasK = (sd.kind == 0 || sd.kind == 1 || (sd.kind == 2 && opts->thermal_model));
    std::vector<int64_t> rowptr(sd.ndofs + 1, 0);
    if (hasK) {
      // rows in dof order: kinds sorted by base
      std::vector<int> order(sd.nc);
      for (int b = 0; b < sd.nc; ++b) order[sd.blk_pos[b]] = b;
      int64_t row = 0;
      for (int ob = 0; ob < sd.nc; ++ob)
        for (int64_t r = 0; r < cnt; ++r, ++row) rowptr[row + 1] = rowptr[row] + (int64_t)sd.nc * (nbr_ptr[r + 1] - nbr_ptr[r]);
      sd.nnz = rowptr[sd.ndofs];
      if (sd.nnz > INT32_MAX) throw Err{IFEM_ERR_CAPACITY, "more than 2^31 nonzeros (PetscInt is 32-bit)"};
      std::vector<int32_t> col(sd.nnz);
      row = 0;
      for (int ob = 0; ob < sd.nc; ++ob)
        for (int64_t r = 0; r < cnt; ++r, ++row) {
          int64_t o = rowptr[row];
          for (int cb = 0; cb < sd.nc; ++cb) {
            const int32_t base = sd.row_base[order[cb]];
            for (int k = nbr_ptr[r]; k < nbr_ptr[r + 1]; ++k) col[o++] = base + nbr[k];
          }
        }
      sd.colidx = dupload(col);
    }
    sd.rowptr = dupload(rowptr);
    for (int k = 0; k < 4; ++k) { sd.state[k] = dalloc<double>(sd.ndofs); CK(cudaMemset(sd.state[k], 0, sd.ndofs * sizeof(double))); }
    sd.f = dalloc<double>(sd.ndofs);
    CK(cudaMemset(sd.f, 0, sd.ndofs * sizeof(double)));
    sd.vals = dalloc<double>(sd.nnz);
    CK(cudaMemset(sd.vals, 0, std::max<int64_t>(1, sd.nnz) * sizeof(double)));
    sd.stats_d = dalloc<unsigned long long>(kStatWords);
    sd.lcrack_d = dalloc<double>(1);
  }
  // device mesh and maps
  c->X = dupload(std::vector<double>(mesh->coords, mesh->coords + (size_t)c->nn * dim));
  if (dim == 3 && mesh->node_weights) {
    // B-spline meshes carry unit weights: skip them (identical results, less traffic)
    bool ones = true;
    for (int64_t i = 0; i < c->nn && ones; ++i) ones = mesh->node_weights[i] == 1.0;
    if (!ones) c->W = dupload(std::vector<double>(mesh->node_weights, mesh->node_weights + c->nn));
  }
  c->conn = dupload(conn);
  c->ext = dupload(ext);
  if (!c->emat_h.empty()) c->emat = dupload(c->emat_h);
  c->mats_d = dupload(c->mats_h);
  c->node_rank = dupload(rank);
  c->nbr_ptr = dupload(nbr_ptr);
  c->inc_ptr = dupload(inc_ptr);
  c->inc_el = dupload(inc_el);
  c->inc_loc = dupload(inc_loc);
  // history (zero, PhaseField.cpp:58-93)
  const size_t nh = (size_t)c->nh;
  auto z = [&](size_t n) { double* p = dalloc<double>(n); CK(cudaMemset(p, 0, std::max<size_t>(1, n) * sizeof(double))); return p; };
  c->h.EP = z(c->ncs * nh); c->h.EPo = z(c->ncs * nh);
  c->h.EH = z(nh); c->h.EHo = z(nh); c->h.VD = z(nh); c->h.VDo = z(nh);
  c->h.DVD = z(nh); c->h.DVDo = z(nh); c->h.MH = z(c->mh * nh); c->h.MHo = z(c->mh * nh);
  // element scratch
  c->Fe = z((size_t)c->nel * (c->coss ? 3 * (dim - 1) : dim) * nen);   // Cosserat: ux uy oz (2D)
  c->Fe2 = z((size_t)c->nel * nen);
  c->WLe = z((size_t)c->nel * nen);
  c->lc_el = z((size_t)c->nel);
  CK(cudaDeviceSynchronize());
}

static void ensure_scratch(ifem_ctx* c, bool f32) {
  const size_t es = f32 ? 4 : 8;
  const size_t cq = 36 * (size_t)c->nh * es;
  const int ncu = c->coss ? 3 * (c->dim - 1) : c->dim;   // u-step components per node
  const size_t ke = (size_t)c->nel * (size_t)c->nen * (size_t)ke_block(ncu, c->nen) * es;
  if (cq > c->Cq_bytes) { if (c->Cq) cudaFree(c->Cq); c->Cq = dalloc<unsigned char>(cq); c->Cq_bytes = cq; }
  if (ke > c->Ke_bytes) { if (c->Ke) cudaFree(c->Ke); c->Ke = dalloc<unsigned char>(ke); c->Ke_bytes = ke; }
  if (c->coss) {   // Cosserat u-step ip outputs, phase-step energies
    if (!c->Sc) c->Sc = dalloc<double>((size_t)c->nh * 18);
    if (!c->Cc) c->Cc = dalloc<double>((size_t)c->nh * 324);
    if (!c->Ec) c->Ec = dalloc<double>((size_t)c->nh);
    if (!c->V2c) c->V2c = dalloc<double>((size_t)c->nh);
  }
  if (c->nlag > 0) {   // phase element systems with multipliers
    const int nc = 1 + c->nlag;
    const size_t ke2 = (size_t)c->nel * (size_t)c->nen * (size_t)ke_block(nc, c->nen) * es;
    if (ke2 > c->Ke2_bytes) { if (c->Ke2) cudaFree(c->Ke2); c->Ke2 = dalloc<unsigned char>(ke2); c->Ke2_bytes = ke2; }
    if (!c->WLp) c->WLp = dalloc<double>((size_t)c->nel * c->nen);
    if (!c->Fl) c->Fl = dalloc<double>((size_t)c->nel * c->nen * nc);
  }
}

static Geo geo_of(const ifem_ctx* c) {
  Geo g;
  g.dim = c->dim; g.nen = c->nen; g.nip = c->nip; g.kron = c->kron;
  g.nel = c->nel; g.nn = c->nn;
  g.X = c->X; g.W = c->W; g.conn = c->conn; g.ext = c->ext; g.emat = c->emat; g.mats = c->mats_d;
  g.el0 = 0; g.el1 = c->nel;
  return g;
}

static DofMap dm_of(const ifem_ctx* c) {
  DofMap d;
  d.node_rank = c->node_rank;
  for (int k = 0; k < IFEM_N_DOF_KINDS; ++k) { d.base[k] = c->kind_base[k]; d.step[k] = c->kind_step[k]; }
  return d;
}

static StepState ss_of(const ifem_ctx* c, int step) {
  StepState s{nullptr, nullptr, nullptr, nullptr};
  if (step < 0) return s;
  const StepDev& sd = c->steps[step];
  s.cur = sd.state[0]; s.old = sd.state[1]; s.d = sd.state[2]; s.dd = sd.state[3];
  return s;
}

static GParams gather_params(ifem_ctx* c, StepDev& sd) {
  GParams g{};
  g.nc = sd.nc; g.nen = c->nen; g.n_nodes = c->n_unique;
  g.nbr_ptr = c->nbr_ptr; g.inc_ptr = c->inc_ptr; g.inc_el = c->inc_el; g.inc_loc = c->inc_loc;
  g.emap = c->emap; g.emap16 = c->emap16;
  g.rowptr = sd.rowptr;
  for (int b = 0; b < 6; ++b) { g.row_base[b] = sd.row_base[b]; g.blk_pos[b] = sd.blk_pos[b]; }
  g.f = sd.f;
  g.vals = sd.vals;
  g.inc_em = c->inc_em; g.max_inc = c->max_inc; g.max_deg = c->max_deg; g.err = sd.stats_d + 4;
  g.acc_stride = sd.nc * sd.nc * c->max_deg;
  if (sd.nc > 3) g.acc_stride = sd.nc * c->max_deg;   // the row-split gather holds one component row per warp
  if (g.acc_stride < 1) g.acc_stride = 1;
  if ((size_t)g.acc_stride * 8 * 8 > 200 * 1024) throw Err{IFEM_ERR_CAPACITY, "node degree too large for the gather"};
  return g;
}

static CossParams coss_params(ifem_ctx* c, const ifem_time& tm) {
  CossParams cp{};
  cp.geo = geo_of(c); cp.rule = c->rule; cp.dm = dm_of(c); cp.mo = c->mo; cp.h = c->h;
  cp.su = ss_of(c, c->step_u); cp.sp = ss_of(c, c->step_ph); cp.sT = ss_of(c, c->step_T);
  cp.t = tm.t; cp.dt = tm.dt; cp.du_dt = tm.du_dt; cp.ddu_dt = tm.ddu_dt;
  cp.Sc = c->Sc; cp.Cc = c->Cc; cp.Ec = c->Ec; cp.V2c = c->V2c; cp.mh = c->mh;
  return cp;
}

static FaceParams face_params(ifem_ctx* c, StepDev& sd) {
  FaceParams fp{};
  fp.dim = c->dim; fp.nfn = c->dim == 2 ? 3 : 9;
  fp.nside = c->tri_nside; fp.ntop = c->tri_ntop;
  fp.rule = c->rule; fp.X = c->X; fp.W = c->W;
  fp.faces = c->tri_faces; fp.C = c->tri_C; fp.dm = dm_of(c);
  fp.ucur = c->steps[c->step_u].state[0];
  fp.phase = (c->tri_prm.damaged_forces && c->step_ph >= 0) ? c->steps[c->step_ph].state[0] : nullptr;
  fp.p0 = c->tri_st.p0; fp.du = c->tri_prm.du; fp.u0 = c->tri_st.u0; fp.penalty = c->tri_prm.penalty;
  fp.F = c->tri_F; fp.K = c->tri_K; fp.sums = c->tri_sums;
  fp.nnodes = c->tri_nnodes; fp.node = c->tri_node; fp.inc_ptr = c->tri_inc_ptr; fp.inc = c->tri_inc;
  fp.kpos = c->tri_kpos; fp.rowptr = sd.rowptr; fp.colidx = sd.colidx;
  fp.f = sd.f; fp.vals = sd.vals; fp.vals_f32 = sd.vals_f32;
  fp.err = sd.stats_d + 4;
  return fp;
}

// Physics::Assemble(step) for this context's models (physics.cpp:255-304)
static void assemble_async(ifem_ctx* c, int step, const ifem_time& tm) {
  if (step < 0 || step >= c->nsteps) throw Err{IFEM_ERR_INVALID, "step"};
  if (!(tm.dt > 0) && step == c->step_ph) throw Err{IFEM_ERR_INVALID, "dt must be positive"};
  if (!(tm.dt > 0) && c->coss && step == c->step_u) throw Err{IFEM_ERR_INVALID, "dt must be positive"};
  StepDev& sd = c->steps[step];
  const bool f32 = c->opt.tangent_precision != IFEM_PREC_FP64;
  ensure_scratch(c, f32);
  CK(cudaMemsetAsync(sd.stats_d, 0, kStatWords * sizeof(unsigned long long), c->stream));
  if (!c->capturing) CK(cudaEventRecord(c->ev[0], c->stream));
  const Geo geo = geo_of(c);
  const DofMap dm = dm_of(c);
  GParams gp = gather_params(c, sd);
  sd.vals_f32 = f32 ? 1 : 0;
  gp.vals_f32 = sd.vals_f32;
  if (sd.kind == 0 && c->coss) {   // CossPhaseField::Assemble_U
    CossParams cp = coss_params(c, tm);
    cp.Fe = c->Fe; cp.Ke = c->Ke; cp.ke_f32 = f32 ? 1 : 0; cp.stats = sd.stats_d;
    launch_coss_u(cp, c->stream);
    if (!c->capturing) CK(cudaEventRecord(c->ev[1], c->stream));
    gp.Ke = c->Ke; gp.ke_f32 = f32 ? 1 : 0; gp.Fe1 = c->Fe; gp.Fe2 = nullptr;
    launch_gather(gp, c->stream);
    sd.slabbed = false;
    if (c->tri_on) {
      if (c->tri_st.t_break > 0.0) c->tri_st.p0 = 0.0;
      FaceParams fp = face_params(c, sd);
      fp.t = tm.t + tm.dt;
      launch_face_loads(fp, c->stream);
      for (int k = 0; k < 3; ++k) launch_reduce_sum(c->tri_sums + k * c->tri_ntop, c->tri_ntop, c->tri_tot + k, c->stream);
      launch_face_gather(fp, c->stream);
      c->tri_assembled = true;
    }
  } else if (sd.kind == 0) {
    UParams p{};
    p.geo = geo; p.rule = c->rule; p.dm = dm; p.mo = c->mo; p.h = c->h;
    p.su = ss_of(c, c->step_u); p.sp = ss_of(c, c->step_ph); p.sT = ss_of(c, c->step_T);
    p.dt = tm.dt; p.du_dt = tm.du_dt; p.ddu_dt = tm.ddu_dt;
    p.Fe = c->Fe; p.WLe = c->WLe; p.Cq = c->Cq; p.cq_f32 = f32 ? 1 : 0; p.stats = sd.stats_d;
    p.vep = c->general ? 1 : 0;
    p.spec = (c->spec && !c->capturing) ? 1 : 0;   // a graph keeps the run-time selection (ifem_set_param)
    // the tensor-core tangent takes its inputs from the sum-factorised points kernel, which has neither the VEP
    // branch nor the SpecStrains / DruckerPrager splits
    const bool tc = c->opt.tangent_precision == IFEM_PREC_TC_SPLIT && c->dim == 3 && c->kron && !c->general;
    if (tc && !c->geoq) c->geoq = dalloc<float>((size_t)kTcGeo * c->nel);
    if (tc && !c->Kd) c->Kd = dalloc<double>((size_t)kTcKd * c->nel);
    if (tc && !c->nxq) c->nxq = dalloc<float>((size_t)kTcNx * c->nel);
    p.geoq = tc ? c->geoq : nullptr;
    p.Kd = tc ? c->Kd : nullptr;
    p.nxq = tc ? c->nxq : nullptr;
    TParams t{};
    t.geo = geo; t.rule = c->rule; t.mo = c->mo; t.Cq = c->Cq; t.nh = c->nh; t.WLe = c->WLe;
    t.phase_cur = c->steps[c->step_ph].state[0]; t.dm = dm; t.du_dt = tm.du_dt; t.ddu_dt = tm.ddu_dt; t.Ke = c->Ke;
    t.geoq = c->geoq;
    t.Kd = c->Kd;
    t.nxq = c->nxq;
    gp.Ke = c->Ke; gp.ke_f32 = f32 ? 1 : 0; gp.Fe1 = c->Fe; gp.Fe2 = nullptr;
    if (c->opt.ocean_bc) {   // OceanBC after the phase-field model: the gather's second residual source
      if (!c->Fo) c->Fo = dalloc<double>((size_t)c->nel * 2 * c->nen);
      OceanParams op{};
      op.geo = geo; op.rule = c->rule; op.dm = dm; op.phase_cur = c->steps[c->step_ph].state[0];
      op.hw = c->opt.ocean_hw; op.density = c->opt.ocean_density; op.Fo = c->Fo;
      launch_ocean_u(op, c->stream);
      gp.Fe2 = c->Fo;
    }
    // one pass over all elements, or (outside graph capture) slabs whose rows the read-back copies as each
    // slab finishes; every launch sees the same data, so the results are identical either way
    const int ns = (c->capturing || c->tri_on) ? 1 : c->slabs;
    for (int k = 0; k < ns; ++k) {
      if (ns > 1) {
        p.geo.el0 = t.geo.el0 = c->slab_el[k];
        p.geo.el1 = t.geo.el1 = c->slab_el[k + 1];
        gp.node0 = c->slab_node[k];
        gp.n_nodes = c->slab_node[k + 1];
      }
      launch_u_points(p, c->stream);
      if (!c->capturing && ns == 1) CK(cudaEventRecord(c->ev[3], c->stream));
      if (tc)
        launch_u_tangent_tc(t, sd.stats_d + 3, c->n_sm, c->stream);
      else
        launch_u_tangent(t, f32 ? 1 : 0, c->stream);
      if (!c->capturing && k == ns - 1) CK(cudaEventRecord(c->ev[1], c->stream));
      launch_gather(gp, c->stream);
      if (ns > 1) CK(cudaEventRecord(c->slab_ev[k], c->stream));
    }
    sd.slabbed = ns > 1;
    if (c->tri_on) {   // TriAxial after the phase-field model (the order of the Models list)
      if (c->tri_st.t_break > 0.0) c->tri_st.p0 = 0.0;   // TriAxial.cpp:140-142
      FaceParams fp = face_params(c, sd);
      fp.t = tm.t + tm.dt;
      launch_face_loads(fp, c->stream);
      for (int k = 0; k < 3; ++k) launch_reduce_sum(c->tri_sums + k * c->tri_ntop, c->tri_ntop, c->tri_tot + k, c->stream);
      launch_face_gather(fp, c->stream);
      c->tri_assembled = true;
    }
  } else if (sd.kind == 1) {
    PParams p{};
    p.geo = geo; p.rule = c->rule; p.dm = dm; p.mo = c->mo; p.h = c->h;
    p.su = ss_of(c, c->step_u); p.sp = ss_of(c, c->step_ph); p.sT = ss_of(c, c->step_T);
    p.dt = tm.dt; p.Fe = c->Fe; p.Ke = c->Ke; p.ke_f32 = f32 ? 1 : 0; p.write_hist = 1;
    p.lcrack_el = c->lc_el; p.stats = sd.stats_d;
    p.general = c->ph_general ? 1 : 0;
    p.spec = (c->spec && !c->capturing) ? 1 : 0;
    p.wl_out = c->nlag ? c->WLp : nullptr;
    if (c->coss) {   // the Cosserat split's driving energy (CossPhaseField.cpp:670-701)
      CossParams cp = coss_params(c, tm);
      launch_coss_energy(cp, c->stream);
      p.e_in = c->Ec; p.v2_in = c->V2c;
    }
    launch_phase(p, c->stream);
    launch_reduce_sum(c->lc_el, c->nel, sd.lcrack_d, c->stream);
    gp.Ke = c->Ke; gp.ke_f32 = f32 ? 1 : 0; gp.Fe1 = c->Fe; gp.Fe2 = nullptr;
    if (c->nlag) {
      LagParams lp{};
      lp.geo = geo; lp.dm = dm; lp.mo = c->mo;
      lp.phase_cur = sd.state[0]; lp.phase_old = sd.state[1];
      lp.nlag = c->nlag; lp.Ke1 = c->Ke; lp.Fe1 = c->Fe; lp.WL = c->WLp;
      lp.Ke = c->Ke2; lp.Fe = c->Fl; lp.ke_f32 = f32 ? 1 : 0;
      launch_phase_lagrange(lp, c->stream);
      gp.Ke = c->Ke2; gp.Fe1 = c->Fl;
    }
    if (!c->capturing) CK(cudaEventRecord(c->ev[1], c->stream));
    launch_gather(gp, c->stream);
  } else if (sd.kind == 2) {
    const bool vh = c->opt.viscous_heating != 0, th = c->opt.thermal_model != 0;
    if (vh || th) {
      ThParams p{};
      p.geo = geo; p.rule = c->rule; p.dm = dm; p.h = c->h; p.sT = ss_of(c, step);
      p.dt = tm.dt; p.du_dt = tm.du_dt; p.visc_heat = vh; p.thermal = th;
      p.Fvh = c->Fe2; p.Fth = c->Fe; p.Ke = c->Ke; p.ke_f32 = f32 ? 1 : 0; p.stats = sd.stats_d;
      launch_thermal(p, c->stream);
    }
    if (!c->capturing) CK(cudaEventRecord(c->ev[1], c->stream));
    if (vh || th) {
      gp.Ke = th ? c->Ke : nullptr; gp.ke_f32 = f32 ? 1 : 0;
      gp.Fe1 = vh ? c->Fe2 : c->Fe;
      gp.Fe2 = (vh && th) ? c->Fe : nullptr;
      launch_gather(gp, c->stream);
    } else {
      CK(cudaMemsetAsync(sd.f, 0, sd.ndofs * sizeof(double), c->stream));
    }
  } else {
    if (!c->capturing) CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaMemsetAsync(sd.f, 0, std::max<int64_t>(1, sd.ndofs) * sizeof(double), c->stream));
  }
  if (!c->capturing) {
    CK(cudaEventRecord(c->ev[2], c->stream));
    CK(cudaEventRecord(c->done_ev[step], c->stream));
  }
  CK(cudaGetLastError());
  sd.assembled = true;
}

static void finish(ifem_ctx* c, int step) {
  StepDev& sd = c->steps[step];
  CK(cudaStreamSynchronize(c->stream));
  unsigned long long st[kStatWords];
  CK(cudaMemcpy(st, sd.stats_d, sizeof(st), cudaMemcpyDeviceToHost));
  float ms_e = 0, ms_s = 0, ms_p = 0, ms_t = 0;
  cudaEventElapsedTime(&ms_e, c->ev[0], c->ev[1]);
  cudaEventElapsedTime(&ms_s, c->ev[1], c->ev[2]);
  if (sd.kind == 0 && !sd.slabbed) {   // the points / tangent split is timed when the step runs as one pass
    cudaEventElapsedTime(&ms_p, c->ev[0], c->ev[3]);
    cudaEventElapsedTime(&ms_t, c->ev[3], c->ev[1]);
  }
  (void)cudaGetLastError();   // events not recorded (graph replays) only leave a non-sticky error here
  sd.stats.ms_element = ms_e; sd.stats.ms_scatter = ms_s; sd.stats.ms_total = ms_e + ms_s;
  sd.stats.ms_points = ms_p; sd.stats.ms_tangent = ms_t;
  sd.stats.rm_iterations = (int64_t)st[0];
  sd.stats.rm_capped = (int64_t)st[1];
  sd.stats.nonfinite = (int64_t)st[2];
  if (sd.kind == 1) CK(cudaMemcpy(&sd.stats.crack_length, sd.lcrack_d, sizeof(double), cudaMemcpyDeviceToHost));
  if (st[3]) throw Err{IFEM_ERR_CUDA, "tensor-core tangent: MMA completion wait timed out"};
  if (st[4]) throw Err{IFEM_ERR_CUDA, "gather: bulk-copy completion wait timed out"};
  if (sd.stats.nonfinite) throw Err{IFEM_ERR_NUMERIC, "non-finite values in the element residuals"};
}

template <class F>
static int guarded(ifem_ctx* c, F&& fn) {
  try {
    if (c) cudaSetDevice(c->device);
    fn();
    return IFEM_OK;
  } catch (const Err& e) {
    if (c) c->err = e.msg; else g_create_err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    if (c) c->err = e.what(); else g_create_err = e.what();
    return IFEM_ERR_INVALID;
  }
}

static double* hist_field(ifem_ctx* c, int field, int old, size_t& n) {
  n = (size_t)c->nh;
  switch (field) {
    case IFEM_HIST_ENERGY: return old ? c->h.EHo : c->h.EH;
    case IFEM_HIST_PLASTIC_STRAIN: n = (size_t)c->ncs * c->nh; return old ? c->h.EPo : c->h.EP;
    case IFEM_HIST_VISC_DISS: return old ? c->h.VDo : c->h.VD;
    case IFEM_HIST_DAM_VISC_DISS: return old ? c->h.DVDo : c->h.DVD;
    case IFEM_HIST_MAT: n = (size_t)c->mh * c->nh; return old ? c->h.MHo : c->h.MH;
  }
  throw Err{IFEM_ERR_INVALID, "history field"};
}

}  // namespace ifem

// ==========================================================================================
// C-ABI
// ==========================================================================================
extern "C" {

int ifem_abi_version(void) { return IFEM_ABI_VERSION; }

int ifem_ctx_create(const ifem_mesh_desc* mesh, const ifem_material* mats, int32_t n_mats, const ifem_options* opts,
                    int32_t device, ifem_ctx** out) {
  if (!out) return IFEM_ERR_INVALID;
  *out = nullptr;
  ifem_ctx* c = new ifem_ctx();
  const int rc = guarded(nullptr, [&] { create(c, mesh, mats, n_mats, opts, device); });
  if (rc != IFEM_OK) { destroy(c); return rc; }
  *out = c;
  return IFEM_OK;
}

int ifem_ctx_destroy(ifem_ctx* ctx) {
  if (!ctx) return IFEM_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  destroy(ctx);
  return IFEM_OK;
}

int ifem_last_error(const ifem_ctx* ctx, char* buf, size_t len) {
  const std::string& m = ctx ? ctx->err : g_create_err;
  if (buf && len) { std::strncpy(buf, m.c_str(), len - 1); buf[len - 1] = 0; }
  return IFEM_OK;
}

int ifem_step_info(const ifem_ctx* ctx, int32_t step, int64_t* n_dofs, int64_t* nnz) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  if (n_dofs) *n_dofs = ctx->steps[step].ndofs;
  if (nnz) *nnz = ctx->steps[step].nnz;
  return IFEM_OK;
}

int ifem_get_dof_numbers(const ifem_ctx* ctx, int32_t kind, int64_t* out) {
  if (!ctx || kind < 0 || kind >= IFEM_N_DOF_KINDS || !out) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    std::vector<int32_t> rank(c->nn);
    CK(cudaMemcpy(rank.data(), c->node_rank, c->nn * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (int64_t n = 0; n < c->nn; ++n)
      out[n] = (c->kind_base[kind] < 0 || rank[n] < 0) ? -1 : (int64_t)c->kind_base[kind] + rank[n];
  });
}

int ifem_build_pattern(const ifem_ctx* ctx, int32_t step, int32_t* row_ptr, int32_t* col_idx) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    const StepDev& sd = c->steps[step];
    if (row_ptr) {
      std::vector<int64_t> rp(sd.ndofs + 1);
      CK(cudaMemcpy(rp.data(), sd.rowptr, rp.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < rp.size(); ++i) row_ptr[i] = (int32_t)rp[i];
    }
    if (col_idx && sd.nnz) CK(cudaMemcpy(col_idx, sd.colidx, sd.nnz * sizeof(int32_t), cudaMemcpyDefault));
  });
}

int ifem_set_state(ifem_ctx* ctx, int32_t step, int32_t kind, const double* src, int64_t n) {
  if (!ctx || step < 0 || step >= ctx->nsteps || kind < 0 || kind > 3 || !src) return IFEM_ERR_INVALID;
  if (n != ctx->steps[step].ndofs) { ctx->err = "state size mismatch"; return IFEM_ERR_INVALID; }
  return guarded(ctx, [&] {
    CK(cudaMemcpyAsync(ctx->steps[step].state[kind], src, n * sizeof(double), cudaMemcpyDefault, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  });
}

int ifem_get_state(const ifem_ctx* ctx, int32_t step, int32_t kind, double* dst, int64_t n) {
  if (!ctx || step < 0 || step >= ctx->nsteps || kind < 0 || kind > 3 || !dst) return IFEM_ERR_INVALID;
  if (n != ctx->steps[step].ndofs) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    CK(cudaMemcpyAsync(dst, c->steps[step].state[kind], n * sizeof(double), cudaMemcpyDefault, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int ifem_assemble(ifem_ctx* ctx, int32_t step, const ifem_time* tm) {
  if (!ctx || !tm) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] { assemble_async(ctx, step, *tm); finish(ctx, step); });
}

int ifem_assemble_async(ifem_ctx* ctx, int32_t step, const ifem_time* tm) {
  if (!ctx || !tm) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] { assemble_async(ctx, step, *tm); });
}

int ifem_sync(ifem_ctx* ctx, int32_t step) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] { finish(ctx, step); });
}

int ifem_get_stream(const ifem_ctx* ctx, void** stream) {
  if (!ctx || !stream) return IFEM_ERR_INVALID;
  *stream = (void*)ctx->stream;
  return IFEM_OK;
}

int ifem_get_residual(const ifem_ctx* ctx, int32_t step, double* dst, int64_t n) {
  if (!ctx || step < 0 || step >= ctx->nsteps || !dst) return IFEM_ERR_INVALID;
  if (n != ctx->steps[step].ndofs) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    const StepDev& sd = c->steps[step];
    if (sd.slabbed) {
      // each slab's rows of every component block as soon as the slab's gather is done
      for (int k = 0; k < c->slabs; ++k) {
        CK(cudaStreamWaitEvent(c->cstream, c->slab_ev[k], 0));
        const int64_t r0 = c->slab_node[k], r1 = c->slab_node[k + 1];
        for (int b = 0; b < sd.nc && r1 > r0; ++b)
          CK(cudaMemcpyAsync(dst + sd.row_base[b] + r0, sd.f + sd.row_base[b] + r0, (r1 - r0) * sizeof(double),
                             cudaMemcpyDefault, c->cstream));
      }
    } else {
      CK(cudaStreamWaitEvent(c->cstream, c->done_ev[step], 0));
      CK(cudaMemcpyAsync(dst, sd.f, n * sizeof(double), cudaMemcpyDefault, c->cstream));
    }
    CK(cudaStreamSynchronize(c->cstream));
  });
}

int ifem_get_matrix(const ifem_ctx* ctx, int32_t step, void* dst, int64_t nnz, int32_t dtype) {
  if (!ctx || step < 0 || step >= ctx->nsteps || !dst) return IFEM_ERR_INVALID;
  if (nnz != ctx->steps[step].nnz || (dtype != IFEM_F64 && dtype != IFEM_F32)) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    const StepDev& sd = c->steps[step];
    if (nnz == 0) return;
    const int src32 = sd.vals_f32;
    if ((dtype == IFEM_F32) == (src32 == 1) && sd.slabbed) {
      const size_t es = src32 ? 4 : 8;
      for (int k = 0; k < c->slabs; ++k) {
        CK(cudaStreamWaitEvent(c->cstream, c->slab_ev[k], 0));
        for (int b = 0; b < sd.nc; ++b) {
          const int64_t o0 = c->slab_off[k * 3 + b], o1 = c->slab_off[(k + 1) * 3 + b];
          if (o1 > o0)
            CK(cudaMemcpyAsync((char*)dst + o0 * es, (const char*)sd.vals + o0 * es, (o1 - o0) * es,
                               cudaMemcpyDefault, c->cstream));
        }
      }
      CK(cudaStreamSynchronize(c->cstream));
      return;
    }
    CK(cudaStreamWaitEvent(c->cstream, c->done_ev[step], 0));
    if ((dtype == IFEM_F32) == (src32 == 1)) {
      CK(cudaMemcpyAsync(dst, sd.vals, nnz * (src32 ? 4 : 8), cudaMemcpyDefault, c->cstream));
      CK(cudaStreamSynchronize(c->cstream));
      return;
    }
    if (src32) {
      std::vector<float> tmp(nnz);
      CK(cudaMemcpyAsync(tmp.data(), sd.vals, nnz * 4, cudaMemcpyDeviceToHost, c->cstream));
      CK(cudaStreamSynchronize(c->cstream));
      std::vector<double> out(tmp.begin(), tmp.end());
      CK(cudaMemcpy(dst, out.data(), nnz * 8, cudaMemcpyDefault));
    } else {
      std::vector<double> tmp(nnz);
      CK(cudaMemcpyAsync(tmp.data(), sd.vals, nnz * 8, cudaMemcpyDeviceToHost, c->cstream));
      CK(cudaStreamSynchronize(c->cstream));
      std::vector<float> out(nnz);
      for (int64_t i = 0; i < nnz; ++i) out[i] = (float)tmp[i];
      CK(cudaMemcpy(dst, out.data(), nnz * 4, cudaMemcpyDefault));
    }
  });
}

int ifem_device_outputs(const ifem_ctx* ctx, int32_t step, const double** f_dev, const void** vals_dev,
                        int32_t* dtype_out) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  const StepDev& sd = ctx->steps[step];
  if (f_dev) *f_dev = sd.f;
  if (vals_dev) *vals_dev = sd.vals;
  if (dtype_out) *dtype_out = sd.vals_f32 ? IFEM_F32 : IFEM_F64;
  return IFEM_OK;
}

int ifem_commit(ifem_ctx* ctx, int32_t commit_type) {
  if (!ctx) return IFEM_ERR_INVALID;
  if (commit_type != IFEM_COMMIT_TIMEDEP) return IFEM_OK;  // PATHDEP: nothing (PhaseField.cpp:124)
  return guarded(ctx, [&] {
    const size_t nh = (size_t)ctx->nh * sizeof(double);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->h.EHo, ctx->h.EH, nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.EPo, ctx->h.EP, ctx->ncs * nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.VDo, ctx->h.VD, nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.DVDo, ctx->h.DVD, nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.MHo, ctx->h.MH, ctx->mh * nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
  });
}

int ifem_reset_step(ifem_ctx* ctx) {
  if (!ctx) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    const size_t nh = (size_t)ctx->nh * sizeof(double);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->h.EH, ctx->h.EHo, nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.EP, ctx->h.EPo, ctx->ncs * nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.VD, ctx->h.VDo, nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.DVD, ctx->h.DVDo, nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->h.MH, ctx->h.MHo, ctx->mh * nh, cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
  });
}

// Plastic strain crosses the ABI as [nel*nip][6] (Plastic_Strain[el][ip], PhaseField.h:118);
// on the device it is stored component-major for coalesced access.
int ifem_get_history(const ifem_ctx* ctx, int32_t field, int32_t old, double* dst, int64_t n) {
  if (!ctx || !dst) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    size_t m;
    double* src = hist_field(c, field, old, m);
    if ((size_t)n != m) throw Err{IFEM_ERR_INVALID, "history size mismatch"};
    CK(cudaStreamSynchronize(c->stream));
    std::vector<double> tmp(m);
    CK(cudaMemcpy(tmp.data(), src, m * sizeof(double), cudaMemcpyDeviceToHost));
    const int comps = field == IFEM_HIST_PLASTIC_STRAIN ? c->ncs : (field == IFEM_HIST_MAT ? c->mh : 1);
    if (comps > 1) {   // device planes [comps][nh] -> ip-major [nh][comps]
      std::vector<double> t2(m);
      const size_t nh = (size_t)c->nh;
      for (size_t i = 0; i < nh; ++i) for (int r = 0; r < comps; ++r) t2[i * comps + r] = tmp[r * nh + i];
      tmp.swap(t2);
    }
    CK(cudaMemcpy(dst, tmp.data(), m * sizeof(double), cudaMemcpyDefault));
  });
}

int ifem_set_history(ifem_ctx* ctx, int32_t field, int32_t old, const double* src, int64_t n) {
  if (!ctx || !src) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    size_t m;
    double* dst = hist_field(ctx, field, old, m);
    if ((size_t)n != m) throw Err{IFEM_ERR_INVALID, "history size mismatch"};
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<double> tmp(m);
    CK(cudaMemcpy(tmp.data(), src, m * sizeof(double), cudaMemcpyDefault));
    const int comps = field == IFEM_HIST_PLASTIC_STRAIN ? ctx->ncs : (field == IFEM_HIST_MAT ? ctx->mh : 1);
    if (comps > 1) {   // ip-major [nh][comps] -> device planes [comps][nh]
      std::vector<double> t2(m);
      const size_t nh = (size_t)ctx->nh;
      for (size_t i = 0; i < nh; ++i) for (int r = 0; r < comps; ++r) t2[r * nh + i] = tmp[i * comps + r];
      tmp.swap(t2);
    }
    CK(cudaMemcpy(dst, tmp.data(), m * sizeof(double), cudaMemcpyHostToDevice));
  });
}

int ifem_set_tangent(ifem_ctx* ctx, int32_t mode, int32_t prec) {
  if (!ctx || mode < 0 || mode > 1 || prec < 0 || prec > 2) return IFEM_ERR_INVALID;
  ctx->opt.tangent_mode = mode;
  ctx->opt.tangent_precision = prec;
  ctx->mo.tangent_mode = mode;
  return IFEM_OK;
}

int ifem_set_readback_slabs(ifem_ctx* ctx, int32_t n_slabs) {
  if (!ctx || n_slabs < 1 || n_slabs > kMaxSlabs) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    ifem_ctx* c = ctx;
    if (c->step_u < 0) throw Err{IFEM_ERR_STATE, "no displacement step"};
    const StepDev& sd = c->steps[c->step_u];
    if (sd.ndofs != (int64_t)sd.nc * c->n_unique) throw Err{IFEM_ERR_UNSUPPORTED, "slabs need a step of displacement rows only"};
    const int n = (int)std::min<int64_t>(n_slabs, std::max<int64_t>(1, c->nel));
    std::vector<int64_t> el(n + 1), node(n + 1), off((size_t)(n + 1) * 3, 0);
    for (int k = 0; k <= n; ++k) {
      // boundaries at nel (k / n)^2: the first slab is small, so the copy-out starts early, and later slabs,
      // which finish while earlier rows are still being copied, are larger
      el[k] = (int64_t)((double)c->nel * ((double)k * k) / ((double)n * n));
      // node ranks whose incident elements all lie below el[k]: a prefix, as node_last is non-decreasing
      node[k] = k == n ? c->n_unique
                       : std::lower_bound(c->node_last.begin(), c->node_last.end(), (int32_t)el[k]) - c->node_last.begin();
      for (int b = 0; b < sd.nc; ++b)
        CK(cudaMemcpy(&off[(size_t)k * 3 + b], sd.rowptr + sd.row_base[b] + node[k], sizeof(int64_t),
                      cudaMemcpyDeviceToHost));
    }
    CK(cudaStreamSynchronize(c->stream));   // no slab of an earlier assembly is still running
    c->slabs = n;
    c->slab_el.swap(el);
    c->slab_node.swap(node);
    c->slab_off.swap(off);
  });
}

int ifem_get_stats(const ifem_ctx* ctx, int32_t step, ifem_stats* out) {
  if (!ctx || step < 0 || step >= ctx->nsteps || !out) return IFEM_ERR_INVALID;
  *out = ctx->steps[step].stats;
  return IFEM_OK;
}

// ---- constraints ----
static void free_cons(StepDev& sd) {
  auto F = [](void* p) { if (p) cudaFree(p); };
  F(sd.fmap); F(sd.row_src); F(sd.con_dof); F(sd.con_val); F(sd.cv); F(sd.rowptr_con); F(sd.colidx_con);
  F(sd.vals_con); F(sd.f_con); F(sd.dx); F(sd.kw); F(sd.kbinv); F(sd.ktbl);
  amg_free(sd.amg); sd.amg = nullptr;
  sd.kw = nullptr; sd.kw_len = 0; sd.kcon_ready = false; sd.kbinv = nullptr; sd.ktbl = nullptr;
  sd.fmap = nullptr; sd.row_src = nullptr; sd.con_dof = nullptr; sd.con_val = nullptr; sd.cv = nullptr;
  sd.rowptr_con = nullptr; sd.colidx_con = nullptr; sd.vals_con = nullptr; sd.f_con = nullptr; sd.dx = nullptr;
  sd.n_cons = sd.n_free = sd.nnz_con = 0;
  sd.cons_set = sd.cons_built = false;
}

// Constrainer::AddConstraint semantics (std::map: ascending dofs, equal duplicates merged) and the
// reduced numbering/pattern, built on the host once per constraint set (the reference's symbolic PtAP).
static void set_constraints(ifem_ctx* c, int step, int64_t n, const int64_t* dofs, const double* values) {
  StepDev& sd = c->steps[step];
  std::vector<int64_t> dh(n);
  std::vector<double> vh(n);
  if (n) {
    CK(cudaMemcpy(dh.data(), dofs, n * sizeof(int64_t), cudaMemcpyDefault));
    CK(cudaMemcpy(vh.data(), values, n * sizeof(double), cudaMemcpyDefault));
  }
  std::map<int64_t, double> m;
  for (int64_t i = 0; i < n; ++i) {
    if (dh[i] < 0 || dh[i] >= sd.ndofs) throw Err{IFEM_ERR_INVALID, "constrained dof out of range"};
    auto it = m.find(dh[i]);
    if (it != m.end()) {
      if (it->second != vh[i]) throw Err{IFEM_ERR_INVALID, "dof doubly constrained with different values"};
    } else {
      m.insert({dh[i], vh[i]});
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  free_cons(sd);
  const int64_t nd = sd.ndofs;
  std::vector<int32_t> fmap(nd);
  std::vector<int32_t> row_src;
  std::vector<int64_t> cd;
  std::vector<double> cvals;
  row_src.reserve(nd - (int64_t)m.size());
  for (int64_t d = 0; d < nd; ++d) {
    auto it = m.find(d);
    if (it != m.end()) { fmap[d] = -1 - (int32_t)cd.size(); cd.push_back(d); cvals.push_back(it->second); }
    else { fmap[d] = (int32_t)row_src.size(); row_src.push_back((int32_t)d); }
  }
  const int64_t nf = (int64_t)row_src.size();
  std::vector<int64_t> rpc(nf + 1, 0);
  std::vector<int32_t> cic;
  if (sd.nnz) {
    std::vector<int64_t> rp(nd + 1);
    std::vector<int32_t> ci(sd.nnz);
    CK(cudaMemcpy(rp.data(), sd.rowptr, rp.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ci.data(), sd.colidx, ci.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nf; ++i) {
      const int64_t r = row_src[i];
      for (int64_t j = rp[r]; j < rp[r + 1]; ++j)
        if (fmap[ci[j]] >= 0) cic.push_back(fmap[ci[j]]);
      rpc[i + 1] = (int64_t)cic.size();
    }
  }
  sd.n_cons = (int64_t)cd.size(); sd.n_free = nf; sd.nnz_con = (int64_t)cic.size();
  sd.fmap = dupload(fmap);
  sd.row_src = dupload(row_src);
  sd.con_dof = dupload(cd);
  sd.con_val = dupload(cvals);
  sd.cv = dalloc<double>(sd.n_cons);
  CK(cudaMemset(sd.cv, 0, std::max<int64_t>(1, sd.n_cons) * sizeof(double)));
  sd.rowptr_con = dupload(rpc);
  sd.colidx_con = dupload(cic);
  sd.vals_con = dalloc<double>(sd.nnz_con);
  sd.f_con = dalloc<double>(nf);
  sd.dx = dalloc<double>(nf);
  sd.cons_set = true;
}

static void constrain(ifem_ctx* c, int step, bool want_matrix) {
  StepDev& sd = c->steps[step];
  if (!sd.cons_set) throw Err{IFEM_ERR_STATE, "no constraints set for this step"};
  if (!sd.assembled) throw Err{IFEM_ERR_STATE, "constrain before assemble"};
  launch_cons_cv(sd.con_dof, sd.con_val, sd.n_cons, sd.state[0], sd.cv, c->stream);
  ConsParams p{};
  p.n_free = sd.n_free; p.row_src = sd.row_src; p.fmap = sd.fmap;
  p.rowptr = sd.rowptr; p.colidx = sd.colidx;
  p.vals = sd.nnz ? sd.vals : nullptr; p.vals_f32 = sd.vals_f32;
  p.f = sd.f; p.cv = sd.cv; p.rowptr_con = sd.rowptr_con;
  p.vals_con = sd.vals_con; p.want_matrix = (want_matrix && sd.nnz) ? 1 : 0; p.f_con = sd.f_con;
  launch_constrain(p, c->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  if (want_matrix) sd.vals_con_f32 = sd.vals_f32;
  if (want_matrix) sd.kcon_ready = true;
  sd.cons_built = true;
}

// Restarted GMRES(m) with right node-block Jacobi preconditioning on K_con dx = f_con (the inverse of each node's
// block of components; the diagonal where a step's DOFs are not one block per node), all vectors on the
// device; classical Gram-Schmidt applied twice (two reductions per step instead of one per basis vector) and
// Givens rotations on the host.  Stops on the true residual ||f_con - K_con dx|| <= rtol ||f_con||.
// Near-null space of a step's free rows for the multigrid set-up: rigid-body modes of the displacement step
// (translations and rotations about the centroid; in the Cosserat model the micro-rotations follow the rotation,
// oy with the sign ConstructBMatCoss gives it), one constant per component for the other steps.
static void amg_setup(ifem_ctx* c, int step) {
  StepDev& sd = c->steps[step];
  for (int k = 0; k < sd.nc; ++k)
    if (sd.comp_kind[k] == IFEM_DOF_LMULT || sd.comp_kind[k] == IFEM_DOF_LMULT2)
      throw Err{IFEM_ERR_UNSUPPORTED, "multigrid: the step has Lagrange-multiplier DOFs (an indefinite system)"};
  const int64_t n = sd.n_free;
  std::vector<int64_t> rp(n + 1);
  std::vector<int32_t> ci(sd.nnz_con);
  CK(cudaMemcpy(rp.data(), sd.rowptr_con, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ci.data(), sd.colidx_con, sd.nnz_con * sizeof(int32_t), cudaMemcpyDeviceToHost));
  std::vector<double> v(sd.nnz_con);
  if (sd.vals_con_f32) {
    std::vector<float> f(sd.nnz_con);
    CK(cudaMemcpy(f.data(), sd.vals_con, sd.nnz_con * sizeof(float), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < sd.nnz_con; ++i) v[i] = f[i];
  } else {
    CK(cudaMemcpy(v.data(), sd.vals_con, sd.nnz_con * sizeof(double), cudaMemcpyDeviceToHost));
  }
  std::vector<int32_t> src(n);
  CK(cudaMemcpy(src.data(), sd.row_src, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  const int64_t nu = c->n_unique;
  std::vector<int32_t> node(n), comp(n);
  for (int64_t i = 0; i < n; ++i) {
    int b = -1;
    for (int k = 0; k < sd.nc; ++k)
      if (src[i] >= sd.row_base[k] && src[i] < sd.row_base[k] + nu) b = k;
    if (b < 0) throw Err{IFEM_ERR_UNSUPPORTED, "multigrid: the step has rows that are not node rows"};
    comp[i] = b; node[i] = src[i] - sd.row_base[b];
  }
  // node coordinates by rank, centred
  std::vector<int32_t> rank(c->nn);
  CK(cudaMemcpy(rank.data(), c->node_rank, c->nn * sizeof(int32_t), cudaMemcpyDeviceToHost));
  std::vector<double> X((size_t)c->nn * c->dim), xr((size_t)nu * 3, 0.0), ctr(3, 0.0);
  CK(cudaMemcpy(X.data(), c->X, X.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int64_t nd = 0; nd < c->nn; ++nd)
    if (rank[nd] >= 0) for (int d = 0; d < c->dim; ++d) xr[(size_t)rank[nd] * 3 + d] = X[(size_t)nd * c->dim + d];
  for (int64_t r = 0; r < nu; ++r) for (int d = 0; d < 3; ++d) ctr[d] += xr[(size_t)r * 3 + d] / (double)nu;
  const bool disp = sd.kind == 0;
  const int dim = c->dim;
  const int nm = disp ? (dim == 2 ? 3 : 6) : sd.nc;
  std::vector<double> B((size_t)n * nm, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    double* Bi = &B[(size_t)i * nm];
    const int kind = sd.comp_kind[comp[i]];
    if (!disp) { Bi[comp[i]] = 1.0; continue; }
    const double x = xr[(size_t)node[i] * 3] - ctr[0], y = xr[(size_t)node[i] * 3 + 1] - ctr[1],
                 z = xr[(size_t)node[i] * 3 + 2] - ctr[2];
    if (dim == 2) {   // modes: translation x, translation y, rotation about z
      if (kind == IFEM_DOF_UX) { Bi[0] = 1.0; Bi[2] = -y; }
      else if (kind == IFEM_DOF_UY) { Bi[1] = 1.0; Bi[2] = x; }
      else if (kind == IFEM_DOF_OZ) Bi[2] = 1.0;
    } else {          // translations x, y, z; rotations about x, y, z (u = w times x)
      if (kind == IFEM_DOF_UX) { Bi[0] = 1.0; Bi[4] = z; Bi[5] = -y; }
      else if (kind == IFEM_DOF_UY) { Bi[1] = 1.0; Bi[3] = -z; Bi[5] = x; }
      else if (kind == IFEM_DOF_UZ) { Bi[2] = 1.0; Bi[3] = y; Bi[4] = -x; }
      else if (kind == IFEM_DOF_OX) Bi[3] = 1.0;
      else if (kind == IFEM_DOF_OY) Bi[4] = -1.0;
      else if (kind == IFEM_DOF_OZ) Bi[5] = 1.0;
    }
  }
  amg_free(sd.amg);
  sd.amg = nullptr;
  sd.amg = amg_build(n, rp, ci, v, node, nu, nm, B, sd.amg_opt);
}

static bool solve_constrained(ifem_ctx* c, int step, double rtol, int max_it, int m, double* dx_out, int* its,
                              double* relres) {
  StepDev& sd = c->steps[step];
  if (!sd.cons_built || !sd.kcon_ready) throw Err{IFEM_ERR_STATE, "call ifem_constrain with want_matrix = 1 first"};
  const int64_t n = sd.n_free;
  *its = 0; *relres = 0.0;
  if (n == 0) return true;
  const size_t need = (size_t)(m + 1) * n + 4 * (size_t)n + 2 * (size_t)(m + 2);
  if (need > sd.kw_len) { if (sd.kw) cudaFree(sd.kw); sd.kw = dalloc<double>(need); sd.kw_len = need; }
  double* V = sd.kw;
  double* w = V + (size_t)(m + 1) * n;
  double* z = w + n;
  double* x = z + n;
  double* dinv = x + n;
  double* hd = dinv + n;            // m + 2 coefficients, then m + 2 more
  cudaStream_t s = c->stream;
  const int64_t* rp = sd.rowptr_con;
  const int32_t* ci = sd.colidx_con;
  auto spmv = [&](const double* in, double* out) { launch_spmv(n, rp, ci, sd.vals_con, sd.vals_con_f32, in, out, s); };
  auto fetch = [&](double* h, int k) {
    CK(cudaMemcpyAsync(h, hd, k * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  };
  auto norm = [&](const double* v) { double r; launch_dots(n, v, n, 1, v, hd, s); fetch(&r, 1); return std::sqrt(r); };
  // preconditioner M^-1: node blocks when the step's DOFs are nc per node (component-major), else the diagonal
  const int64_t nu = c->n_unique;
  // the node-block table maps dof c*nu + rank to (node rank, component c): only valid for that layout
  bool node_major_blocks = sd.nc >= 1 && sd.nc <= 3 && sd.ndofs == (int64_t)sd.nc * nu;
  if (node_major_blocks) {
    int32_t rb[3] = {sd.row_base[0], sd.row_base[1], sd.row_base[2]};
    std::sort(rb, rb + sd.nc);
    for (int b = 0; b < sd.nc; ++b) node_major_blocks = node_major_blocks && rb[b] == (int64_t)b * nu;
  }
  const bool use_amg = sd.pc_kind == IFEM_PC_AMG || sd.pc_kind == IFEM_PC_AMG_REUSE;
  const bool blocks = node_major_blocks && !use_amg;
  if (use_amg) {
    if (sd.pc_kind == IFEM_PC_AMG || !sd.amg) amg_setup(c, step);
  } else if (blocks) {
    if (!sd.kbinv) sd.kbinv = dalloc<double>((size_t)nu * 9);
    if (!sd.ktbl) sd.ktbl = dalloc<int32_t>((size_t)nu * sd.nc);
    launch_block_setup(n, sd.row_src, nu, sd.nc, sd.ktbl, rp, ci, sd.vals_con, sd.vals_con_f32, sd.kbinv, s);
  } else {
    launch_diag_inv(n, rp, ci, sd.vals_con, sd.vals_con_f32, dinv, s);
  }
  auto prec = [&](const double* in, double* out) {   // out = M^-1 in (out may be in)
    if (use_amg) amg_apply(sd.amg, in, out, s);
    else if (blocks) launch_block_apply(nu, sd.nc, sd.ktbl, sd.kbinv, in, out, s);
    else launch_scale(n, 1.0, in, dinv, out, s);
  };
  CK(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  const double bnorm = norm(sd.f_con);
  const double one = 1.0;
  bool conv = bnorm == 0.0;
  std::vector<double> H((size_t)(m + 1) * m), g(m + 1), cs(m), sn(m), h(m + 1), h2(m + 2), y(m);
  while (!conv && *its < max_it) {
    spmv(x, z);
    launch_sub(n, sd.f_con, z, w, s);                       // r = b - K x
    const double beta = norm(w);
    if (beta <= rtol * bnorm) { conv = true; break; }
    launch_scale(n, 1.0 / beta, w, nullptr, V, s);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int jend = 0;
    for (int j = 0; j < m && *its < max_it; ++j) {
      prec(V + (size_t)j * n, z);                             // z = M^-1 V_j
      spmv(z, w);
      launch_dots(n, V, n, j + 1, w, hd, s); fetch(h.data(), j + 1);   // the coefficients stay in hd for the update
      launch_comb(n, V, n, hd, j + 1, -1.0, w, s);
      launch_dots(n, V, n, j + 1, w, hd, s, true); fetch(h2.data(), j + 2);   // + w.w in h2[j + 1]
      launch_comb(n, V, n, hd, j + 1, -1.0, w, s);
      // ||w - V h2||^2 = w.w - |h2|^2 for orthonormal V; the explicit norm where that cancels (near breakdown)
      double hn2 = h2[j + 1];
      for (int i = 0; i <= j; ++i) hn2 -= h2[i] * h2[i];
      const double hn = hn2 >= 1e-4 * h2[j + 1] ? std::sqrt(hn2) : norm(w);
      for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = h[i] + h2[i];
      H[(size_t)(j + 1) * m + j] = hn;
      if (hn > 0.0) launch_scale(n, 1.0 / hn, w, nullptr, V + (size_t)(j + 1) * n, s);
      for (int i = 0; i < j; ++i) {                          // earlier rotations on column j
        const double a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
      }
      const double a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
      if (b == 0.0) { cs[j] = 1.0; sn[j] = 0.0; }
      else if (std::fabs(b) > std::fabs(a)) { const double t = a / b; sn[j] = 1.0 / std::sqrt(1.0 + t * t); cs[j] = t * sn[j]; }
      else { const double t = b / a; cs[j] = 1.0 / std::sqrt(1.0 + t * t); sn[j] = t * cs[j]; }
      H[(size_t)j * m + j] = cs[j] * a + sn[j] * b;
      H[(size_t)(j + 1) * m + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++*its;
      jend = j + 1;
      if (std::fabs(g[j + 1]) <= rtol * bnorm || hn == 0.0) break;
    }
    for (int i = jend - 1; i >= 0; --i) {                    // H y = g
      double t = g[i];
      for (int k = i + 1; k < jend; ++k) t -= H[(size_t)i * m + k] * y[k];
      const double piv = H[(size_t)i * m + i];
      if (!(std::fabs(piv) > 0.0) || !std::isfinite(piv))
        throw Err{IFEM_ERR_NUMERIC, "GMRES: zero or non-finite pivot of the Hessenberg matrix at column " +
                                        std::to_string(i) + " (K_con singular or inconsistent)"};
      y[i] = t / piv;
    }
    CK(cudaMemcpyAsync(hd, y.data(), jend * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(z, 0, n * sizeof(double), s));
    launch_comb(n, V, n, hd, jend, 1.0, z, s);                 // z = V y
    prec(z, z);                                                 // z = M^-1 V y
    CK(cudaMemcpyAsync(hd + m + 2, &one, sizeof(double), cudaMemcpyHostToDevice, s));
    launch_comb(n, z, n, hd + m + 2, 1, 1.0, x, s);            // x += z
  }
  spmv(x, z);
  launch_sub(n, sd.f_con, z, w, s);
  const double rn = norm(w);
  *relres = bnorm > 0.0 ? rn / bnorm : 0.0;
  conv = *relres <= rtol;
  CK(cudaMemcpyAsync(dx_out, x, n * sizeof(double), cudaMemcpyDefault, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return conv;
}

int ifem_set_constraints(ifem_ctx* ctx, int32_t step, int64_t n, const int64_t* dofs, const double* values) {
  if (!ctx || step < 0 || step >= ctx->nsteps || n < 0 || (n > 0 && (!dofs || !values))) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] { set_constraints(ctx, step, n, dofs, values); });
}

int ifem_constrained_info(const ifem_ctx* ctx, int32_t step, int64_t* n_free, int64_t* nnz) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  const StepDev& sd = ctx->steps[step];
  if (n_free) *n_free = sd.cons_set ? sd.n_free : sd.ndofs;
  if (nnz) *nnz = sd.cons_set ? sd.nnz_con : sd.nnz;
  return IFEM_OK;
}

int ifem_build_constrained_pattern(const ifem_ctx* ctx, int32_t step, int32_t* row_ptr, int32_t* col_idx) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    const StepDev& sd = c->steps[step];
    if (!sd.cons_set) throw Err{IFEM_ERR_STATE, "no constraints set for this step"};
    if (row_ptr) {
      std::vector<int64_t> rp(sd.n_free + 1);
      CK(cudaMemcpy(rp.data(), sd.rowptr_con, rp.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < rp.size(); ++i) row_ptr[i] = (int32_t)rp[i];
    }
    if (col_idx && sd.nnz_con) CK(cudaMemcpy(col_idx, sd.colidx_con, sd.nnz_con * sizeof(int32_t), cudaMemcpyDefault));
  });
}

int ifem_constrain(ifem_ctx* ctx, int32_t step, int32_t want_matrix) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] { constrain(ctx, step, want_matrix != 0); });
}

int ifem_get_constrained(const ifem_ctx* ctx, int32_t step, double* f_con, void* vals, int64_t nnz, int32_t dtype) {
  if (!ctx || step < 0 || step >= ctx->nsteps || (dtype != IFEM_F64 && dtype != IFEM_F32)) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    const StepDev& sd = c->steps[step];
    if (!sd.cons_built) throw Err{IFEM_ERR_STATE, "ifem_constrain has not run"};
    CK(cudaStreamSynchronize(c->stream));
    if (f_con && sd.n_free) CK(cudaMemcpy(f_con, sd.f_con, sd.n_free * sizeof(double), cudaMemcpyDefault));
    if (vals) {
      if (nnz != sd.nnz_con) throw Err{IFEM_ERR_INVALID, "nnz mismatch"};
      if (!nnz) return;
      const bool src32 = sd.vals_con_f32 != 0, dst32 = dtype == IFEM_F32;
      if (src32 == dst32) {
        CK(cudaMemcpy(vals, sd.vals_con, nnz * (dst32 ? 4 : 8), cudaMemcpyDefault));
      } else if (src32) {
        std::vector<float> t(nnz);
        CK(cudaMemcpy(t.data(), sd.vals_con, nnz * 4, cudaMemcpyDeviceToHost));
        std::vector<double> d(t.begin(), t.end());
        CK(cudaMemcpy(vals, d.data(), nnz * 8, cudaMemcpyDefault));
      } else {
        std::vector<double> t(nnz);
        CK(cudaMemcpy(t.data(), sd.vals_con, nnz * 8, cudaMemcpyDeviceToHost));
        std::vector<float> d(t.begin(), t.end());
        CK(cudaMemcpy(vals, d.data(), nnz * 4, cudaMemcpyDefault));
      }
    }
  });
}

int ifem_device_constrained(const ifem_ctx* ctx, int32_t step, const double** f_con, const void** vals,
                            int32_t* dtype_out) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  const StepDev& sd = ctx->steps[step];
  if (!sd.cons_built) return IFEM_ERR_STATE;
  if (f_con) *f_con = sd.f_con;
  if (vals) *vals = sd.vals_con;
  if (dtype_out) *dtype_out = sd.vals_con_f32 ? IFEM_F32 : IFEM_F64;
  return IFEM_OK;
}

int ifem_set_preconditioner(ifem_ctx* ctx, int32_t step, int32_t kind) {
  if (!ctx || step < 0 || step >= ctx->nsteps || kind < IFEM_PC_BLOCK_JACOBI || kind > IFEM_PC_AMG_REUSE)
    return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    StepDev& sd = ctx->steps[step];
    sd.pc_kind = kind;
    amg_free(sd.amg);
    sd.amg = nullptr;
  });
}

int ifem_set_multigrid(ifem_ctx* ctx, int32_t step, double strength_threshold, int32_t sweeps) {
  if (!ctx || step < 0 || step >= ctx->nsteps || !(strength_threshold >= 0.0 && strength_threshold < 1.0) ||
      sweeps < 1 || sweeps > 8)
    return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    StepDev& sd = ctx->steps[step];
    sd.amg_opt.theta = strength_threshold;
    sd.amg_opt.sweeps = sweeps;
    amg_free(sd.amg);
    sd.amg = nullptr;
  });
}

int ifem_preconditioner_info(const ifem_ctx* ctx, int32_t step, int32_t* levels, int64_t* sizes, double* setup_ms) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  const StepDev& sd = ctx->steps[step];
  if (!sd.amg) { if (levels) *levels = 0; if (setup_ms) *setup_ms = 0.0; return IFEM_OK; }
  int64_t tmp[16];
  const int nl = amg_levels(sd.amg, tmp, 16);
  if (levels) *levels = nl;
  if (sizes) for (int i = 0; i < nl && i < 8; ++i) sizes[i] = tmp[i];
  if (setup_ms) *setup_ms = amg_setup_ms(sd.amg);
  return IFEM_OK;
}

int ifem_solve_constrained(ifem_ctx* ctx, int32_t step, double rtol, int32_t max_it, int32_t restart, double* dx,
                           int32_t* iterations, double* rel_residual) {
  if (!ctx || step < 0 || step >= ctx->nsteps || !dx || !(rtol > 0) || max_it < 1 || restart < 1 || restart > 200)
    return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    int its = 0;
    double rr = 0.0;
    const bool ok = solve_constrained(ctx, step, rtol, max_it, restart, dx, &its, &rr);
    if (iterations) *iterations = its;
    if (rel_residual) *rel_residual = rr;
    if (!ok) throw Err{IFEM_ERR_NUMERIC, "GMRES did not reach the tolerance within max_it (dx holds the last iterate)"};
  });
}

int ifem_update_state(ifem_ctx* ctx, int32_t step, const double* dx) {
  if (!ctx || step < 0 || step >= ctx->nsteps || !dx) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    StepDev& sd = ctx->steps[step];
    if (!sd.cons_built) throw Err{IFEM_ERR_STATE, "ifem_constrain has not run"};
    if (sd.n_free) CK(cudaMemcpyAsync(sd.dx, dx, sd.n_free * sizeof(double), cudaMemcpyDefault, ctx->stream));
    launch_update_state(sd.fmap, sd.ndofs, sd.dx, sd.cv, sd.state[0], ctx->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
  });
}

// TriAxialModel::init / Setup (TriAxial.cpp:22-71): the groups are uploaded once; the gather lists put each face
// node's incidences in face order, side faces first, as the model's two element loops add them
int ifem_set_triaxial(ifem_ctx* ctx, const ifem_face_group* side, const ifem_face_group* top, const ifem_triaxial* prm) {
  if (!ctx || !side || !top || !prm) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    ifem_ctx* c = ctx;
    if (c->step_u < 0) throw Err{IFEM_ERR_INVALID, "TriAxial needs displacement dofs"};
    const int nfn = c->dim == 2 ? 3 : 9;
    const ifem_face_group* g[2] = {side, top};
    for (int k = 0; k < 2; ++k)
      if (g[k]->n_faces < 1 || !g[k]->faces || !g[k]->face_data) throw Err{IFEM_ERR_INVALID, "empty face group"};
    if (!(prm->penalty >= 0.0) || !std::isfinite(prm->p0) || !std::isfinite(prm->du) || !std::isfinite(prm->penalty))
      throw Err{IFEM_ERR_INVALID, "TriAxial parameters"};
    if (prm->damaged_forces && c->step_ph < 0) throw Err{IFEM_ERR_INVALID, "DamagedForces needs a phase field"};
    const int64_t nf = side->n_faces + top->n_faces;
    if (nf * nfn > INT32_MAX) throw Err{IFEM_ERR_CAPACITY, "face groups too large"};
    std::vector<int32_t> rank(c->nn);
    CK(cudaMemcpy(rank.data(), c->node_rank, c->nn * sizeof(int32_t), cudaMemcpyDeviceToHost));
    std::vector<int32_t> faces((size_t)nf * nfn);
    std::vector<double> C((size_t)nf * nfn * nfn);
    int64_t off = 0;
    for (int k = 0; k < 2; ++k) {
      for (int64_t i = 0; i < g[k]->n_faces * nfn; ++i) {
        const int64_t nd = g[k]->faces[i];
        if (nd < 0 || nd >= c->nn || rank[nd] < 0) throw Err{IFEM_ERR_INVALID, "face node without displacement dofs"};
        faces[off * nfn + i] = (int32_t)nd;
      }
      for (int64_t i = 0; i < g[k]->n_faces * nfn * nfn; ++i) {
        if (!std::isfinite(g[k]->face_data[i])) throw Err{IFEM_ERR_INVALID, "face extraction operator"};
        C[off * nfn * nfn + i] = g[k]->face_data[i];
      }
      off += g[k]->n_faces;
    }
    // incidences sorted by node, then by face (stable: faces are already in order)
    std::vector<std::pair<int32_t, int32_t>> inc((size_t)nf * nfn);
    for (int64_t i = 0; i < nf * nfn; ++i) inc[i] = {faces[i], (int32_t)i};
    std::stable_sort(inc.begin(), inc.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<int32_t> node, inc_ptr{0}, inc_e;
    for (size_t i = 0; i < inc.size(); ++i) {
      if (i == 0 || inc[i].first != inc[i - 1].first) { if (i) inc_ptr.push_back((int32_t)i); node.push_back(inc[i].first); }
      inc_e.push_back(inc[i].second);
    }
    inc_ptr.push_back((int32_t)inc.size());
    // a captured graph may reference the buffers replaced below
    CK(cudaStreamSynchronize(c->stream));
    if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    c->graph_steps.clear();
    auto F = [](void* p) { if (p) cudaFree(p); };
    F(c->tri_faces); F(c->tri_node); F(c->tri_inc_ptr); F(c->tri_inc); F(c->tri_C); F(c->tri_F); F(c->tri_K);
    F(c->tri_sums); F(c->tri_tot); F(c->tri_kpos);
    c->tri_faces = c->tri_node = c->tri_inc_ptr = c->tri_inc = nullptr;
    c->tri_C = c->tri_F = c->tri_K = c->tri_sums = c->tri_tot = nullptr;
    c->tri_kpos = nullptr;
    c->tri_on = false;
    c->tri_nside = side->n_faces; c->tri_ntop = top->n_faces; c->tri_nnodes = (int64_t)node.size();
    c->tri_faces = dupload(faces); c->tri_C = dupload(C);
    c->tri_node = dupload(node); c->tri_inc_ptr = dupload(inc_ptr); c->tri_inc = dupload(inc_e);
    c->tri_F = dalloc<double>((size_t)nf * c->dim * nfn);
    c->tri_K = dalloc<double>((size_t)top->n_faces * nfn * nfn);
    c->tri_sums = dalloc<double>((size_t)3 * top->n_faces);
    c->tri_tot = dalloc<double>(3);
    c->tri_kpos = dalloc<int64_t>((size_t)top->n_faces * nfn * nfn);
    StepDev& sd = c->steps[c->step_u];
    FaceParams fp = face_params(c, sd);
    unsigned long long* err = dalloc<unsigned long long>(1);
    CK(cudaMemsetAsync(err, 0, sizeof(unsigned long long), c->stream));
    fp.err = err;
    launch_face_kpos(fp, c->tri_kpos, c->stream);
    CK(cudaGetLastError());
    unsigned long long e = 0;
    CK(cudaMemcpyAsync(&e, err, sizeof(e), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(err);
    if (e) throw Err{IFEM_ERR_INVALID, "top-group node pairs outside the displacement matrix pattern"};
    c->tri_prm = *prm;
    ifem_triaxial_state st{};
    st.area = 1.0; st.f_ext = 0.0; st.uz_sum = 0.0; st.u0 = -1.0e8; st.t_break = 0.0; st.max_load = -1e9;
    st.p0 = prm->p0; st.min_load_passed = 0;
    c->tri_st = st;
    c->tri_assembled = false;
    c->tri_on = true;
  });
}

// the sums of the last displacement-step assembly (TriAxial.cpp:218-276)
static void tri_read_sums(ifem_ctx* c) {
  if (!c->tri_assembled) return;
  double t[3];
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(t, c->tri_tot, sizeof(t), cudaMemcpyDeviceToHost));
  c->tri_st.area = t[0]; c->tri_st.f_ext = t[1]; c->tri_st.uz_sum = t[2];
  c->tri_assembled = false;
}

static double sgn(double v) { return (double)((0.0 < v) - (v < 0.0)); }

// TriAxialModel::Commit (TriAxial.cpp:75-122)
int ifem_triaxial_commit(ifem_ctx* ctx, int32_t commit_type, double time, double* max_time) {
  if (!ctx) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    if (!ctx->tri_on) throw Err{IFEM_ERR_STATE, "no TriAxial model"};
    if (commit_type != IFEM_COMMIT_TIMEDEP) return;
    tri_read_sums(ctx);
    ifem_triaxial_state& s = ctx->tri_st;
    const double du = ctx->tri_prm.du, p0 = ctx->tri_prm.p0;
    const double load = s.f_ext / s.area;
    s.max_load = std::max(s.max_load, load * sgn(du));
    auto broken = [&](double min_load) {
      if (s.min_load_passed && std::fabs(load) < min_load && s.t_break < 1e-8) {
        s.t_break = time;
        if (max_time) *max_time = s.t_break + ctx->tri_prm.t_post_fail;
      }
    };
    if (sgn(du) < 0) {   // loaded downwards
      if (!s.min_load_passed && load * sgn(du) > std::max(1.0e3, std::fabs(p0)) && time > 0.0) s.min_load_passed = 1;
      broken(std::max(0.05 * std::fabs(p0), 0.05 * s.max_load));
    } else {             // loaded upwards
      broken(std::max(0.0, 0.25 * s.max_load));
      if (!s.min_load_passed && load * sgn(du) > 0.0 && time > 0.0) s.min_load_passed = 1;
    }
    if (time < 0.0) s.u0 = s.uz_sum / s.area;
  });
}

int ifem_triaxial_get_state(const ifem_ctx* ctx, ifem_triaxial_state* out) {
  if (!ctx || !out) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  return guarded(c, [&] {
    if (!c->tri_on) throw Err{IFEM_ERR_STATE, "no TriAxial model"};
    tri_read_sums(c);
    *out = c->tri_st;
  });
}

int ifem_triaxial_set_state(ifem_ctx* ctx, const ifem_triaxial_state* in) {
  if (!ctx || !in) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    if (!ctx->tri_on) throw Err{IFEM_ERR_STATE, "no TriAxial model"};
    tri_read_sums(ctx);
    ctx->tri_st = *in;
  });
}

int ifem_set_param(ifem_ctx* ctx, int32_t mat, int32_t theta, double value) {
  if (!ctx || mat < 0 || mat >= (int)ctx->mats_in.size()) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    ifem_material& m = ctx->mats_in[mat];
    switch (theta) {
      case 0: m.gc = value; break;
      case 1: m.pf_l = value; break;
      case 2: m.creep_a = value; break;
      case 3: m.creep_n = value; break;
      default: throw Err{IFEM_ERR_INVALID, "theta index"};
    }
    ctx->mats_h[mat] = make_mat(m, ctx->opt);
    set_spec(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(ctx->mats_d + mat, &ctx->mats_h[mat], sizeof(MatDev), cudaMemcpyHostToDevice));
  });
}

// Adjoint buffers (allocated once; never inside a graph capture).
static void adjoint_alloc(ifem_ctx* c) {
  if (c->adj_dF) return;
  const int n_mats = (int)c->mats_h.size();
  c->adj_dF = dalloc<double>(4 * (size_t)c->nel * (size_t)c->dim * c->nen);
  int64_t fmax = 1;
  for (const auto& st : c->steps) fmax = std::max<int64_t>(fmax, st.ndofs);
  c->adj_lam = dalloc<double>((size_t)fmax);
  c->adj_el = dalloc<double>(4 * (size_t)c->nel);
  for (const auto& st : c->steps) {
    c->adj_f.push_back(dalloc<double>(4 * (size_t)std::max<int64_t>(1, st.ndofs)));
    c->adj_out.push_back(dalloc<double>(4 * (size_t)n_mats));
    CK(cudaMemset(c->adj_out.back(), 0, 4 * (size_t)n_mats * sizeof(double)));
    CK(cudaMemset(c->adj_f.back(), 0, 4 * (size_t)std::max<int64_t>(1, st.ndofs) * sizeof(double)));
  }
  // elements of each material set, ascending
  std::vector<int32_t> ptr(n_mats + 1, 0), els((size_t)c->nel);
  for (int64_t e = 0; e < c->nel; ++e) ptr[(c->emat_h.empty() ? 0 : c->emat_h[e]) + 1]++;
  for (int m = 0; m < n_mats; ++m) ptr[m + 1] += ptr[m];
  std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
  for (int64_t e = 0; e < c->nel; ++e) els[fill[c->emat_h.empty() ? 0 : c->emat_h[e]]++] = (int32_t)e;
  c->adj_mat_ptr = dupload(ptr);
  c->adj_mat_el = dupload(els);
}

// dR/dtheta of one step's residual at the stored state and history (nothing is written back), enqueued on
// the context's stream: element kernels give dF[theta][el][comp*nen+node]; the deterministic gather turns
// each theta's element vectors into a global vector in element order (adj_f[step]); lambda^T dF is summed
// per element and then per material set in ascending element order (adj_out[step]).  lam_d: device
// vector or nullptr (ones).
static void adjoint_enqueue(ifem_ctx* c, int step, const ifem_time& tm, const double* lam_d, bool full, bool per_set) {
  StepDev& sd = c->steps[step];
  // the implicit differentiation is of the viscoelastic local system (SolidMaterial.cpp:278-301)
  if (c->coss) throw Err{IFEM_ERR_UNSUPPORTED, "adjoint of the Cosserat model"};
  if (c->mh == 4) throw Err{IFEM_ERR_UNSUPPORTED, "adjoint of the viscoelastic-plastic return map"};
  if (c->general || c->ph_general)
    throw Err{IFEM_ERR_UNSUPPORTED, "adjoint with a SpecStrains / DruckerPrager split or Lagrange multipliers"};
  if (dist_second_gradient(c->mo.dist) && step == c->step_ph)
    throw Err{IFEM_ERR_UNSUPPORTED, "phase-step adjoint of a second-gradient distribution function"};
  if (!(tm.dt > 0) && step == c->step_ph) throw Err{IFEM_ERR_INVALID, "dt must be positive"};
  const int n_mats = (int)c->mats_h.size();
  const int64_t n = sd.ndofs;
  const Geo geo = geo_of(c);
  const DofMap dm = dm_of(c);
  int nc = 0, kind0 = 0;
  if (sd.kind == 0) {
    UParams p{};
    p.geo = geo; p.rule = c->rule; p.dm = dm; p.mo = c->mo; p.h = c->h;
    p.su = ss_of(c, c->step_u); p.sp = ss_of(c, c->step_ph); p.sT = ss_of(c, c->step_T);
    p.dt = tm.dt; p.du_dt = tm.du_dt; p.ddu_dt = tm.ddu_dt;
    launch_adjoint_u(p, c->adj_dF, nullptr, nullptr, c->adj_f32, c->stream);
    nc = c->dim; kind0 = IFEM_DOF_UX;
  } else if (sd.kind == 1) {
    PParams p{};
    p.geo = geo; p.rule = c->rule; p.dm = dm; p.mo = c->mo; p.h = c->h;
    p.su = ss_of(c, c->step_u); p.sp = ss_of(c, c->step_ph); p.sT = ss_of(c, c->step_T);
    p.dt = tm.dt;
    launch_adjoint_phase(p, c->adj_dF, nullptr, nullptr, c->adj_f32, c->stream);
    nc = 1; kind0 = IFEM_DOF_PHASE;
  }
  if (nc == 0) {   // the T step does not depend on theta
    CK(cudaMemsetAsync(c->adj_f[step], 0, 4 * (size_t)std::max<int64_t>(1, n) * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->adj_out[step], 0, 4 * (size_t)n_mats * sizeof(double), c->stream));
    return;
  }
  const int64_t per_theta = c->nel * (int64_t)nc * c->nen;
  if (full) {
    GParams gp = gather_params(c, sd);
    gp.Ke = nullptr; gp.Fe2 = nullptr; gp.vals = nullptr;
    for (int th = 0; th < 4; ++th) {
      gp.Fe1 = c->adj_dF + th * per_theta;
      gp.f = c->adj_f[step] + th * n;
      launch_gather(gp, c->stream);
    }
  }
  if (per_set)
    launch_adjoint_lambda(c->adj_dF, c->nel, nc, c->nen, c->conn, dm, kind0, lam_d, c->adj_el, c->adj_mat_ptr,
                          c->adj_mat_el, n_mats, c->adj_out[step], c->stream);
  CK(cudaGetLastError());
}

static void adjoint_copy_out(ifem_ctx* c, int step, double* dr_dtheta, double* lam_dr) {
  CK(cudaStreamSynchronize(c->stream));
  const int64_t n = c->steps[step].ndofs;
  if (dr_dtheta && n) CK(cudaMemcpy(dr_dtheta, c->adj_f[step], 4 * n * sizeof(double), cudaMemcpyDefault));
  if (lam_dr) CK(cudaMemcpy(lam_dr, c->adj_out[step], 4 * c->mats_h.size() * sizeof(double), cudaMemcpyDefault));
}

int ifem_adjoint(ifem_ctx* ctx, int32_t step, const ifem_time* tm, const double* lambda, double* dr_dtheta,
                 double* lam_dr) {
  if (!ctx || !tm || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    ifem_ctx* c = ctx;
    adjoint_alloc(c);
    const double* lam_d = nullptr;
    if (lambda && lam_dr) {
      CK(cudaMemcpyAsync(c->adj_lam, lambda, c->steps[step].ndofs * sizeof(double), cudaMemcpyDefault, c->stream));
      lam_d = c->adj_lam;
    }
    adjoint_enqueue(c, step, *tm, lam_d, dr_dtheta != nullptr, lam_dr != nullptr);
    adjoint_copy_out(c, step, dr_dtheta, lam_dr);
  });
}

int ifem_set_adjoint_precision(ifem_ctx* ctx, int32_t dtype) {
  if (!ctx || (dtype != IFEM_F64 && dtype != IFEM_F32)) return IFEM_ERR_INVALID;
  ctx->adj_f32 = dtype == IFEM_F32 ? 1 : 0;
  return IFEM_OK;
}

// dR_step/dT . dT through A(T) (u step) and Gc(T) (phase step), evaluated like the adjoint at the stored state
// and start-of-assembly history; element vectors gathered in element order like a residual.
int ifem_temperature_sensitivity(ifem_ctx* ctx, int32_t step, const ifem_time* tm, const double* dT, double* dr_out) {
  if (!ctx || !tm || step < 0 || step >= ctx->nsteps || !dr_out) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    ifem_ctx* c = ctx;
    StepDev& sd = c->steps[step];
    if (sd.kind == 2)
      throw Err{IFEM_ERR_INVALID, "the temperature step's derivative with respect to its own DOFs is its tangent"};
    if (c->hasT != (dT != nullptr))
      throw Err{IFEM_ERR_INVALID, c->hasT ? "dT [n_T] is required: the context has a temperature DOF"
                                          : "dT must be NULL: the derivative is with respect to the pinned temperature"};
    if (c->coss) throw Err{IFEM_ERR_UNSUPPORTED, "temperature sensitivity of the Cosserat model"};
    if (c->mh == 4) throw Err{IFEM_ERR_UNSUPPORTED, "temperature sensitivity of the viscoelastic-plastic return map"};
    if (c->general || c->ph_general)
      throw Err{IFEM_ERR_UNSUPPORTED, "temperature sensitivity with a SpecStrains / DruckerPrager split or Lagrange multipliers"};
    for (const MatDev& m : c->mats_h)
      if (m.split == IFEM_SPLIT_ICE) throw Err{IFEM_ERR_UNSUPPORTED, "temperature sensitivity of the ICE split"};
    if (dist_second_gradient(c->mo.dist) && step == c->step_ph)
      throw Err{IFEM_ERR_UNSUPPORTED, "phase-step temperature sensitivity of a second-gradient distribution function"};
    if (!(tm->dt > 0) && step == c->step_ph) throw Err{IFEM_ERR_INVALID, "dt must be positive"};
    const int nc = sd.kind == 0 ? c->dim : 1;
    if (!c->sens_dF) c->sens_dF = dalloc<double>((size_t)c->nel * c->dim * c->nen);
    const int64_t n = sd.ndofs;
    if (c->sens_f_len < n) {
      if (c->sens_f) cudaFree(c->sens_f);
      c->sens_f = dalloc<double>((size_t)std::max<int64_t>(1, n));
      c->sens_f_len = n;
    }
    const double* dT_d = nullptr;
    if (dT) {
      const int64_t nT = c->steps[c->step_T].ndofs;
      if (!c->sens_dT) c->sens_dT = dalloc<double>((size_t)std::max<int64_t>(1, nT));
      CK(cudaMemcpyAsync(c->sens_dT, dT, nT * sizeof(double), cudaMemcpyDefault, c->stream));
      dT_d = c->sens_dT;
    }
    const Geo geo = geo_of(c);
    const DofMap dm = dm_of(c);
    if (sd.kind == 0) {
      UParams p{};
      p.geo = geo; p.rule = c->rule; p.dm = dm; p.mo = c->mo; p.h = c->h;
      p.su = ss_of(c, c->step_u); p.sp = ss_of(c, c->step_ph); p.sT = ss_of(c, c->step_T);
      p.dt = tm->dt; p.du_dt = tm->du_dt; p.ddu_dt = tm->ddu_dt;
      launch_adjoint_u(p, nullptr, dT_d, c->sens_dF, c->adj_f32, c->stream);
    } else {
      PParams p{};
      p.geo = geo; p.rule = c->rule; p.dm = dm; p.mo = c->mo; p.h = c->h;
      p.su = ss_of(c, c->step_u); p.sp = ss_of(c, c->step_ph); p.sT = ss_of(c, c->step_T);
      p.dt = tm->dt;
      launch_adjoint_phase(p, nullptr, dT_d, c->sens_dF, c->adj_f32, c->stream);
    }
    (void)nc;
    GParams gp = gather_params(c, sd);
    gp.Ke = nullptr; gp.Fe2 = nullptr; gp.vals = nullptr;
    gp.Fe1 = c->sens_dF;
    gp.f = c->sens_f;
    launch_gather(gp, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dr_out, c->sens_f, n * sizeof(double), cudaMemcpyDefault, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int ifem_adjoint_results(const ifem_ctx* ctx, int32_t step, double* dr_dtheta, double* lam_dr) {
  if (!ctx || step < 0 || step >= ctx->nsteps) return IFEM_ERR_INVALID;
  ifem_ctx* c = const_cast<ifem_ctx*>(ctx);
  if (!c->adj_dF) { c->err = "no adjoint has run"; return IFEM_ERR_STATE; }
  return guarded(c, [&] { adjoint_copy_out(c, step, dr_dtheta, lam_dr); });
}

// ---- CUDA graph of a sequence of assemblies (+ adjoints) ----
int ifem_graph_capture(ifem_ctx* ctx, int32_t n_steps, const int32_t* steps, const ifem_time* tm,
                       int32_t with_adjoint) {
  if (!ctx || !tm || n_steps <= 0 || !steps) return IFEM_ERR_INVALID;
  for (int i = 0; i < n_steps; ++i) if (steps[i] < 0 || steps[i] >= ctx->nsteps) return IFEM_ERR_INVALID;
  return guarded(ctx, [&] {
    ifem_ctx* c = ctx;
    // every buffer the captured work uses exists before the capture starts
    const bool f32 = c->opt.tangent_precision != IFEM_PREC_FP64;
    ensure_scratch(c, f32);
    if (c->opt.tangent_precision == IFEM_PREC_TC_SPLIT && c->dim == 3 && c->kron) {
      if (!c->geoq) c->geoq = dalloc<float>((size_t)kTcGeo * c->nel);
      if (!c->Kd) c->Kd = dalloc<double>((size_t)kTcKd * c->nel);
      if (!c->nxq) c->nxq = dalloc<float>((size_t)kTcNx * c->nel);
    }
    if (with_adjoint) adjoint_alloc(c);
    if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    c->capturing = true;
    try {
      for (int i = 0; i < n_steps; ++i) {
        assemble_async(c, steps[i], *tm);
        if (with_adjoint) adjoint_enqueue(c, steps[i], *tm, nullptr, true, true);
      }
    } catch (...) {
      c->capturing = false;
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    c->capturing = false;
    CK(cudaStreamEndCapture(c->stream, &c->graph));
    CK(cudaGraphInstantiate(&c->gexec, c->graph, 0));
    c->graph_steps.assign(steps, steps + n_steps);
  });
}

int ifem_graph_launch(ifem_ctx* ctx) {
  if (!ctx) return IFEM_ERR_INVALID;
  if (!ctx->gexec) { ctx->err = "no graph captured"; return IFEM_ERR_STATE; }
  return guarded(ctx, [&] {
    CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
    for (int s : ctx->graph_steps) {
      ctx->steps[s].assembled = true;
      ctx->steps[s].slabbed = false;
      CK(cudaEventRecord(ctx->done_ev[s], ctx->stream));
      if (s == ctx->step_u && ctx->tri_on) ctx->tri_assembled = true;
    }
  });
}

}  // extern "C"
