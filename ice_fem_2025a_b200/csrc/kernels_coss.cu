// Fracture/CossPhaseField (CossPhaseField.cpp:337-800) on the device: ux, uy, oz per node in 2D, ux, uy, uz, ox, oy,
// oz in 3D.
//
//   k_coss_points  one warp per element, lane = integration point: strains B_coss U (ConstructBMatCoss,
//                  CossPhaseField.cpp:1168-1223), UpdatePlasticStrains with the Cosserat return map, the
//                  Cosserat split; writes the history, w (Dam sigma_d + sigma_u) and w (Dam D_d + D_u) DPlast.
//   k_coss_elem    one CTA per element: F_e = sum_q B^T (w sigma), K_e = sum_q B^T (w C) B through the
//                  structure of B (every entry of B is a coefficient times N or a gradient component), then the
//                  lumped inertia, damping and gravity terms in the reference's order; stored in the gathers'
//                  element layout.
//   k_coss_energy  phase step: the driving energy of the Cosserat split of B_coss U - plastic strain, zero
//                  before t = 0, with the history maximum, and |N_uu dU|^2 with the micro-rotation rates.
//
// Every loop is bounded (the return map at 501 iterations); no kernel waits or traps.

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "device_coss.cuh"
#include "icefem_internal.h"

namespace ifem {
namespace {

__device__ __forceinline__ int cdof(const DofMap& dm, int kind, int node) { return dm.base[kind] + dm.node_rank[node]; }

// B_coss entries per displacement component c (ConstructBMatCoss): (strain row, basis kind, coefficient); kind
// 0..DIM-1 is the gradient component, DIM the shape value; coefficient 2 stands for l_coss.  Components: ux, uy,
// oz in 2D; ux, uy, uz, ox, oy, oz in 3D.
struct BEnt { int row, kind; double coef; };
__constant__ BEnt kB2[3][5] = {
    {{0, 0, 1.0}, {4, 1, 1.0}, {-1, 0, 0.0}, {-1, 0, 0.0}, {-1, 0, 0.0}},
    {{1, 1, 1.0}, {3, 0, 1.0}, {-1, 0, 0.0}, {-1, 0, 0.0}, {-1, 0, 0.0}},
    {{3, 2, -1.0}, {4, 2, 1.0}, {14, 0, 2.0}, {16, 1, 2.0}, {-1, 0, 0.0}},
};
__constant__ BEnt kB3[6][5] = {
    {{0, 0, 1.0}, {4, 1, 1.0}, {8, 2, 1.0}, {-1, 0, 0.0}, {-1, 0, 0.0}},
    {{1, 1, 1.0}, {3, 0, 1.0}, {6, 2, 1.0}, {-1, 0, 0.0}, {-1, 0, 0.0}},
    {{2, 2, 1.0}, {5, 1, 1.0}, {7, 0, 1.0}, {-1, 0, 0.0}, {-1, 0, 0.0}},
    {{5, 3, -1.0}, {6, 3, 1.0}, {9, 0, 2.0}, {12, 0, 2.0}, {16, 0, 2.0}},
    {{7, 3, -1.0}, {8, 3, 1.0}, {10, 1, 2.0}, {13, 1, 2.0}, {14, 1, 2.0}},
    {{3, 3, -1.0}, {4, 3, 1.0}, {11, 2, 2.0}, {15, 2, 2.0}, {17, 2, 2.0}},
};
template <int DIM>
__device__ __forceinline__ BEnt bent(int c, int k) { return DIM == 2 ? kB2[c][k] : kB3[c][k]; }
__host__ __device__ constexpr int coss_nc(int dim) { return dim == 2 ? 3 : 6; }
// the u-step's dof kinds in DofNames_u order
template <int DIM>
__device__ __forceinline__ int ukind(int c) {
  if (DIM == 2) return c == 0 ? IFEM_DOF_UX : (c == 1 ? IFEM_DOF_UY : IFEM_DOF_OZ);
  return c < 3 ? IFEM_DOF_UX + c : IFEM_DOF_OX + (c - 3);
}
constexpr int kCWarps = 4;

template <int DIM, bool KRON>
struct CPSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN, NC = coss_nc(DIM);
  ElemSm<DIM, KRON> e;
  double U[NC][NEN];
  double Ph[NEN];
  double T[NEN];
};

template <int DIM, bool KRON>
__device__ __forceinline__ void coss_strain(const CPSm<DIM, KRON>& s, const Rule& R, const IpGeo<DIM>& g, int q,
                                            double lc, double* eps, double& phi, double& Tip) {
  constexpr int NEN = ElemTraits<DIM>::NEN;
  for (int r = 0; r < 18; ++r) eps[r] = 0.0;
  phi = 0; Tip = 0;
  for (int a = 0; a < NEN; ++a) {
    double N, G[DIM];
    shape_at<DIM, KRON>(s.e, R, g, q, a, N, G);
    phi += N * s.Ph[a];
    Tip += N * s.T[a];
    for (int c = 0; c < coss_nc(DIM); ++c)
      for (int k = 0; k < 5; ++k) {
        const BEnt b = bent<DIM>(c, k);
        if (b.row < 0) continue;
        const double gv = b.kind < DIM ? G[b.kind] : N;
        const double cf = b.coef == 2.0 ? lc : b.coef;
        eps[b.row] += cf * gv * s.U[c][a];
      }
  }
}

template <int DIM, bool KRON>
__global__ void __launch_bounds__(128) k_coss_points(const CossParams p) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, NC = coss_nc(DIM);
  extern __shared__ __align__(16) unsigned char smraw[];
  CPSm<DIM, KRON>* sm = reinterpret_cast<CPSm<DIM, KRON>*>(smraw);
  const int warp = threadIdx.x >> 5, q = threadIdx.x & 31;
  const int64_t el = (int64_t)blockIdx.x * kCWarps + warp;
  if (el >= p.geo.nel) return;   // whole warp
  CPSm<DIM, KRON>& s = sm[warp];
  const Geo& geo = p.geo;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const int64_t nh = geo.nel * NIP;
  fill_elem<DIM, KRON>(s.e, geo, p.rule, el, q, 32);
  if (q < NEN) {
    const int node = geo.conn[el * NEN + q];
    for (int c = 0; c < NC; ++c) s.U[c][q] = p.su.cur[cdof(dm, ukind<DIM>(c), node)];
    s.Ph[q] = p.sp.cur[cdof(dm, IFEM_DOF_PHASE, node)];
    s.T[q] = mo.hasT ? p.sT.cur[cdof(dm, IFEM_DOF_T, node)] : 0.0;
  }
  __syncwarp();
  unsigned its = 0, capped = 0, bad = 0;
  if (q < NIP) {
    IpGeo<DIM> g;
    ip_geometry<DIM, KRON>(s.e, p.rule, q, g);
    const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
    PtMat M;
    double eps[18], phi, Tip;
    coss_strain<DIM, KRON>(s, p.rule, g, q, m.l_coss, eps, phi, Tip);
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    CossMat c;
    coss_mat(m, M, c);
    const int64_t hi = el * NIP + q;
    double epl[18], eplO[18], hist[4] = {0, 0, 0, 0}, histO[4] = {0, 0, 0, 0};
    for (int r = 0; r < 18; ++r) { epl[r] = p.h.EP[r * nh + hi]; eplO[r] = p.h.EPo[r * nh + hi]; }
    if (p.mh == 4) for (int k = 0; k < 4; ++k) { hist[k] = p.h.MH[k * nh + hi]; histO[k] = p.h.MHo[k * nh + hi]; }
    double* Co = p.Cc + hi * 324;   // first DPlast of the return map, then w (Dam D_d + D_u) DPlast
    double diss = 0, damdiss = 0;
    bool ident = true;
    if (c.rheo != IFEM_RHEO_LE && !(phi > c.phi_lim)) {   // UpdatePlasticStrains (CosseratMaterial.cpp:450-514)
      double dam = 1.0, u1, u2;
      if (c.rheo == IFEM_RHEO_DVEP) damage_function(fmin(1.0, fmax(0.0, phi)), mo.dam_f, mo.k0, mo.porder_p, dam, u1, u2);
      CossRM ro{0, 0, 0};
      coss_return_map(c, dam, p.dt, eps, eplO, epl, hist, histO, Co, diss, damdiss, mo.rm_tol_mode == IFEM_RM_TIGHT, ro);
      its = ro.iters; capped = ro.capped; bad |= ro.singular;
      ident = false;
    } else {
      for (int r = 0; r < 18; ++r) epl[r] = eplO[r];
    }
    for (int r = 0; r < 18; ++r) p.h.EP[r * nh + hi] = epl[r];
    p.h.VD[hi] = p.h.VDo[hi] + diss * p.dt;
    p.h.DVD[hi] = p.h.DVDo[hi] + damdiss * p.dt;
    if (p.mh == 4) for (int k = 0; k < 4; ++k) p.h.MH[k * nh + hi] = hist[k];
    double Dam, dDam, u3;
    damage_function(phi, mo.dam_f, mo.k0, mo.porder_p, Dam, dDam, u3);
    double ee[18];
    for (int r = 0; r < 18; ++r) ee[r] = eps[r] - epl[r];
    double Dd[324], Du[324], Sd[18], Su[18];
    coss_split(c, ee, Dd, Du, Sd, Su, true);
    const double w = g.w;
    double* So = p.Sc + hi * 18;
    for (int r = 0; r < 18; ++r) { So[r] = w * (Dam * Sd[r] + Su[r]); if (!isfinite(So[r])) bad = 1; }
    if (ident) {
      for (int i = 0; i < 324; ++i) Co[i] = w * (Dam * Dd[i] + Du[i]);
    } else {
      // column j of (Dam D_d + D_u) DPlast needs column j of DPlast only, so it overwrites it in place
      for (int j = 0; j < 18; ++j) {
        double x[18];
        for (int k = 0; k < 18; ++k) x[k] = Co[k * 18 + j];
        for (int i = 0; i < 18; ++i) {
          double v = 0;
          for (int k = 0; k < 18; ++k) v += (Dam * Dd[i * 18 + k] + Du[i * 18 + k]) * x[k];
          Co[i * 18 + j] = w * v;
        }
      }
    }
  }
  const unsigned ti = __reduce_add_sync(0xffffffffu, its), tc = __reduce_add_sync(0xffffffffu, capped),
                 tb = __reduce_add_sync(0xffffffffu, bad);
  if (q == 0) {
    if (ti) atomicAdd(&p.stats[0], (unsigned long long)ti);
    if (tc) atomicAdd(&p.stats[1], (unsigned long long)tc);
    if (tb) atomicAdd(&p.stats[2], (unsigned long long)tb);
  }
}


template <int DIM, bool KRON>
struct CESm {
  static constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, NC = coss_nc(DIM), NG = DIM + 1;
  ElemSm<DIM, KRON> e;
  IpGeo<DIM> g[NIP];
  double bas[NIP][NG][NEN];          // G_0 .. G_{DIM-1}, N per ip and node
  double E[NIP][NC][NC][NG][NG];     // B^T (w C) B of each ip in basis-kind form
  double U[NC][NEN], dU[NC][NEN], ddU[NC][NEN], Ph[NEN];
  double DamI[NIP], DamG[NIP];
  double WLI[NEN], WLG[NEN];
};

// CossPhaseField::Assemble_U element sums (CossPhaseField.cpp:392-531).  Entry (c a, d b) of K_e is
// sum_q sum_{k,m} E_q[c][d][k][m] g_k(a) g_m(b), with E_q the ip's tangent contracted with the structure of B.
template <int DIM, bool KRON, typename KT>
__global__ void __launch_bounds__(128) k_coss_elem(const CossParams p) {
  using S = CESm<DIM, KRON>;
  constexpr int NEN = S::NEN, NIP = S::NIP, NC = S::NC, NG = S::NG, NU = NC * NEN;
  extern __shared__ __align__(16) unsigned char smraw[];
  S& s = *reinterpret_cast<S*>(smraw);
  const int64_t el = blockIdx.x;
  const int t = threadIdx.x;
  const Geo& geo = p.geo;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
  fill_elem<DIM, KRON>(s.e, geo, p.rule, el, t, blockDim.x);
  if (t < NEN) {
    const int node = geo.conn[el * NEN + t];
    for (int c = 0; c < NC; ++c) {
      const int d = cdof(dm, ukind<DIM>(c), node);
      s.U[c][t] = p.su.cur[d]; s.dU[c][t] = p.su.d[d]; s.ddU[c][t] = p.su.dd[d];
    }
    s.Ph[t] = p.sp.cur[cdof(dm, IFEM_DOF_PHASE, node)];
  }
  __syncthreads();
  if (t < NIP) ip_geometry<DIM, KRON>(s.e, p.rule, t, s.g[t]);
  __syncthreads();
  for (int i = t; i < NIP * NEN; i += blockDim.x) {
    const int q = i / NEN, a = i % NEN;
    double N, G[DIM];
    shape_at<DIM, KRON>(s.e, p.rule, s.g[q], q, a, N, G);
    for (int d = 0; d < DIM; ++d) s.bas[q][d][a] = G[d];
    s.bas[q][DIM][a] = N;
  }
  // E_q for every ip from the ip tangents
  for (int i = t; i < NIP * NC * NC * NG * NG; i += blockDim.x) {
    const int q = i / (NC * NC * NG * NG), rem = i % (NC * NC * NG * NG);
    const int c = rem / (NC * NG * NG), d = (rem / (NG * NG)) % NC, k = (rem / NG) % NG, mm = rem % NG;
    const double* Cq = p.Cc + (el * NIP + q) * 324;
    double v = 0;
    for (int x = 0; x < 5; ++x) {
      const BEnt b1 = bent<DIM>(c, x);
      if (b1.row < 0 || b1.kind != k) continue;
      const double c1 = b1.coef == 2.0 ? m.l_coss : b1.coef;
      for (int y = 0; y < 5; ++y) {
        const BEnt b2 = bent<DIM>(d, y);
        if (b2.row < 0 || b2.kind != mm) continue;
        const double c2 = b2.coef == 2.0 ? m.l_coss : b2.coef;
        v += c1 * c2 * Cq[b1.row * 18 + b2.row];
      }
    }
    s.E[q][c][d][k][mm] = v;
  }
  __syncthreads();
  if (t < NIP) {
    double phi = 0;
    for (int a = 0; a < NEN; ++a) phi += s.bas[t][DIM][a] * s.Ph[a];
    double D, dD, ddD;
    damage_function(phi, mo.dens_f, mo.k0, mo.porder_p, D, dD, ddD);
    s.DamI[t] = D;
    damage_function(phi, mo.grav_f, mo.k0, mo.porder_p, D, dD, ddD);
    s.DamG[t] = D;
  }
  __syncthreads();
  if (t < NEN) {   // lumped weights, ips in order
    double wi = 0, wg = 0;
    for (int q = 0; q < NIP; ++q) {
      const double wN = s.g[q].w * s.bas[q][DIM][t];
      wi += wN * s.DamI[q];
      wg += wN * (1.0 - 0.0) * s.DamG[q];
    }
    s.WLI[t] = wi; s.WLG[t] = wg;
  }
  __syncthreads();
  // lumped inertia, damping and gravity (CossPhaseField.cpp:455-526) of component c at node n; in 3D the
  // tangent of the ox and oy inertia terms uses the density, as the reference's
  const double rho = m.density, lc = m.l_coss, rhoC = 2 * lc * lc * rho / (1 + m.nu), dmp = m.damping;
  auto lumped = [&](int c, int n, double& f, double& k) {
    const double W = s.WLI[n];
    f = 0; k = 0;
    const bool rot = c >= DIM;
    if (mo.inertia) {
      f += W * (rot ? rhoC : rho) * s.ddU[c][n];
      k += W * ((rot && c == NC - 1) ? rhoC : rho) * p.ddu_dt;
    }
    if (dmp > 0.0) {
      const double dr = rot ? 2 * lc * lc * dmp : dmp;
      f += W * dr * s.dU[c][n]; k += W * dr * p.du_dt;
    }
    if (!rot) f += -s.WLG[n] * rho * mo.g[c];
  };
  const int64_t hi0 = el * NIP;
  for (int i = t; i < NU; i += blockDim.x) {   // residual rows, ips in order
    const int c = i / NEN, a = i % NEN;
    double F = 0;
    for (int q = 0; q < NIP; ++q) {
      const double* Sq = p.Sc + (hi0 + q) * 18;
      for (int k = 0; k < 5; ++k) {
        const BEnt b = bent<DIM>(c, k);
        if (b.row < 0) continue;
        const double cf = b.coef == 2.0 ? m.l_coss : b.coef;
        F += cf * s.bas[q][b.kind][a] * Sq[b.row];
      }
    }
    double f, k;
    lumped(c, a, f, k);
    p.Fe[el * NU + i] = F + f;
  }
  KT* Ke = reinterpret_cast<KT*>(p.Ke) + el * NEN * ke_block(NC, NEN);
  for (int i = t; i < NU * NU; i += blockDim.x) {
    const int r = i / NU, col = i % NU;
    const int c = r / NEN, a = r % NEN, d = col / NEN, b = col % NEN;
    double v = 0;
    for (int q = 0; q < NIP; ++q) {
      double u = 0;
      for (int k = 0; k < NG; ++k) {
        const double ga = s.bas[q][k][a];
        double w2 = 0;
        for (int mm = 0; mm < NG; ++mm) w2 += s.E[q][c][d][k][mm] * s.bas[q][mm][b];
        u += ga * w2;
      }
      v += u;
    }
    if (r == col) { double f, k; lumped(c, a, f, k); v += k; }
    Ke[a * ke_block(NC, NEN) + (c * NC + d) * NEN + b] = (KT)v;
  }
}

template <int DIM, bool KRON>
struct CESmE {
  static constexpr int NEN = ElemTraits<DIM>::NEN, NC = coss_nc(DIM);
  CPSm<DIM, KRON> b;
  double dU[NC][NEN];
};

// CossPhaseField::Assemble_Phase, the driving energy (CossPhaseField.cpp:670-701): Cosserat split of the elastic
// strain, zero while t < 0, history maximum for Hist irreversibility; and |N_uu dU|^2 of the inertia term
template <int DIM, bool KRON>
__global__ void __launch_bounds__(128) k_coss_energy(const CossParams p) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, NC = coss_nc(DIM);
  extern __shared__ __align__(16) unsigned char smraw[];
  CESmE<DIM, KRON>* sm = reinterpret_cast<CESmE<DIM, KRON>*>(smraw);
  const int warp = threadIdx.x >> 5, q = threadIdx.x & 31;
  const int64_t el = (int64_t)blockIdx.x * kCWarps + warp;
  if (el >= p.geo.nel) return;
  CESmE<DIM, KRON>& s = sm[warp];
  const Geo& geo = p.geo;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const int64_t nh = geo.nel * NIP;
  fill_elem<DIM, KRON>(s.b.e, geo, p.rule, el, q, 32);
  if (q < NEN) {
    const int node = geo.conn[el * NEN + q];
    for (int c = 0; c < NC; ++c) {
      const int d = cdof(dm, ukind<DIM>(c), node);
      s.b.U[c][q] = p.su.cur[d];
      s.dU[c][q] = p.su.d[d];
    }
    s.b.Ph[q] = p.sp.cur[cdof(dm, IFEM_DOF_PHASE, node)];
    // the phase step reads the T state at DOF 0 for every node when RefCompatPhaseT is on (CossPhaseField.cpp:615)
    s.b.T[q] = mo.hasT ? (mo.ref_compat_T ? p.sT.cur[0] : p.sT.cur[cdof(dm, IFEM_DOF_T, node)]) : 0.0;
  }
  __syncwarp();
  if (q < NIP) {
    IpGeo<DIM> g;
    ip_geometry<DIM, KRON>(s.b.e, p.rule, q, g);
    const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
    double eps[18], phi, Tip;
    coss_strain<DIM, KRON>(s.b, p.rule, g, q, m.l_coss, eps, phi, Tip);
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    CossMat c;
    coss_mat(m, M, c);
    const int64_t hi = el * NIP + q;
    for (int r = 0; r < 18; ++r) eps[r] -= p.h.EP[r * nh + hi];
    double Sd[18], Su[18];
    double Energy = coss_split(c, eps, nullptr, nullptr, Sd, Su, false);
    if (p.t < 0.0) Energy = 0.0;   // initialisation period
    if (mo.irr == IFEM_IRR_HIST) {
      const double Eo = p.h.EHo[hi];
      if (Eo > Energy) { p.h.EH[hi] = Eo; Energy = Eo; }
      else p.h.EH[hi] = Energy;
    } else {
      p.h.EH[hi] = Energy;
    }
    p.Ec[hi] = Energy;
    double v2 = 0;
    for (int cc = 0; cc < NC; ++cc) {
      double v = 0;
      for (int a = 0; a < NEN; ++a) {
        double N, G[DIM];
        shape_at<DIM, KRON>(s.b.e, p.rule, g, q, a, N, G);
        v += N * s.dU[cc][a];
      }
      v2 += v * v;
    }
    p.V2c[hi] = v2;
  }
}

// Gather of steps with more than 3 components per node: one warp per (node r, component b1) owns that CSR row,
// accumulates the row blocks (b1, b2, a2) of r's incident elements in ascending element order in shared memory,
// and adds the element residual entries in the same order.
constexpr int kRWarps = 8;
template <int NC, int NEN, typename KT, typename VT, typename MT>
__global__ void __launch_bounds__(256) k_gather_rows(const GParams p) {
  constexpr int KB = ke_block(NC, NEN);
  extern __shared__ __align__(16) double racc[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kRWarps + warp;
  const int64_t r = p.node0 + w / NC;
  const int b1 = (int)(w % NC);
  if (r >= p.n_nodes) return;
  double* acc = racc + warp * p.acc_stride;
  const int deg = p.nbr_ptr[r + 1] - p.nbr_ptr[r];
  const int rowlen = NC * deg;
  const bool withK = p.Ke != nullptr;
  if (withK) for (int i = lane; i < rowlen; i += 32) acc[i] = 0.0;
  __syncwarp();
  double fsum = 0.0;
  const MT* emap = reinterpret_cast<const MT*>(p.emap);
  for (int k = p.inc_ptr[r]; k < p.inc_ptr[r + 1]; ++k) {
    const int64_t e = p.inc_el[k];
    const int a1 = p.inc_loc[k];
    if (lane == 0) {
      if (p.Fe1) fsum += p.Fe1[e * NC * NEN + b1 * NEN + a1];
    }
    if (withK) {
      const KT* blk = reinterpret_cast<const KT*>(p.Ke) + (e * NEN + a1) * KB + b1 * NC * NEN;
      const MT* em = emap + (e * NEN + a1) * NEN;
      for (int i = lane; i < NC * NEN; i += 32) {
        const int b2 = i / NEN, a2 = i % NEN;
        acc[p.blk_pos[b2] * deg + (int)em[a2]] += (double)blk[i];
      }
      __syncwarp();
    }
  }
  if (p.Fe2 && lane == 0)   // a second residual source, summed after the first over all elements
    for (int k = p.inc_ptr[r]; k < p.inc_ptr[r + 1]; ++k) fsum += p.Fe2[(int64_t)p.inc_el[k] * NC * NEN + b1 * NEN + p.inc_loc[k]];
  const int64_t row = p.row_base[b1] + r;
  if (lane == 0) p.f[row] = fsum;
  if (withK) {
    VT* vals = reinterpret_cast<VT*>(p.vals) + p.rowptr[row];
    for (int i = lane; i < rowlen; i += 32) vals[i] = (VT)acc[i];
  }
}

template <int NC, int NEN, typename KT, typename VT>
void gather_rows_go(const GParams& p, cudaStream_t s) {
  const int64_t rows = (p.n_nodes - p.node0) * NC;
  const unsigned blocks = (unsigned)((rows + kRWarps - 1) / kRWarps);
  const size_t smem = (size_t)kRWarps * p.acc_stride * sizeof(double);
  if (p.emap16) {
    auto k = k_gather_rows<NC, NEN, KT, VT, uint16_t>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<blocks, 32 * kRWarps, smem, s>>>(p);
  } else {
    auto k = k_gather_rows<NC, NEN, KT, VT, uint8_t>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<blocks, 32 * kRWarps, smem, s>>>(p);
  }
}

template <int DIM, bool KRON>
void coss_u_go(const CossParams& p, cudaStream_t s) {
  const unsigned blocks = (unsigned)((p.geo.nel + kCWarps - 1) / kCWarps);
  const size_t smem = sizeof(CPSm<DIM, KRON>) * kCWarps;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_coss_points<DIM, KRON>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_coss_points<DIM, KRON><<<blocks, 32 * kCWarps, smem, s>>>(p);
  const size_t es = sizeof(CESm<DIM, KRON>);
  if (p.ke_f32) {
    if (es > 48 * 1024) cudaFuncSetAttribute(k_coss_elem<DIM, KRON, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)es);
    k_coss_elem<DIM, KRON, float><<<(unsigned)p.geo.nel, 128, es, s>>>(p);
  } else {
    if (es > 48 * 1024) cudaFuncSetAttribute(k_coss_elem<DIM, KRON, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)es);
    k_coss_elem<DIM, KRON, double><<<(unsigned)p.geo.nel, 128, es, s>>>(p);
  }
}

template <int DIM, bool KRON>
void coss_energy_go(const CossParams& p, cudaStream_t s) {
  const unsigned blocks = (unsigned)((p.geo.nel + kCWarps - 1) / kCWarps);
  const size_t smem = sizeof(CESmE<DIM, KRON>) * kCWarps;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_coss_energy<DIM, KRON>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_coss_energy<DIM, KRON><<<blocks, 32 * kCWarps, smem, s>>>(p);
}

}  // namespace

void launch_coss_u(const CossParams& p, cudaStream_t s) {
  if (p.geo.nel <= 0) return;
  if (p.geo.dim == 2) { if (p.geo.kron) coss_u_go<2, true>(p, s); else coss_u_go<2, false>(p, s); }
  else { if (p.geo.kron) coss_u_go<3, true>(p, s); else coss_u_go<3, false>(p, s); }
}

void launch_gather_rows(const GParams& p, cudaStream_t s) {
  if (p.nc != 6 || p.nen != 27) return;   // the 3D Cosserat u-step is the only such step
  if (p.ke_f32) {
    if (p.vals_f32) gather_rows_go<6, 27, float, float>(p, s); else gather_rows_go<6, 27, float, double>(p, s);
  } else {
    if (p.vals_f32) gather_rows_go<6, 27, double, float>(p, s); else gather_rows_go<6, 27, double, double>(p, s);
  }
}

void launch_coss_energy(const CossParams& p, cudaStream_t s) {
  if (p.geo.nel <= 0) return;
  if (p.geo.dim == 2) { if (p.geo.kron) coss_energy_go<2, true>(p, s); else coss_energy_go<2, false>(p, s); }
  else { if (p.geo.kron) coss_energy_go<3, true>(p, s); else coss_energy_go<3, false>(p, s); }
}

}  // namespace ifem
