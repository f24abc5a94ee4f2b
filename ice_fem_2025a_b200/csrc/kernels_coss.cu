// Fracture/CossPhaseField (CossPhaseField.cpp:337-800) on the device, 2D (ux, uy, oz per node).
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

// B_coss entries per displacement component c: (strain row, basis kind, coefficient); kind 0..DIM-1 is the
// gradient component, DIM the shape value; coefficient 2 stands for l_coss.  2D components: ux, uy, oz.
struct BEnt { int row, kind; double coef; };
__constant__ BEnt kB2[3][4] = {
    {{0, 0, 1.0}, {4, 1, 1.0}, {-1, 0, 0.0}, {-1, 0, 0.0}},
    {{1, 1, 1.0}, {3, 0, 1.0}, {-1, 0, 0.0}, {-1, 0, 0.0}},
    {{3, 2, -1.0}, {4, 2, 1.0}, {14, 0, 2.0}, {16, 1, 2.0}},
};
__host__ __device__ constexpr int coss_nc(int dim) { return dim == 2 ? 3 : 6; }
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
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 4; ++k) {
        const BEnt b = kB2[c][k];
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
    const int kinds[3] = {IFEM_DOF_UX, IFEM_DOF_UY, IFEM_DOF_OZ};
    for (int c = 0; c < NC; ++c) s.U[c][q] = p.su.cur[cdof(dm, kinds[c], node)];
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
    double DPl[324], diss = 0, damdiss = 0;
    bool ident = true;
    if (c.rheo != IFEM_RHEO_LE && !(phi > c.phi_lim)) {   // UpdatePlasticStrains (CosseratMaterial.cpp:450-514)
      double dam = 1.0, u1, u2;
      if (c.rheo == IFEM_RHEO_DVEP) damage_function(fmin(1.0, fmax(0.0, phi)), mo.dam_f, mo.k0, mo.porder_p, dam, u1, u2);
      CossRM ro{0, 0, 0};
      coss_return_map(c, dam, p.dt, eps, eplO, epl, hist, histO, DPl, diss, damdiss, mo.rm_tol_mode == IFEM_RM_TIGHT, ro);
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
    double* Co = p.Cc + hi * 324;
    for (int i = 0; i < 18; ++i)
      for (int j = 0; j < 18; ++j) {
        double v;
        if (ident) v = Dam * Dd[i * 18 + j] + Du[i * 18 + j];
        else {
          v = 0;
          for (int k = 0; k < 18; ++k) v += (Dam * Dd[i * 18 + k] + Du[i * 18 + k]) * DPl[k * 18 + j];
        }
        Co[i * 18 + j] = w * v;
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
  double U[NC][NEN], dU[NC][NEN], ddU[NC][NEN], Ph[NEN];
  double DamI[NIP], DamG[NIP];
  double E[NC][NC][NG][NG];          // B^T C B of one ip in basis-kind form
  double WLI[NEN], WLG[NEN];
};

// CossPhaseField::Assemble_U element sums (CossPhaseField.cpp:392-531)
template <int DIM, bool KRON, typename KT>
__global__ void __launch_bounds__(128) k_coss_elem(const CossParams p) {
  using S = CESm<DIM, KRON>;
  constexpr int NEN = S::NEN, NIP = S::NIP, NC = S::NC, NG = S::NG, NU = NC * NEN;
  __shared__ S s;
  const int64_t el = blockIdx.x;
  const int t = threadIdx.x;
  const Geo& geo = p.geo;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
  fill_elem<DIM, KRON>(s.e, geo, p.rule, el, t, blockDim.x);
  if (t < NEN) {
    const int node = geo.conn[el * NEN + t];
    const int kinds[3] = {IFEM_DOF_UX, IFEM_DOF_UY, IFEM_DOF_OZ};
    for (int c = 0; c < NC; ++c) {
      const int d = cdof(dm, kinds[c], node);
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
  const int64_t hi0 = el * NIP;
  // residual rows and lumped weights, ips in order
  double Fr[(NU + 127) / 128];
  for (int j = 0; j < (NU + 127) / 128; ++j) {
    const int i = t + 128 * j;
    double F = 0;
    if (i < NU) {
      const int c = i / NEN, a = i % NEN;
      for (int q = 0; q < NIP; ++q) {
        const double* Sq = p.Sc + (hi0 + q) * 18;
        for (int k = 0; k < 4; ++k) {
          const BEnt b = kB2[c][k];
          if (b.row < 0) continue;
          const double cf = b.coef == 2.0 ? m.l_coss : b.coef;
          F += cf * s.bas[q][b.kind][a] * Sq[b.row];
        }
      }
    }
    Fr[j] = F;
  }
  if (t < NEN) {
    double wi = 0, wg = 0;
    for (int q = 0; q < NIP; ++q) {
      const double wN = s.g[q].w * s.bas[q][DIM][t];
      wi += wN * s.DamI[q];
      wg += wN * (1.0 - 0.0) * s.DamG[q];
    }
    s.WLI[t] = wi; s.WLG[t] = wg;
  }
  // tangent: entries (c a, d b) = sum_q sum_{k,m} E_q[c][d][k][m] g_k[a] g_m[b]
  constexpr int NE = NU * NU, PER = (NE + 127) / 128;
  double acc[PER];
  for (int j = 0; j < PER; ++j) acc[j] = 0.0;
  for (int q = 0; q < NIP; ++q) {
    __syncthreads();
    const double* Cq = p.Cc + (hi0 + q) * 324;
    for (int i = t; i < NC * NC * NG * NG; i += blockDim.x) {
      const int c = i / (NC * NG * NG), d = (i / (NG * NG)) % NC, k = (i / NG) % NG, mm = i % NG;
      double v = 0;
      for (int x = 0; x < 4; ++x) {
        const BEnt b1 = kB2[c][x];
        if (b1.row < 0 || b1.kind != k) continue;
        const double c1 = b1.coef == 2.0 ? m.l_coss : b1.coef;
        for (int y = 0; y < 4; ++y) {
          const BEnt b2 = kB2[d][y];
          if (b2.row < 0 || b2.kind != mm) continue;
          const double c2 = b2.coef == 2.0 ? m.l_coss : b2.coef;
          v += c1 * c2 * Cq[b1.row * 18 + b2.row];
        }
      }
      s.E[c][d][k][mm] = v;
    }
    __syncthreads();
    for (int j = 0; j < PER; ++j) {
      const int i = t + 128 * j;
      if (i >= NE) break;
      const int r = i / NU, col = i % NU;
      const int c = r / NEN, a = r % NEN, d = col / NEN, b = col % NEN;
      double v = 0;
      for (int k = 0; k < NG; ++k) {
        const double ga = s.bas[q][k][a];
        if (ga == 0.0) continue;
        double u = 0;
        for (int mm = 0; mm < NG; ++mm) u += s.E[c][d][k][mm] * s.bas[q][mm][b];
        v += ga * u;
      }
      acc[j] += v;
    }
  }
  __syncthreads();
  // lumped inertia, damping and gravity (CossPhaseField.cpp:455-526): node n's rows n (ux), ny (uy), oz
  const double rho = m.density, lc = m.l_coss, rhoC = 2 * lc * lc * rho / (1 + m.nu), dmp = m.damping;
  auto lumped = [&](int c, int n, double& f, double& k) {
    const double W = s.WLI[n];
    f = 0; k = 0;
    if (mo.inertia) {
      const double r = c < 2 ? rho : rhoC;
      f += W * r * s.ddU[c][n]; k += W * r * p.ddu_dt;
    }
    if (dmp > 0.0) {
      const double dr = c < 2 ? dmp : 2 * lc * lc * dmp;
      f += W * dr * s.dU[c][n]; k += W * dr * p.du_dt;
    }
    if (c < 2) f += -s.WLG[n] * rho * mo.g[c];
  };
  for (int j = 0; j < (NU + 127) / 128; ++j) {
    const int i = t + 128 * j;
    if (i >= NU) break;
    const int c = i / NEN, n = i % NEN;
    double f, k;
    lumped(c, n, f, k);
    p.Fe[el * NU + i] = Fr[j] + f;
  }
  KT* Ke = reinterpret_cast<KT*>(p.Ke) + el * NEN * ke_block(NC, NEN);
  for (int j = 0; j < PER; ++j) {
    const int i = t + 128 * j;
    if (i >= NE) break;
    const int r = i / NU, col = i % NU;
    const int c = r / NEN, a = r % NEN, d = col / NEN, b = col % NEN;
    double v = acc[j];
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
    const int kinds[3] = {IFEM_DOF_UX, IFEM_DOF_UY, IFEM_DOF_OZ};
    for (int c = 0; c < NC; ++c) {
      const int d = cdof(dm, kinds[c], node);
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

template <int DIM, bool KRON>
void coss_u_go(const CossParams& p, cudaStream_t s) {
  const unsigned blocks = (unsigned)((p.geo.nel + kCWarps - 1) / kCWarps);
  const size_t smem = sizeof(CPSm<DIM, KRON>) * kCWarps;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_coss_points<DIM, KRON>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_coss_points<DIM, KRON><<<blocks, 32 * kCWarps, smem, s>>>(p);
  if (p.ke_f32) k_coss_elem<DIM, KRON, float><<<(unsigned)p.geo.nel, 128, 0, s>>>(p);
  else k_coss_elem<DIM, KRON, double><<<(unsigned)p.geo.nel, 128, 0, s>>>(p);
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
  if (p.geo.kron) coss_u_go<2, true>(p, s); else coss_u_go<2, false>(p, s);
}

void launch_coss_energy(const CossParams& p, cudaStream_t s) {
  if (p.geo.nel <= 0) return;
  if (p.geo.kron) coss_energy_go<2, true>(p, s); else coss_energy_go<2, false>(p, s);
}

}  // namespace ifem
