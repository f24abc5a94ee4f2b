// Element-assembly kernels for sm_100a.
//
//   k_u_points   FP64 U-step integration points (PhaseField.cpp:382-435, SolidMaterial.cpp:123-301):
//                one warp per 3D element (lane = integration point), three 2D elements per warp.
//                Writes history, the element residual (per-node sums over ips in ip order, i.e. a
//                lane-per-node transpose through shared memory instead of a shuffle tree so the
//                summation order is the reference's), lumped weights and the per-ip material
//                tangent C_q = w (g D+ + D-) DPlast.
//   k_u_tangent  K_e = sum_q B_q^T C_q B_q (PhaseField.cpp:422) in FP32 or FP64 on CUDA cores,
//                one CTA per 3D element; each thread owns one (node a1, comp b1, comp b2) row of
//                27 columns; staged through shared memory for coalesced stores.
//   k_phase      FP64 phase step (PhaseField.cpp:541-712): residual + tangent + history max.
//   k_thermal    thermal model (ThermalModel.cpp:94-133) and viscous heating (PhaseField.cpp:748-767).
//   k_gather     deterministic scatter: one warp per mesh node owns that node's CSR rows and adds
//                the contributions of its incident elements in ascending element order, the
//                order in which serial MatSetValues/VecSetValues(ADD_VALUES) accumulates them.
//
// No kernel spins or traps; every loop is bounded (the return map by rm_max_it).

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <type_traits>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

__device__ __forceinline__ int elem_mat(const Geo& g, int64_t el) { return g.emat ? g.emat[el] : 0; }

__device__ __forceinline__ int dof_of(const DofMap& dm, int kind, int node) {
  return dm.base[kind] + dm.node_rank[node];
}

// ============================================================================================
// U step: integration points (FP64)
// ============================================================================================
template <int DIM, bool KRON>
struct USm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, KRON> e;
  double U[DIM][NEN];
  double UO[DIM][NEN];
  double Ph[NEN];
  double PhO[NEN];
  double T[NEN];
  IpGeo<DIM> g[NEN];
  double sw[NEN][6];
};

constexpr int kUWarps = 4;

// VEP: the variant for contexts with a viscoelastic-plastic material set or a DruckerPrager / SpecStrains split
// (full 6x6 return-map and split tangents)
// SPL, NI, DAMF >= 0 / > 0: energy split, integral creep exponent and degradation function fixed at compile time
// (every material set shares them; the same arithmetic as the run-time selection, in less code)
template <int DIM, bool KRON, typename CT, bool CONS, bool VEP, int SPL = -1, int NI = 0, int DAMF = -1>
__global__ void __launch_bounds__(128) k_u_points(const UParams p) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  USm<DIM, KRON>* sm = reinterpret_cast<USm<DIM, KRON>*>(smraw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP;
  const int q = lane - sub * NIP;
  const int64_t el = p.geo.el0 + ((int64_t)blockIdx.x * kUWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < p.geo.el1);
  USm<DIM, KRON>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
  const Geo& geo = p.geo;
  const int64_t nh = geo.nel * NIP;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const bool expl_rheo = true;

  if (act) {
    fill_elem<DIM, KRON>(s.e, geo, p.rule, el, q, NIP);
    const int a = q;
    const int node = geo.conn[el * NEN + a];
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      const int d = dof_of(dm, IFEM_DOF_UX + b, node);
      s.U[b][a] = p.su.cur[d];
      s.UO[b][a] = p.su.old[d];
    }
    const int dph = dof_of(dm, IFEM_DOF_PHASE, node);
    s.Ph[a] = p.sp.cur[dph];
    s.PhO[a] = p.sp.old[dph];
    s.T[a] = mo.hasT ? p.sT.cur[dof_of(dm, IFEM_DOF_T, node)] : 0.0;
  }
  __syncwarp();

  unsigned it_count = 0, capped = 0, bad = 0;
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, KRON>(s.e, p.rule, q, g);
    s.g[q] = g;
    if (DIM == 3 && p.geoq) {
      float* gq = p.geoq + el * kTcGeo + q;
#pragma unroll
      for (int i = 0; i < DIM * DIM; ++i) gq[i * 27] = (float)g.Jinv[i];
      gq[9 * 27] = (float)g.wFun;
#pragma unroll
      for (int d = 0; d < DIM; ++d) gq[(10 + d) * 27] = (float)g.dW[d];
    }
    double eps[6] = {0, 0, 0, 0, 0, 0}, epsO[6] = {0, 0, 0, 0, 0, 0};
    double phi = 0, phiO = 0, Tip = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, KRON>(s.e, p.rule, g, q, a, N, G);
      phi += N * s.Ph[a];
      phiO += N * s.PhO[a];
      Tip += N * s.T[a];
      if (DIM == 2) {
        const double ux = s.U[0][a], uy = s.U[1][a];
        eps[0] += G[0] * ux; eps[1] += G[1] * uy; eps[3] += G[1] * ux + G[0] * uy;
        if (expl_rheo) {
          const double ox = s.UO[0][a], oy = s.UO[1][a];
          epsO[0] += G[0] * ox; epsO[1] += G[1] * oy; epsO[3] += G[1] * ox + G[0] * oy;
        }
      } else {
        const double ux = s.U[0][a], uy = s.U[1][a], uz = s.U[DIM - 1][a];
        eps[0] += G[0] * ux; eps[1] += G[1] * uy; eps[2] += G[DIM - 1] * uz;
        eps[3] += G[1] * ux + G[0] * uy; eps[4] += G[DIM - 1] * uy + G[1] * uz; eps[5] += G[DIM - 1] * ux + G[0] * uz;
        if (expl_rheo) {
          const double ox = s.UO[0][a], oy = s.UO[1][a], oz = s.UO[DIM - 1][a];
          epsO[0] += G[0] * ox; epsO[1] += G[1] * oy; epsO[2] += G[DIM - 1] * oz;
          epsO[3] += G[1] * ox + G[0] * oy; epsO[4] += G[DIM - 1] * oy + G[1] * oz; epsO[5] += G[DIM - 1] * ox + G[0] * oz;
        }
      }
    }
    const MatDev& m = geo.mats[elem_mat(geo, el)];
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    double Dam, dDam, unused;
    damage_function<DAMF>(phi, mo.dam_f, mo.k0, mo.porder_p, Dam, dDam, unused);
    const int64_t hi = el * NIP + q;
    double epl[6], eplo[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) { epl[r] = p.h.EP[r * nh + hi]; eplo[r] = p.h.EPo[r * nh + hi]; }
    double hist0 = (M.rheo != IFEM_RHEO_LE) ? p.h.MH[hi] : 0.0;
    // tangent of the return map: identity, factored reference form, or full (consistent)
    int tkind = 0;            // 0 identity, 1 reference factored, 2 full DPl
    RMTan tan;
    constexpr bool kFull = CONS || VEP;
    double DPl[kFull ? 36 : 1];
    double diss = 0.0;
    double damdiss = 0.0;
    RMResult rr{0, false, true};
    const bool vis = (M.rheo == IFEM_RHEO_VE || M.rheo == IFEM_RHEO_DVE);
    const bool vexp = (M.rheo == IFEM_RHEO_VE_EXPL || M.rheo == IFEM_RHEO_DVE_EXPL);
    if (vis && !(phi > M.phi_lim)) {
      double dmg = 1.0, u1, u2;
      if (M.rheo == IFEM_RHEO_DVE) damage_function<DAMF>(phi, mo.dam_f, mo.k0, mo.porder_p, dmg, u1, u2);
      rr = return_mapping_viscous<NI>(M, DPl, epl, eps, eplo, dmg, p.dt, hist0, mo.rm_tol_mode, mo.rm_max_it,
                                  CONS ? IFEM_TANGENT_CONSISTENT : IFEM_TANGENT_REFERENCE, diss, CONS ? nullptr : &tan);
      tkind = CONS ? 2 : 1;
    } else if (vexp && !(phiO > M.phi_lim)) {
      double dmg = 1.0, u1, u2;
      if (M.rheo == IFEM_RHEO_DVE_EXPL) damage_function<DAMF>(phiO, mo.dam_f, mo.k0, mo.porder_p, dmg, u1, u2);
      rr = return_mapping_viscous<NI>(M, DPl, epl, epsO, eplo, dmg, p.dt, hist0, mo.rm_tol_mode, mo.rm_max_it,
                                  IFEM_TANGENT_REFERENCE, diss, &tan);   // explicit: DMat = I afterwards
    } else if (VEP && M.rheo == IFEM_RHEO_VEP && !(phiO > M.phi_lim)) {
      // SolidMaterial.cpp:174-182: damage fixed at 1; MatHist [hardening, dLambda_v, dLambda_p] in planes 0..2
      double vh[3] = {hist0, p.h.MH[nh + hi], p.h.MH[2 * nh + hi]};
      rr = return_mapping_vep(M, DPl, epl, eps, eplo, p.dt, 1.0, vh, p.h.MHo[hi], mo.rm_tol_mode, mo.rm_max_it,
                              diss, damdiss);
      hist0 = vh[0];
      p.h.MH[nh + hi] = vh[1];
      p.h.MH[2 * nh + hi] = vh[2];
      tkind = 2;
    } else {
#pragma unroll
      for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplo[r];
    }
    it_count = rr.iters;
    capped = rr.capped ? 1u : 0u;
#pragma unroll
    for (int r = 0; r < 6; ++r) p.h.EP[r * nh + hi] = epl[r];
    p.h.VD[hi] = p.h.VDo[hi] + diss * p.dt;
    p.h.DVD[hi] = p.h.DVDo[hi] + damdiss * p.dt;
    if (M.rheo != IFEM_RHEO_LE) p.h.MH[hi] = hist0;

    double ee[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) ee[r] = eps[r] - epl[r];
    double Sd[6], Su[6];
    energy_split<false, VEP, SPL>(M, ee, Sd, Su, nullptr, nullptr, false);
#pragma unroll
    for (int r = 0; r < 6; ++r) s.sw[q][r] = g.w * (Dam * Sd[r] + Su[r]);
    // C_q = w (Dam Dd + Du) DPlast with (Dam Dd + Du) = alpha 11^T + gamma VC
    double alpha, gamma;
    split_tangent<SPL>(M, ee, Dam, alpha, gamma);
    const double VC[6] = {1, 1, 1, 0.5, 0.5, 0.5};
    CT* Cq = reinterpret_cast<CT*>(p.Cq);
    // [36][nh], or element-major [nel][36][27] for the tensor-core tangent
    auto cq_at = [&](int k) -> int64_t { return p.geoq ? el * kTcCq + k * 27 + q : (int64_t)k * nh + hi; };
    if (VEP && M.ce && (M.split == IFEM_SPLIT_SPECSTRAINS || M.split == IFEM_SPLIT_DRUCKERPRAGER)) {
      // C_q = w (Dam Dd + Du) T, T the return map's tangent: I, I - a b^T / den, or DPl
      double Dd[36], Du[36], t1[6], t2[6];
      split_full(M, ee, t1, t2, Dd, Du, true);
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
          double v = 0;
          for (int k = 0; k < 6; ++k) {
            const double dt = Dam * Dd[i * 6 + k] + Du[i * 6 + k];
            const double T = tkind == 2 ? DPl[(k * 6 + j) % (kFull ? 36 : 1)]
                           : (tkind == 1 ? (k == j ? 1.0 : 0.0) - tan.a[k] * tan.b[j] / tan.den : (k == j ? 1.0 : 0.0));
            v += dt * T;
          }
          Cq[cq_at(i * 6 + j)] = (CT)(g.w * v);
        }
    } else if (tkind == 1) {
      const double sa = tan.a[0] + tan.a[1] + tan.a[2];
      double bj[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) bj[j] = tan.b[j] / tan.den;
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          const double v = (i < 3 ? alpha * ((j < 3 ? 1.0 : 0.0) - sa * bj[j]) : 0.0) +
                           gamma * VC[i] * ((i == j ? 1.0 : 0.0) - tan.a[i] * bj[j]);
          Cq[cq_at(i * 6 + j)] = (CT)(g.w * v);
        }
    } else if (kFull && tkind == 2) {
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          const double v = (i < 3 ? alpha * (DPl[(0 * 6 + j) % (kFull ? 36 : 1)] + DPl[(1 * 6 + j) % (kFull ? 36 : 1)] +
                                             DPl[(2 * 6 + j) % (kFull ? 36 : 1)])
                                  : 0.0) +
                           gamma * VC[i] * DPl[(i * 6 + j) % (kFull ? 36 : 1)];
          Cq[cq_at(i * 6 + j)] = (CT)(g.w * v);
        }
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          const double v = ((i < 3 && j < 3) ? alpha : 0.0) + (i == j ? gamma * VC[i] : 0.0);
          Cq[cq_at(i * 6 + j)] = (CT)(g.w * v);
        }
    }
    if (!rr.ok) bad = 1;
  }
  __syncwarp();

  // element residual: lane a sums node a's contribution over ips in ip order
  if (act) {
    const int a = q;
    double F[DIM], WL = 0;
#pragma unroll
    for (int b = 0; b < DIM; ++b) F[b] = 0;
    for (int qq = 0; qq < NIP; ++qq) {
      double N, G[DIM];
      shape_at<DIM, KRON>(s.e, p.rule, s.g[qq], qq, a, N, G);
      const double* S = s.sw[qq];
      if (DIM == 2) {
        F[0] += G[0] * S[0] + G[1] * S[3];
        F[1] += G[1] * S[1] + G[0] * S[3];
      } else {
        F[0] += G[0] * S[0] + G[1] * S[3] + G[DIM - 1] * S[5];
        F[1] += G[1] * S[1] + G[0] * S[3] + G[DIM - 1] * S[4];
        F[DIM - 1] += G[DIM - 1] * S[2] + G[1] * S[4] + G[0] * S[5];
      }
      WL += s.g[qq].w * N;
    }
    const MatDev& m = geo.mats[elem_mat(geo, el)];
    const int node = geo.conn[el * NEN + a];
    double DamI, dDamI, u;
    double kd = 0.0;   // lumped diagonal tangent terms of this node (PhaseField.cpp:441-468)
    if (mo.inertia) {
      damage_function(s.Ph[a], mo.dens_f, mo.k0, mo.porder_p, DamI, dDamI, u);
#pragma unroll
      for (int b = 0; b < DIM; ++b) F[b] += WL * DamI * m.density * p.su.dd[dof_of(dm, IFEM_DOF_UX + b, node)];
      kd += WL * DamI * m.density * p.ddu_dt;
    }
    if (m.damping > 0.0) {
#pragma unroll
      for (int b = 0; b < DIM; ++b) F[b] += WL * m.damping * p.su.d[dof_of(dm, IFEM_DOF_UX + b, node)];
      kd += WL * m.damping * p.du_dt;
    }
    if (p.Kd) p.Kd[el * kTcKd + a] = kd;
    double DamG, dDamG;
    damage_function(s.Ph[a], mo.dens_f, mo.k0, mo.porder_p, DamG, dDamG, u);
#pragma unroll
    for (int b = 0; b < DIM; ++b) F[b] += -WL * DamG * m.density * mo.g[b];
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      p.Fe[el * (DIM * NEN) + b * NEN + a] = F[b];
      if (!isfinite(F[b])) bad = 1;
    }
    p.WLe[el * NEN + a] = WL;
  }
  const unsigned tot_it = __reduce_add_sync(0xffffffffu, it_count);
  const unsigned tot_cap = __reduce_add_sync(0xffffffffu, capped);
  const unsigned tot_bad = __reduce_add_sync(0xffffffffu, bad);
  if (lane == 0) {
    if (tot_it) atomicAdd(&p.stats[0], (unsigned long long)tot_it);
    if (tot_cap) atomicAdd(&p.stats[1], (unsigned long long)tot_cap);
    if (tot_bad) atomicAdd(&p.stats[2], (unsigned long long)tot_bad);
  }
}

// ============================================================================================
// U step: element tangent K_e = sum_q B_q^T C_q B_q
// ============================================================================================
template <int DIM, bool KRON, typename T>
struct TSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, KRON> e;
  IpGeo<DIM> g[NEN];
  double WL[NEN];
  double Ph[NEN];
  T G[NEN][NEN][4];          // [q][a][d]
  T C[NEN][36];              // [q][ij]
  T stage[DIM * NEN * DIM * NEN];
};

template <int DIM> struct TCfg;
template <> struct TCfg<2> { static constexpr int EPC = 3, NT = 128; };
template <> struct TCfg<3> { static constexpr int EPC = 1, NT = 256; };

template <int DIM, bool KRON, typename T>
__global__ void __launch_bounds__(TCfg<DIM>::NT) k_u_tangent(const TParams p) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPC = TCfg<DIM>::EPC, NT = TCfg<DIM>::NT;
  constexpr int R = NEN * DIM * DIM;          // rows of work per element
  constexpr int KE = DIM * NEN * DIM * NEN;   // entries per element
  extern __shared__ __align__(16) unsigned char smraw[];
  TSm<DIM, KRON, T>* sm = reinterpret_cast<TSm<DIM, KRON, T>*>(smraw);
  const int t = threadIdx.x;
  const int64_t el0 = p.geo.el0 + (int64_t)blockIdx.x * EPC;
  const Geo& geo = p.geo;

  for (int sub = 0; sub < EPC; ++sub) {
    const int64_t el = el0 + sub;
    if (el >= geo.el1) break;
    fill_elem<DIM, KRON>(sm[sub].e, geo, p.rule, el, t, NT);
    for (int a = t; a < NEN; a += NT) {
      sm[sub].WL[a] = p.WLe[el * NEN + a];
      const int node = geo.conn[el * NEN + a];
      sm[sub].Ph[a] = p.phase_cur[dof_of(p.dm, IFEM_DOF_PHASE, node)];
    }
  }
  __syncthreads();
  for (int i = t; i < EPC * NIP; i += NT) {
    const int sub = i / NIP, q = i % NIP;
    const int64_t el = el0 + sub;
    if (el >= geo.el1) continue;
    ip_geometry<DIM, KRON>(sm[sub].e, p.rule, q, sm[sub].g[q]);
  }
  for (int i = t; i < EPC * NIP * 36; i += NT) {
    const int sub = i / (NIP * 36), rem = i % (NIP * 36), k = rem / NIP, q = rem % NIP;
    const int64_t el = el0 + sub;
    if (el >= geo.el1) continue;
    sm[sub].C[q][k] = reinterpret_cast<const T*>(p.Cq)[(int64_t)k * p.nh + el * NIP + q];
  }
  __syncthreads();
  for (int i = t; i < EPC * NIP * NEN; i += NT) {
    const int sub = i / (NIP * NEN), rem = i % (NIP * NEN), q = rem / NEN, a = rem % NEN;
    const int64_t el = el0 + sub;
    if (el >= geo.el1) continue;
    double N, G[DIM];
    shape_at<DIM, KRON>(sm[sub].e, p.rule, sm[sub].g[q], q, a, N, G);
#pragma unroll
    for (int d = 0; d < 4; ++d) sm[sub].G[q][a][d] = (T)(d < DIM ? G[d] : 0.0);
  }
  __syncthreads();

  const int sub = t / R, r = t % R;
  const int64_t el = el0 + sub;
  const bool act = sub < EPC && el < geo.el1;
  if (act) {
    TSm<DIM, KRON, T>& s = sm[sub];
    const int a1 = r / (DIM * DIM), b1 = (r / DIM) % DIM, b2 = r % DIM;
    int vi[DIM], vj[DIM];
#pragma unroll
    for (int pp = 0; pp < DIM; ++pp) { vi[pp] = voigt_idx(b1, pp); vj[pp] = voigt_idx(b2, pp); }
    T acc[NEN];
#pragma unroll
    for (int a2 = 0; a2 < NEN; ++a2) acc[a2] = (T)0;
    for (int q = 0; q < NIP; ++q) {
      T g1[DIM];
#pragma unroll
      for (int pp = 0; pp < DIM; ++pp) g1[pp] = s.G[q][a1][pp];
      T v[DIM];
#pragma unroll
      for (int rr = 0; rr < DIM; ++rr) {
        T sacc = (T)0;
#pragma unroll
        for (int pp = 0; pp < DIM; ++pp) sacc += g1[pp] * s.C[q][vi[pp] * 6 + vj[rr]];
        v[rr] = sacc;
      }
#pragma unroll
      for (int a2 = 0; a2 < NEN; ++a2) {
        T sacc = acc[a2];
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr) sacc += v[rr] * s.G[q][a2][rr];
        acc[a2] = sacc;
      }
    }
    double add = 0.0;   // diagonal lumped inertia / damping terms, added to entry a2 == a1
    if (b1 == b2) {
      const MatDev& m = geo.mats[elem_mat(geo, el)];
      if (p.mo.inertia) {
        double DamI, d1, d2;
        damage_function(s.Ph[a1], p.mo.dens_f, p.mo.k0, p.mo.porder_p, DamI, d1, d2);
        add += s.WL[a1] * DamI * m.density * p.ddu_dt;
      }
      if (m.damping > 0.0) add += s.WL[a1] * m.damping * p.du_dt;
    }
    // stage (stride NEN is odd -> conflict-free), then coalesced copy-out; static indices keep acc in
    // registers
#pragma unroll
    for (int a2 = 0; a2 < NEN; ++a2)
      s.stage[r * NEN + a2] = (a2 == a1 && add != 0.0) ? (T)((double)acc[a2] + add) : acc[a2];
  }
  __syncthreads();
  constexpr int RB = DIM * DIM * NEN, KB = ke_block(DIM, NEN);
  for (int sub2 = 0; sub2 < EPC; ++sub2) {
    const int64_t e2 = el0 + sub2;
    if (e2 >= geo.el1) break;
    T* dst = reinterpret_cast<T*>(p.Ke) + e2 * (NEN * KB);
    for (int i = t; i < KE; i += NT) dst[(i / RB) * KB + (i % RB)] = sm[sub2].stage[i];
  }
}

// ============================================================================================
// Phase step (FP64 points; tangent stored in T)
// ============================================================================================
template <int DIM, bool KRON, typename T>
struct PSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, KRON> e;
  double U[DIM][NEN];
  double Ph[NEN], PhO[NEN], Tn[NEN], dU[DIM][NEN];
  IpGeo<DIM> g[NEN];
  // (N, Gx, Gy, Gz) per (ip, node) in the tangent's precision; the residual recomputes in FP64
  typename std::conditional<sizeof(T) == 4, float4, double4>::type pk[NEN][NEN];
  double kNF[NEN], kGF[NEN], kNN[NEN], kGG[NEN], kLD[NEN];
  double dphi[NEN][DIM];
  double lc[NEN];
  double last_Gc, last_l, last_visc;
};

constexpr int kPWarps = 4;

template <int DIM, bool KRON, typename T, int SPL = -1, int DAMF = -1>
__global__ void __launch_bounds__(128) k_phase(const PParams p) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  using V4 = typename std::conditional<sizeof(T) == 4, float4, double4>::type;
  extern __shared__ __align__(16) unsigned char smraw[];
  PSm<DIM, KRON, T>* sm = reinterpret_cast<PSm<DIM, KRON, T>*>(smraw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP;
  const int q = lane - sub * NIP;
  const int64_t el = ((int64_t)blockIdx.x * kPWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < p.geo.nel);
  PSm<DIM, KRON, T>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
  const Geo& geo = p.geo;
  const int64_t nh = geo.nel * NIP;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  unsigned bad = 0;

  if (act) {
    fill_elem<DIM, KRON>(s.e, geo, p.rule, el, q, NIP);
    const int a = q;
    const int node = geo.conn[el * NEN + a];
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      const int d = dof_of(dm, IFEM_DOF_UX + b, node);
      s.U[b][a] = p.su.cur[d];
      s.dU[b][a] = p.su.d[d];
    }
    const int dph = dof_of(dm, IFEM_DOF_PHASE, node);
    s.Ph[a] = p.sp.cur[dph];
    s.PhO[a] = p.sp.old[dph];
    if (mo.hasT) s.Tn[a] = mo.ref_compat_T ? p.sT.cur[0] : p.sT.cur[dof_of(dm, IFEM_DOF_T, node)];
    else s.Tn[a] = 0.0;
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, KRON>(s.e, p.rule, q, g);
    s.g[q] = g;
    double phi = 0, Tip = 0, gphi[DIM], eps[6] = {0, 0, 0, 0, 0, 0}, uip[DIM], vip[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) { gphi[d] = 0; uip[d] = 0; vip[d] = 0; }
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, KRON>(s.e, p.rule, g, q, a, N, G);
      V4 v;
      v.x = (T)N; v.y = (T)G[0]; v.z = (T)G[1]; v.w = (T)(DIM == 3 ? G[DIM - 1] : 0.0);
      s.pk[q][a] = v;
#pragma unroll
      for (int d = 0; d < DIM; ++d) { gphi[d] += G[d] * s.Ph[a]; uip[d] += N * s.U[d][a]; vip[d] += N * s.dU[d][a]; }
      phi += N * s.Ph[a];
      Tip += N * s.Tn[a];
      if (DIM == 2) {
        const double ux = s.U[0][a], uy = s.U[1][a];
        eps[0] += G[0] * ux; eps[1] += G[1] * uy; eps[3] += G[1] * ux + G[0] * uy;
      } else {
        const double ux = s.U[0][a], uy = s.U[1][a], uz = s.U[DIM - 1][a];
        eps[0] += G[0] * ux; eps[1] += G[1] * uy; eps[2] += G[DIM - 1] * uz;
        eps[3] += G[1] * ux + G[0] * uy; eps[4] += G[DIM - 1] * uy + G[1] * uz; eps[5] += G[DIM - 1] * ux + G[0] * uz;
      }
    }
    const MatDev& m = geo.mats[elem_mat(geo, el)];
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    double Dam, dDam, ddDam, DamI, dDamI, ddDamI, DamG, dDamG, ddDamG;
    damage_function<DAMF>(phi, mo.dam_f, mo.k0, mo.porder_p, Dam, dDam, ddDam);
    damage_function(phi, mo.dens_f, mo.k0, mo.porder_p, DamI, dDamI, ddDamI);
    damage_function(phi, mo.grav_f, mo.k0, mo.porder_p, DamG, dDamG, ddDamG);
    const int64_t hi = el * NIP + q;
    double ee[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) ee[r] = eps[r] - p.h.EP[r * nh + hi];
    double Sd[6], Su[6];
    double Energy;
    if (p.e_in) {   // Cosserat model: split, initialisation period and history applied by k_coss_energy
      Energy = p.e_in[hi];
    } else {
      Energy = energy_split<true, true, SPL>(M, ee, Sd, Su, nullptr, nullptr, false);
      if (mo.irr == IFEM_IRR_HIST) {
        const double Eo = p.h.EHo[hi];
        if (Eo > Energy) { if (p.write_hist) p.h.EH[hi] = Eo; Energy = Eo; }
        else if (p.write_hist) p.h.EH[hi] = Energy;
      } else if (p.write_hist) p.h.EH[hi] = Energy;
    }
    // distribution function (PhaseFieldUtil.cpp:185-221): Dist_a = c (nF N_a + grad G_a.dphi)
    const double l = M.l;
    double dGdG = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) dGdG += gphi[d] * gphi[d];
    double c = 0, nF = 0, nK = 0, grad = 0, gamma = 0;
    switch (mo.dist) {
      case IFEM_DIST_QUADRATIC: c = 1.0 / (2.0 * l); gamma = c * (phi * phi + l * l * dGdG); nF = 2.0 * phi; nK = 2.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LINEAR: c = 3.0 / (8.0 * l); gamma = c * (phi + l * l * dGdG); nF = 1.0; nK = 0.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LINEAR2: c = 1.0 / (4.0 * l); gamma = c * (2.0 * phi + l * l * dGdG); nF = 2.0; nK = 0.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LOCAL: c = 1.0 / l; gamma = c * (phi * phi); nF = 2.0 * phi; nK = 2.0; grad = 0.0; break;
      case IFEM_DIST_CZM: c = 1.0 / (3.141592 * l); gamma = c * (2.0 * phi - phi * phi + l * l * dGdG); nF = 2.0 * (1.0 - phi); nK = -2.0; grad = 2.0 * l * l; break;
      default: break;
    }
    double capF = 0, capK = 0;   // DistCap_a = capF N_a, dDistCap_ab = capK N_a N_b (GetCapacityOnly)
    if (mo.lumped_cap) {
      switch (mo.dist) {
        case IFEM_DIST_QUADRATIC: capF = 1.0 / (2.0 * l) * 2.0 * phi; capK = 1.0 / (2.0 * l) * 2.0; break;
        case IFEM_DIST_CZM: capF = 1.0 / (3.141592 * l) * 2.0 * (1.0 - phi); capK = 1.0 / (3.141592 * l) * -2.0; break;
        case IFEM_DIST_LINEAR: capF = 3.0 / (8.0 * l); break;
        case IFEM_DIST_LINEAR2: capF = 1.0 / (4.0 * l) * 2.0; break;
        case IFEM_DIST_LOCAL: capF = 1.0 / l * 2 * phi; capK = 1.0 / l * 2; break;
        default: break;
      }
    }
    const double w = g.w;
    double kNF = w * M.Gc * (c * nF - capF);
    double kNN = w * M.Gc * (c * nK - capK);
    const double kG = w * M.Gc * c * grad;
    double kLD = 0;
    if (!mo.lumped_drive) { kNF += w * dDam * Energy; kNN += w * ddDam * Energy; }
    else kLD = w * Energy;
    if (mo.visco_fact > 1.0e-9) {
      double DamV, dDamV, ddDamV;
      const double PD = mo.visco_fact * p.h.DVD[hi];
      damage_function(phi, mo.visc_f, mo.k0, mo.porder_p, DamV, dDamV, ddDamV);
      kNF += w * dDamV * PD; kNN += w * ddDamV * PD;
    }
    if (mo.inertia && mo.consistent_deg) {
      double v2 = 0;
      for (int d = 0; d < DIM; ++d) v2 += vip[d] * vip[d];
      if (p.v2_in) v2 = p.v2_in[hi];   // Cosserat model: the micro-rotation rates are part of N_uu dU
      kNF += -w * 0.5 * m.density * v2 * dDamI; kNN += -w * 0.5 * m.density * v2 * ddDamI;
    }
    if (mo.consistent_deg) {
      double gu = 0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) gu += mo.g[d] * uip[d];
      kNF += -w * m.density * gu * dDamG; kNN += -w * m.density * gu * ddDamG;
    }
    s.kNF[q] = kNF; s.kGF[q] = kG; s.kNN[q] = kNN; s.kGG[q] = kG; s.kLD[q] = kLD;
#pragma unroll
    for (int d = 0; d < DIM; ++d) s.dphi[q][d] = gphi[d];
    s.lc[q] = gamma * w;
    if (q == NIP - 1) { s.last_Gc = M.Gc; s.last_l = M.l; s.last_visc = M.visc; }
  }
  __syncwarp();
  if (act) {
    const int b = q;   // lane = node b
    double F = 0, WL = 0, LD = 0;
    for (int qq = 0; qq < NIP; ++qq) {   // FP64 residual, ips in order
      double N, G[DIM];
      shape_at<DIM, KRON>(s.e, p.rule, s.g[qq], qq, b, N, G);
      double gd = 0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) gd += G[d] * s.dphi[qq][d];
      F += s.kNF[qq] * N + s.kGF[qq] * gd;
      WL += s.g[qq].w * N;
      LD += s.kLD[qq] * N;
    }
    const double Gc = s.last_Gc, l = s.last_l, visc = s.last_visc;
    const MatDev& m = geo.mats[elem_mat(geo, el)];
    double diag = 0;
    if (mo.lumped_drive) {
      double D, dD, ddD;
      damage_function<DAMF>(s.Ph[b], mo.dam_f, mo.k0, mo.porder_p, D, dD, ddD);
      F += LD * dD; diag += LD * ddD;
    }
    if (mo.lumped_cap) {
      const double ph = s.Ph[b];
      double DL = 0, dDL = 0;
      switch (mo.dist) {
        case IFEM_DIST_QUADRATIC: DL = 1.0 / l * ph; dDL = 1.0 / l; break;
        case IFEM_DIST_CZM: DL = 2.0 / (3.141592 * l) * (1.0 - ph); dDL = -2.0 / (3.141592 * l); break;
        case IFEM_DIST_LINEAR: DL = 3.0 / (8.0 * l); break;
        case IFEM_DIST_LINEAR2: DL = 1.0 / (4.0 * l); break;
        case IFEM_DIST_LOCAL: DL = 2.0 / l * ph; dDL = 2.0 / l; break;
        default: break;
      }
      F += WL * Gc * DL; diag += WL * Gc * dDL;
    }
    F += WL * visc / p.dt * (s.Ph[b] - s.PhO[b]);
    const double stab = (mo.tangent_mode == IFEM_TANGENT_CONSISTENT) ? 0.0 : mo.visc_num * Gc / l;
    diag += WL * (visc / p.dt + stab);
    if (mo.irr == IFEM_IRR_PENALTY) {
      const double ph = s.Ph[b];
      const double lim0 = fmin(1.0 - 1.0e-3, fmax(0.0, s.PhO[b])), lim1 = 1.0 + 1e-1;
      if (ph < lim0) { F += WL * m.gc_input * mo.penalty * (ph - lim0); diag += WL * m.gc_input * mo.penalty; }
      if (ph > lim1) { F += WL * m.gc_input * mo.penalty * (ph - lim1); diag += WL * m.gc_input * mo.penalty; }
    }
    p.Fe[el * NEN + b] = F;
    if (p.wl_out) p.wl_out[el * NEN + b] = WL;
    if (!isfinite(F)) bad = 1;
    // tangent column b: K_ab = sum_q kNN N_a N_b + kGG G_a . G_b  (register-blocked over a)
    T acc[NEN];
#pragma unroll
    for (int a = 0; a < NEN; ++a) acc[a] = (T)0;
    for (int qq = 0; qq < NIP; ++qq) {
      const V4 mb = s.pk[qq][b];
      const T cn = (T)s.kNN[qq], cg = (T)s.kGG[qq];
      const T bx = cn * mb.x, by = cg * mb.y, bz = cg * mb.z, bw = cg * mb.w;
#pragma unroll
      for (int a = 0; a < NEN; ++a) {
        const V4 ma = s.pk[qq][a];
        acc[a] += bx * ma.x + by * ma.y + bz * ma.z + bw * ma.w;
      }
    }
    constexpr int KB = ke_block(1, NEN);
    T* Ke = reinterpret_cast<T*>(p.Ke) + el * NEN * KB;
#pragma unroll
    for (int a = 0; a < NEN; ++a) {
      double k = (double)acc[a];
      if (a == b) k += diag;
      Ke[a * KB + b] = (T)k;
    }
    if (b == 0) {
      double lc = 0;
      for (int qq = 0; qq < NIP; ++qq) lc += s.lc[qq];
      p.lcrack_el[el] = lc;
    }
  }
  const unsigned tot_bad = __reduce_add_sync(0xffffffffu, bad);
  if (lane == 0 && tot_bad) atomicAdd(&p.stats[2], (unsigned long long)tot_bad);
}

// ============================================================================================
// T step: viscous heating residual and thermal model
// ============================================================================================
template <int DIM, bool KRON>
struct HSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, KRON> e;
  double T[NEN], dT[NEN];
  double N[NEN][NEN];
  double G[NEN][NEN][DIM];
  double w[NEN], rate[NEN], k[NEN];
  double gT[NEN][DIM];
};

constexpr int kHWarps = 2;

template <int DIM, bool KRON, typename T>
__global__ void __launch_bounds__(64) k_thermal(const ThParams p) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  HSm<DIM, KRON>* sm = reinterpret_cast<HSm<DIM, KRON>*>(smraw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP;
  const int q = lane - sub * NIP;
  const int64_t el = ((int64_t)blockIdx.x * kHWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < p.geo.nel);
  HSm<DIM, KRON>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
  const Geo& geo = p.geo;
  const int64_t nh = geo.nel * NIP;
  unsigned bad = 0;
  if (act) {
    fill_elem<DIM, KRON>(s.e, geo, p.rule, el, q, NIP);
    const int node = geo.conn[el * NEN + q];
    const int d = dof_of(p.dm, IFEM_DOF_T, node);
    s.T[q] = p.sT.cur[d];
    s.dT[q] = p.sT.d[d];
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, KRON>(s.e, p.rule, q, g);
    double gT[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) gT[d] = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, KRON>(s.e, p.rule, g, q, a, N, G);
      s.N[q][a] = N;
#pragma unroll
      for (int d = 0; d < DIM; ++d) { s.G[q][a][d] = G[d]; gT[d] += G[d] * s.T[a]; }
    }
    s.w[q] = g.w;
#pragma unroll
    for (int d = 0; d < DIM; ++d) s.gT[q][d] = gT[d];
    const int64_t hi = el * NIP + q;
    s.rate[q] = p.visc_heat ? (p.h.VD[hi] - p.h.VDo[hi]) / p.dt : 0.0;
    s.k[q] = geo.mats[elem_mat(geo, el)].k_thermal;
  }
  __syncwarp();
  if (act) {
    const int b = q;
    const MatDev& m = geo.mats[elem_mat(geo, el)];
    if (p.visc_heat) {
      double F = 0;
      for (int qq = 0; qq < NIP; ++qq) F += -s.w[qq] * s.N[qq][b] * s.rate[qq];
      p.Fvh[el * NEN + b] = F;
      if (!isfinite(F)) bad = 1;
    }
    if (p.thermal) {
      double F = 0, WL = 0;
      for (int qq = 0; qq < NIP; ++qq) {
        double gd = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) gd += s.G[qq][b][d] * s.gT[qq][d];
        F += s.w[qq] * s.k[qq] * gd;
        WL += s.w[qq] * s.N[qq][b];
      }
      F += WL * m.density * m.cp * s.dT[b];
      p.Fth[el * NEN + b] = F;
      if (!isfinite(F)) bad = 1;
      constexpr int KB = ke_block(1, NEN);
      T* Ke = reinterpret_cast<T*>(p.Ke) + el * NEN * KB;
      for (int a = 0; a < NEN; ++a) {
        double k = 0;
        for (int qq = 0; qq < NIP; ++qq) {
          double gg = 0;
#pragma unroll
          for (int d = 0; d < DIM; ++d) gg += s.G[qq][a][d] * s.G[qq][b][d];
          k += s.w[qq] * s.k[qq] * gg;
        }
        if (a == b) k += WL * m.density * m.cp * p.du_dt;
        Ke[a * KB + b] = (T)k;
      }
    }
  }
  const unsigned tot_bad = __reduce_add_sync(0xffffffffu, bad);
  if (lane == 0 && tot_bad) atomicAdd(&p.stats[2], (unsigned long long)tot_bad);
}

// ============================================================================================
// Deterministic node-row gather
// ============================================================================================
constexpr int kGWarps = 8;

template <int NC, int NEN, typename KT, typename VT, typename MT>
__global__ void __launch_bounds__(256, 2) k_gather(const GParams p) {
  constexpr int BLK = NC * NC * NEN;          // values of one (element, local node) row block
  constexpr int KB = ke_block(NC, NEN);       // its padded stride
  // 3-component blocks (3D u-step) are read with 16-byte loads; small blocks element-wise
  constexpr bool VLD = (NC * NC * NEN) >= 64;
  using V16 = typename std::conditional<!VLD, KT, typename std::conditional<sizeof(KT) == 4, float4, double2>::type>::type;
  constexpr int VEC = VLD ? 16 / (int)sizeof(KT) : 1;
  constexpr int NV = KB / VEC;                // 16-byte vectors per block
  constexpr int PERV = (NV + 31) / 32;        // per lane
  constexpr int UNR = VLD ? 4 : 8;            // element blocks in flight per warp
  extern __shared__ __align__(16) double acc_all[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = p.node0 + (int64_t)blockIdx.x * kGWarps + warp;
  if (r >= p.n_nodes) return;
  double* acc = acc_all + warp * p.acc_stride;
  const int deg = p.nbr_ptr[r + 1] - p.nbr_ptr[r];
  const int rowlen = NC * deg;
  const bool withK = p.Ke != nullptr;
  if (withK)
    for (int i = lane; i < NC * rowlen; i += 32) acc[i] = 0.0;
  // per-lane slot offsets inside a row block (independent of the element)
  int slot_base[PERV][VEC], slot_a2[PERV][VEC];
#pragma unroll
  for (int j = 0; j < PERV; ++j)
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      const int i = (lane + 32 * j) * VEC + c;
      const int b1 = i / (NC * NEN), rem = i - b1 * (NC * NEN), b2 = rem / NEN, a2 = rem - b2 * NEN;
      slot_base[j][c] = (i < BLK) ? b1 * rowlen + p.blk_pos[b2 < NC ? b2 : 0] * deg : -1;
      slot_a2[j][c] = a2;
    }
  double fa = 0.0;
  __syncwarp();
  const int k0 = p.inc_ptr[r], nk = p.inc_ptr[r + 1] - k0;
  const KT* Ke = reinterpret_cast<const KT*>(p.Ke);
  const MT* emap = reinterpret_cast<const MT*>(p.emap);
  for (int kc = 0; kc < nk; kc += 32) {
    const int cnt = min(32, nk - kc);
    const int my_el = lane < cnt ? p.inc_el[k0 + kc + lane] : 0;
    const int my_loc = lane < cnt ? (int)p.inc_loc[k0 + kc + lane] : 0;
    for (int kk = 0; kk < cnt; kk += UNR) {
      V16 kv[UNR][PERV];
      double fv[UNR];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {        // issue the loads of UNR element blocks
        const bool live = kk + u < cnt;
        const int64_t el = __shfl_sync(0xffffffffu, my_el, live ? kk + u : 0);
        const int a1 = __shfl_sync(0xffffffffu, my_loc, live ? kk + u : 0);
        fv[u] = (live && lane < NC) ? p.Fe1[el * (NC * NEN) + lane * NEN + a1] : 0.0;
        const V16* blk = reinterpret_cast<const V16*>(Ke + (el * NEN + a1) * KB);
#pragma unroll
        for (int j = 0; j < PERV; ++j) {
          if (withK && live && lane + 32 * j < NV) kv[u][j] = blk[lane + 32 * j];
          else { V16 z; memset(&z, 0, sizeof(V16)); kv[u][j] = z; }
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u) {        // then add them in ascending element order
        const bool live = kk + u < cnt;
        if (withK && live) {
          const int64_t el = __shfl_sync(0xffffffffu, my_el, kk + u);
          const int a1 = __shfl_sync(0xffffffffu, my_loc, kk + u);
          const MT* em = emap + (el * NEN + a1) * NEN;
#pragma unroll
          for (int j = 0; j < PERV; ++j) {
            const KT* vv = reinterpret_cast<const KT*>(&kv[u][j]);
#pragma unroll
            for (int c = 0; c < VEC; ++c)
              if (slot_base[j][c] >= 0) acc[slot_base[j][c] + (int)em[slot_a2[j][c]]] += (double)vv[c];
          }
        }
        fa += fv[u];
        __syncwarp();
      }
    }
  }
  if (p.Fe2)
    for (int k = k0; k < k0 + nk; ++k) {
      const int64_t el = p.inc_el[k];
      const int a1 = p.inc_loc[k];
      if (lane < NC) fa += p.Fe2[el * (NC * NEN) + lane * NEN + a1];
    }
  __syncwarp();
  if (withK) {
    VT* vals = reinterpret_cast<VT*>(p.vals);
#pragma unroll
    for (int b1 = 0; b1 < NC; ++b1) {
      const int64_t off = p.rowptr[p.row_base[b1] + r];
      for (int i = lane; i < rowlen; i += 32) vals[off + i] = (VT)acc[b1 * rowlen + i];
    }
  }
  if (lane < NC) p.f[p.row_base[lane] + r] = fa;
}

// Small row blocks (phase and thermal steps, 2D u-step): one lane per block entry, incident elements
// one after another.  Many resident warps hide the load latency better than deeper per-warp
// batching for these 9..36-entry blocks.
template <int NC, int NEN, typename KT, typename VT, typename MT>
__global__ void __launch_bounds__(256) k_gather_small(const GParams p) {
  constexpr int BLK = NC * NC * NEN;
  constexpr int KB = ke_block(NC, NEN);
  static_assert(BLK <= 64, "small-block gather");
  extern __shared__ __align__(16) double acc_all[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = p.node0 + (int64_t)blockIdx.x * kGWarps + warp;
  if (r >= p.n_nodes) return;
  double* acc = acc_all + warp * p.acc_stride;
  const int deg = p.nbr_ptr[r + 1] - p.nbr_ptr[r];
  const int rowlen = NC * deg;
  const bool withK = p.Ke != nullptr;
  if (withK)
    for (int i = lane; i < NC * rowlen; i += 32) acc[i] = 0.0;
  int sb[2], sa[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int i = lane + 32 * j;
    const int b1 = i / (NC * NEN), rem = i - b1 * (NC * NEN), b2 = rem / NEN, a2 = rem - b2 * NEN;
    sb[j] = (i < BLK) ? b1 * rowlen + p.blk_pos[b2 < NC ? b2 : 0] * deg : -1;
    sa[j] = a2;
  }
  double fa = 0.0;
  __syncwarp();
  const int k0 = p.inc_ptr[r], k1 = p.inc_ptr[r + 1];
  const KT* Ke = reinterpret_cast<const KT*>(p.Ke);
  const MT* emap = reinterpret_cast<const MT*>(p.emap);
  for (int k = k0; k < k1; ++k) {
    const int64_t el = p.inc_el[k];
    const int a1 = p.inc_loc[k];
    if (withK) {
      const KT* blk = Ke + (el * NEN + a1) * KB;
      const MT* em = emap + (el * NEN + a1) * NEN;
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (sb[j] >= 0) acc[sb[j] + (int)em[sa[j]]] += (double)blk[lane + 32 * j];
    }
    if (lane < NC) fa += p.Fe1[el * (NC * NEN) + lane * NEN + a1];
    __syncwarp();
  }
  if (p.Fe2)
    for (int k = k0; k < k1; ++k) {
      const int64_t el = p.inc_el[k];
      const int a1 = p.inc_loc[k];
      if (lane < NC) fa += p.Fe2[el * (NC * NEN) + lane * NEN + a1];
    }
  __syncwarp();
  if (withK) {
    VT* vals = reinterpret_cast<VT*>(p.vals);
#pragma unroll
    for (int b1 = 0; b1 < NC; ++b1) {
      const int64_t off = p.rowptr[p.row_base[b1] + r];
      for (int i = lane; i < rowlen; i += 32) vals[off + i] = (VT)acc[b1 * rowlen + i];
    }
  }
  if (lane < NC) p.f[p.row_base[lane] + r] = fa;
}

// fixed-order block reduction (deterministic)
// one CTA, fixed order: four interleaved accumulators per thread (independent loads in flight), then warp and
// CTA trees; deterministic, and no storage beyond the output
__global__ void __launch_bounds__(1024) k_reduce_sum(const double* x, int64_t n, double* out) {
  __shared__ double sh[32];
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int64_t i = threadIdx.x;
  for (; i + 3 * 1024 < n; i += 4 * 1024) { s0 += x[i]; s1 += x[i + 1024]; s2 += x[i + 2048]; s3 += x[i + 3072]; }
  for (; i < n; i += 1024) s0 += x[i];
  double s = (s0 + s1) + (s2 + s3);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = sh[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) *out = t;
  }
}

template <typename K>
void set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------------
template <int DIM, bool KRON>
static void u_points_dispatch(const UParams& p, cudaStream_t s) {
  constexpr int EPW = (DIM == 2) ? 3 : 1;
  const size_t smem = sizeof(USm<DIM, KRON>) * kUWarps * EPW;
  const int64_t per_block = (int64_t)kUWarps * EPW;
  const int64_t blocks = (p.geo.el1 - p.geo.el0 + per_block - 1) / per_block;
  const bool cons = p.mo.tangent_mode == IFEM_TANGENT_CONSISTENT;
  void (*k)(const UParams);
  if (p.vep)
    k = p.cq_f32 ? (cons ? k_u_points<DIM, KRON, float, true, true> : k_u_points<DIM, KRON, float, false, true>)
                 : (cons ? k_u_points<DIM, KRON, double, true, true> : k_u_points<DIM, KRON, double, false, true>);
  else if (p.spec) {
    constexpr int VS = IFEM_SPLIT_VOLSTRAINS, QD = IFEM_DAM_QUADRATIC;
    k = p.cq_f32 ? (cons ? k_u_points<DIM, KRON, float, true, false, VS, 3, QD> : k_u_points<DIM, KRON, float, false, false, VS, 3, QD>)
                 : (cons ? k_u_points<DIM, KRON, double, true, false, VS, 3, QD> : k_u_points<DIM, KRON, double, false, false, VS, 3, QD>);
  } else
    k = p.cq_f32 ? (cons ? k_u_points<DIM, KRON, float, true, false> : k_u_points<DIM, KRON, float, false, false>)
                 : (cons ? k_u_points<DIM, KRON, double, true, false> : k_u_points<DIM, KRON, double, false, false>);
  set_smem(k, smem);
  k<<<(unsigned)blocks, 128, smem, s>>>(p);
}

void launch_u_points(const UParams& p, cudaStream_t s) {
  if (p.geo.el1 <= p.geo.el0) return;
  if (!p.vep && launch_u_points_hex(p, s)) return;   // the sum-factorised kernel has no VEP branch
  if (p.geo.dim == 2) { if (p.geo.kron) u_points_dispatch<2, true>(p, s); else u_points_dispatch<2, false>(p, s); }
  else { if (p.geo.kron) u_points_dispatch<3, true>(p, s); else u_points_dispatch<3, false>(p, s); }
}

template <int DIM, bool KRON, typename T>
static void u_tangent_dispatch(const TParams& p, cudaStream_t s) {
  constexpr int EPC = TCfg<DIM>::EPC, NT = TCfg<DIM>::NT;
  const size_t smem = sizeof(TSm<DIM, KRON, T>) * EPC;
  const int64_t blocks = (p.geo.el1 - p.geo.el0 + EPC - 1) / EPC;
  auto k = k_u_tangent<DIM, KRON, T>;
  set_smem(k, smem);
  k<<<(unsigned)blocks, NT, smem, s>>>(p);
}

void launch_u_tangent(const TParams& p, int f32, cudaStream_t s) {
  if (p.geo.el1 <= p.geo.el0) return;
  if (p.geo.dim == 2) {
    if (p.geo.kron) { if (f32) u_tangent_dispatch<2, true, float>(p, s); else u_tangent_dispatch<2, true, double>(p, s); }
    else { if (f32) u_tangent_dispatch<2, false, float>(p, s); else u_tangent_dispatch<2, false, double>(p, s); }
  } else {
    if (p.geo.kron) { if (f32) u_tangent_dispatch<3, true, float>(p, s); else u_tangent_dispatch<3, true, double>(p, s); }
    else { if (f32) u_tangent_dispatch<3, false, float>(p, s); else u_tangent_dispatch<3, false, double>(p, s); }
  }
}

template <int DIM, bool KRON, typename T>
static void phase_dispatch(const PParams& p, cudaStream_t s) {
  constexpr int EPW = (DIM == 2) ? 3 : 1;
  const size_t smem = sizeof(PSm<DIM, KRON, T>) * kPWarps * EPW;
  const int64_t per_block = (int64_t)kPWarps * EPW;
  const int64_t blocks = (p.geo.nel + per_block - 1) / per_block;
  void (*k)(const PParams) = (p.spec && !p.general) ? k_phase<DIM, KRON, T, IFEM_SPLIT_VOLSTRAINS, IFEM_DAM_QUADRATIC>
                                                      : k_phase<DIM, KRON, T>;
  set_smem(k, smem);
  k<<<(unsigned)blocks, 32 * kPWarps, smem, s>>>(p);
}

void launch_phase(const PParams& p, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  if (dist_second_gradient(p.mo.dist)) { launch_phase_ho(p, s); return; }
  if (!p.general && launch_phase_hex(p, s)) return;   // the sum-factorised kernel has no SpecStrains/DruckerPrager
  if (p.geo.dim == 2) {
    if (p.geo.kron) { if (p.ke_f32) phase_dispatch<2, true, float>(p, s); else phase_dispatch<2, true, double>(p, s); }
    else { if (p.ke_f32) phase_dispatch<2, false, float>(p, s); else phase_dispatch<2, false, double>(p, s); }
  } else {
    if (p.geo.kron) { if (p.ke_f32) phase_dispatch<3, true, float>(p, s); else phase_dispatch<3, true, double>(p, s); }
    else { if (p.ke_f32) phase_dispatch<3, false, float>(p, s); else phase_dispatch<3, false, double>(p, s); }
  }
}

template <int DIM, bool KRON, typename T>
static void thermal_dispatch(const ThParams& p, cudaStream_t s) {
  constexpr int EPW = (DIM == 2) ? 3 : 1;
  const size_t smem = sizeof(HSm<DIM, KRON>) * kHWarps * EPW;
  const int64_t per_block = (int64_t)kHWarps * EPW;
  const int64_t blocks = (p.geo.nel + per_block - 1) / per_block;
  auto k = k_thermal<DIM, KRON, T>;
  set_smem(k, smem);
  k<<<(unsigned)blocks, 32 * kHWarps, smem, s>>>(p);
}

void launch_thermal(const ThParams& p, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  if (p.geo.dim == 2) {
    if (p.geo.kron) { if (p.ke_f32) thermal_dispatch<2, true, float>(p, s); else thermal_dispatch<2, true, double>(p, s); }
    else { if (p.ke_f32) thermal_dispatch<2, false, float>(p, s); else thermal_dispatch<2, false, double>(p, s); }
  } else {
    if (p.geo.kron) { if (p.ke_f32) thermal_dispatch<3, true, float>(p, s); else thermal_dispatch<3, true, double>(p, s); }
    else { if (p.ke_f32) thermal_dispatch<3, false, float>(p, s); else thermal_dispatch<3, false, double>(p, s); }
  }
}

template <int NC, int NEN, typename KT, typename VT>
static void gather_dispatch2(const GParams& p, cudaStream_t s) {
  const size_t smem = sizeof(double) * (size_t)p.acc_stride * kGWarps;
  const int64_t blocks = (p.n_nodes - p.node0 + kGWarps - 1) / kGWarps;
  void (*k)(const GParams);
  if constexpr (NC * NC * NEN <= 64)
    k = p.emap16 ? k_gather_small<NC, NEN, KT, VT, uint16_t> : k_gather_small<NC, NEN, KT, VT, uint8_t>;
  else
    k = p.emap16 ? k_gather<NC, NEN, KT, VT, uint16_t> : k_gather<NC, NEN, KT, VT, uint8_t>;
  set_smem(k, smem);
  k<<<(unsigned)blocks, 32 * kGWarps, smem, s>>>(p);
}

template <int NC, int NEN>
static void gather_dispatch(const GParams& p, cudaStream_t s) {
  if (p.ke_f32) {
    if (p.vals_f32) gather_dispatch2<NC, NEN, float, float>(p, s); else gather_dispatch2<NC, NEN, float, double>(p, s);
  } else {
    if (p.vals_f32) gather_dispatch2<NC, NEN, double, float>(p, s); else gather_dispatch2<NC, NEN, double, double>(p, s);
  }
}

void launch_gather(const GParams& p, cudaStream_t s) {
  if (p.n_nodes <= p.node0) return;
  if (p.nc > 3) { launch_gather_rows(p, s); return; }
  if (launch_gather_bulk(p, s)) return;
  // 2D u-step: 2 components; 3D u-step: 3; phase step: 1, or 2-3 with Lagrange multipliers
  if (p.nen == 9) {
    if (p.nc == 1) gather_dispatch<1, 9>(p, s); else if (p.nc == 2) gather_dispatch<2, 9>(p, s); else gather_dispatch<3, 9>(p, s);
  } else {
    if (p.nc == 1) gather_dispatch<1, 27>(p, s); else if (p.nc == 2) gather_dispatch<2, 27>(p, s); else gather_dispatch<3, 27>(p, s);
  }
}

// EnforceIrreversible with Lagrange multipliers (PhaseFieldUtil.cpp:350-484, PhaseField.cpp:712-729).  One thread
// per element node a: the phase element's row a (Ke1, Fe1 from the phase kernel, which ran without an
// irreversibility term) grown to the rows of [phase, L(, L2)] x nodes, with the nodal multiplier terms added
// after all other phase terms, in the reference's order.  The utility's own Gc and l scale the augmented methods.
template <typename T>
__global__ void __launch_bounds__(128) k_phase_lagrange(const LagParams p) {
  const int nen = p.geo.nen;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.geo.nel * nen) return;
  const int64_t el = t / nen;
  const int a = (int)(t - el * nen);
  const int nc = 1 + p.nlag;
  const int KB1 = ke_block(1, nen), KB = ke_block(nc, nen);
  const int node = p.geo.conn[el * nen + a];
  const int dph = dof_of(p.dm, IFEM_DOF_PHASE, node);
  const double Ph = p.phase_cur[dph], PhO = p.phase_old[dph];
  const double L = p.phase_cur[dof_of(p.dm, IFEM_DOF_LMULT, node)];
  const double L2 = p.nlag == 2 ? p.phase_cur[dof_of(p.dm, IFEM_DOF_LMULT2, node)] : 0.0;
  const double W = p.WL[el * nen + a];
  const MatDev& m = p.geo.mats[elem_mat(p.geo, el)];
  const T* K1 = reinterpret_cast<const T*>(p.Ke1) + (el * nen + a) * KB1;
  double FPh = p.Fe1[el * nen + a], FL = 0, FL2 = 0;
  double kpp = (double)K1[a], kpq = 0, kqp = 0, kqq = 0, kpq2 = 0, kq2p = 0, kq2q2 = 0;
  const double lim0 = fmin(1.0 - 1.0e-3, fmax(0.0, PhO)), lim1 = 1.0 + 1e-1;
  const double LF = p.mo.lag_fact;
  switch (p.mo.irr) {
    case IFEM_IRR_LAGRANGE:   // LagrMultIrr (:383-399)
      FPh += W * L; kpq += W;
      if (Ph >= 1.0) { FL += W * (Ph - lim1); kqp += W; }
      else if (Ph < PhO) { FL += W * (Ph - lim0); kqp += W; }
      else { FL += W * L; kqq += W; }
      break;
    case IFEM_IRR_AUGLAG: {   // AugLagrIrr (:401-441)
      const double sc = m.gc_input / m.l / LF, d = LF;
      FL += -W * sc * L * (1.0 + 1.0e-10); kqq += -W * sc * (1.0 + 1.0e-10);
      const double pre = L + LF * (Ph - lim0);
      FPh += W * sc * L * d; kpq += W * sc * d;
      if (pre <= 0) { FPh += W * sc * (pre - L) * d; kpp += W * sc * d * d; FL += W * sc * pre; kqq += W * sc; kqp += W * sc * d; }
    } break;
    case IFEM_IRR_AUGLAG2: {  // AugLagrIrr2 (:444-484)
      const double c = m.gc_input / m.l / LF, d = LF;
      FL += -W * c * L * (1.0 - 1.0e-8); kqq += -W * c * (1.0 - 1.0e-8);
      FL2 += -W * c * L2 * (1.0 - 1.0e-8); kq2q2 += -W * c * (1.0 - 1.0e-8);
      FPh += W * c * L * d; kpq += W * c * d;
      FPh += W * c * L2 * d; kpq2 += W * c * d;
      const double pre = L + LF * (Ph - lim0);
      if (pre <= 0) { FPh += W * c * (pre - L) * d; kpp += W * c * d * d; FL += W * c * pre; kqq += W * c; kqp += W * c * d; }
      const double pre2 = L2 + LF * (Ph - lim1);
      if (pre2 >= 0) { FPh += W * c * (pre2 - L2) * d; kpp += W * c * d * d; FL2 += W * c * pre2; kq2q2 += W * c; kq2p += W * c * d; }
    } break;
    default: break;
  }
  // couplings of row (node a, c1) with column (node a, c2); the phase-phase block keeps Ke1's other columns
  const double cpl[3][3] = {{kpp, kpq, kpq2}, {kqp, kqq, 0.0}, {kq2p, 0.0, kq2q2}};
  T* K = reinterpret_cast<T*>(p.Ke) + (el * nen + a) * KB;
  for (int c1 = 0; c1 < nc; ++c1)
    for (int c2 = 0; c2 < nc; ++c2)
      for (int b = 0; b < nen; ++b) {
        const T v = (b == a) ? (T)cpl[c1][c2] : ((c1 == 0 && c2 == 0) ? K1[b] : (T)0);
        K[(c1 * nc + c2) * nen + b] = v;
      }
  for (int i = nc * nc * nen; i < KB; ++i) K[i] = (T)0;
  double* F = p.Fe + el * nc * nen;
  F[a] = FPh;
  F[nen + a] = FL;
  if (nc == 3) F[2 * nen + a] = FL2;
}

void launch_phase_lagrange(const LagParams& p, cudaStream_t s) {
  const int64_t n = p.geo.nel * p.geo.nen;
  if (n == 0) return;
  const unsigned blocks = (unsigned)((n + 127) / 128);
  if (p.ke_f32) k_phase_lagrange<float><<<blocks, 128, 0, s>>>(p);
  else k_phase_lagrange<double><<<blocks, 128, 0, s>>>(p);
}

// OceanBCModel::Assemble_U (OceanBC.cpp:96-150), 2D quadratic elements: one warp per element; lanes 0..8 are
// the ips, then the nodes.  F_ux(n) = W(n) rho g max(0, hw - y_n), W(n) = sum_q w_q (N_q . Phase) N_q,n, summed
// over q in order; the uy rows get nothing.
template <bool KRON>
__global__ void __launch_bounds__(128) k_ocean_u(const OceanParams p) {
  __shared__ ElemSm<2, KRON> es[4];
  __shared__ IpGeo<2> ig[4][9];
  __shared__ double phq[4][9];
  __shared__ double ph[4][9];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t el = (int64_t)blockIdx.x * 4 + warp;
  if (el >= p.geo.nel) return;                   // whole warp; only warp-level synchronisation below
  fill_elem<2, KRON>(es[warp], p.geo, p.rule, el, lane, 32);
  if (lane < 9) ph[warp][lane] = p.phase_cur[dof_of(p.dm, IFEM_DOF_PHASE, p.geo.conn[el * 9 + lane])];
  __syncwarp();
  if (lane < 9) ip_geometry<2, KRON>(es[warp], p.rule, lane, ig[warp][lane]);
  __syncwarp();
  if (lane < 9) {
    double phi = 0;
    for (int a = 0; a < 9; ++a) {
      double N, G[2];
      shape_at<2, KRON>(es[warp], p.rule, ig[warp][lane], lane, a, N, G);
      phi += N * ph[warp][a];
    }
    phq[warp][lane] = phi;
  }
  __syncwarp();
  if (lane < 9) {
    const int n = lane;
    double WL = 0;
    for (int q = 0; q < 9; ++q) {
      double N, G[2];
      shape_at<2, KRON>(es[warp], p.rule, ig[warp][q], q, n, N, G);
      WL += ig[warp][q].w * phq[warp][q] * N;
    }
    const double hIP = p.hw - es[warp].X[n][1];
    const double pTarget = hIP < 0.0 ? 0.0 : 9.81 * p.density * hIP;   // g = 9.81 (OceanBC.h:43)
    p.Fo[el * 18 + n] = WL * pTarget;
    p.Fo[el * 18 + 9 + n] = 0.0;
  }
}

void launch_ocean_u(const OceanParams& p, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  const unsigned blocks = (unsigned)((p.geo.nel + 3) / 4);
  if (p.geo.kron) k_ocean_u<true><<<blocks, 128, 0, s>>>(p);
  else k_ocean_u<false><<<blocks, 128, 0, s>>>(p);
}

void launch_reduce_sum(const double* x, int64_t n, double* out, cudaStream_t s) {
  k_reduce_sum<<<1, 1024, 0, s>>>(x, n, out);
}

}  // namespace ifem
