// Adjoint of the residual kernels with respect to the material parameters theta = (Gc, l, A, n).
// The reference has no sensitivities; this is the analytic derivative of the residual the
// assembly kernels compute (checked against central finite differences of that residual).
//
//   u step:     R_U = sum_q w B^T sigma(eps - eps_p(theta)).  eps_p comes from the converged Glen
//               return map (SolidMaterial.cpp:200-269): implicit differentiation of its local
//               system gives d eps_e / d(A, n) (rm_param_sensitivity), mapped through the split
//               tangent (g D+ + D-) and B^T.  dR_U/dGc = dR_U/dl = 0.
//   phase step: R_ph = sum_q w Gc (Dist - DistCap) + driving + nodal terms (PhaseField.cpp:652-712):
//               Dist scales as 1/l and its gradient part as l (PhaseFieldUtil.cpp:185-221); with the
//               reference's derived fracture energy Gc = 2 ft^2 l / E (IceMaterial.cpp:71-72) the
//               l-derivative also carries dGc/dl = Gc / l.  dR_ph/dA = dR_ph/dn = 0.
// Outputs per element: dF[theta][el][comp*nen + node] (fp64), gathered into global vectors by the
// deterministic gather, and lambda^T dF per element reduced per material set in element order.
// History and state are read, never written.
//
// Temperature (the thermal Arrhenius coupling, IceMaterial.cpp:49-84).  With dFT set, the same kernels also
// give the directional derivative dR/dT . dT of the residual with respect to the temperature field:
//   u step:     A(T) = A0 exp(-Q/R (1/TAbs - 1/TRef)), dA/dT = A Q / (R TAbs^2) below the melting clamp, so
//               d eps_e/dT = (d eps_e/dA0) A0 Q / (R TAbs^2) (the same implicit differentiation);
//   phase step: Gc(T) = 2 ft(T)^2 l / E with ft = ft0 - ftdeg (TAbs - TRef), dGc/dT = -4 ft ftdeg l / E, through
//               every term that carries Gc (the crack density and the lumped capacity, which uses the last
//               ip's Gc, PhaseField.cpp:702-706).
// dT_ip is the interpolated nodal perturbation (the phase step's ref-compat mode reads DOF 0 for every node,
// PhaseField.cpp:562-565, so its perturbation is dT[0]), or 1 for the pinned temperature of a context without
// a T DOF.
//
// Precision.  R = double is the FP64 adjoint.  R = float keeps the return map and its 7x7 sensitivity solve
// in FP64 (the converged local system) and forms the per-ip sensitivity stresses and their contraction with
// the shape gradients in FP32, the FP32 variant of the calibration sweeps.

#include <cuda_runtime.h>
#include <cstdint>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

__device__ __forceinline__ int amat(const Geo& g, int64_t el) { return g.emat ? g.emat[el] : 0; }
__device__ __forceinline__ int adof(const DofMap& dm, int kind, int node) { return dm.base[kind] + dm.node_rank[node]; }

template <int DIM, typename R>
struct AUSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, true> e;
  double U[DIM][NEN], UO[DIM][NEN];
  double Ph[NEN], PhO[NEN], T[NEN], dT[NEN];
  IpGeo<DIM> g[NEN];
  R sA[NEN][6], sN[NEN][6], sT[NEN][6];
};

constexpr int kAWarps = 4;

// TAbs of IceMaterial::SetTemperature and the derivative of TAbs with respect to T (0 above the melting clamp)
__device__ __forceinline__ double tabs_of(const MatDev& m, double T, double& dTabs) {
  double TAbs = T + m.t_offset;
  dTabs = 1.0;
  if (TAbs > 273.15) { TAbs = 273.15; dTabs = 0.0; }
  return TAbs;
}

template <int DIM, typename R>
__global__ void __launch_bounds__(128) k_adjoint_u(const UParams p, double* dF, const double* dTv, double* dFT) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  __shared__ AUSm<DIM, R> sm[kAWarps * EPW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP, q = lane - sub * NIP;
  const int64_t el = ((int64_t)blockIdx.x * kAWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < p.geo.nel);
  AUSm<DIM, R>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
  const Geo& geo = p.geo;
  const int64_t nh = geo.nel * NIP;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  if (act) {
    fill_elem<DIM, true>(s.e, geo, p.rule, el, q, NIP);
    const int node = geo.conn[el * NEN + q];
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      const int d = adof(dm, IFEM_DOF_UX + b, node);
      s.U[b][q] = p.su.cur[d];
      s.UO[b][q] = p.su.old[d];
    }
    const int dph = adof(dm, IFEM_DOF_PHASE, node);
    s.Ph[q] = p.sp.cur[dph];
    s.PhO[q] = p.sp.old[dph];
    s.T[q] = mo.hasT ? p.sT.cur[adof(dm, IFEM_DOF_T, node)] : 0.0;
    s.dT[q] = (dFT && mo.hasT) ? dTv[adof(dm, IFEM_DOF_T, node)] : 0.0;
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, true>(s.e, p.rule, q, g);
    s.g[q] = g;
    double eps[6] = {0, 0, 0, 0, 0, 0}, epsO[6] = {0, 0, 0, 0, 0, 0};
    double phi = 0, phiO = 0, Tip = 0, dTip = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, true>(s.e, p.rule, g, q, a, N, G);
      phi += N * s.Ph[a]; phiO += N * s.PhO[a]; Tip += N * s.T[a]; dTip += N * s.dT[a];
      const double ux = s.U[0][a], uy = s.U[1][a], uz = s.U[DIM - 1][a];
      const double ox = s.UO[0][a], oy = s.UO[1][a], oz = s.UO[DIM - 1][a];
      if (DIM == 2) {
        eps[0] += G[0] * ux; eps[1] += G[1] * uy; eps[3] += G[1] * ux + G[0] * uy;
        epsO[0] += G[0] * ox; epsO[1] += G[1] * oy; epsO[3] += G[1] * ox + G[0] * oy;
      } else {
        eps[0] += G[0] * ux; eps[1] += G[1] * uy; eps[2] += G[DIM - 1] * uz;
        eps[3] += G[1] * ux + G[0] * uy; eps[4] += G[DIM - 1] * uy + G[1] * uz; eps[5] += G[DIM - 1] * ux + G[0] * uz;
        epsO[0] += G[0] * ox; epsO[1] += G[1] * oy; epsO[2] += G[DIM - 1] * oz;
        epsO[3] += G[1] * ox + G[0] * oy; epsO[4] += G[DIM - 1] * oy + G[1] * oz; epsO[5] += G[DIM - 1] * ox + G[0] * oz;
      }
    }
    const MatDev& m = geo.mats[amat(geo, el)];
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    double Dam, dDam, unused;
    damage_function(phi, mo.dam_f, mo.k0, mo.porder_p, Dam, dDam, unused);
    const int64_t hi = el * NIP + q;
    double epl[6], eplo[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) { epl[r] = p.h.EP[r * nh + hi]; eplo[r] = p.h.EPo[r * nh + hi]; }
    double hist0 = (M.rheo != IFEM_RHEO_LE) ? p.h.MH[hi] : 0.0;
    double dA[6] = {0, 0, 0, 0, 0, 0}, dn[6] = {0, 0, 0, 0, 0, 0};
    double DPl[1], diss = 0, sol[7];
    const bool vis = (M.rheo == IFEM_RHEO_VE || M.rheo == IFEM_RHEO_DVE);
    const bool vexp = (M.rheo == IFEM_RHEO_VE_EXPL || M.rheo == IFEM_RHEO_DVE_EXPL);
    RMTan tan;
    const double A_over_A0 = (m.A0 != 0.0) ? M.A / m.A0 : 0.0;
    if (vis && !(phi > M.phi_lim)) {
      double dmg = 1.0, u1, u2;
      if (M.rheo == IFEM_RHEO_DVE) damage_function(phi, mo.dam_f, mo.k0, mo.porder_p, dmg, u1, u2);
      return_mapping_viscous(M, DPl, epl, eps, eplo, dmg, p.dt, hist0, mo.rm_tol_mode, mo.rm_max_it,
                             IFEM_TANGENT_REFERENCE, diss, &tan, sol);
      rm_param_sensitivity(M, A_over_A0, sol, p.dt, dA, dn);
    } else if (vexp && !(phiO > M.phi_lim)) {
      double dmg = 1.0, u1, u2;
      if (M.rheo == IFEM_RHEO_DVE_EXPL) damage_function(phiO, mo.dam_f, mo.k0, mo.porder_p, dmg, u1, u2);
      return_mapping_viscous(M, DPl, epl, epsO, eplo, dmg, p.dt, hist0, mo.rm_tol_mode, mo.rm_max_it,
                             IFEM_TANGENT_REFERENCE, diss, &tan, sol);
      // eps_p = eps_old - sol(0:5) at convergence, so d(eps - eps_p) = d sol(0:5) here too
      rm_param_sensitivity(M, A_over_A0, sol, p.dt, dA, dn);
    } else {
#pragma unroll
      for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplo[r];
    }
    double ee[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) ee[r] = eps[r] - epl[r];
    double alpha, gamma;
    split_tangent(M, ee, Dam, alpha, gamma);
    // sigma(eps - eps_p) has the split tangent alpha 11^T + gamma VC; eps - eps_p = sol(0:5)
    const double VC[6] = {1, 1, 1, 0.5, 0.5, 0.5};
    const double trA = dA[0] + dA[1] + dA[2], trN = dn[0] + dn[1] + dn[2];
    // d eps_e / dT = (d eps_e / dA0) A0 Q / (R TAbs^2) dTAbs/dT, times the ip's temperature perturbation
    double kT = 0.0;
    if (dFT) {
      double dTabs;
      const double TAbs = tabs_of(m, mo.hasT ? Tip : mo.pinned_T, dTabs);
      kT = m.A0 * m.q_creep / (kR * TAbs * TAbs) * dTabs * (mo.hasT ? dTip : 1.0);
    }
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const double sa = g.w * ((r < 3 ? alpha * trA : 0.0) + gamma * VC[r] * dA[r]);
      s.sA[q][r] = (R)sa;
      s.sN[q][r] = (R)(g.w * ((r < 3 ? alpha * trN : 0.0) + gamma * VC[r] * dn[r]));
      s.sT[q][r] = (R)(sa * kT);
    }
  }
  __syncwarp();
  if (act) {
    const int a = q;
    R FA[DIM], FN[DIM], FT[DIM];
#pragma unroll
    for (int b = 0; b < DIM; ++b) { FA[b] = 0; FN[b] = 0; FT[b] = 0; }
    auto contract = [&](const R* S, R* Fo, const R G[DIM]) {
      if (DIM == 2) {
        Fo[0] += G[0] * S[0] + G[1] * S[3]; Fo[1] += G[1] * S[1] + G[0] * S[3];
      } else {
        Fo[0] += G[0] * S[0] + G[1] * S[3] + G[DIM - 1] * S[5];
        Fo[1] += G[1] * S[1] + G[0] * S[3] + G[DIM - 1] * S[4];
        Fo[DIM - 1] += G[DIM - 1] * S[2] + G[1] * S[4] + G[0] * S[5];
      }
    };
    for (int qq = 0; qq < NIP; ++qq) {
      double N, Gd[DIM];
      shape_at<DIM, true>(s.e, p.rule, s.g[qq], qq, a, N, Gd);
      R G[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) G[d] = (R)Gd[d];
      contract(s.sA[qq], FA, G);
      contract(s.sN[qq], FN, G);
      if (dFT) contract(s.sT[qq], FT, G);
    }
    const int64_t stride = geo.nel * (DIM * NEN);
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      const int64_t o = el * (DIM * NEN) + b * NEN + a;
      if (dF) {
        dF[0 * stride + o] = 0.0;
        dF[1 * stride + o] = 0.0;
        dF[2 * stride + o] = (double)FA[b];
        dF[3 * stride + o] = (double)FN[b];
      }
      if (dFT) dFT[o] = (double)FT[b];
    }
  }
}

template <int DIM, typename R>
struct APSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, true> e;
  double Ph[NEN], Tn[NEN], dTn[NEN];
  IpGeo<DIM> g[NEN];
  R cNG[NEN], cGG[NEN], cNL[NEN], cGL[NEN];   // coefficients of N and G.dphi in dF/dGc, dF/dl
  R cNT[NEN], cGT[NEN];                       // ... and in dF/dT . dT
  R dphi[NEN][DIM];
  double last_Gc, last_dGcdl, last_l, last_dGcdT;
};

template <int DIM, typename R>
__global__ void __launch_bounds__(128) k_adjoint_phase(const PParams p, double* dF, const double* dTv, double* dFT) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  __shared__ APSm<DIM, R> sm[kAWarps * EPW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP, q = lane - sub * NIP;
  const int64_t el = ((int64_t)blockIdx.x * kAWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < p.geo.nel);
  APSm<DIM, R>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
  const Geo& geo = p.geo;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  if (act) {
    fill_elem<DIM, true>(s.e, geo, p.rule, el, q, NIP);
    const int node = geo.conn[el * NEN + q];
    s.Ph[q] = p.sp.cur[adof(dm, IFEM_DOF_PHASE, node)];
    if (mo.hasT) s.Tn[q] = mo.ref_compat_T ? p.sT.cur[0] : p.sT.cur[adof(dm, IFEM_DOF_T, node)];
    else s.Tn[q] = 0.0;
    s.dTn[q] = (dFT && mo.hasT) ? (mo.ref_compat_T ? dTv[0] : dTv[adof(dm, IFEM_DOF_T, node)]) : 0.0;
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, true>(s.e, p.rule, q, g);
    s.g[q] = g;
    double phi = 0, Tip = 0, dTip = 0, gphi[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) gphi[d] = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, true>(s.e, p.rule, g, q, a, N, G);
      phi += N * s.Ph[a];
      Tip += N * s.Tn[a];
      dTip += N * s.dTn[a];
#pragma unroll
      for (int d = 0; d < DIM; ++d) gphi[d] += G[d] * s.Ph[a];
    }
    const MatDev& m = geo.mats[amat(geo, el)];
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    const double l = M.l;
    double c = 0, nF = 0, grad = 0;
    switch (mo.dist) {
      case IFEM_DIST_QUADRATIC: c = 1.0 / (2.0 * l); nF = 2.0 * phi; grad = 2.0 * l * l; break;
      case IFEM_DIST_LINEAR: c = 3.0 / (8.0 * l); nF = 1.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LINEAR2: c = 1.0 / (4.0 * l); nF = 2.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LOCAL: c = 1.0 / l; nF = 2.0 * phi; grad = 0.0; break;
      case IFEM_DIST_CZM: c = 1.0 / (3.141592 * l); nF = 2.0 * (1.0 - phi); grad = 2.0 * l * l; break;
      default: break;
    }
    double capF = 0;
    if (mo.lumped_cap) {
      switch (mo.dist) {
        case IFEM_DIST_QUADRATIC: capF = 1.0 / (2.0 * l) * 2.0 * phi; break;
        case IFEM_DIST_CZM: capF = 1.0 / (3.141592 * l) * 2.0 * (1.0 - phi); break;
        case IFEM_DIST_LINEAR: capF = 3.0 / (8.0 * l); break;
        case IFEM_DIST_LINEAR2: capF = 1.0 / (4.0 * l) * 2.0; break;
        case IFEM_DIST_LOCAL: capF = 1.0 / l * 2 * phi; break;
        default: break;
      }
    }
    const double w = g.w;
    const double dGc_dgc = (m.gc_mode == 1) ? 1.0 : 0.0;
    const double dGc_dl = (m.gc_mode == 1) ? 0.0 : M.Gc / l;
    const double fN = c * nF - capF;          // scales as 1/l
    const double fG = c * grad;               // scales as l
    // dGc/dT . dT_ip for the derived fracture energy Gc = 2 ft(T)^2 l / E
    double dGc_dT = 0.0;
    if (dFT && m.gc_mode != 1) {
      double dTabs;
      const double TAbs = tabs_of(m, mo.hasT ? Tip : mo.pinned_T, dTabs);
      const double ft = m.ft0 - m.ftdeg * (TAbs - m.t_ref);
      dGc_dT = -4.0 * ft * m.ftdeg * l / m.E * dTabs * (mo.hasT ? dTip : 1.0);
    }
    s.cNG[q] = (R)(w * dGc_dgc * fN);
    s.cGG[q] = (R)(w * dGc_dgc * fG);
    s.cNL[q] = (R)(w * (dGc_dl * fN - M.Gc * fN / l));
    s.cGL[q] = (R)(w * (dGc_dl * fG + (grad != 0.0 ? M.Gc * fG / l : 0.0)));
    s.cNT[q] = (R)(w * dGc_dT * fN);
    s.cGT[q] = (R)(w * dGc_dT * fG);
#pragma unroll
    for (int d = 0; d < DIM; ++d) s.dphi[q][d] = (R)gphi[d];
    if (q == NIP - 1) { s.last_Gc = M.Gc; s.last_dGcdl = dGc_dl; s.last_l = l; s.last_dGcdT = dGc_dT; }
  }
  __syncwarp();
  if (act) {
    const int b = q;
    R FG = 0, FL = 0, FT = 0;
    double WL = 0;
    for (int qq = 0; qq < NIP; ++qq) {
      double Nd, Gd[DIM];
      shape_at<DIM, true>(s.e, p.rule, s.g[qq], qq, b, Nd, Gd);
      const R N = (R)Nd;
      R gd = 0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) gd += (R)Gd[d] * s.dphi[qq][d];
      FG += s.cNG[qq] * N + s.cGG[qq] * gd;
      FL += s.cNL[qq] * N + s.cGL[qq] * gd;
      FT += s.cNT[qq] * N + s.cGT[qq] * gd;
      WL += s.g[qq].w * Nd;
    }
    const MatDev& m = geo.mats[amat(geo, el)];
    if (mo.lumped_cap) {   // WL Gc DL with DL ~ 1/l, Gc of the last ip (PhaseField.cpp:702-706)
      const double ph = s.Ph[b], l = s.last_l;
      double DL = 0;
      switch (mo.dist) {
        case IFEM_DIST_QUADRATIC: DL = 1.0 / l * ph; break;
        case IFEM_DIST_CZM: DL = 2.0 / (3.141592 * l) * (1.0 - ph); break;
        case IFEM_DIST_LINEAR: DL = 3.0 / (8.0 * l); break;
        case IFEM_DIST_LINEAR2: DL = 1.0 / (4.0 * l); break;
        case IFEM_DIST_LOCAL: DL = 2.0 / l * ph; break;
        default: break;
      }
      FG += (R)(WL * ((m.gc_mode == 1) ? 1.0 : 0.0) * DL);
      FL += (R)(WL * (s.last_dGcdl * DL - s.last_Gc * DL / l));
      FT += (R)(WL * s.last_dGcdT * DL);
    }
    if (mo.irr == IFEM_IRR_PENALTY) {   // PenaltyIrr uses the utility's own Gc = the input gc
      const double ph = s.Ph[b];
      const double PhO = p.sp.old[adof(dm, IFEM_DOF_PHASE, geo.conn[el * NEN + b])];
      const double lim0 = fmin(1.0 - 1.0e-3, fmax(0.0, PhO)), lim1 = 1.0 + 1e-1;
      if (ph < lim0) FG += (R)(WL * mo.penalty * (ph - lim0));
      if (ph > lim1) FG += (R)(WL * mo.penalty * (ph - lim1));
    }
    const int64_t stride = geo.nel * NEN;
    const int64_t o = el * NEN + b;
    if (dF) {
      dF[0 * stride + o] = (double)FG;
      dF[1 * stride + o] = (double)FL;
      dF[2 * stride + o] = 0.0;
      dF[3 * stride + o] = 0.0;
    }
    if (dFT) dFT[o] = (double)FT;
  }
}

// lambda^T dF per element and parameter (element-local sums in node order)
__global__ void k_adjoint_lambda(const double* dF, int64_t nel, int nc, int nen, const int32_t* conn, DofMap dm,
                                 int kind0, const double* lambda, double* out /* [nel][4] */) {
  const int64_t el = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (el >= nel) return;
  const int64_t stride = nel * nc * nen;
  for (int th = 0; th < 4; ++th) {
    double sum = 0;
    for (int b = 0; b < nc; ++b)
      for (int a = 0; a < nen; ++a) {
        const double lam = lambda ? lambda[dm.base[kind0 + b] + dm.node_rank[conn[el * nen + a]]] : 1.0;
        sum += lam * dF[th * stride + el * nc * nen + b * nen + a];
      }
    out[el * 4 + th] = sum;
  }
}

// per material set, elements in ascending order (deterministic)
__global__ void k_adjoint_reduce(const double* per_el, const int32_t* mat_ptr, const int32_t* mat_el, int n_mats,
                                 double* out /* [n_mats][4] */) {
  const int mset = blockIdx.x;
  if (mset >= n_mats) return;
  __shared__ double sh[4][128];
  double acc[4] = {0, 0, 0, 0};
  const int b = mat_ptr[mset], e = mat_ptr[mset + 1];
  for (int k = b + (int)threadIdx.x; k < e; k += 128)
#pragma unroll
    for (int th = 0; th < 4; ++th) acc[th] += per_el[(int64_t)mat_el[k] * 4 + th];
#pragma unroll
  for (int th = 0; th < 4; ++th) sh[th][threadIdx.x] = acc[th];
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int th = 0; th < 4; ++th) sh[th][threadIdx.x] += sh[th][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int th = 0; th < 4; ++th) out[mset * 4 + th] = sh[th][0];
}

}  // namespace

void launch_adjoint_u(const UParams& p, double* dF, const double* dT, double* dFT, int f32, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  const int EPW = p.geo.dim == 2 ? 3 : 1;
  const int64_t blocks = (p.geo.nel + kAWarps * EPW - 1) / (kAWarps * EPW);
  if (p.geo.dim == 2) {
    if (f32) k_adjoint_u<2, float><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
    else k_adjoint_u<2, double><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
  } else {
    if (f32) k_adjoint_u<3, float><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
    else k_adjoint_u<3, double><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
  }
}

void launch_adjoint_phase(const PParams& p, double* dF, const double* dT, double* dFT, int f32, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  const int EPW = p.geo.dim == 2 ? 3 : 1;
  const int64_t blocks = (p.geo.nel + kAWarps * EPW - 1) / (kAWarps * EPW);
  if (p.geo.dim == 2) {
    if (f32) k_adjoint_phase<2, float><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
    else k_adjoint_phase<2, double><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
  } else {
    if (f32) k_adjoint_phase<3, float><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
    else k_adjoint_phase<3, double><<<(unsigned)blocks, 128, 0, s>>>(p, dF, dT, dFT);
  }
}

void launch_adjoint_lambda(const double* dF, int64_t nel, int nc, int nen, const int32_t* conn, const DofMap& dm,
                           int kind0, const double* lambda, double* per_el, const int32_t* mat_ptr,
                           const int32_t* mat_el, int n_mats, double* out, cudaStream_t s) {
  if (nel > 0) k_adjoint_lambda<<<(unsigned)((nel + 127) / 128), 128, 0, s>>>(dF, nel, nc, nen, conn, dm, kind0, lambda, per_el);
  k_adjoint_reduce<<<n_mats, 128, 0, s>>>(per_el, mat_ptr, mat_el, n_mats, out);
}

}  // namespace ifem
