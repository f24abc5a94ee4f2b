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

#include <cuda_runtime.h>
#include <cstdint>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

__device__ __forceinline__ int amat(const Geo& g, int64_t el) { return g.emat ? g.emat[el] : 0; }
__device__ __forceinline__ int adof(const DofMap& dm, int kind, int node) { return dm.base[kind] + dm.node_rank[node]; }

template <int DIM>
struct AUSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, true> e;
  double U[DIM][NEN], UO[DIM][NEN];
  double Ph[NEN], PhO[NEN], T[NEN];
  IpGeo<DIM> g[NEN];
  double sA[NEN][6], sN[NEN][6];
};

constexpr int kAWarps = 4;

template <int DIM>
__global__ void __launch_bounds__(128) k_adjoint_u(const UParams p, double* dF) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  __shared__ AUSm<DIM> sm[kAWarps * EPW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP, q = lane - sub * NIP;
  const int64_t el = ((int64_t)blockIdx.x * kAWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < p.geo.nel);
  AUSm<DIM>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
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
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, true>(s.e, p.rule, q, g);
    s.g[q] = g;
    double eps[6] = {0, 0, 0, 0, 0, 0}, epsO[6] = {0, 0, 0, 0, 0, 0};
    double phi = 0, phiO = 0, Tip = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, true>(s.e, p.rule, g, q, a, N, G);
      phi += N * s.Ph[a]; phiO += N * s.PhO[a]; Tip += N * s.T[a];
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
    damage_function(phi, mo.dam_f, mo.k0, Dam, dDam, unused);
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
      if (M.rheo == IFEM_RHEO_DVE) damage_function(phi, mo.dam_f, mo.k0, dmg, u1, u2);
      return_mapping_viscous(M, DPl, epl, eps, eplo, dmg, p.dt, hist0, mo.rm_tol_mode, mo.rm_max_it,
                             IFEM_TANGENT_REFERENCE, diss, &tan, sol);
      rm_param_sensitivity(M, A_over_A0, sol, p.dt, dA, dn);
    } else if (vexp && !(phiO > M.phi_lim)) {
      double dmg = 1.0, u1, u2;
      if (M.rheo == IFEM_RHEO_DVE_EXPL) damage_function(phiO, mo.dam_f, mo.k0, dmg, u1, u2);
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
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      s.sA[q][r] = g.w * ((r < 3 ? alpha * trA : 0.0) + gamma * VC[r] * dA[r]);
      s.sN[q][r] = g.w * ((r < 3 ? alpha * trN : 0.0) + gamma * VC[r] * dn[r]);
    }
  }
  __syncwarp();
  if (act) {
    const int a = q;
    double FA[DIM], FN[DIM];
#pragma unroll
    for (int b = 0; b < DIM; ++b) { FA[b] = 0; FN[b] = 0; }
    for (int qq = 0; qq < NIP; ++qq) {
      double N, G[DIM];
      shape_at<DIM, true>(s.e, p.rule, s.g[qq], qq, a, N, G);
      const double* A = s.sA[qq];
      const double* Nn = s.sN[qq];
      if (DIM == 2) {
        FA[0] += G[0] * A[0] + G[1] * A[3]; FA[1] += G[1] * A[1] + G[0] * A[3];
        FN[0] += G[0] * Nn[0] + G[1] * Nn[3]; FN[1] += G[1] * Nn[1] + G[0] * Nn[3];
      } else {
        FA[0] += G[0] * A[0] + G[1] * A[3] + G[DIM - 1] * A[5];
        FA[1] += G[1] * A[1] + G[0] * A[3] + G[DIM - 1] * A[4];
        FA[DIM - 1] += G[DIM - 1] * A[2] + G[1] * A[4] + G[0] * A[5];
        FN[0] += G[0] * Nn[0] + G[1] * Nn[3] + G[DIM - 1] * Nn[5];
        FN[1] += G[1] * Nn[1] + G[0] * Nn[3] + G[DIM - 1] * Nn[4];
        FN[DIM - 1] += G[DIM - 1] * Nn[2] + G[1] * Nn[4] + G[0] * Nn[5];
      }
    }
    const int64_t stride = geo.nel * (DIM * NEN);
#pragma unroll
    for (int b = 0; b < DIM; ++b) {
      const int64_t o = el * (DIM * NEN) + b * NEN + a;
      dF[0 * stride + o] = 0.0;
      dF[1 * stride + o] = 0.0;
      dF[2 * stride + o] = FA[b];
      dF[3 * stride + o] = FN[b];
    }
  }
}

template <int DIM>
struct APSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, true> e;
  double Ph[NEN], Tn[NEN];
  IpGeo<DIM> g[NEN];
  double cNG[NEN], cGG[NEN], cNL[NEN], cGL[NEN];   // coefficients of N and G.dphi in dF/dGc, dF/dl
  double dphi[NEN][DIM];
  double last_Gc, last_dGcdl, last_l;
};

template <int DIM>
__global__ void __launch_bounds__(128) k_adjoint_phase(const PParams p, double* dF) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  __shared__ APSm<DIM> sm[kAWarps * EPW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP, q = lane - sub * NIP;
  const int64_t el = ((int64_t)blockIdx.x * kAWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < p.geo.nel);
  APSm<DIM>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
  const Geo& geo = p.geo;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  if (act) {
    fill_elem<DIM, true>(s.e, geo, p.rule, el, q, NIP);
    const int node = geo.conn[el * NEN + q];
    s.Ph[q] = p.sp.cur[adof(dm, IFEM_DOF_PHASE, node)];
    if (mo.hasT) s.Tn[q] = mo.ref_compat_T ? p.sT.cur[0] : p.sT.cur[adof(dm, IFEM_DOF_T, node)];
    else s.Tn[q] = 0.0;
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, true>(s.e, p.rule, q, g);
    s.g[q] = g;
    double phi = 0, Tip = 0, gphi[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) gphi[d] = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, true>(s.e, p.rule, g, q, a, N, G);
      phi += N * s.Ph[a];
      Tip += N * s.Tn[a];
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
    s.cNG[q] = w * dGc_dgc * fN;
    s.cGG[q] = w * dGc_dgc * fG;
    s.cNL[q] = w * (dGc_dl * fN - M.Gc * fN / l);
    s.cGL[q] = w * (dGc_dl * fG + (grad != 0.0 ? M.Gc * fG / l : 0.0));
#pragma unroll
    for (int d = 0; d < DIM; ++d) s.dphi[q][d] = gphi[d];
    if (q == NIP - 1) { s.last_Gc = M.Gc; s.last_dGcdl = dGc_dl; s.last_l = l; }
  }
  __syncwarp();
  if (act) {
    const int b = q;
    double FG = 0, FL = 0, WL = 0;
    for (int qq = 0; qq < NIP; ++qq) {
      double N, G[DIM];
      shape_at<DIM, true>(s.e, p.rule, s.g[qq], qq, b, N, G);
      double gd = 0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) gd += G[d] * s.dphi[qq][d];
      FG += s.cNG[qq] * N + s.cGG[qq] * gd;
      FL += s.cNL[qq] * N + s.cGL[qq] * gd;
      WL += s.g[qq].w * N;
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
      FG += WL * ((m.gc_mode == 1) ? 1.0 : 0.0) * DL;
      FL += WL * (s.last_dGcdl * DL - s.last_Gc * DL / l);
    }
    if (mo.irr == IFEM_IRR_PENALTY) {   // PenaltyIrr uses the utility's own Gc = the input gc
      const double ph = s.Ph[b];
      const double PhO = p.sp.old[adof(dm, IFEM_DOF_PHASE, geo.conn[el * NEN + b])];
      const double lim0 = fmin(1.0 - 1.0e-3, fmax(0.0, PhO)), lim1 = 1.0 + 1e-1;
      if (ph < lim0) FG += WL * mo.penalty * (ph - lim0);
      if (ph > lim1) FG += WL * mo.penalty * (ph - lim1);
    }
    const int64_t stride = geo.nel * NEN;
    const int64_t o = el * NEN + b;
    dF[0 * stride + o] = FG;
    dF[1 * stride + o] = FL;
    dF[2 * stride + o] = 0.0;
    dF[3 * stride + o] = 0.0;
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

void launch_adjoint_u(const UParams& p, double* dF, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  const int EPW = p.geo.dim == 2 ? 3 : 1;
  const int64_t blocks = (p.geo.nel + kAWarps * EPW - 1) / (kAWarps * EPW);
  if (p.geo.dim == 2) k_adjoint_u<2><<<(unsigned)blocks, 128, 0, s>>>(p, dF);
  else k_adjoint_u<3><<<(unsigned)blocks, 128, 0, s>>>(p, dF);
}

void launch_adjoint_phase(const PParams& p, double* dF, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  const int EPW = p.geo.dim == 2 ? 3 : 1;
  const int64_t blocks = (p.geo.nel + kAWarps * EPW - 1) / (kAWarps * EPW);
  if (p.geo.dim == 2) k_adjoint_phase<2><<<(unsigned)blocks, 128, 0, s>>>(p, dF);
  else k_adjoint_phase<3><<<(unsigned)blocks, 128, 0, s>>>(p, dF);
}

void launch_adjoint_lambda(const double* dF, int64_t nel, int nc, int nen, const int32_t* conn, const DofMap& dm,
                           int kind0, const double* lambda, double* per_el, const int32_t* mat_ptr,
                           const int32_t* mat_el, int n_mats, double* out, cudaStream_t s) {
  if (nel > 0) k_adjoint_lambda<<<(unsigned)((nel + 127) / 128), 128, 0, s>>>(dF, nel, nc, nen, conn, dm, kind0, lambda, per_el);
  k_adjoint_reduce<<<n_mats, 128, 0, s>>>(per_el, mat_ptr, mat_el, n_mats, out);
}

}  // namespace ifem
