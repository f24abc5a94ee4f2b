// U-step integration points of the 3D quadratic hex with Kronecker-factored extraction, by sum
// factorisation (FP64).
//
// The element basis is separable in the reference coordinates: with C_e = Cz (x) Cy (x) Cx the extracted
// Bernstein function of node a = (ia, ja, ka) at ip q = (qx, qy, qz) is NX[qx][ia] NY[qy][ja] NZ[qz][ka]
// (NX = Cx B, B the 1-D Bernstein values at the Gauss points), and its reference gradient replaces one
// factor by the derivative table.  Interpolating a nodal field to all 27 ips therefore takes three 1-D
// contractions of 3 terms (x, then y, then z) instead of 27 x 27 products, and the residual
// F_a = sum_q B_a(q)^T sigma_q w_q is the transposed contraction (z, then y, then x) of per-ip quantities.
//
// Rational basis (NURBS3_Cube2.cpp:89-115): R_a = W_a N_a / w with w = sum_a W_a N_a, so every nodal field is
// contracted premultiplied by W_a, and
//     sum_a f_a grad R_a = J^{-1} (rw grad(Wf) - (Wf) dW rw^2),  rw = 1/w,
// (the same quotient rule as the node-by-node evaluation, applied to the sums).  The Jacobian comes from the
// same contraction of W X.  For the residual, sum_q G_a(q) . S_q = W_a sum_q [GB_a . (rw P_q) - CB_a (dWr . P_q)]
// with P_q = J_q^{-T} S_q.
//
// The integration-point physics (return map, split, history, C_q) is the same code as the general kernel
// in kernels.cu; only the geometry and the residual assembly change, so results agree with it to
// rounding (sums are taken in a different order).  One warp per element, lane = ip in the ip phase and
// lane = node in the residual phase; the 1-D passes use lanes as (ip, node, node), (ip, ip, node) index
// triples.

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

constexpr int kHWarpsPts = 4;
constexpr int kNF = 13;   // W, W X (3), W U (3), W U_old (3), W phi, W phi_old, W T

constexpr int kNG = 10;                  // fields 0..9 need gradients (W, W X, W U, W U_old)
constexpr int kNA = kNF + kNG, kNB = kNF + 2 * kNG;
struct HexSm {
  double NX[3][3][3], GX[3][3][3];   // [axis][ip coordinate][function]
  // The nodal fields are dead once the x pass has read them, and the y pass output once the z pass has: the two
  // share storage (as do the per-ip residual fields and the transposed y pass output), which keeps four CTAs of
  // four warps within one SM's shared memory.
  union {
    double f[kNF][27];               // nodal fields; reused for the per-ip residual fields
    double B[kNB][27];               // y pass: (qx, qy, ka) rows [0, kNF) N N; kNF + 2 g (+1): N dN, dN N of g < kNG
  } u;
  double A[kNA][27];                 // x pass: (qx, ja, ka) rows [0, kNF) function, kNF + g derivative in x
  double Ph[27];                     // nodal phase (lumped node terms)
  double W[27];
  float tcb[3][32];                  // tensor-core tangent: per-ip ||Jinv|| |rw|, ||Jinv|| max |dWr|, max |C_q|
};

__device__ __forceinline__ int hdof(const DofMap& dm, int kind, int node) { return dm.base[kind] + dm.node_rank[node]; }

// SPL, NI, DAMF >= 0 / > 0: energy split, integral creep exponent and degradation function fixed at compile time
// (every material set shares them; the same arithmetic as the run-time selection, in less code)
// The specialised instance with the reference tangent fits 128 registers with a few spills: four CTAs per SM.
template <typename CT, bool CONS, int SPL, int NI, int DAMF>
__global__ void __launch_bounds__(128, (SPL >= 0 && !CONS) ? 4 : 3) k_u_points_hex(const UParams p) {
  extern __shared__ __align__(16) unsigned char smraw[];
  HexSm* sm = reinterpret_cast<HexSm*>(smraw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t el = p.geo.el0 + (int64_t)blockIdx.x * kHWarpsPts + warp;
  const Geo& geo = p.geo;
  if (el >= geo.el1) return;                     // whole warp; no CTA-wide barrier in this kernel
  HexSm& s = sm[warp];
  const int64_t nh = geo.nel * 27;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const bool act = lane < 27;
  const int q = lane;                             // ip (ip phase) / node (residual phase)

  // ---- nodal fields and 1-D tables ----
  if (act) {
    const int a = lane;
    const int node = geo.conn[el * 27 + a];
    const double W = geo.W ? geo.W[node] : 1.0;
    s.W[a] = W;
    s.u.f[0][a] = W;
#pragma unroll
    for (int c = 0; c < 3; ++c) s.u.f[1 + c][a] = W * geo.X[(int64_t)node * 3 + c];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int d = hdof(dm, IFEM_DOF_UX + c, node);
      s.u.f[4 + c][a] = W * p.su.cur[d];
      s.u.f[7 + c][a] = W * p.su.old[d];
    }
    const int dph = hdof(dm, IFEM_DOF_PHASE, node);
    const double ph = p.sp.cur[dph];
    s.Ph[a] = ph;
    s.u.f[10][a] = W * ph;
    s.u.f[11][a] = W * p.sp.old[dph];
    s.u.f[12][a] = mo.hasT ? W * p.sT.cur[hdof(dm, IFEM_DOF_T, node)] : 0.0;
    const int ax = a / 9, pt = (a / 3) % 3, fn = a % 3;
    const double* Ce = geo.ext + (el * 3 + ax) * 9;
    double sN = 0, sG = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) { sN += Ce[fn * 3 + k] * p.rule.B[pt][k]; sG += Ce[fn * 3 + k] * p.rule.dB[pt][k]; }
    s.NX[ax][pt][fn] = sN;
    s.GX[ax][pt][fn] = sG;
    if (p.nxq) {
      p.nxq[el * kTcNx + a] = (float)sN;
      p.nxq[el * kTcNx + 27 + a] = (float)sG;
      p.nxq[el * kTcNx + 54 + a] = (float)W;
    }
  }
  __syncwarp();
  // ---- x pass: lane = (qx, ja, ka) ----
  if (act) {
    const int qx = lane % 3, jk = lane / 3;       // jk = ja + 3 ka
    const double n0 = s.NX[0][qx][0], n1 = s.NX[0][qx][1], n2 = s.NX[0][qx][2];
    const double g0 = s.GX[0][qx][0], g1 = s.GX[0][qx][1], g2 = s.GX[0][qx][2];
#pragma unroll
    for (int f = 0; f < kNF; ++f) {
      const double v0 = s.u.f[f][3 * jk], v1 = s.u.f[f][3 * jk + 1], v2 = s.u.f[f][3 * jk + 2];
      s.A[f][lane] = n0 * v0 + n1 * v1 + n2 * v2;
      if (f < kNG) s.A[kNF + f][lane] = g0 * v0 + g1 * v1 + g2 * v2;
    }
  }
  __syncwarp();
  // ---- y pass: lane = (qx, qy, ka) ----
  if (act) {
    const int qx = lane % 3, qy = (lane / 3) % 3, ka = lane / 9;
    const double n0 = s.NX[1][qy][0], n1 = s.NX[1][qy][1], n2 = s.NX[1][qy][2];
    const double g0 = s.GX[1][qy][0], g1 = s.GX[1][qy][1], g2 = s.GX[1][qy][2];
    const int i0 = qx + 9 * ka;                   // A index (qx, ja, ka) = qx + 3 ja + 9 ka
#pragma unroll
    for (int f = 0; f < kNF; ++f) {
      const double a0 = s.A[f][i0], a1 = s.A[f][i0 + 3], a2 = s.A[f][i0 + 6];
      s.u.B[f][lane] = n0 * a0 + n1 * a1 + n2 * a2;
      if (f < kNG) {
        s.u.B[kNF + 2 * f][lane] = g0 * a0 + g1 * a1 + g2 * a2;
        const double d0 = s.A[kNF + f][i0], d1 = s.A[kNF + f][i0 + 3], d2 = s.A[kNF + f][i0 + 6];
        s.u.B[kNF + 2 * f + 1][lane] = n0 * d0 + n1 * d1 + n2 * d2;
      }
    }
  }
  __syncwarp();

  unsigned it_count = 0, capped = 0, bad = 0;
  double Jinv[9], rw = 1.0, dWr[3] = {0, 0, 0}, w = 0.0;
  if (act) {
    // ---- z pass: lane = ip (qx, qy, qz) ----
    const int qz = q / 9, i0 = q % 9;             // B index (qx, qy, ka) = qx + 3 qy + 9 ka
    const double n0 = s.NX[2][qz][0], n1 = s.NX[2][qz][1], n2 = s.NX[2][qz][2];
    const double g0 = s.GX[2][qz][0], g1 = s.GX[2][qz][1], g2 = s.GX[2][qz][2];
    double val[kNF], dr[kNG][3];
#pragma unroll
    for (int f = 0; f < kNF; ++f) {
      const double b0 = s.u.B[f][i0], b1 = s.u.B[f][i0 + 9], b2 = s.u.B[f][i0 + 18];
      val[f] = n0 * b0 + n1 * b1 + n2 * b2;
      if (f < kNG) {
        const double* B1 = s.u.B[kNF + 2 * f];
        const double* B2 = s.u.B[kNF + 2 * f + 1];
        dr[f][2] = g0 * b0 + g1 * b1 + g2 * b2;
        dr[f][1] = n0 * B1[i0] + n1 * B1[i0 + 9] + n2 * B1[i0 + 18];
        dr[f][0] = n0 * B2[i0] + n1 * B2[i0 + 9] + n2 * B2[i0 + 18];
      }
    }
    __syncwarp(0x07ffffffu);                      // every ip has read the y pass output: f (its storage) is free
    // ---- geometry at the ip (ip_geometry's quotient rule, applied to the sums) ----
    rw = 1.0 / val[0];
    const double rw2 = rw * rw;
#pragma unroll
    for (int d = 0; d < 3; ++d) dWr[d] = dr[0][d] * rw2;
    double J[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int c = 0; c < 3; ++c) J[d][c] = dr[1 + c][d] * rw - val[1 + c] * dWr[d];
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c10 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c20 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c10 + J[0][2] * c20;
    const double id = 1.0 / det;
    Jinv[0] = c00 * id; Jinv[1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id; Jinv[2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    Jinv[3] = c10 * id; Jinv[4] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id; Jinv[5] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    Jinv[6] = c20 * id; Jinv[7] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id; Jinv[8] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    w = p.rule.wip[q] * fabs(det);
    if (p.geoq) {
      float* gq = p.geoq + el * kTcGeo + q;
#pragma unroll
      for (int i = 0; i < 9; ++i) gq[i * 27] = (float)Jinv[i];
      gq[9 * 27] = (float)rw;
#pragma unroll
      for (int d = 0; d < 3; ++d) gq[(10 + d) * 27] = (float)dWr[d];
      // per-ip factors of the element's bound of max |G| (reduced after the ip phase)
      float jn = 0.0f;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        jn = fmaxf(jn, fabsf((float)Jinv[3 * d]) + fabsf((float)Jinv[3 * d + 1]) + fabsf((float)Jinv[3 * d + 2]));
      s.tcb[0][q] = jn * fabsf((float)rw);
      s.tcb[1][q] = jn * fmaxf(fabsf((float)dWr[0]), fmaxf(fabsf((float)dWr[1]), fabsf((float)dWr[2])));
    }
    // displacement gradients: du^c/dx_d = sum_e Jinv[d][e] (rw d(WU^c)/dxi_e - WU^c dWr_e)
    double gu[3][3], guo[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double H[3], Ho[3];
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        H[e] = dr[4 + c][e] * rw - val[4 + c] * dWr[e];
        Ho[e] = dr[7 + c][e] * rw - val[7 + c] * dWr[e];
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        gu[c][d] = Jinv[d * 3 + 0] * H[0] + Jinv[d * 3 + 1] * H[1] + Jinv[d * 3 + 2] * H[2];
        guo[c][d] = Jinv[d * 3 + 0] * Ho[0] + Jinv[d * 3 + 1] * Ho[1] + Jinv[d * 3 + 2] * Ho[2];
      }
    }
    double eps[6], epsO[6];
    eps[0] = gu[0][0]; eps[1] = gu[1][1]; eps[2] = gu[2][2];
    eps[3] = gu[0][1] + gu[1][0]; eps[4] = gu[1][2] + gu[2][1]; eps[5] = gu[0][2] + gu[2][0];
    epsO[0] = guo[0][0]; epsO[1] = guo[1][1]; epsO[2] = guo[2][2];
    epsO[3] = guo[0][1] + guo[1][0]; epsO[4] = guo[1][2] + guo[2][1]; epsO[5] = guo[0][2] + guo[2][0];
    const double phi = val[10] * rw, phiO = val[11] * rw, Tip = val[12] * rw;

    // ---- integration-point physics (as k_u_points, PhaseField.cpp:382-435, SolidMaterial.cpp:123-301) ----
    const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    double Dam, dDam, unused;
    damage_function<DAMF>(phi, mo.dam_f, mo.k0, mo.porder_p, Dam, dDam, unused);
    const int64_t hi = el * 27 + q;
    double epl[6], eplo[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) { epl[r] = p.h.EP[r * nh + hi]; eplo[r] = p.h.EPo[r * nh + hi]; }
    double hist0 = (M.rheo != IFEM_RHEO_LE) ? p.h.MH[hi] : 0.0;
    int tkind = 0;            // 0 identity, 1 reference factored, 2 full DPl
    RMTan tan;
    double DPl[CONS ? 36 : 1];
    double diss = 0.0;
    const double damdiss = 0.0;
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
    energy_split<false, false, SPL>(M, ee, Sd, Su, nullptr, nullptr, false);
    double sw[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) sw[r] = w * (Dam * Sd[r] + Su[r]);
    double alpha, gamma;
    split_tangent<SPL>(M, ee, Dam, alpha, gamma);
    const double VC[6] = {1, 1, 1, 0.5, 0.5, 0.5};
    CT* Cq = reinterpret_cast<CT*>(p.Cq);
    // [36][nh], or element-major [nel][36][27] for the tensor-core tangent
    auto cq_at = [&](int k) -> int64_t { return p.geoq ? el * kTcCq + k * 27 + q : (int64_t)k * nh + hi; };
    float cmax = 0.0f;                             // max |C_q| of this ip (tensor-core tangent)
    auto cq_put = [&](int k, double v) {
      const CT c = (CT)v;
      Cq[cq_at(k)] = c;
      cmax = fmaxf(cmax, fabsf((float)c));
    };
    if (tkind == 1) {
      const double sa = tan.a[0] + tan.a[1] + tan.a[2];
      double bj[6];
#pragma unroll
      for (int jj = 0; jj < 6; ++jj) bj[jj] = tan.b[jj] / tan.den;
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int jj = 0; jj < 6; ++jj) {
          const double v = (i < 3 ? alpha * ((jj < 3 ? 1.0 : 0.0) - sa * bj[jj]) : 0.0) +
                           gamma * VC[i] * ((i == jj ? 1.0 : 0.0) - tan.a[i] * bj[jj]);
          cq_put(i * 6 + jj, w * v);
        }
    } else if (CONS && tkind == 2) {
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int jj = 0; jj < 6; ++jj) {
          const double v = (i < 3 ? alpha * (DPl[0 * 6 + jj] + DPl[1 * 6 + jj] + DPl[2 * 6 + jj]) : 0.0) +
                           gamma * VC[i] * DPl[(i * 6 + jj) % (CONS ? 36 : 1)];
          cq_put(i * 6 + jj, w * v);
        }
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int jj = 0; jj < 6; ++jj) {
          const double v = ((i < 3 && jj < 3) ? alpha : 0.0) + (i == jj ? gamma * VC[i] : 0.0);
          cq_put(i * 6 + jj, w * v);
        }
    }
    if (p.nxq) s.tcb[2][q] = cmax;
    if (!rr.ok) bad = 1;

    // ---- per-ip residual fields: P = J^{-T} S (S the symmetric stress tensor of sw), Q = rw P, R = P dWr ----
    const double S[3][3] = {{sw[0], sw[3], sw[5]}, {sw[3], sw[1], sw[4]}, {sw[5], sw[4], sw[2]}};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double P[3];
#pragma unroll
      for (int e = 0; e < 3; ++e) P[e] = Jinv[0 * 3 + e] * S[c][0] + Jinv[1 * 3 + e] * S[c][1] + Jinv[2 * 3 + e] * S[c][2];
#pragma unroll
      for (int e = 0; e < 3; ++e) s.u.f[3 * c + e][q] = rw * P[e];
      s.u.f[9 + c][q] = P[0] * dWr[0] + P[1] * dWr[1] + P[2] * dWr[2];
    }
    s.u.f[12][q] = w * rw;
  }
  __syncwarp();
  if (p.nxq) {
    // the element's operand bounds for the tensor-core tangent, in the basis block's padding:
    //   |G_d(node; q)| <= sum_e |Jinv[d][e]| W |GB_e rw - CB dWr_e|
    //                  <= W_max (mG mN^2 max_q ||Jinv||_inf |rw| + mN^3 max_q ||Jinv||_inf max_e |dWr_e|)
    // with mN, mG the largest 1-D basis value and derivative of the element
    float jr = act ? s.tcb[0][lane] : 0.0f, jd = act ? s.tcb[1][lane] : 0.0f, cm = act ? s.tcb[2][lane] : 0.0f;
    float mn = act ? fabsf((float)(&s.NX[0][0][0])[lane]) : 0.0f;
    float mg = act ? fabsf((float)(&s.GX[0][0][0])[lane]) : 0.0f;
    float mw = act ? fabsf((float)s.W[lane]) : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      jr = fmaxf(jr, __shfl_xor_sync(0xffffffffu, jr, o));
      jd = fmaxf(jd, __shfl_xor_sync(0xffffffffu, jd, o));
      cm = fmaxf(cm, __shfl_xor_sync(0xffffffffu, cm, o));
      mn = fmaxf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mg = fmaxf(mg, __shfl_xor_sync(0xffffffffu, mg, o));
      mw = fmaxf(mw, __shfl_xor_sync(0xffffffffu, mw, o));
    }
    if (lane == 0) {
      p.nxq[el * kTcNx + 81] = cm;
      p.nxq[el * kTcNx + 82] = mw * (mg * mn * mn * jr + mn * mn * mn * jd);
    }
  }
  // ---- transposed contraction.  z pass: lane = (qx, qy, ka); Q[c][2] pairs with dN in z ----
  if (act) {
    const int i0 = lane % 9, ka = lane / 9;       // ip index (qx, qy, qz) = i0 + 9 qz
    const double n0 = s.NX[2][0][ka], n1 = s.NX[2][1][ka], n2 = s.NX[2][2][ka];
    const double g0 = s.GX[2][0][ka], g1 = s.GX[2][1][ka], g2 = s.GX[2][2][ka];
#pragma unroll
    for (int k = 0; k < kNF; ++k) {
      const double y0 = s.u.f[k][i0], y1 = s.u.f[k][i0 + 9], y2 = s.u.f[k][i0 + 18];
      const bool dz = (k < 9) && (k % 3 == 2);
      s.A[k][lane] = dz ? (g0 * y0 + g1 * y1 + g2 * y2) : (n0 * y0 + n1 * y1 + n2 * y2);
    }
  }
  __syncwarp();
  // ---- y pass: lane = (qx, ja, ka); Q[c][1] pairs with dN in y ----
  if (act) {
    const int qx = lane % 3, ja = (lane / 3) % 3, ka = lane / 9;
    const double n0 = s.NX[1][0][ja], n1 = s.NX[1][1][ja], n2 = s.NX[1][2][ja];
    const double g0 = s.GX[1][0][ja], g1 = s.GX[1][1][ja], g2 = s.GX[1][2][ja];
    const int i0 = qx + 9 * ka;                   // z-pass index (qx, qy, ka) = qx + 3 qy + 9 ka
#pragma unroll
    for (int k = 0; k < kNF; ++k) {
      const double y0 = s.A[k][i0], y1 = s.A[k][i0 + 3], y2 = s.A[k][i0 + 6];
      const bool dy = (k < 9) && (k % 3 == 1);
      s.u.B[k][lane] = dy ? (g0 * y0 + g1 * y1 + g2 * y2) : (n0 * y0 + n1 * y1 + n2 * y2);
    }
  }
  __syncwarp();
  // ---- x pass: lane = node a = (ia, ja, ka); element residual and lumped node terms ----
  if (act) {
    const int a = lane, ia = a % 3, i0 = a - ia;  // y-pass index (qx, ja, ka) = qx + 3 ja + 9 ka
    const double n0 = s.NX[0][0][ia], n1 = s.NX[0][1][ia], n2 = s.NX[0][2][ia];
    const double g0 = s.GX[0][0][ia], g1 = s.GX[0][1][ia], g2 = s.GX[0][2][ia];
    auto xn = [&](int k) { return n0 * s.u.B[k][i0] + n1 * s.u.B[k][i0 + 1] + n2 * s.u.B[k][i0 + 2]; };
    auto xg = [&](int k) { return g0 * s.u.B[k][i0] + g1 * s.u.B[k][i0 + 1] + g2 * s.u.B[k][i0 + 2]; };
    const double Wa = s.W[a];
    double F[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) F[c] = Wa * (xg(3 * c) + xn(3 * c + 1) + xn(3 * c + 2) - xn(9 + c));
    const double WL = Wa * xn(12);
    const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
    const int node = geo.conn[el * 27 + a];
    double DamI, dDamI, u;
    double kd = 0.0;   // lumped diagonal tangent terms of this node (PhaseField.cpp:441-468)
    if (mo.inertia) {
      damage_function(s.Ph[a], mo.dens_f, mo.k0, mo.porder_p, DamI, dDamI, u);
#pragma unroll
      for (int b = 0; b < 3; ++b) F[b] += WL * DamI * m.density * p.su.dd[hdof(dm, IFEM_DOF_UX + b, node)];
      kd += WL * DamI * m.density * p.ddu_dt;
    }
    if (m.damping > 0.0) {
#pragma unroll
      for (int b = 0; b < 3; ++b) F[b] += WL * m.damping * p.su.d[hdof(dm, IFEM_DOF_UX + b, node)];
      kd += WL * m.damping * p.du_dt;
    }
    if (p.Kd) p.Kd[el * kTcKd + a] = kd;
    double DamG, dDamG;
    damage_function(s.Ph[a], mo.dens_f, mo.k0, mo.porder_p, DamG, dDamG, u);
#pragma unroll
    for (int b = 0; b < 3; ++b) F[b] += -WL * DamG * m.density * mo.g[b];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      p.Fe[el * 81 + b * 27 + a] = F[b];
      if (!isfinite(F[b])) bad = 1;
    }
    p.WLe[el * 27 + a] = WL;
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
// Phase step of the 3D hex by sum factorisation (PhaseField.cpp:541-712): nodal fields to the ips and the
// residual back to the nodes by 1-D passes; the Gram-form tangent keeps per-(ip, node) shape values in the
// tangent's precision, evaluated from the same 1-D tables.
// ============================================================================================
constexpr int kPF = 12;   // W, W X (3), W U (3), W phi, W dU (3), W T; fields 0..7 need gradients

template <typename T>
struct PhexSm {
  using V4 = typename std::conditional<sizeof(T) == 4, float4, double4>::type;
  double NX[3][3][3], GX[3][3][3];
  double f[kPF][27];                 // nodal fields; reused for the per-ip residual fields
  union {
    struct {
      double A[kPF][2][27];
      double B[kPF][3][27];
    } ab;                            // 1-D pass buffers (forward passes, then the transposed ones)
    V4 pk[27][27];                   // (N, G) per (ip, node) in the tangent's precision, between the two
    float pkT[27][116];              // FP32 tangent: per ip the rows N, G0, G1, G2 over the nodes (28 with the pad
                                     // node), 16-byte aligned; the ip stride of 116 keeps 16-byte stores of 8
                                     // consecutive ips in distinct banks
  } u;
  double Ph[27], PhO[27], W[27];
  double kNN[27], kGG[27], lc[27];
  double dg[27];                     // FP32 tangent: the nodes' lumped diagonal terms, for the tile owners
  double last_Gc, last_l, last_visc;
  float fNX[3][3][3], fGX[3][3][3], fW[27];   // the 1-D tables and weights in FP32 (the FP32 tangent's rows)
  float fkNN[27], fkGG[27];                   // the per-ip tangent coefficients in FP32
};

constexpr int kPWarpsHex = 4;

template <typename T, int SPL, int DAMF>
__global__ void __launch_bounds__(128) k_phase_hex(const PParams p) {
  using V4 = typename PhexSm<T>::V4;
  extern __shared__ __align__(16) unsigned char smraw[];
  PhexSm<T>* sm = reinterpret_cast<PhexSm<T>*>(smraw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t el = (int64_t)blockIdx.x * kPWarpsHex + warp;
  const Geo& geo = p.geo;
  if (el >= geo.nel) return;
  PhexSm<T>& s = sm[warp];
  const int64_t nh = geo.nel * 27;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const bool act = lane < 27;
  const int q = lane;
  unsigned bad = 0;

  if (act) {
    const int a = lane;
    const int node = geo.conn[el * 27 + a];
    const double W = geo.W ? geo.W[node] : 1.0;
    s.W[a] = W;
    s.f[0][a] = W;
#pragma unroll
    for (int c = 0; c < 3; ++c) s.f[1 + c][a] = W * geo.X[(int64_t)node * 3 + c];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int d = hdof(dm, IFEM_DOF_UX + c, node);
      s.f[4 + c][a] = W * p.su.cur[d];
      s.f[8 + c][a] = W * p.su.d[d];
    }
    const int dph = hdof(dm, IFEM_DOF_PHASE, node);
    const double ph = p.sp.cur[dph];
    s.Ph[a] = ph;
    s.PhO[a] = p.sp.old[dph];
    s.f[7][a] = W * ph;
    const double Tn = mo.hasT ? (mo.ref_compat_T ? p.sT.cur[0] : p.sT.cur[hdof(dm, IFEM_DOF_T, node)]) : 0.0;
    s.f[11][a] = W * Tn;
    const int ax = a / 9, pt = (a / 3) % 3, fn = a % 3;
    const double* Ce = geo.ext + (el * 3 + ax) * 9;
    double sN = 0, sG = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) { sN += Ce[fn * 3 + k] * p.rule.B[pt][k]; sG += Ce[fn * 3 + k] * p.rule.dB[pt][k]; }
    s.NX[ax][pt][fn] = sN;
    s.GX[ax][pt][fn] = sG;
    s.fNX[ax][pt][fn] = (float)sN;
    s.fGX[ax][pt][fn] = (float)sG;
    s.fW[a] = (float)W;
  }
  __syncwarp();
  if (act) {   // x pass
    const int qx = lane % 3, jk = lane / 3;
    const double n0 = s.NX[0][qx][0], n1 = s.NX[0][qx][1], n2 = s.NX[0][qx][2];
    const double g0 = s.GX[0][qx][0], g1 = s.GX[0][qx][1], g2 = s.GX[0][qx][2];
#pragma unroll
    for (int f = 0; f < kPF; ++f) {
      const double v0 = s.f[f][3 * jk], v1 = s.f[f][3 * jk + 1], v2 = s.f[f][3 * jk + 2];
      s.u.ab.A[f][0][lane] = n0 * v0 + n1 * v1 + n2 * v2;
      if (f < 8) s.u.ab.A[f][1][lane] = g0 * v0 + g1 * v1 + g2 * v2;
    }
  }
  __syncwarp();
  if (act) {   // y pass
    const int qx = lane % 3, qy = (lane / 3) % 3, ka = lane / 9;
    const double n0 = s.NX[1][qy][0], n1 = s.NX[1][qy][1], n2 = s.NX[1][qy][2];
    const double g0 = s.GX[1][qy][0], g1 = s.GX[1][qy][1], g2 = s.GX[1][qy][2];
    const int i0 = qx + 9 * ka;
#pragma unroll
    for (int f = 0; f < kPF; ++f) {
      const double a0 = s.u.ab.A[f][0][i0], a1 = s.u.ab.A[f][0][i0 + 3], a2 = s.u.ab.A[f][0][i0 + 6];
      s.u.ab.B[f][0][lane] = n0 * a0 + n1 * a1 + n2 * a2;
      if (f < 8) {
        s.u.ab.B[f][1][lane] = g0 * a0 + g1 * a1 + g2 * a2;
        s.u.ab.B[f][2][lane] = n0 * s.u.ab.A[f][1][i0] + n1 * s.u.ab.A[f][1][i0 + 3] + n2 * s.u.ab.A[f][1][i0 + 6];
      }
    }
  }
  __syncwarp();
  const int qz = q / 9;
  double val[kPF], dr[8][3];
  if (act) {
    // ---- z pass (into registers) ----
    const int i0 = q % 9;
    const double n0 = s.NX[2][qz][0], n1 = s.NX[2][qz][1], n2 = s.NX[2][qz][2];
    const double g0 = s.GX[2][qz][0], g1 = s.GX[2][qz][1], g2 = s.GX[2][qz][2];
#pragma unroll
    for (int f = 0; f < kPF; ++f) {
      const double b0 = s.u.ab.B[f][0][i0], b1 = s.u.ab.B[f][0][i0 + 9], b2 = s.u.ab.B[f][0][i0 + 18];
      val[f] = n0 * b0 + n1 * b1 + n2 * b2;
      if (f < 8) {
        dr[f][2] = g0 * b0 + g1 * b1 + g2 * b2;
        dr[f][1] = n0 * s.u.ab.B[f][1][i0] + n1 * s.u.ab.B[f][1][i0 + 9] + n2 * s.u.ab.B[f][1][i0 + 18];
        dr[f][0] = n0 * s.u.ab.B[f][2][i0] + n1 * s.u.ab.B[f][2][i0 + 9] + n2 * s.u.ab.B[f][2][i0 + 18];
      }
    }
  }
  __syncwarp();                                   // pass buffers free: pk overwrites them
  if (act) {
    // ---- ip geometry ----
    const double rw = 1.0 / val[0], rw2 = rw * rw;
    double dWr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) dWr[d] = dr[0][d] * rw2;
    double J[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int c = 0; c < 3; ++c) J[d][c] = dr[1 + c][d] * rw - val[1 + c] * dWr[d];
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c10 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c20 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c10 + J[0][2] * c20;
    const double id = 1.0 / det;
    double Jinv[9];
    Jinv[0] = c00 * id; Jinv[1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id; Jinv[2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    Jinv[3] = c10 * id; Jinv[4] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id; Jinv[5] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    Jinv[6] = c20 * id; Jinv[7] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id; Jinv[8] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    const double w = p.rule.wip[q] * fabs(det);
    // physical gradients of u and phi at the ip
    auto pgrad = [&](int f, double out[3]) {
      double H[3];
#pragma unroll
      for (int e = 0; e < 3; ++e) H[e] = dr[f][e] * rw - val[f] * dWr[e];
#pragma unroll
      for (int d = 0; d < 3; ++d) out[d] = Jinv[d * 3 + 0] * H[0] + Jinv[d * 3 + 1] * H[1] + Jinv[d * 3 + 2] * H[2];
    };
    double gu[3][3], gphi[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) pgrad(4 + c, gu[c]);
    pgrad(7, gphi);
    double eps[6];
    eps[0] = gu[0][0]; eps[1] = gu[1][1]; eps[2] = gu[2][2];
    eps[3] = gu[0][1] + gu[1][0]; eps[4] = gu[1][2] + gu[2][1]; eps[5] = gu[0][2] + gu[2][0];
    double uip[3], vip[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { uip[d] = val[4 + d] * rw; vip[d] = val[8 + d] * rw; }
    const double phi = val[7] * rw, Tip = val[11] * rw;
    // ---- ip physics (as k_phase) ----
    const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    double Dam, dDam, ddDam, DamI, dDamI, ddDamI, DamG, dDamG, ddDamG;
    damage_function<DAMF>(phi, mo.dam_f, mo.k0, mo.porder_p, Dam, dDam, ddDam);
    damage_function(phi, mo.dens_f, mo.k0, mo.porder_p, DamI, dDamI, ddDamI);
    damage_function(phi, mo.grav_f, mo.k0, mo.porder_p, DamG, dDamG, ddDamG);
    const int64_t hi = el * 27 + q;
    double ee[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) ee[r] = eps[r] - p.h.EP[r * nh + hi];
    double Sd[6], Su[6];
    double Energy = energy_split<true, false, SPL>(M, ee, Sd, Su, nullptr, nullptr, false);
    if (mo.irr == IFEM_IRR_HIST) {
      const double Eo = p.h.EHo[hi];
      if (Eo > Energy) { if (p.write_hist) p.h.EH[hi] = Eo; Energy = Eo; }
      else if (p.write_hist) p.h.EH[hi] = Energy;
    } else if (p.write_hist) p.h.EH[hi] = Energy;
    const double l = M.l;
    const double dGdG = gphi[0] * gphi[0] + gphi[1] * gphi[1] + gphi[2] * gphi[2];
    double c = 0, nF = 0, nK = 0, grad = 0, gamma = 0;
    switch (mo.dist) {
      case IFEM_DIST_QUADRATIC: c = 1.0 / (2.0 * l); gamma = c * (phi * phi + l * l * dGdG); nF = 2.0 * phi; nK = 2.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LINEAR: c = 3.0 / (8.0 * l); gamma = c * (phi + l * l * dGdG); nF = 1.0; nK = 0.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LINEAR2: c = 1.0 / (4.0 * l); gamma = c * (2.0 * phi + l * l * dGdG); nF = 2.0; nK = 0.0; grad = 2.0 * l * l; break;
      case IFEM_DIST_LOCAL: c = 1.0 / l; gamma = c * (phi * phi); nF = 2.0 * phi; nK = 2.0; grad = 0.0; break;
      case IFEM_DIST_CZM: c = 1.0 / (3.141592 * l); gamma = c * (2.0 * phi - phi * phi + l * l * dGdG); nF = 2.0 * (1.0 - phi); nK = -2.0; grad = 2.0 * l * l; break;
      default: break;
    }
    double capF = 0, capK = 0;
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
      const double v2 = vip[0] * vip[0] + vip[1] * vip[1] + vip[2] * vip[2];
      kNF += -w * 0.5 * m.density * v2 * dDamI; kNN += -w * 0.5 * m.density * v2 * ddDamI;
    }
    if (mo.consistent_deg) {
      const double gu2 = mo.g[0] * uip[0] + mo.g[1] * uip[1] + mo.g[2] * uip[2];
      kNF += -w * m.density * gu2 * dDamG; kNN += -w * m.density * gu2 * ddDamG;
    }
    s.kNN[q] = kNN; s.kGG[q] = kG;
    s.fkNN[q] = (float)kNN; s.fkGG[q] = (float)kG;
    s.lc[q] = gamma * w;
    if (q == 26) { s.last_Gc = M.Gc; s.last_l = M.l; s.last_visc = M.visc; }
    // ---- per-ip residual fields: F_b = W_b sum_q [CB_b Y0 + GB_b . (Y1, Y2, Y3)] ----
    double P[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) P[e] = Jinv[0 * 3 + e] * gphi[0] + Jinv[1 * 3 + e] * gphi[1] + Jinv[2 * 3 + e] * gphi[2];
    s.f[0][q] = kNF * rw - kG * (P[0] * dWr[0] + P[1] * dWr[1] + P[2] * dWr[2]);
#pragma unroll
    for (int e = 0; e < 3; ++e) s.f[1 + e][q] = kG * rw * P[e];
    s.f[4][q] = w * rw;      // lumped weight
    s.f[5][q] = kLD * rw;    // lumped driving
    // (N, G) per node in the tangent's precision, from the same 1-D tables (after the ip physics, whose
    // values are then dead: fewer live registers)
    {
      const int qx = q % 3, qy = (q / 3) % 3;
      const T trw = (T)rw, tw0 = (T)dWr[0], tw1 = (T)dWr[1], tw2 = (T)dWr[2];
      T tJ[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) tJ[i] = (T)Jinv[i];
      auto ng = [&](int a) {
        const int ia = a % 3, ja = (a / 3) % 3, ka = a / 9;
        const T nx = (T)s.NX[0][qx][ia], ny = (T)s.NX[1][qy][ja], nz = (T)s.NX[2][qz][ka];
        const T CB = nx * ny * nz;
        const T GB0 = (T)s.GX[0][qx][ia] * ny * nz, GB1 = nx * (T)s.GX[1][qy][ja] * nz, GB2 = nx * ny * (T)s.GX[2][qz][ka];
        const T Wa = (T)s.W[a];
        const T x0 = Wa * (GB0 * trw - CB * tw0), x1 = Wa * (GB1 * trw - CB * tw1), x2 = Wa * (GB2 * trw - CB * tw2);
        V4 v;
        v.x = Wa * CB * trw;
        v.y = tJ[0] * x0 + tJ[1] * x1 + tJ[2] * x2;
        v.z = tJ[3] * x0 + tJ[4] * x1 + tJ[5] * x2;
        v.w = tJ[6] * x0 + tJ[7] * x1 + tJ[8] * x2;
        return v;
      };
      if constexpr (sizeof(T) == 4) {
        // FP32 tables (no conversions); the lane's 1-D values in registers, the node loop unrolled
        float tnx[3], tny[3], tnz[3], tgx[3], tgy[3], tgz[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          tnx[i] = s.fNX[0][qx][i]; tny[i] = s.fNX[1][qy][i]; tnz[i] = s.fNX[2][qz][i];
          tgx[i] = s.fGX[0][qx][i]; tgy[i] = s.fGX[1][qy][i]; tgz[i] = s.fGX[2][qz][i];
        }
        auto ngf = [&](int a) {
          const int ia = a % 3, ja = (a / 3) % 3, ka = a / 9;
          const float nx = tnx[ia], ny = tny[ja], nz = tnz[ka];
          const float nyz = ny * nz, CB = nx * nyz;
          const float GB0 = tgx[ia] * nyz, GB1 = nx * tgy[ja] * nz, GB2 = nx * ny * tgz[ka];
          const float Wa = s.fW[a];
          const float x0 = Wa * (GB0 * trw - CB * tw0), x1 = Wa * (GB1 * trw - CB * tw1), x2 = Wa * (GB2 * trw - CB * tw2);
          V4 v;
          v.x = Wa * CB * trw;
          v.y = tJ[0] * x0 + tJ[1] * x1 + tJ[2] * x2;
          v.z = tJ[3] * x0 + tJ[4] * x1 + tJ[5] * x2;
          v.w = tJ[6] * x0 + tJ[7] * x1 + tJ[8] * x2;
          return v;
        };
#pragma unroll
        for (int g = 0; g < 7; ++g) {            // nodes 4 g .. 4 g + 3 (node 27 is a zero pad)
          V4 v[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) v[i] = (4 * g + i < 27) ? ngf(4 * g + i) : V4{0, 0, 0, 0};
          float* row = s.u.pkT[q] + 4 * g;
          *reinterpret_cast<float4*>(row) = make_float4(v[0].x, v[1].x, v[2].x, v[3].x);
          *reinterpret_cast<float4*>(row + 28) = make_float4(v[0].y, v[1].y, v[2].y, v[3].y);
          *reinterpret_cast<float4*>(row + 56) = make_float4(v[0].z, v[1].z, v[2].z, v[3].z);
          *reinterpret_cast<float4*>(row + 84) = make_float4(v[0].w, v[1].w, v[2].w, v[3].w);
        }
      } else {
        for (int a = 0; a < 27; ++a) s.u.pk[q][a] = ng(a);
      }
    }
  }
  __syncwarp();
  // ---- tangent K_ab = sum_q kNN N_a N_b + kGG G_a . G_b, before pk is overwritten ----
  // FP32: lane t < 28 owns the 4 x 8 tile of rows 4 (t / 4) .. + 3 and columns 8 (t % 4) .. + 7 (row 27 and the
  // columns past 27 are padding and not stored); per ip and shape row, one 16-byte load of the tile's rows
  // (7 distinct addresses in the warp) and two of its columns (4 distinct), then 16 packed FP32x2 FMAs.
  // FP64: lane b accumulates column b.
  float2 tacc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) tacc[i][j] = make_float2(0.0f, 0.0f);
  T acc[27];
#pragma unroll
  for (int a = 0; a < 27; ++a) acc[a] = (T)0;
  if constexpr (sizeof(T) == 4) {
    if (lane < 28) {
      const int ia = lane >> 2, ib = lane & 3;
      for (int qq = 0; qq < 27; ++qq) {
        const float* row = s.u.pkT[qq];
        const float cn = s.fkNN[qq], cg = s.fkGG[qq];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float cf = c == 0 ? cn : cg;
          const float4 r = *reinterpret_cast<const float4*>(row + 28 * c + 4 * ia);
          const float4 c0 = *reinterpret_cast<const float4*>(row + 28 * c + 8 * ib);
          const float4 c1 = *reinterpret_cast<const float4*>(row + 28 * c + 8 * ib + 4);
          const float rr[4] = {cf * r.x, cf * r.y, cf * r.z, cf * r.w};
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float2 ri = make_float2(rr[i], rr[i]);
            tacc[i][0] = __ffma2_rn(ri, make_float2(c0.x, c0.y), tacc[i][0]);
            tacc[i][1] = __ffma2_rn(ri, make_float2(c0.z, c0.w), tacc[i][1]);
            tacc[i][2] = __ffma2_rn(ri, make_float2(c1.x, c1.y), tacc[i][2]);
            tacc[i][3] = __ffma2_rn(ri, make_float2(c1.z, c1.w), tacc[i][3]);
          }
        }
      }
    }
  } else if (act) {
    const int b = lane;
    {
      for (int qq = 0; qq < 27; ++qq) {
        const V4 mb = s.u.pk[qq][b];
        const T cn = (T)s.kNN[qq], cg = (T)s.kGG[qq];
        const T bx = cn * mb.x, by = cg * mb.y, bz = cg * mb.z, bw = cg * mb.w;
#pragma unroll
        for (int a = 0; a < 27; ++a) {
          const V4 ma = s.u.pk[qq][a];
          acc[a] += bx * ma.x + by * ma.y + bz * ma.z + bw * ma.w;
        }
      }
    }
  }
  __syncwarp();                                   // pk no longer needed: the transposed passes reuse its space
  constexpr int NY = 6;
  if (act) {   // transposed z pass: Y3 pairs with dN in z
    const int i0 = lane % 9, ka = lane / 9;
    const double n0 = s.NX[2][0][ka], n1 = s.NX[2][1][ka], n2 = s.NX[2][2][ka];
    const double g0 = s.GX[2][0][ka], g1 = s.GX[2][1][ka], g2 = s.GX[2][2][ka];
#pragma unroll
    for (int k = 0; k < NY; ++k) {
      const double y0 = s.f[k][i0], y1 = s.f[k][i0 + 9], y2 = s.f[k][i0 + 18];
      s.u.ab.A[k][0][lane] = (k == 3) ? (g0 * y0 + g1 * y1 + g2 * y2) : (n0 * y0 + n1 * y1 + n2 * y2);
    }
  }
  __syncwarp();
  if (act) {   // transposed y pass: Y2 pairs with dN in y
    const int qx = lane % 3, ja = (lane / 3) % 3, ka = lane / 9;
    const double n0 = s.NX[1][0][ja], n1 = s.NX[1][1][ja], n2 = s.NX[1][2][ja];
    const double g0 = s.GX[1][0][ja], g1 = s.GX[1][1][ja], g2 = s.GX[1][2][ja];
    const int i0 = qx + 9 * ka;
#pragma unroll
    for (int k = 0; k < NY; ++k) {
      const double y0 = s.u.ab.A[k][0][i0], y1 = s.u.ab.A[k][0][i0 + 3], y2 = s.u.ab.A[k][0][i0 + 6];
      s.u.ab.B[k][0][lane] = (k == 2) ? (g0 * y0 + g1 * y1 + g2 * y2) : (n0 * y0 + n1 * y1 + n2 * y2);
    }
  }
  __syncwarp();
  if (act) {   // transposed x pass (Y1 pairs with dN in x), node terms, tangent column b
    const int b = lane, ib = b % 3, i0 = b - ib;
    const double n0 = s.NX[0][0][ib], n1 = s.NX[0][1][ib], n2 = s.NX[0][2][ib];
    const double g0 = s.GX[0][0][ib], g1 = s.GX[0][1][ib], g2 = s.GX[0][2][ib];
    auto xn = [&](int k) { return n0 * s.u.ab.B[k][0][i0] + n1 * s.u.ab.B[k][0][i0 + 1] + n2 * s.u.ab.B[k][0][i0 + 2]; };
    auto xg = [&](int k) { return g0 * s.u.ab.B[k][0][i0] + g1 * s.u.ab.B[k][0][i0 + 1] + g2 * s.u.ab.B[k][0][i0 + 2]; };
    const double Wb = s.W[b];
    double F = Wb * (xn(0) + xg(1) + xn(2) + xn(3));
    const double WL = Wb * xn(4), LD = Wb * xn(5);
    const double Gc = s.last_Gc, l = s.last_l, visc = s.last_visc;
    const MatDev& m = geo.mats[geo.emat ? geo.emat[el] : 0];
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
    p.Fe[el * 27 + b] = F;
    if (!isfinite(F)) bad = 1;
    constexpr int KB = ke_block(1, 27);
    T* Ke = reinterpret_cast<T*>(p.Ke) + el * 27 * KB;
    if constexpr (sizeof(T) == 4) {
      s.dg[b] = diag;
    } else {
#pragma unroll
      for (int a = 0; a < 27; ++a) {
        // the diagonal term in FP64, the rest stored as accumulated (one conversion per column)
        Ke[a * KB + b] = (a == b) ? (T)((double)acc[a] + diag) : acc[a];
      }
    }
    if (b == 0) {
      double lcs = 0;
      for (int qq = 0; qq < 27; ++qq) lcs += s.lc[qq];
      p.lcrack_el[el] = lcs;
    }
  }
  if constexpr (sizeof(T) == 4) {
    __syncwarp();
    if (lane < 28) {   // the lane's tile: rows 4 ia + i < 27, columns 8 ib .. 8 ib + 7 (through the pad column 27)
      const int ia = lane >> 2, ib = lane & 3;
      constexpr int KB = ke_block(1, 27);
      float* Ke = reinterpret_cast<float*>(p.Ke) + el * 27 * KB;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int a = 4 * ia + i;
        if (a < 27) {
          float v[8] = {tacc[i][0].x, tacc[i][0].y, tacc[i][1].x, tacc[i][1].y,
                        tacc[i][2].x, tacc[i][2].y, tacc[i][3].x, tacc[i][3].y};
          // the diagonal term in FP64, the rest stored as accumulated
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (8 * ib + j == a) v[j] = (float)((double)v[j] + s.dg[a]);
          float* dst = Ke + a * KB + 8 * ib;
          *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
          if (ib < 3) *reinterpret_cast<float4*>(dst + 4) = make_float4(v[4], v[5], v[6], v[7]);
        }
      }
    }
  }
  const unsigned tot_bad = __reduce_add_sync(0xffffffffu, bad);
  if (lane == 0 && tot_bad) atomicAdd(&p.stats[2], (unsigned long long)tot_bad);
}

template <typename K>
void set_smem_pts(K kernel, size_t bytes) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

template <typename T>
void phase_hex_go(const PParams& p, cudaStream_t s) {
  const int64_t blocks = (p.geo.nel + kPWarpsHex - 1) / kPWarpsHex;
  const size_t smem = sizeof(PhexSm<T>) * kPWarpsHex;
  void (*k)(const PParams) = p.spec ? k_phase_hex<T, IFEM_SPLIT_VOLSTRAINS, IFEM_DAM_QUADRATIC> : k_phase_hex<T, -1, -1>;
  set_smem_pts(k, smem);
  k<<<(unsigned)blocks, 32 * kPWarpsHex, smem, s>>>(p);
}

bool launch_phase_hex(const PParams& p, cudaStream_t s) {
  if (p.geo.dim != 3 || !p.geo.kron || p.geo.nel == 0) return false;
  if (p.ke_f32) phase_hex_go<float>(p, s);
  else phase_hex_go<double>(p, s);
  return true;
}

template <typename CT, bool CONS>
void u_points_hex_go(const UParams& p, cudaStream_t s) {
  const size_t smem = sizeof(HexSm) * kHWarpsPts;
  const int64_t blocks = (p.geo.el1 - p.geo.el0 + kHWarpsPts - 1) / kHWarpsPts;
  void (*k)(const UParams) = p.spec ? k_u_points_hex<CT, CONS, IFEM_SPLIT_VOLSTRAINS, 3, IFEM_DAM_QUADRATIC>
                                    : k_u_points_hex<CT, CONS, -1, 0, -1>;
  set_smem_pts(k, smem);
  cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);   // four CTAs per SM
  k<<<(unsigned)blocks, 32 * kHWarpsPts, smem, s>>>(p);
}

// 3D Kronecker-factored meshes: the sum-factorised points kernel
bool launch_u_points_hex(const UParams& p, cudaStream_t s) {
  if (p.geo.dim != 3 || !p.geo.kron) return false;
  const bool cons = p.mo.tangent_mode == IFEM_TANGENT_CONSISTENT;
  if (p.cq_f32) { if (cons) u_points_hex_go<float, true>(p, s); else u_points_hex_go<float, false>(p, s); }
  else { if (cons) u_points_hex_go<double, true>(p, s); else u_points_hex_go<double, false>(p, s); }
  return true;
}

}  // namespace ifem
