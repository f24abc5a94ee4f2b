// Device-side building blocks shared by the assembly kernels: element geometry (Bezier
// extraction + rational Jacobian), material point laws, energy splits and the Glen return map.
// Each routine cites the reference function it restates.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "icefem_internal.h"

namespace ifem {

template <int DIM> struct ElemTraits;
template <> struct ElemTraits<2> { static constexpr int NEN = 9, NIP = 9; };
template <> struct ElemTraits<3> { static constexpr int NEN = 27, NIP = 27; };

__device__ __forceinline__ int voigt_idx(int b, int p) {
  // strain component of displacement b differentiated along p (ConstructBMat, math.cpp:3-26)
  return b == p ? b : (b + p == 1 ? 3 : (b + p == 3 ? 4 : 5));
}

// ---------------------------------------------------------------------------------------
// Element geometry cache (shared memory), filled cooperatively by the lanes of one element.
// ---------------------------------------------------------------------------------------
template <int DIM, bool KRON>
struct ElemSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  double X[NEN][DIM];
  double W[NEN];
  // KRON: NX[axis][point][i] = sum_k Cax[i][k] B[point][k]; GX likewise with dB
  double NX[DIM][3][3];
  double GX[DIM][3][3];
  double C[KRON ? 1 : NEN * NEN];
};

// per-ip geometry kept to re-evaluate shape gradients node by node
// (3D: wFun holds 1/wFun and dW holds dW/wFun^2)
template <int DIM>
struct IpGeo {
  double Jinv[DIM * DIM];
  double wFun;
  double dW[DIM];
  double w;
};

template <int DIM, bool KRON>
__device__ __forceinline__ void fill_elem(ElemSm<DIM, KRON>& e, const Geo& g, const Rule& R, int64_t el, int t,
                                          int nthr) {
  constexpr int NEN = ElemTraits<DIM>::NEN;
  for (int i = t; i < NEN; i += nthr) {
    const int node = g.conn[el * NEN + i];
#pragma unroll
    for (int d = 0; d < DIM; ++d) e.X[i][d] = g.X[(int64_t)node * DIM + d];
    e.W[i] = (DIM == 3 && g.W) ? g.W[node] : 1.0;
  }
  if (KRON) {
    for (int i = t; i < DIM * 9; i += nthr) {
      const int ax = i / 9, pt = (i / 3) % 3, fn = i % 3;
      const double* Ce = g.ext + (el * DIM + ax) * 9;
      double sN = 0, sG = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) { sN += Ce[fn * 3 + k] * R.B[pt][k]; sG += Ce[fn * 3 + k] * R.dB[pt][k]; }
      e.NX[ax][pt][fn] = sN;
      e.GX[ax][pt][fn] = sG;
    }
  } else {
    for (int i = t; i < NEN * NEN; i += nthr) e.C[i] = g.ext[el * NEN * NEN + i];
  }
}

// CB_a (extraction applied to the Bernstein values) and its parametric gradient GB_a at ip q.
template <int DIM, bool KRON>
__device__ __forceinline__ void bern_at(const ElemSm<DIM, KRON>& e, const Rule& R, int q, int a, double& CB,
                                        double GB[DIM]) {
  if (KRON) {
    if (DIM == 2) {
      const int qx = q % 3, qy = q / 3, ia = a % 3, ja = a / 3;
      CB = e.NX[0][qx][ia] * e.NX[1][qy][ja];
      GB[0] = e.GX[0][qx][ia] * e.NX[1][qy][ja];
      GB[1] = e.NX[0][qx][ia] * e.GX[1][qy][ja];
    } else {
      const int qx = q % 3, qy = (q / 3) % 3, qz = q / 9, ia = a % 3, ja = (a / 3) % 3, ka = a / 9;
      const double nx = e.NX[0][qx][ia], ny = e.NX[1][qy][ja], nz = e.NX[2 % DIM][qz][ka];
      CB = nx * ny * nz;
      GB[0] = e.GX[0][qx][ia] * ny * nz;
      GB[1] = nx * e.GX[1][qy][ja] * nz;
      if (DIM == 3) GB[DIM - 1] = nx * ny * e.GX[DIM - 1][qz][ka];
    }
  } else {
    constexpr int NEN = ElemTraits<DIM>::NEN;
    CB = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) GB[d] = 0;
    if (DIM == 2) {
      const int qx = q % 3, qy = q / 3;
      for (int k = 0; k < NEN; ++k) {
        const int kx = k % 3, ky = k / 3;
        const double c = e.C[a * NEN + k];
        CB += c * (R.B[qx][kx] * R.B[qy][ky]);
        GB[0] += c * (R.dB[qx][kx] * R.B[qy][ky]);
        GB[1] += c * (R.B[qx][kx] * R.dB[qy][ky]);
      }
    } else {
      const int qx = q % 3, qy = (q / 3) % 3, qz = q / 9;
      for (int k = 0; k < NEN; ++k) {
        const int kx = k % 3, ky = (k / 3) % 3, kz = k / 9;
        const double c = e.C[a * NEN + k];
        const double bx = R.B[qx][kx], by = R.B[qy][ky], bz = R.B[qz][kz];
        CB += c * (bx * by * bz);
        GB[0] += c * (R.dB[qx][kx] * by * bz);
        GB[1] += c * (bx * R.dB[qy][ky] * bz);
        GB[DIM - 1] += c * (bx * by * R.dB[qz][kz]);
      }
    }
  }
}

// B2_2::getShapeGrads (B2_2.cpp:72-88) / NURBS3_Cube2::getShapeGrads (NURBS3_Cube2.cpp:89-115):
// Jacobian, its inverse and the ip weight.
template <int DIM, bool KRON>
__device__ void ip_geometry(const ElemSm<DIM, KRON>& e, const Rule& R, int q, IpGeo<DIM>& g) {
  constexpr int NEN = ElemTraits<DIM>::NEN;
  if (DIM == 2) {
    double J[2][2] = {{0, 0}, {0, 0}};  // J(d,e) = sum_a GB(d,a) X(a,e)
    for (int a = 0; a < NEN; ++a) {
      double CB, GB[DIM];
      bern_at<DIM, KRON>(e, R, q, a, CB, GB);
      J[0][0] += GB[0] * e.X[a][0]; J[0][1] += GB[0] * e.X[a][1];
      J[1][0] += GB[1] * e.X[a][0]; J[1][1] += GB[1] * e.X[a][1];
    }
    // transposeInPlace, then Jinv = inverse (the reference's B2_2 applies inv(J^T) to GB)
    const double Jt00 = J[0][0], Jt01 = J[1][0], Jt10 = J[0][1], Jt11 = J[1][1];
    const double det = Jt00 * Jt11 - Jt10 * Jt01;
    const double id = 1.0 / det;
    g.Jinv[0] = Jt11 * id; g.Jinv[1] = -Jt01 * id; g.Jinv[2] = -Jt10 * id; g.Jinv[3] = Jt00 * id;
    g.wFun = 1.0;
    g.dW[0] = g.dW[1] = 0.0;
    g.w = R.wip[q] * fabs(det);
  } else {
    double wFun = 0, dW[3] = {0, 0, 0};
    for (int a = 0; a < NEN; ++a) {
      double CB, GB[DIM];
      bern_at<DIM, KRON>(e, R, q, a, CB, GB);
      wFun += CB * e.W[a];
#pragma unroll
      for (int d = 0; d < DIM; ++d) dW[d] += GB[d] * e.W[a];
    }
    double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    // one reciprocal instead of the quotient-rule divisions (NURBS3_Cube2.cpp:105)
    const double rw = 1.0 / wFun, rw2 = rw * rw;
    double dWr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) dWr[d] = dW[d] * rw2;
    for (int a = 0; a < NEN; ++a) {
      double CB, GB[DIM];
      bern_at<DIM, KRON>(e, R, q, a, CB, GB);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double gx = e.W[a] * (GB[d] * rw - CB * dWr[d]);
#pragma unroll
        for (int c = 0; c < 3; ++c) J[d][c] += gx * e.X[a][c];
      }
    }
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c10 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c20 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c10 + J[0][2] * c20;
    const double id = 1.0 / det;
    g.Jinv[0] = c00 * id; g.Jinv[1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id; g.Jinv[2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    g.Jinv[3] = c10 * id; g.Jinv[4] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id; g.Jinv[5] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    g.Jinv[6] = c20 * id; g.Jinv[7] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id; g.Jinv[8] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    g.wFun = rw;                         // stored as 1/wFun
    g.dW[0] = dWr[0]; g.dW[1] = dWr[1]; g.dW[2] = dWr[2];   // stored as dW/wFun^2
    g.w = R.wip[q] * fabs(det);
  }
}

// Shape function N_a and physical gradient G_a at ip q from the cached ip geometry.
template <int DIM, bool KRON>
__device__ __forceinline__ void shape_at(const ElemSm<DIM, KRON>& e, const Rule& R, const IpGeo<DIM>& g, int q,
                                         int a, double& N, double G[DIM]) {
  double CB, GB[DIM];
  bern_at<DIM, KRON>(e, R, q, a, CB, GB);
  if (DIM == 2) {
    N = CB;
    G[0] = g.Jinv[0] * GB[0] + g.Jinv[1] * GB[1];
    G[1] = g.Jinv[2] * GB[0] + g.Jinv[3] * GB[1];
  } else {
    N = e.W[a] * CB * g.wFun;
    double gx[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) gx[d] = e.W[a] * (GB[d] * g.wFun - CB * g.dW[d]);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      double s = 0;
#pragma unroll
      for (int c = 0; c < DIM; ++c) s += g.Jinv[d * DIM + c] * gx[c];
      G[d] = s;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Material point
// ---------------------------------------------------------------------------------------
struct PtMat {
  double G, lame, K, A, n, Gc, l, visc, phi_lim, star, eref, cred;
  double sy, ya, pa, hard, plv;   // viscoelastic-plastic: yield stress, friction factors, hardening, plastic viscosity
  double bdp;                     // DruckerPrager split
  int rheo, split, ce;
};

// IceMaterial::SetTemperature (IceMaterial.cpp:49-84) with porosity 0.
__device__ __forceinline__ void set_temperature(const MatDev& m, bool pinned, double T, PtMat& p) {
  p.G = m.G; p.lame = m.lame; p.K = m.K; p.n = m.n; p.l = m.l; p.visc = m.visc;
  p.phi_lim = m.phi_visc_lim; p.star = m.star_gamma;
  p.rheo = m.rheology; p.split = m.split; p.ce = m.consistent_energy;
  p.ya = m.yield_alpha; p.pa = m.pot_alpha; p.hard = m.hardening; p.plv = m.pl_visc; p.bdp = m.b_dp;
  if (pinned) {
    p.A = m.A_pin; p.Gc = m.Gc_pin; p.eref = m.eref_pin; p.cred = m.cred_pin; p.sy = m.sy_pin;
    return;
  }
  double TAbs = T + m.t_offset;
  if (TAbs > 273.15) TAbs = 273.15;
  const double ExpTerm = -m.q_creep / kR * (1 / TAbs - 1 / m.t_ref);
  p.A = m.A0 * exp(ExpTerm);
  const double ft = 1.0 * (m.ft0 - m.ftdeg * (TAbs - m.t_ref));
  p.Gc = (m.gc_mode == 1) ? m.gc_input : 2.0 * ft * ft / m.E * m.l;
  p.eref = m.ice_eref; p.cred = m.ice_creduce;
  p.sy = 1.0 * (m.sy0 - m.sydeg * (TAbs - m.t_ref));
  if (m.split == IFEM_SPLIT_ICE) {
    p.eref = m.ice_eref + m.ice_ereduce_fact * sqrt(fmax(1e-3, -(TAbs - m.t_ref)));
    p.cred = m.ice_creduce - (TAbs - m.t_ref) * m.ice_creduce_fact;
  }
}

// PhaseFieldUtility::GenericDamageFunction (PhaseFieldUtil.cpp:77-183)
// DAMF >= 0 fixes the function at compile time (the kernels' specialised instances); -1 reads f.
template <int DAMF = -1>
__device__ __forceinline__ void damage_function(double phi, int f, double k0, double p, double& D, double& dD,
                                                double& ddD) {
  double pl = phi;
  if (pl < 0.0) pl = 0.0;
  if (pl > 1.0) pl = 1.0;
  switch (DAMF >= 0 ? DAMF : f) {
    case IFEM_DAM_NONE: D = 1.0; dD = 0.0; ddD = 0.0; break;
    case IFEM_DAM_LINEAR: D = (1.0 - k0) * (1.0 - pl) + k0; dD = -1.0 * (1.0 - k0); ddD = 0.0; break;
    case IFEM_DAM_LINEAR_NR: D = (1.0 - pl); dD = -1.0; ddD = 0.0; break;
    case IFEM_DAM_QUADRATIC: D = (1.0 - k0) * ((1.0 - pl) * (1.0 - pl)) + k0; dD = -2.0 * (1.0 - k0) * (1.0 - phi); ddD = 2.0 * (1.0 - k0); break;
    case IFEM_DAM_QUADRATIC_NR: D = (1.0 - pl) * (1.0 - pl); dD = -2.0 * (1.0 - phi); ddD = 2.0; break;
    case IFEM_DAM_CUBIC: D = (1.0 - k0) * ((1.0 - pl) * (1.0 - pl) * (1.0 - pl)) + k0; dD = -3.0 * (1.0 - k0) * (1.0 - phi) * (1.0 - phi); ddD = 6.0 * (1.0 - k0) * (1.0 - phi); break;
    case IFEM_DAM_CUBIC_NR: D = (1.0 - pl) * (1.0 - pl) * (1.0 - pl); dD = -3.0 * (1.0 - phi) * (1.0 - phi); ddD = 6.0 * (1.0 - phi); break;
    case IFEM_DAM_PORDER:
      D = (1.0 - k0) * pow((1.0 - pl), p) + k0; dD = -p * (1.0 - k0) * pow((1.0 - phi), p - 1);
      ddD = p > 1 ? p * (p - 1) * (1.0 - k0) * pow((1.0 - phi), p - 2) : 0.0; break;
    case IFEM_DAM_CZM:
      D = (1.0 - k0) * (2.0 * (1 - phi) * (1 - phi) - 1.0 * (1 - phi) * (1 - phi) * (1 - phi)) + k0;
      dD = (1.0 - k0) * (3.0 * (1 - phi) * (1 - phi) - 4.0 * (1 - phi));
      ddD = (1.0 - k0) * (-6.0 * (1 - phi) + 4.0); break;
    case IFEM_DAM_STEP2: D = phi < 0.2 ? 1.0 : 0.0; dD = 0.0; ddD = 0.0; break;
    case IFEM_DAM_STEP5: D = phi < 0.5 ? 1.0 : 0.0; dD = 0.0; ddD = 0.0; break;
    case IFEM_DAM_STEP8: D = phi < 0.8 ? 1.0 : 0.0; dD = 0.0; ddD = 0.0; break;
    default: D = 1.0; dD = 0.0; ddD = 0.0; break;
  }
}

// sigma = D eps for the isotropic D of SolidMaterial.cpp:90-94
__device__ __forceinline__ void apply_D(const PtMat& M, const double e[6], double s[6]) {
  const double tr = e[0] + e[1] + e[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) s[i] = M.lame * tr + 2 * M.G * e[i];
#pragma unroll
  for (int i = 3; i < 6; ++i) s[i] = M.G * e[i];
}

__device__ __forceinline__ double Dij(const PtMat& M, int i, int j) {
  double v = (i < 3 && j < 3) ? M.lame : 0.0;
  if (i == j) v += (i < 3) ? 2 * M.G : M.G;
  return v;
}

// SpecStressSplit energy (PhaseFieldMaterial.cpp:118-151): positive principal part of sigma = D e (with the
// reference's perturbation of near-zero normal and xy components) contracted with the strain.  The symmetric
// 3x3 eigen-decomposition is the cyclic Jacobi method (Golub & Van Loan, Matrix Computations, sec. 8.5); the
// positive part it feeds is the same for any accurate solver.  Not inlined and with scalar arguments: only
// SpecStress contexts call it, and the kernels that contain the call keep their registers and stack.
static __device__ __noinline__ double spec_stress_energy(double lame, double G, double e0, double e1, double e2, double e3,
                                                  double e4, double e5) {
  const double e[6] = {e0, e1, e2, e3, e4, e5};
  const double tr = e0 + e1 + e2;
  double S[6] = {lame * tr + 2 * G * e0, lame * tr + 2 * G * e1, lame * tr + 2 * G * e2, G * e3, G * e4, G * e5};
  for (int i = 0; i < 4; ++i) if (S[i] * S[i] < 1.0e-9) S[i] = (i + 1) * 1e-9;
  double A[3][3] = {{S[0], S[3], S[5]}, {S[3], S[1], S[4]}, {S[5], S[4], S[2]}};
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 16; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (off == 0.0 || off <= 1e-36 * dia) break;
    for (int k = 0; k < 3; ++k) {
      const int p = k == 2 ? 1 : 0, q = k == 0 ? 1 : 2;
      const double apq = A[p][q];
      if (apq == 0.0) continue;
      const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
      const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
      A[p][p] -= t * apq;
      A[q][q] += t * apq;
      A[p][q] = A[q][p] = 0.0;
      const int r = 3 - p - q;
      const double arp = A[r][p], arq = A[r][q];
      A[r][p] = A[p][r] = c * arp - sn * arq;
      A[r][q] = A[q][r] = sn * arp + c * arq;
      for (int i = 0; i < 3; ++i) {
        const double vip = V[i][p], viq = V[i][q];
        V[i][p] = c * vip - sn * viq;
        V[i][q] = sn * vip + c * viq;
      }
    }
  }
  double Sp[6] = {0, 0, 0, 0, 0, 0};   // positive part, Voigt order xx yy zz xy yz xz
  for (int k = 0; k < 3; ++k) {
    const double l = A[k][k];
    if (l > 0) {
      Sp[0] += l * V[0][k] * V[0][k]; Sp[1] += l * V[1][k] * V[1][k]; Sp[2] += l * V[2][k] * V[2][k];
      Sp[3] += l * V[0][k] * V[1][k]; Sp[4] += l * V[1][k] * V[2][k]; Sp[5] += l * V[0][k] * V[2][k];
    }
  }
  double Energy = 0;
  for (int i = 0; i < 6; ++i) Energy += Sp[i] * e[i];
  return 0.5 * Energy;
}

// SpecStrainSplit (PhaseFieldMaterial.cpp:239-290) with GetEigenValues2D (:408-448), and DruckerPragerSplit
// (:292-343): energy, split stresses and (want_D) their full tangents.  Their tangents are not of the
// alpha 11^T + gamma VC form, so only the general kernels' full-tangent variants contain this code.
__device__ inline double split_full(const PtMat& M, const double e[6], double Sd[6], double Su[6], double* Dd,
                                   double* Du, bool want_D) {
  double Energy = 0;
  double dd[36], du[36];
  for (int i = 0; i < 36; ++i) { dd[i] = 0; du[i] = 0; }
  for (int i = 0; i < 6; ++i) { Sd[i] = 0; Su[i] = 0; }
  if (M.split == IFEM_SPLIT_SPECSTRAINS) {
    const double kVC[6] = {1, 1, 1, 0.5, 0.5, 0.5};
    double su[6], sn[6];
    for (int i = 0; i < 6; ++i) { su[i] = kVC[i] * e[i]; sn[i] = su[i]; }
    for (int i = 0; i < 3; ++i) if (fabs(sn[i]) < 1.0e-6) sn[i] = (i + 1.0) * 1.0e-6;
    // principal strains: zz and (xx + yy -/+ sqrt((xx - yy)^2 + 4 xy^2)) / 2; derivatives from the moved values
    double s[3], ds[3][6], h[3][3];   // h[k]: (c2, c1, c3) coefficients of the second derivative
    const double sq = sn[0] * sn[0] + sn[1] * sn[1] - 2.0 * sn[0] * sn[1] + 4 * sn[3] * sn[3];
    const double squ = su[0] * su[0] + su[1] * su[1] - 2.0 * su[0] * su[1] + 4 * su[3] * su[3];
    const double r1 = pow(sq + 2.220446049250313e-16, -0.5), r3 = pow(sq + 2.220446049250313e-16, -1.5);
    const double c1 = 2.0 * sn[3] * (sn[0] - sn[1]) * r3, c2 = 2.0 * sn[3] * sn[3] * r3;
    const double c3 = 2.0 * (sn[0] - sn[1]) * (sn[0] - sn[1]) * r3;
    for (int k = 0; k < 3; ++k) for (int i = 0; i < 6; ++i) ds[k][i] = 0;
    s[0] = su[2]; ds[0][2] = 1.0; h[0][0] = h[0][1] = h[0][2] = 0;
    for (int k = 1; k < 3; ++k) {
      const double sg = 2.0 * k - 3.0;
      s[k] = 0.5 * (su[0] + su[1] + sg * pow(squ, 0.5));
      ds[k][0] = 0.5 + 0.5 * sg * (sn[0] - sn[1]) * r1;
      ds[k][1] = 0.5 + 0.5 * sg * (-sn[0] + sn[1]) * r1;
      ds[k][3] = 2.0 * sg * sn[3] * r1;
      h[k][0] = sg * c2; h[k][1] = sg * c1; h[k][2] = sg * c3;
    }
    // second derivative of principal value k: rows/cols (0, 1, 3) = [[c2, -c2, -c1], [-c2, c2, c1], [-c1, c1, c3]]
    auto dds = [&](int k, int i, int j) -> double {
      const int a = i == 0 ? 0 : (i == 1 ? 1 : (i == 3 ? 2 : -1)), b = j == 0 ? 0 : (j == 1 ? 1 : (j == 3 ? 2 : -1));
      if (a < 0 || b < 0) return 0.0;
      const double C2 = h[k][0], C1 = h[k][1], C3 = h[k][2];
      const double t[3][3] = {{C2, -C2, -C1}, {-C2, C2, C1}, {-C1, C1, C3}};
      return t[a][b];
    };
    const double p0 = s[0] + s[1] + s[2];
    double p1[6];
    for (int i = 0; i < 6; ++i) p1[i] = ds[0][i] + ds[1][i] + ds[2][i];
    if (p0 >= 0) Energy += 0.5 * M.lame * p0 * p0;
    double* Dm = p0 >= 0 ? dd : du;
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j)
      Dm[i * 6 + j] += M.lame * (p0 * (dds(0, i, j) + dds(1, i, j) + dds(2, i, j)) + p1[i] * p1[j]);
    for (int k = 0; k < 3; ++k) {
      if (s[k] >= 0) Energy += M.G * s[k] * s[k];
      double* Dk = s[k] >= 0 ? dd : du;
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j)
        Dk[i * 6 + j] += M.G * (2 * s[k] * dds(k, i, j) + 2 * ds[k][i] * ds[k][j]);
    }
    // back to engineering shears; stresses from the tangents (PhaseFieldMaterial.cpp:281-288)
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) {
      dd[i * 6 + j] *= kVC[i] * kVC[j];
      du[i * 6 + j] *= kVC[i] * kVC[j];
    }
    for (int i = 0; i < 6; ++i) {
      double a = 0, b = 0;
      for (int j = 0; j < 6; ++j) { a += dd[i * 6 + j] * e[j]; b += du[i * 6 + j] * e[j]; }
      Sd[i] = a; Su[i] = b;
    }
  } else {   // DruckerPrager
    const double J2D[6] = {1, 1, 1, 0.5, 0.5, 0.5};
    auto j2m = [&](int i, int j) { return (i == j ? J2D[i] : 0.0) - ((i < 3 && j < 3) ? 1.0 / 3.0 : 0.0); };
    const double B = M.bdp, K = M.K, G = M.G;
    const double I1 = e[0] + e[1] + e[2];
    double dJ2[6];
    for (int i = 0; i < 6; ++i) { double t = 0; for (int j = 0; j < 6; ++j) t += j2m(i, j) * e[j]; dJ2[i] = t; }
    double J2 = 0;
    for (int i = 0; i < 6; ++i) J2 += e[i] * dJ2[i];
    J2 *= 0.5;
    const double sq = sqrt(J2 + 1.0e-16);
    auto ddsq = [&](int i, int j) { return 0.5 / sq * j2m(i, j) - 0.25 / sq / sq / sq * dJ2[i] * dJ2[j]; };
    const bool dam = -6.0 * B * sqrt(J2) < I1;
    if (dam || 2 * G * sqrt(J2) < 3 * B * K * I1) {
      double* S = dam ? Sd : Su;
      double* Dm = dam ? dd : du;
      if (dam) Energy = 0.5 * K * I1 * I1 + 2.0 * G * J2;
      for (int i = 0; i < 6; ++i) S[i] = K * I1 * (i < 3 ? 1.0 : 0.0) + 2.0 * G * dJ2[i];
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dm[i * 6 + j] = K * ((i < 3 && j < 3) ? 1.0 : 0.0) + 2.0 * G * j2m(i, j);
    } else {
      double pre = 1.0 / (18.0 * B * B * K + 2.0 * G);
      double q = -3.0 * B * K * I1 + 2 * G * sq, dq[6];
      for (int i = 0; i < 6; ++i) dq[i] = -3.0 * B * K * (i < 3 ? 1.0 : 0.0) + 2.0 * G * (0.5 / sq * dJ2[i]);
      Energy = pre * q * q;
      for (int i = 0; i < 6; ++i) Sd[i] = pre * 2.0 * q * dq[i];
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) dd[i * 6 + j] = pre * (2.0 * q * 2.0 * G * ddsq(i, j) + 2.0 * dq[i] * dq[j]);
      pre = K * G / (18.0 * B * B * K + 2.0 * G);
      q = I1 + 6 * B * sq;
      for (int i = 0; i < 6; ++i) dq[i] = (i < 3 ? 1.0 : 0.0) + 6 * B * (0.5 / sq * dJ2[i]);
      for (int i = 0; i < 6; ++i) Su[i] = pre * 2.0 * q * dq[i];
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) du[i * 6 + j] = pre * (2.0 * q * 6 * B * ddsq(i, j) + 2.0 * dq[i] * dq[j]);
    }
  }
  if (want_D) for (int i = 0; i < 36; ++i) { Dd[i] = dd[i]; Du[i] = du[i]; }
  return Energy;
}

// PhaseFieldMaterial::EnergySplit (PhaseFieldMaterial.cpp:47-117,194-245,356-408).
// Dd/Du are only formed when want_D is set.  ENERGY = false: the caller ignores the energy (u-step), so the
// SpecStress energy is not evaluated.  FULLSPLITS: SpecStrains and DruckerPrager are compiled in (general
// kernels' full-tangent variants; other kernels never see them).
template <bool ENERGY = true, bool FULLSPLITS = false, int SPL = -1>
__device__ inline double energy_split(const PtMat& M, const double e[6], double Sd[6], double Su[6], double* Dd,
                               double* Du, bool want_D) {
  const int split = SPL >= 0 ? SPL : M.split;   // SPL >= 0: the split is known at compile time
  const double kVC[6] = {1, 1, 1, 0.5, 0.5, 0.5};
  const double kVDD[6] = {1, 1, 1, 2, 2, 2};
  double Energy = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) { Sd[i] = 0; Su[i] = 0; }
  if (want_D) for (int i = 0; i < 36; ++i) { Dd[i] = 0; Du[i] = 0; }
  auto devproj = [](int r, int c) { return (r == c ? 1.0 : 0.0) - ((r < 3 && c < 3) ? 1.0 / 3.0 : 0.0); };
  switch (split) {
    case IFEM_SPLIT_NONE: {
      apply_D(M, e, Sd);
      if (want_D) for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dd[i * 6 + j] = Dij(M, i, j);
      for (int i = 0; i < 6; ++i) Energy += 0.5 * Sd[i] * e[i];
    } break;
    case IFEM_SPLIT_VOLSTRAINS: {
      const double p = e[0] + e[1] + e[2];
      if (p >= 0) {
        Energy += 0.5 * M.K * p * p;
        for (int i = 0; i < 3; ++i) Sd[i] += M.K * p;
        if (want_D) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Dd[i * 6 + j] += M.K;
      } else {
        for (int i = 0; i < 3; ++i) Su[i] += M.K * p;
        if (want_D) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Du[i * 6 + j] += M.K;
      }
      double dev[6], ed = 0;
      for (int i = 0; i < 6; ++i) dev[i] = kVC[i] * e[i] - 1.0 / 3.0 * p * (i < 3 ? 1.0 : 0.0);
      for (int i = 0; i < 6; ++i) ed += dev[i] * kVDD[i] * dev[i];
      Energy += M.G * ed;
      for (int i = 0; i < 6; ++i) Sd[i] += 2 * M.G * kVC[i] * kVDD[i] * dev[i];
      if (want_D) for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dd[i * 6 + j] += 2 * M.G * kVC[i] * kVDD[i] * kVC[i] * devproj(i, j);
    } break;
    case IFEM_SPLIT_VOLSTRESS: {
      double S[6];
      apply_D(M, e, S);
      const double p = 1.0 / 3.0 * (S[0] + S[1] + S[2]);
      if (p >= 0) { for (int i = 0; i < 3; ++i) Sd[i] += p; }
      else { for (int i = 0; i < 3; ++i) Su[i] += p; }
      for (int i = 0; i < 6; ++i) Sd[i] += S[i] - (i < 3 ? p : 0.0);
      if (want_D) {
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) {
          const double iiD = (i < 3) ? 1.0 / 3.0 * (Dij(M, 0, j) + Dij(M, 1, j) + Dij(M, 2, j)) : 0.0;
          if (p >= 0) Dd[i * 6 + j] += iiD; else Du[i * 6 + j] += iiD;
          double s = 0;
          for (int k = 0; k < 6; ++k) s += devproj(i, k) * Dij(M, k, j);
          Dd[i * 6 + j] += s;
        }
      }
      for (int i = 0; i < 6; ++i) Energy += 0.5 * Sd[i] * e[i];
    } break;
    case IFEM_SPLIT_STARCONVEX:
    case IFEM_SPLIT_ICE: {
      const double p = e[0] + e[1] + e[2];
      double pplus, pmin, dpplus, dpmin;
      if (p >= 0) { pplus = p; dpplus = 1.0; pmin = 0.0; dpmin = 0.0; }
      else { pplus = 0.0; dpplus = 0.0; pmin = p; dpmin = 1.0; }
      double dev[6], ed = 0;
      for (int i = 0; i < 6; ++i) dev[i] = kVC[i] * e[i] - 1.0 / 3.0 * p * (i < 3 ? 1.0 : 0.0);
      for (int i = 0; i < 6; ++i) ed += dev[i] * kVDD[i] * dev[i];
      double Ddl[36], Dul[36];
      for (int i = 0; i < 36; ++i) { Ddl[i] = 0; Dul[i] = 0; }
      if (split == IFEM_SPLIT_STARCONVEX) {
        const double g = M.star;
        Energy += 0.5 * M.K * (pplus * pplus - g * pmin * pmin);
        for (int i = 0; i < 3; ++i) {
          Sd[i] += M.K * (pplus * dpplus - g * pmin * dpmin);
          Su[i] += (1.0 + g) * M.K * pmin * dpmin;
          for (int j = 0; j < 3; ++j) {
            Ddl[i * 6 + j] += M.K * (dpplus * dpplus - g * dpmin * dpmin);
            Dul[i * 6 + j] += (1.0 + g) * M.K * dpmin * dpmin;
          }
        }
        Energy += M.G * ed;
        for (int i = 0; i < 6; ++i) Sd[i] += 2 * M.G * kVC[i] * kVDD[i] * dev[i];
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Ddl[i * 6 + j] += 2 * M.G * kVC[i] * kVDD[i] * kVC[i] * devproj(i, j);
      } else {
        Energy += 0.5 * M.K * pplus * pplus;
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
          Ddl[i * 6 + j] += M.K * dpplus * dpplus;
          Dul[i * 6 + j] += M.K * dpmin * dpmin;
        }
        Energy += M.G * ed;
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Ddl[i * 6 + j] += 2 * M.G * kVC[i] * kVDD[i] * kVC[i] * devproj(i, j);
        Energy += -0.5 * M.K * M.cred * pmin * pmin / (M.eref * M.eref + pmin * pmin);
        for (int i = 0; i < 6; ++i) {
          double s1 = 0, s2 = 0;
          for (int j = 0; j < 6; ++j) { s1 += Ddl[i * 6 + j] * e[j]; s2 += Dul[i * 6 + j] * e[j]; }
          Sd[i] = s1; Su[i] = s2;
        }
        if (Energy < 0.0) Energy = 0.0;
        if (Energy > 1.0e12 || isnan(Energy)) Energy = 1.0e12;
        if (Energy < -1.0e12) Energy = -1.0e12;
      }
      if (want_D) for (int i = 0; i < 36; ++i) { Dd[i] = Ddl[i]; Du[i] = Dul[i]; }
    } break;
    case IFEM_SPLIT_SPECSTRESS:   // energy only; stresses and tangents are D e / D (consistent_energy = 0)
      if (ENERGY) Energy = spec_stress_energy(M.lame, M.G, e[0], e[1], e[2], e[3], e[4], e[5]);
      break;
    case IFEM_SPLIT_SPECSTRAINS:
    case IFEM_SPLIT_DRUCKERPRAGER:
      if (FULLSPLITS) Energy = split_full(M, e, Sd, Su, Dd, Du, want_D);
      break;
    default: break;
  }
  if (M.ce == 0) {
    apply_D(M, e, Sd);
    for (int i = 0; i < 6; ++i) Su[i] = 0;
    if (want_D) for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) { Dd[i * 6 + j] = Dij(M, i, j); Du[i * 6 + j] = 0; }
  }
  return Energy;
}

// (Dam*D_Dam + D_UnDam) of every supported split has the form alpha * 1 1^T (normal block) +
// gamma * VoightCorrect (diagonal): VolStrains/VolStress give K[p>=0] - 2G/3 on the normal block and
// 2G VC; NoSplit gives lame and 2G VC; StarConvex/ICE shift the volumetric part
// (PhaseFieldMaterial.cpp:57-94,97-117,194-245,356-408).
template <int SPL = -1>
__device__ __forceinline__ void split_tangent(const PtMat& M, const double e[6], double Dam, double& alpha,
                                              double& gamma) {
  const int split = SPL >= 0 ? SPL : M.split;
  gamma = Dam * 2.0 * M.G;
  if (M.ce == 0 || split == IFEM_SPLIT_NONE) { alpha = Dam * M.lame; return; }
  double p = e[0] + e[1] + e[2];
  if (split == IFEM_SPLIT_VOLSTRESS) {
    double S[6];
    apply_D(M, e, S);
    p = 1.0 / 3.0 * (S[0] + S[1] + S[2]);
  }
  const double dpp = p >= 0 ? 1.0 : 0.0, dpm = p >= 0 ? 0.0 : 1.0;
  switch (split) {
    case IFEM_SPLIT_STARCONVEX:
      alpha = Dam * (M.K * (dpp * dpp - M.star * dpm * dpm) - M.G * (2.0 / 3.0)) + (1.0 + M.star) * M.K * dpm * dpm;
      break;
    default:   // VolStrains, VolStress, ICE
      alpha = Dam * (M.K * dpp - M.G * (2.0 / 3.0)) + M.K * dpm;
      break;
  }
}

// x^n with exact repeated multiplication for small integral n, pow() otherwise.  NI > 0: n == NI is known at
// compile time (the same products, in the same order).
template <int NI = 0>
__device__ __forceinline__ double pown(double x, double n) {
  if constexpr (NI > 0) {
    double v = 1.0;
#pragma unroll
    for (int i = 0; i < NI; ++i) v *= x;
    return v;
  }
  const double r = rint(n);
  if (r == n && r >= 0.0 && r <= 8.0) {
    double v = 1.0;
    for (int i = 0; i < (int)r; ++i) v *= x;
    return v;
  }
  return pow(x, n);
}

// YieldFunctionVE (SolidMaterial.cpp:477-492): J2Mat_stress applied structurally
// The stress scale sc = 1e6 divides by multiplication with its reciprocal (a double division is a long
// dependent instruction sequence on the GPU; the two differ by at most one rounding).
constexpr double kInvSc = 1.0e-6;

__device__ __forceinline__ double yield_ve(const double S[6], double dF[6], double& J2) {
  const double sc = 1.0e6, eps = 1.0e-12;
  double Ss[6], dJ2[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) Ss[i] = S[i] * kInvSc;
  const double m = (Ss[0] + Ss[1] + Ss[2]) * (1.0 / 3.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) dJ2[i] = Ss[i] - m;
#pragma unroll
  for (int i = 3; i < 6; ++i) dJ2[i] = 2.0 * Ss[i];
  J2 = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) J2 += Ss[i] * dJ2[i];
  J2 *= 0.5;
  const double F = sc * sqrt(2.0 * J2);
  const double c = 0.7071067811865476 * rsqrt(J2 + eps);   // 0.5 sqrt(2) / sqrt(J2 + eps)
#pragma unroll
  for (int i = 0; i < 6; ++i) dF[i] = c * dJ2[i];
  return F;
}

// return_mapping_getKF (SolidMaterial.cpp:278-301): f and K = [[I, a],[b^T, -1]]
template <int NI = 0>
__device__ __forceinline__ void rm_getKF(const PtMat& M, double f[7], double a[6], double b[6], const double sol[7],
                                         const double eps_t[6], const double eplo[6], double damage, double dt) {
  double S[6], dF[6], J2;
  apply_D(M, sol, S);
  const double F = yield_ve(S, dF, J2);
#pragma unroll
  for (int i = 0; i < 6; ++i) { f[i] = sol[i] - eps_t[i] + eplo[i] + sol[6] * dF[i]; a[i] = dF[i]; }
  const double sc = 1.0e6;
  const double PreFac = M.A * dt * pown<NI>(sc, M.n);
  const double Fs = F * kInvSc;
  const double pm1 = pown<(NI > 1 ? NI - 1 : 0)>(Fs, M.n - 1.0);
  f[6] = PreFac * (pm1 * Fs) - sol[6];
  const double coef = M.n * PreFac * kInvSc * pm1;
  double DdF[6];
  double ddF[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) ddF[i] = damage * dF[i];
  apply_D(M, ddF, DdF);  // D symmetric: (damage dF)^T D = D (damage dF)
#pragma unroll
  for (int j = 0; j < 6; ++j) b[j] = coef * DdF[j];
}

// Exact Jacobian of the local system (consistent tangent), row-major 7x7.
__device__ inline void rm_exact_jacobian(const PtMat& M, const double sol[7], double dt, double Kx[49]) {
  const double sc = 1.0e6, eps = 1.0e-12;
  double S[6], dF[6], J2;
  apply_D(M, sol, S);
  yield_ve(S, dF, J2);
  double Ss[6], dJ2[6];
  for (int i = 0; i < 6; ++i) Ss[i] = S[i] * kInvSc;
  const double m = (Ss[0] + Ss[1] + Ss[2]) * (1.0 / 3.0);
  for (int i = 0; i < 3; ++i) dJ2[i] = Ss[i] - m;
  for (int i = 3; i < 6; ++i) dJ2[i] = 2.0 * Ss[i];
  const double c = 0.7071067811865476 * rsqrt(J2 + eps);   // 0.5 sqrt(2) / sqrt(J2 + eps)
  // H = c/sc (J2Mat - 1/(2(J2+eps)) dJ2 dJ2^T);  Kx(0:5,0:5) = I + dl * H D
  for (int i = 0; i < 6; ++i) {
    double HD[6];
    for (int j = 0; j < 6; ++j) {
      double s = 0;
      for (int k = 0; k < 6; ++k) {
        const double j2 = (i == k ? 1.0 : 0.0) - ((i < 3 && k < 3) ? 1.0 / 3.0 : 0.0) + ((i == k && i >= 3) ? 1.0 : 0.0);
        const double H = c * kInvSc * (j2 - 0.5 / (J2 + eps) * dJ2[i] * dJ2[k]);
        s += H * Dij(M, k, j);
      }
      HD[j] = s;
    }
    for (int j = 0; j < 6; ++j) Kx[i * 7 + j] = (i == j ? 1.0 : 0.0) + sol[6] * HD[j];
    Kx[i * 7 + 6] = c * dJ2[i];
  }
  const double F = sc * sqrt(2.0 * J2);
  const double PreFac = M.A * dt * pown(sc, M.n);
  const double coef = (J2 > 0) ? M.n * PreFac * kInvSc * pown(F * kInvSc, M.n - 1.0) / sqrt(2.0 * J2) : 0.0;
  double DdJ[6];
  apply_D(M, dJ2, DdJ);
  for (int j = 0; j < 6; ++j) Kx[6 * 7 + j] = coef * DdJ[j];
  Kx[6 * 7 + 6] = -1.0;
}

// In-register 7x7 inverse by Gauss-Jordan with partial pivoting; returns false if singular.
__device__ inline bool inv7(double A[49], double Ai[49]) {
  for (int i = 0; i < 49; ++i) Ai[i] = (i % 8 == 0) ? 1.0 : 0.0;
  for (int k = 0; k < 7; ++k) {
    int p = k;
    double best = fabs(A[k * 7 + k]);
    for (int i = k + 1; i < 7; ++i) if (fabs(A[i * 7 + k]) > best) { best = fabs(A[i * 7 + k]); p = i; }
    if (best == 0.0) return false;
    if (p != k) for (int j = 0; j < 7; ++j) {
      double t = A[k * 7 + j]; A[k * 7 + j] = A[p * 7 + j]; A[p * 7 + j] = t;
      t = Ai[k * 7 + j]; Ai[k * 7 + j] = Ai[p * 7 + j]; Ai[p * 7 + j] = t;
    }
    const double ip = 1.0 / A[k * 7 + k];
    for (int j = 0; j < 7; ++j) { A[k * 7 + j] *= ip; Ai[k * 7 + j] *= ip; }
    for (int i = 0; i < 7; ++i) {
      if (i == k) continue;
      const double fct = A[i * 7 + k];
      if (fct == 0.0) continue;
      for (int j = 0; j < 7; ++j) { A[i * 7 + j] -= fct * A[k * 7 + j]; Ai[i * 7 + j] -= fct * Ai[k * 7 + j]; }
    }
  }
  return true;
}

struct RMResult { int iters; bool capped; bool ok; };

// Reference return-map tangent in factored form: DPlast = I - a b^T / den
struct RMTan { double a[6], b[6], den; };

// return_mapping_Viscous (SolidMaterial.cpp:200-269).  Newton loop bounded by maxit.
template <int NI = 0>
__device__ inline RMResult return_mapping_viscous(const PtMat& M, double DMat[36], double epl[6], const double eps_t[6],
                                           const double eplo[6], double damage, double dt, double& hist0,
                                           int tol_mode, int maxit, int tangent_mode, double& diss,
                                           RMTan* tan = nullptr, double* sol_out = nullptr) {
  double sol[7], f[7], a[6], b[6], dsol[7];
#pragma unroll
  for (int i = 0; i < 6; ++i) sol[i] = eps_t[i] - epl[i];
  sol[6] = hist0;
  rm_getKF<NI>(M, f, a, b, sol, eps_t, eplo, damage, dt);
  double e0 = 0;
#pragma unroll
  for (int i = 0; i < 7; ++i) e0 += f[i] * f[i];
  e0 = fmax(e0, 1e-12);
  double eprev = 1e300;
  RMResult r{0, false, true};
  bool conv = false;
  int it = 0;
  while (!conv) {
    it += 1;
    // dsol = -K^{-1} f with K = [[I, a],[b^T, -1]] (closed-form Schur complement)
    double bf = 0, ba = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) { bf += b[i] * f[i]; ba += b[i] * a[i]; }
    const double x6 = (bf - f[6]) / (1.0 + ba);
#pragma unroll
    for (int i = 0; i < 6; ++i) { dsol[i] = -(f[i] - a[i] * x6); sol[i] += dsol[i]; }
    dsol[6] = -x6;
    sol[6] += dsol[6];
    double ls2 = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) ls2 += f[i] * dsol[i];
    rm_getKF<NI>(M, f, a, b, sol, eps_t, eplo, damage, dt);
    double ls1 = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) ls1 += f[i] * dsol[i];
    double ls;
    if ((ls1 - ls2) == 0.0) ls = 1.0;
    else {
      const double s = (ls1 - ls2) > 0 ? 1.0 : ((ls1 - ls2) < 0 ? -1.0 : 0.0);
      ls = -(ls2) / (fabs(ls1 - ls2) + 1e-12) * s;
      ls = fmin(fmax(ls, 0.2), 1.0);
    }
#pragma unroll
    for (int i = 0; i < 7; ++i) sol[i] = sol[i] - (1.0 - ls) * dsol[i];
    rm_getKF<NI>(M, f, a, b, sol, eps_t, eplo, damage, dt);
    double e = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) e += f[i] * f[i];
    if (tol_mode == IFEM_RM_REFERENCE) {
      if (e < 1.0e-16 || e < 1.0e-9 * e0) conv = true;   // e / e0 < 1e-9 without the division (e0 > 0)
    } else {
      if (e < 1.0e-36 || (it >= 3 && e >= eprev)) conv = true;
    }
    eprev = e;
    if (it > maxit) { conv = true; r.capped = true; }
  }
  r.iters = it;
  double S[6], dF[6], J2;
  apply_D(M, sol, S);
  yield_ve(S, dF, J2);
#pragma unroll
  for (int i = 0; i < 6; ++i) epl[i] = eplo[i] + sol[6] * dF[i];
  if (tangent_mode == IFEM_TANGENT_REFERENCE) {
    double ba = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) ba += b[i] * a[i];
    const double den = 1.0 + ba;
    if (tan) {
#pragma unroll
      for (int i = 0; i < 6; ++i) { tan->a[i] = a[i]; tan->b[i] = b[i]; }
      tan->den = den;
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) DMat[i * 6 + j] = (i == j ? 1.0 : 0.0) - a[i] * b[j] / den;
    }
  } else {
    double Kx[49], Ki[49];
    rm_exact_jacobian(M, sol, dt, Kx);
    r.ok = inv7(Kx, Ki);
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) DMat[i * 6 + j] = Ki[i * 7 + j];
  }
  double d = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) d += S[i] * (epl[i] - eplo[i]);
  d = damage * d;
  diss = fabs(d) / dt;
  hist0 = sol[6];
  if (sol_out)
#pragma unroll
    for (int i = 0; i < 7; ++i) sol_out[i] = sol[i];
  return r;
}

// Sensitivities of the converged elastic strain to theta = (A at TRef, n): implicit differentiation
// of the local system f(x; theta) = 0 with f6 = A dt sc^n (F/sc)^n - dlambda (SolidMaterial.cpp:295-297):
// dx/dtheta = -Kx^{-1} df/dtheta, df/dtheta = (0,...,0, df6/dtheta).
__device__ inline void rm_param_sensitivity(const PtMat& M, double A_over_A0, const double sol[7], double dt,
                                            double dA[6], double dn[6]) {
  double Kx[49], Ki[49];
  rm_exact_jacobian(M, sol, dt, Kx);
  if (!inv7(Kx, Ki)) {
    for (int i = 0; i < 6; ++i) { dA[i] = 0; dn[i] = 0; }
    return;
  }
  double S[6], dF[6], J2;
  apply_D(M, sol, S);
  const double F = yield_ve(S, dF, J2);
  const double sc = 1.0e6;
  const double Fn = pown(sc, M.n) * pown(F * kInvSc, M.n);
  const double df6_dA0 = A_over_A0 * dt * Fn;
  const double df6_dn = (F > 0) ? M.A * dt * Fn * log(F) : 0.0;
  for (int i = 0; i < 6; ++i) {
    dA[i] = -Ki[i * 7 + 6] * df6_dA0;
    dn[i] = -Ki[i * 7 + 6] * df6_dn;
  }
}

// ---------------------------------------------------------------------------------------
// Viscoelastic-plastic return map (SolidMaterial.cpp:303-521).  Unknowns x = [eps_e (6), dLambda_v,
// dLambda_p], unscaled stresses.  With the isotropic D: P D and J2Mat D are closed forms,
//   (P D)_ij     = 2G (d_ij - 1/3) for i, j < 3, G on the shear diagonal;
//   (J2Mat D)_ij = 2G (d_ij - 1/3) for i, j < 3, 2G on the shear diagonal.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void vep_P(const double S[6], double o[6]) {   // P = I - 1/3 i i^T
  const double m = (S[0] + S[1] + S[2]) * (1.0 / 3.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) o[i] = S[i] - m;
#pragma unroll
  for (int i = 3; i < 6; ++i) o[i] = S[i];
}

// J2 = 1/2 S^T J2Mat S and dJ2 = J2Mat S
__device__ __forceinline__ double vep_J2(const double S[6], double dJ2[6]) {
  const double m = (S[0] + S[1] + S[2]) * (1.0 / 3.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) dJ2[i] = S[i] - m;
#pragma unroll
  for (int i = 3; i < 6; ++i) dJ2[i] = 2.0 * S[i];
  double J2 = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) J2 += S[i] * dJ2[i];
  return 0.5 * J2;
}

// apex branch of YieldFunction / PotentialFunction, decided by the trial stress (SolidMaterial.cpp:459-463)
__device__ __forceinline__ bool vep_apex(const PtMat& M, const double St[6]) {
  return M.ya > 0.0 && (St[0] + St[1] + St[2]) > M.sy * 3.0 / M.ya;
}

// YieldFunction (SolidMaterial.cpp:447-475) value and gradient; the Hessian is not needed by getKF
__device__ inline double vep_yield(const PtMat& M, const double S[6], bool apex, double dF[6]) {
  const double I1 = S[0] + S[1] + S[2];
  if (apex) {
#pragma unroll
    for (int i = 0; i < 6; ++i) dF[i] = i < 3 ? M.ya / 3.0 : 0.0;
    return M.ya / 3.0 * I1 - M.sy;
  }
  double dJ2[6];
  const double J2 = vep_J2(S, dJ2);
  const double c = 0.5 * sqrt(3.0) / sqrt(J2 + 1.0e-6);
#pragma unroll
  for (int i = 0; i < 6; ++i) dF[i] = c * dJ2[i] + (i < 3 ? M.ya / 3.0 : 0.0);
  return sqrt(3.0 * J2 + 1.0e-6) + M.ya / 3.0 * I1 - M.sy;
}

// PotentialFunction (SolidMaterial.cpp:494-521): normalised gradient dG; the Hessian as the factors of
// ddG = c J2Mat - c2 dJ2 dJ2^T (c = c2 = 0 at the apex)
__device__ inline void vep_potential(const PtMat& M, const double S[6], const double St[6], bool apex, double dG[6],
                                     double dJ2[6], double& c, double& c2) {
  if (!apex) {
    const double J2 = vep_J2(S, dJ2);
    c = 0.5 * sqrt(3.0) / sqrt(J2 + 1.0e-6);
    c2 = 0.25 * sqrt(3.0) * pow(J2 + 1.0e-6, -1.5);
#pragma unroll
    for (int i = 0; i < 6; ++i) dG[i] = c * dJ2[i] + (i < 3 ? M.pa / 3.0 : 0.0);
  } else {
    // dG = D^-1 (St - 3 sy / ya i): isotropic compliance, normal block (I - lame/(2G + 3 lame) 11^T) / 2G
    double dS[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) dS[i] = St[i] - (i < 3 ? 3.0 * M.sy / M.ya : 0.0);
    const double tr = dS[0] + dS[1] + dS[2];
    const double k = M.lame / (2.0 * M.G + 3.0 * M.lame);
#pragma unroll
    for (int i = 0; i < 3; ++i) dG[i] = (dS[i] - k * tr) / (2.0 * M.G);
#pragma unroll
    for (int i = 3; i < 6; ++i) dG[i] = dS[i] / M.G;
#pragma unroll
    for (int i = 0; i < 6; ++i) dJ2[i] = 0.0;
    c = 0.0; c2 = 0.0;
  }
  double z = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) z += dG[i] * dG[i];
  if (z > 0.0) {
    const double nrm = sqrt(z);
#pragma unroll
    for (int i = 0; i < 6; ++i) dG[i] /= nrm;
  }
}

// return_mapping_VEP_getKF (SolidMaterial.cpp:358-407): f (8) and K (8x8 row-major).  Also returns the stress
// (damage D x), its deviator and the normalised potential gradient for the strain update.
__device__ inline void vep_getKF(const PtMat& M, double K[64], double f[8], const double x[8], const double eps_t[6],
                                 const double eplo[6], double dt, double damage, double h_old, double S[6],
                                 double Sd[6], double dG[6]) {
  double r[6], St[6], dF[6], dJ2[6], c, c2;
  apply_D(M, x, S);
#pragma unroll
  for (int i = 0; i < 6; ++i) S[i] *= damage;
  vep_P(S, Sd);
#pragma unroll
  for (int i = 0; i < 6; ++i) r[i] = eps_t[i] - eplo[i] - x[6] * Sd[i];
  apply_D(M, r, St);
#pragma unroll
  for (int i = 0; i < 6; ++i) St[i] *= damage;
  const bool apex = vep_apex(M, St);
  const double FTrial = vep_yield(M, St, apex, dF);
  const double F = vep_yield(M, S, apex, dF);
  vep_potential(M, S, St, apex, dG, dJ2, c, c2);
  double h = h_old + M.hard * sqrt(x[7] * x[7]);
  double dh = M.hard * (x[7] > 0 ? 1.0 : (x[7] < 0 ? -1.0 : 0.0));
  if (h < -0.9 * M.sy) { h = -0.9 * M.sy; dh = -0.0; }
#pragma unroll
  for (int i = 0; i < 6; ++i) f[i] = x[i] - eps_t[i] + eplo[i] + x[6] * Sd[i] + x[7] * dG[i];
  // K(0:5,0:5) = I + damage x6 P D + damage x7 ddG D, ddG D = c J2Mat D - c2 dJ2 (D dJ2)^T
  double DdJ[6];
  apply_D(M, dJ2, DdJ);
  const double a6 = damage * x[6], a7 = damage * x[7];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const double pd = (i < 3 && j < 3) ? 2.0 * M.G * ((i == j ? 1.0 : 0.0) - 1.0 / 3.0) : (i == j ? M.G : 0.0);
      const double jd = (i < 3 && j < 3) ? pd : (i == j ? 2.0 * M.G : 0.0);
      K[i * 8 + j] = (i == j ? 1.0 : 0.0) + a6 * pd + a7 * (c * jd - c2 * dJ2[i] * DdJ[j]);
    }
#pragma unroll
  for (int i = 0; i < 6; ++i) { K[i * 8 + 6] = Sd[i]; K[i * 8 + 7] = dG[i]; }
  double ss = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) ss += Sd[i] * Sd[i];
  f[6] = x[6] - M.A * dt * pow(ss, (M.n - 1.0) / 2.0);
  // K(6,0:5) = -A dt ss^((n-3)/2) (n-1)/2 2 damage (D P SDev)^T
  double PS[6], DPS[6];
  vep_P(Sd, PS);
  apply_D(M, PS, DPS);
  const double c6 = -M.A * dt * pow(ss, (M.n - 3.0) / 2.0) * (M.n - 1.0) / 2.0 * 2.0 * damage;
#pragma unroll
  for (int j = 0; j < 6; ++j) K[6 * 8 + j] = c6 * DPS[j];
  K[6 * 8 + 6] = 1.0;
  K[6 * 8 + 7] = 0.0;
  if (FTrial - h_old < 0.0) {
    f[7] = -(M.plv + 1.0e0) / dt * x[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) K[7 * 8 + j] = 0.0;
    K[7 * 8 + 7] = -(M.plv + 1.0e0) / dt;
  } else {
    f[7] = F - h - M.plv / dt * sqrt(x[7] * x[7] + 1.0e-12);
    double DdF[6];
    apply_D(M, dF, DdF);
#pragma unroll
    for (int j = 0; j < 6; ++j) K[7 * 8 + j] = damage * DdF[j];
    K[7 * 8 + 6] = 0.0;
    K[7 * 8 + 7] = -M.plv / dt * (x[7] > 0 ? 1.0 : (x[7] < 0 ? -1.0 : 0.0)) - dh;
  }
}

// Gauss-Jordan inverse with partial pivoting of an 8x8 row-major matrix (A is destroyed); false if singular.
__device__ inline bool inv8(double A[64], double Ai[64]) {
  for (int i = 0; i < 64; ++i) Ai[i] = (i % 9 == 0) ? 1.0 : 0.0;
  for (int k = 0; k < 8; ++k) {
    int p = k;
    double best = fabs(A[k * 8 + k]);
    for (int i = k + 1; i < 8; ++i) if (fabs(A[i * 8 + k]) > best) { best = fabs(A[i * 8 + k]); p = i; }
    if (best == 0.0) return false;
    if (p != k) for (int j = 0; j < 8; ++j) {
      double t = A[k * 8 + j]; A[k * 8 + j] = A[p * 8 + j]; A[p * 8 + j] = t;
      t = Ai[k * 8 + j]; Ai[k * 8 + j] = Ai[p * 8 + j]; Ai[p * 8 + j] = t;
    }
    const double ip = 1.0 / A[k * 8 + k];
    for (int j = 0; j < 8; ++j) { A[k * 8 + j] *= ip; Ai[k * 8 + j] *= ip; }
    for (int i = 0; i < 8; ++i) {
      if (i == k) continue;
      const double fct = A[i * 8 + k];
      if (fct == 0.0) continue;
      for (int j = 0; j < 8; ++j) { A[i * 8 + j] -= fct * A[k * 8 + j]; Ai[i * 8 + j] -= fct * Ai[k * 8 + j]; }
    }
  }
  return true;
}

// return_mapping_VEP (SolidMaterial.cpp:303-356) with return_mapping_VEP_updateStrain (:409-445).
// vh: the ip's current MatHist[0..2] (initial guess x6 = vh[1], x7 = vh[2]; written back); h_old = MatHistOld[0].
// DMat = K^-1(0:5,0:5) of the last evaluated K.  diss = DissRate, damdiss = DamDissRate.
__device__ inline RMResult return_mapping_vep(const PtMat& M, double DMat[36], double epl[6], const double eps_t[6],
                                              const double eplo[6], double dt, double damage, double vh[3],
                                              double h_old, int tol_mode, int maxit, double& diss, double& damdiss) {
  double x[8], f[8], K[64], Ki[64], dx[8], S[6], Sd[6], dG[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) x[i] = eps_t[i] - epl[i];
  x[6] = vh[1];
  x[7] = vh[2];
  vep_getKF(M, K, f, x, eps_t, eplo, dt, damage, h_old, S, Sd, dG);
  double e0 = 0;
  for (int i = 0; i < 8; ++i) e0 += f[i] * f[i];
  e0 = fmax(e0, 1e-12);
  double eprev = 1e300;
  RMResult r{0, false, true};
  bool conv = false;
  int it = 0;
  while (!conv) {
    it += 1;
    if (!inv8(K, Ki)) { r.ok = false; break; }
    double ls2 = 0;
    for (int i = 0; i < 8; ++i) {
      double t = 0;
      for (int j = 0; j < 8; ++j) t += Ki[i * 8 + j] * f[j];
      dx[i] = -t;
      x[i] += dx[i];
      ls2 += f[i] * dx[i];
    }
    vep_getKF(M, K, f, x, eps_t, eplo, dt, damage, h_old, S, Sd, dG);
    double ls1 = 0;
    for (int i = 0; i < 8; ++i) ls1 += f[i] * dx[i];
    double ls;
    if ((ls1 - ls2) == 0.0) ls = 1.0;
    else {
      const double sg = (ls1 - ls2) > 0 ? 1.0 : -1.0;
      ls = -(ls2) / (fabs(ls1 - ls2) + 1e-12) * sg;
      ls = fmin(fmax(ls, 0.2), 1.0);
    }
    for (int i = 0; i < 8; ++i) x[i] = x[i] - (1.0 - ls) * dx[i];
    vep_getKF(M, K, f, x, eps_t, eplo, dt, damage, h_old, S, Sd, dG);
    double e = 0;
    for (int i = 0; i < 8; ++i) e += f[i] * f[i];
    if (tol_mode == IFEM_RM_REFERENCE) {
      if (e < 1.0e-16 || e / e0 < 1.0e-8) conv = true;
    } else {
      if (e < 1.0e-36 || (it >= 3 && e >= eprev)) conv = true;
    }
    eprev = e;
    if (it > maxit) { conv = true; r.capped = true; }
  }
  r.iters = it;
  // updateStrain: S, Sd and dG are those of the last getKF, evaluated at the final x
  double dv = 0, dp = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const double ev = x[6] * Sd[i], ep = x[7] * dG[i];
    epl[i] = eplo[i] + ev + ep;
    dv += 1.0 / dt * fabs(ev * S[i]);
    dp += 1.0 / dt * fabs(ep * S[i]);
  }
  vh[0] = h_old + M.hard * sqrt(x[7] * x[7]);
  vh[1] = x[6];
  vh[2] = x[7];
  diss = dv + dp;
  damdiss = dp;
  if (r.ok) r.ok = inv8(K, Ki);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) DMat[i * 6 + j] = Ki[i * 8 + j];
  return r;
}

}  // namespace ifem
