// Cosserat ice material on the device (CosseratMaterial.cpp): 18-component strains (0-8 the non-symmetric
// strain xx, yy, zz, xy, yx, yz, zy, xz, zx; 9-17 the curvatures times l_coss), D_coss and J2Mat_Coss applied in
// their block form, the four splits the Cosserat material defines, and the viscoelastic-plastic return map with
// its 18 elastic strains and two multipliers.  One thread per integration point; the 18x18 and 20x20 work arrays
// live in the thread's local memory.
#pragma once

#include "device_common.cuh"

namespace ifem {

struct CossMat {
  double lame, G, K, Gc, l, her;           // Lame, Shear, Bulk, G_coss, l_coss, hard_eRef
  double A, n, sy, hard, plv, phi_lim;     // creep, yield, hardening, plastic viscosity, PhiViscLim
  double star_g, b_dp;
  int rheo, split, cons;
};

__device__ __forceinline__ void coss_mat(const MatDev& m, const PtMat& M, CossMat& c) {
  c.lame = M.lame; c.G = M.G; c.K = M.K;
  c.Gc = m.g_coss; c.l = m.l_coss; c.her = m.hard_e_ref;
  c.A = M.A; c.n = M.n; c.sy = M.sy; c.hard = M.hard; c.plv = M.plv; c.phi_lim = M.phi_lim;
  c.star_g = M.star; c.b_dp = M.bdp;
  c.rheo = M.rheo; c.split = M.split; c.cons = M.ce;
}

// y = D_coss x (CosseratMaterial.cpp:68-104)
__device__ __forceinline__ void coss_D(const CossMat& c, const double* x, double* y) {
  const double tr = x[0] + x[1] + x[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) y[i] = c.lame * tr + 2.0 * c.G * x[i];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const int a = 3 + 2 * p, b = 4 + 2 * p;
    y[a] = (c.G + c.Gc) * x[a] + (c.G - c.Gc) * x[b];
    y[b] = (c.G - c.Gc) * x[a] + (c.G + c.Gc) * x[b];
  }
#pragma unroll
  for (int i = 9; i < 18; ++i) y[i] = 2.0 * c.G * x[i];
}

// D_coss(i, j)
__device__ __forceinline__ double coss_Dij(const CossMat& c, int i, int j) {
  if (i < 3 && j < 3) return c.lame + (i == j ? 2.0 * c.G : 0.0);
  if (i >= 3 && i < 9 && j >= 3 && j < 9 && (i - 3) / 2 == (j - 3) / 2) return i == j ? c.G + c.Gc : c.G - c.Gc;
  if (i >= 9 && i == j) return 2.0 * c.G;
  return 0.0;
}

// y = J2Mat_Coss x (CosseratMaterial.cpp:31-66; a1 = a2 = 0.25, a3 = 0.5)
__device__ __forceinline__ void coss_J2(const double* x, double* y) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double s = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) s += ((i == j) ? 2.0 / 3.0 : -1.0 / 3.0) * x[j];
    y[i] = s;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    y[3 + k] = 2 * 0.25 * x[3 + k] + 2 * 0.25 * x[6 + k];
    y[6 + k] = 2 * 0.25 * x[3 + k] + 2 * 0.25 * x[6 + k];
  }
#pragma unroll
  for (int i = 9; i < 18; ++i) y[i] = 2 * 0.5 * x[i];
}

__device__ __forceinline__ double coss_J2ij(int i, int j) {
  if (i < 3 && j < 3) return (i == j) ? 2.0 / 3.0 : -1.0 / 3.0;
  if (i >= 3 && i < 9 && j >= 3 && j < 9 && ((i - 3) % 3) == ((j - 3) % 3)) return 0.5;
  if (i >= 9 && i == j) return 1.0;
  return 0.0;
}

// the cyclic Jacobi eigen-solver of a symmetric 3x3 (Golub and Van Loan, sec. 8.5); eigenvalues on the diagonal
__device__ inline void coss_jacobi3(double A[3][3], double V[3][3]) {
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 16; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (off == 0.0 || off <= 1e-36 * dia) break;
    for (int k = 0; k < 3; ++k) {
      const int p = k < 2 ? 0 : 1, q = k == 0 ? 1 : 2;
      const double apq = A[p][q];
      if (apq == 0.0) continue;
      const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
      const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
      A[p][p] -= t * apq;
      A[q][q] += t * apq;
      A[p][q] = A[q][p] = 0.0;
      const int r = 3 - p - q;
      const double arp = A[r][p], arq = A[r][q];
      A[r][p] = A[p][r] = cs * arp - sn * arq;
      A[r][q] = A[q][r] = sn * arp + cs * arq;
      for (int i = 0; i < 3; ++i) {
        const double vip = V[i][p], viq = V[i][q];
        V[i][p] = cs * vip - sn * viq;
        V[i][q] = sn * vip + cs * viq;
      }
    }
  }
}

// eigen-decomposition of the symmetrised macro stress of D_coss e, near-zero components replaced by (i+1) tiny
__device__ inline void coss_stress_eig(const CossMat& c, const double* e, double tiny, double lam[3], double V[3][3]) {
  double S[18];
  coss_D(c, e, S);
  double sn[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) { sn[i] = S[i]; if (fabs(sn[i]) < tiny) sn[i] = (i + 1) * tiny; }
  const double Sm[3][3] = {{sn[0], sn[3], sn[7]}, {sn[4], sn[1], sn[5]}, {sn[8], sn[6], sn[2]}};
  double A[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = 0.5 * (Sm[i][j] + Sm[j][i]);
  coss_jacobi3(A, V);
  lam[0] = A[0][0]; lam[1] = A[1][1]; lam[2] = A[2][2];
}

// 0.5 (positive principal part) : macro strain
__device__ inline double coss_pos_energy(const double* e, const double lam[3], const double V[3][3]) {
  double P[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int k = 0; k < 3; ++k)
    if (lam[k] > 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) P[i][j] += lam[k] * V[i][k] * V[j][k];
  const double sv[9] = {P[0][0], P[1][1], P[2][2], P[0][1], P[1][0], P[1][2], P[2][1], P[0][2], P[2][0]};
  double E = 0;
#pragma unroll
  for (int i = 0; i < 9; ++i) E += sv[i] * e[i];
  return 0.5 * E;
}


// EnergySplit (CosseratMaterial.cpp:107-154) for the None, SpecStress, DruckerPrager and StarConvex splits; the
// tangents Dd, Du (row-major 18x18) are formed only when want_D.  Without energy-consistent stresses the stresses
// are D_coss e and the tangent D_coss, whatever the split.
__device__ inline double coss_split(const CossMat& c, const double* e, double* Dd, double* Du, double* Sd, double* Su,
                                    bool want_D) {
  for (int i = 0; i < 18; ++i) { Sd[i] = 0; Su[i] = 0; }
  if (want_D) for (int i = 0; i < 324; ++i) { Dd[i] = 0; Du[i] = 0; }
  auto ic = [](int i) { return i < 3 ? 1.0 : 0.0; };
  double E = 0;
  if (c.split == IFEM_SPLIT_NONE) {
    coss_D(c, e, Sd);
    for (int i = 0; i < 18; ++i) E += Sd[i] * e[i];
    E *= 0.5;
    if (want_D) for (int i = 0; i < 18; ++i) for (int j = 0; j < 18; ++j) Dd[i * 18 + j] = coss_Dij(c, i, j);
  } else if (c.split == IFEM_SPLIT_SPECSTRESS) {
    double lam[3], V[3][3];
    if (!c.cons) {   // SpecStressSplit (CosseratMaterial.cpp:378-420)
      coss_stress_eig(c, e, 1.0e-9, lam, V);
      E = fmax(0.0, coss_pos_energy(e, lam, V));
    } else {         // SpecStressSplitConsistent (:263-377)
      coss_stress_eig(c, e, 1.0e-12, lam, V);
      E = coss_pos_energy(e, lam, V);
      if (want_D) {
        // P+ in the reference's row = 3a + b indexing, applied to D_coss (rotations kept whole)
        double P[324];
        for (int i = 0; i < 324; ++i) P[i] = 0;
        for (int k = 0; k < 3; ++k) {
          if (!(lam[k] > 0.0)) continue;
          for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) for (int cc = 0; cc < 3; ++cc) for (int d = 0; d < 3; ++d)
            P[(3 * a + b) * 18 + 3 * cc + d] += V[a][k] * V[b][k] * V[cc][k] * V[d][k];
        }
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
          if (i == j) continue;
          if (lam[i] <= 0.0 && lam[j] <= 0.0) continue;
          const double den = lam[i] - lam[j];
          if (fabs(den) < 1e-12) continue;
          const double coeff = (fmax(lam[i], 0.0) - fmax(lam[j], 0.0)) / den;
          for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) for (int cc = 0; cc < 3; ++cc) for (int d = 0; d < 3; ++d)
            P[(3 * a + b) * 18 + 3 * cc + d] += 0.5 * coeff * (V[a][i] * V[b][j] * V[cc][j] * V[d][i] +
                                                               V[a][j] * V[b][i] * V[cc][i] * V[d][j]);
        }
        for (int i = 9; i < 18; ++i) P[i * 18 + i] = 1.0;
        for (int i = 0; i < 18; ++i) {
          double row[18];
          coss_D(c, P + i * 18, row);   // (P D)_i. = D P_i. (D symmetric)
          for (int j = 0; j < 18; ++j) { Dd[i * 18 + j] = row[j]; Du[i * 18 + j] = coss_Dij(c, i, j) - row[j]; }
        }
        for (int i = 0; i < 18; ++i) {
          double a = 0, b = 0;
          for (int j = 0; j < 18; ++j) { a += Dd[i * 18 + j] * e[j]; b += Du[i * 18 + j] * e[j]; }
          Sd[i] = a; Su[i] = b;
        }
      }
    }
  } else if (c.split == IFEM_SPLIT_DRUCKERPRAGER) {   // DruckerPragerSplit (:206-261)
    const double K = c.K, G = c.G, B = c.b_dp;
    const double I1 = e[0] + e[1] + e[2];
    double dJ2[18];
    coss_J2(e, dJ2);
    double J2 = 0;
    for (int i = 0; i < 18; ++i) J2 += e[i] * dJ2[i];
    J2 *= 0.5;
    const double sq = sqrt(J2 + 1.0e-16);
    auto ddsq = [&](int i, int j) { return 0.5 / sq * coss_J2ij(i, j) - 0.25 / sq / sq / sq * dJ2[i] * dJ2[j]; };
    if (-6.0 * B * sqrt(J2) < I1) {
      E = 0.5 * K * I1 * I1 + 2.0 * G * J2;
      for (int i = 0; i < 18; ++i) Sd[i] = K * I1 * ic(i) + 2.0 * G * dJ2[i];
      if (want_D) for (int i = 0; i < 18; ++i) for (int j = 0; j < 18; ++j) Dd[i * 18 + j] = K * ic(i) * ic(j) + 2.0 * G * coss_J2ij(i, j);
    } else if (2 * G * sqrt(J2) < 3 * B * K * I1) {
      for (int i = 0; i < 18; ++i) Su[i] = K * I1 * ic(i) + 2.0 * G * dJ2[i];
      if (want_D) for (int i = 0; i < 18; ++i) for (int j = 0; j < 18; ++j) Du[i * 18 + j] = K * ic(i) * ic(j) + 2.0 * G * coss_J2ij(i, j);
    } else {
      double pre = 1.0 / (18.0 * B * B * K + 2.0 * G);
      double q = -3.0 * B * K * I1 + 2 * G * sq;
      double dq[18];
      for (int i = 0; i < 18; ++i) dq[i] = -3.0 * B * K * ic(i) + 2.0 * G * (0.5 / sq * dJ2[i]);
      E = pre * q * q;
      for (int i = 0; i < 18; ++i) Sd[i] = pre * 2.0 * q * dq[i];
      if (want_D) for (int i = 0; i < 18; ++i) for (int j = 0; j < 18; ++j) Dd[i * 18 + j] = pre * (2.0 * q * 2.0 * G * ddsq(i, j) + 2.0 * dq[i] * dq[j]);
      pre = K * G / (18.0 * B * B * K + 2.0 * G);
      q = I1 + 6 * B * sq;
      for (int i = 0; i < 18; ++i) dq[i] = ic(i) + 6 * B * (0.5 / sq * dJ2[i]);
      for (int i = 0; i < 18; ++i) Su[i] = pre * 2.0 * q * dq[i];
      if (want_D) for (int i = 0; i < 18; ++i) for (int j = 0; j < 18; ++j) Du[i * 18 + j] = pre * (2.0 * q * 6 * B * ddsq(i, j) + 2.0 * dq[i] * dq[j]);
    }
  } else {   // StarConvexSplit (:156-204)
    const double K = c.K, G = c.G, Gc = c.Gc;
    const double p = e[0] + e[1] + e[2];
    double dev[9];
    for (int i = 0; i < 9; ++i) dev[i] = e[i] - (i < 3 ? p / 3.0 : 0.0);
    const double pplus = p >= 0 ? p : 0.0, dpplus = p >= 0 ? 1.0 : 0.0;
    const double pmin = p >= 0 ? 0.0 : p, dpmin = p >= 0 ? 0.0 : 1.0;
    // dDev dev = dev (trace free); SkewMat dev on the pairs (3,4), (5,6), (7,8)
    double sk[9];
    for (int i = 0; i < 3; ++i) sk[i] = 0.0;
    for (int k = 0; k < 3; ++k) { const int a = 3 + 2 * k, b = 4 + 2 * k; sk[a] = dev[a] - dev[b]; sk[b] = dev[b] - dev[a]; }
    double dd = 0, sks = 0;
    for (int i = 0; i < 9; ++i) { dd += dev[i] * dev[i]; sks += dev[i] * sk[i]; }
    E = 0.5 * K * pplus * pplus + G * dd + 0.5 * (G - Gc) * sks;
    for (int i = 0; i < 3; ++i) { Sd[i] += K * pplus * dpplus; Su[i] += K * pmin * dpmin; }
    for (int i = 0; i < 9; ++i) {
      const double ddev = dev[i] - (i < 3 ? (dev[0] + dev[1] + dev[2]) / 3.0 : 0.0);
      const double dsk = sk[i] - (i < 3 ? (sk[0] + sk[1] + sk[2]) / 3.0 : 0.0);
      Sd[i] += 2 * G * ddev + (G - Gc) * dsk;
    }
    for (int i = 9; i < 18; ++i) Sd[i] += 2 * Gc * e[i];
    if (want_D) {
      auto dD = [](int i, int j) { return (i == j ? 1.0 : 0.0) - ((i < 3 && j < 3) ? 1.0 / 3.0 : 0.0); };
      auto Sk = [](int i, int j) {
        if (i < 3 || j < 3 || (i - 3) / 2 != (j - 3) / 2) return 0.0;
        return i == j ? 1.0 : -1.0;
      };
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { Dd[i * 18 + j] += K * dpplus * dpplus; Du[i * 18 + j] += K * dpmin * dpmin; }
      for (int i = 0; i < 9; ++i) for (int j = 0; j < 9; ++j) {
        double a = 0, b = 0;
        for (int k = 0; k < 9; ++k) {
          a += dD(i, k) * dD(k, j);
          double u = 0;
          for (int l = 0; l < 9; ++l) u += Sk(k, l) * dD(l, j);
          b += dD(i, k) * u;
        }
        Dd[i * 18 + j] += 2 * G * a + (G - Gc) * b;
      }
      for (int i = 9; i < 18; ++i) Dd[i * 18 + i] += 2 * Gc;
    }
    E += -0.5 * K * c.star_g * pmin * pmin;
    E = fmax(0.0, E);
  }
  if (!c.cons) {   // stresses not using the same split as energies
    coss_D(c, e, Sd);
    for (int i = 0; i < 18; ++i) Su[i] = 0.0;
    if (want_D) for (int i = 0; i < 18; ++i) for (int j = 0; j < 18; ++j) { Dd[i * 18 + j] = coss_Dij(c, i, j); Du[i * 18 + j] = 0.0; }
  }
  return E;
}


// ---- viscoelastic-plastic return map (CosseratMaterial.cpp:516-842) ----
constexpr double kCsc = 1e6, kCs1 = 1.0e3, kCs2 = -1.0e-6, kCs3 = -1.0e-6, kCeps = 1.0e-12;

// J2 of the stress / sc and its gradient J2Mat_Coss S / sc (YieldFunction, YieldFunctionVE, PotentialFunction)
__device__ __forceinline__ double coss_j2(const double* S, double* dJ2) {
  double ss[18];
  for (int i = 0; i < 18; ++i) ss[i] = S[i] / kCsc;
  coss_J2(ss, dJ2);
  double J2 = 0;
  for (int i = 0; i < 18; ++i) J2 += ss[i] * dJ2[i];
  return 0.5 * J2;
}

// return_mapping_VEP_getKF (:684-734).  The viscous surface and the potential are evaluated at the same stress,
// so their second derivatives (both with the reference's sqrt(3) prefactor) coincide.
__device__ inline void coss_getKF(const CossMat& c, const double* sol, const double* eps, const double* eplO, double dt,
                                  double Dam, double h_old, double* K, double* f) {
  double S[18], dJ2[18];
  coss_D(c, sol, S);
  for (int i = 0; i < 18; ++i) S[i] *= Dam;
  const double J2 = coss_j2(S, dJ2);
  const double r = 1.0 / sqrt(J2 + kCeps);
  const double Fve = kCsc * sqrt(2.0 * J2), Fy = kCsc * sqrt(3.0 * J2) - c.sy;
  double dFve[18], dG[18];
  for (int i = 0; i < 18; ++i) { dFve[i] = 0.5 * sqrt(2.0) * r * dJ2[i]; dG[i] = 0.5 * sqrt(3.0) * r * dJ2[i]; }
  const double a = 0.5 / kCsc * sqrt(3.0) * r, b = 0.5 / (J2 + kCeps);
  double St[18], et[18], dJ2t[18];
  for (int i = 0; i < 18; ++i) et[i] = eps[i] - eplO[i] - sol[18] * dFve[i];
  coss_D(c, et, St);
  for (int i = 0; i < 18; ++i) St[i] *= Dam;
  const double FTrial = kCsc * sqrt(3.0 * coss_j2(St, dJ2t)) - c.sy;
  const double h = c.hard * c.sy * (1.0 - exp(-h_old * c.l / c.her));   // explicit hardening: h = hOld
  const double ml = sol[18] + sol[19];
  for (int i = 0; i < 18; ++i) {
    f[i] = kCs1 * (sol[i] - eps[i] + eplO[i] + sol[18] * dFve[i] + sol[19] * dG[i]);
    double row[18], y[18];
    for (int k = 0; k < 18; ++k) row[k] = ml * a * (coss_J2ij(i, k) - b * dJ2[i] * dJ2[k]);
    coss_D(c, row, y);
    for (int j = 0; j < 18; ++j) K[i * 20 + j] = kCs1 * ((i == j ? 1.0 : 0.0) + Dam * y[j]);
    K[i * 20 + 18] = kCs1 * dFve[i];
    K[i * 20 + 19] = kCs1 * dG[i];
  }
  const double pre = c.A * dt * pow(kCsc, c.n);
  f[18] = kCs2 * (pre * pow(Fve / kCsc, c.n) - sol[18]);
  const double kf = kCs2 * c.n * pre / kCsc * pow(Fve / kCsc, c.n - 1.0);
  double Dv[18], Dg[18];
  coss_D(c, dFve, Dv);
  coss_D(c, dG, Dg);
  for (int j = 0; j < 18; ++j) K[18 * 20 + j] = kf * (Dam * Dv[j]);
  K[18 * 20 + 18] = -kCs2;
  K[18 * 20 + 19] = 0.0;
  const double lv = c.l * c.plv;
  if (FTrial - h < 0.0) {
    f[19] = -kCs3 * (lv + 1.0e-6) / dt * sol[19];
    for (int j = 0; j < 19; ++j) K[19 * 20 + j] = 0.0;
    K[19 * 20 + 19] = -kCs3 * (lv + 1.0e-6) / dt;
  } else {
    f[19] = kCs3 * (Fy - h - lv / dt * sol[19]);
    for (int j = 0; j < 18; ++j) K[19 * 20 + j] = kCs3 * (Dam * Dg[j]);
    K[19 * 20 + 18] = 0.0;
    K[19 * 20 + 19] = kCs3 * (-lv / dt);
  }
}

// in-place LU with partial pivoting of a 20x20 system; false when singular
__device__ inline bool coss_lu20(double* A, int* piv) {
  for (int k = 0; k < 20; ++k) {
    int p = k;
    double best = fabs(A[k * 20 + k]);
    for (int i = k + 1; i < 20; ++i) if (fabs(A[i * 20 + k]) > best) { best = fabs(A[i * 20 + k]); p = i; }
    piv[k] = p;
    if (best == 0.0) return false;
    if (p != k) for (int j = 0; j < 20; ++j) { const double t = A[k * 20 + j]; A[k * 20 + j] = A[p * 20 + j]; A[p * 20 + j] = t; }
    const double inv = 1.0 / A[k * 20 + k];
    for (int i = k + 1; i < 20; ++i) {
      const double l = A[i * 20 + k] * inv;
      A[i * 20 + k] = l;
      for (int j = k + 1; j < 20; ++j) A[i * 20 + j] -= l * A[k * 20 + j];
    }
  }
  return true;
}

__device__ inline void coss_lu20_solve(const double* A, const int* piv, double* x) {
  for (int k = 0; k < 20; ++k) { const int p = piv[k]; if (p != k) { const double t = x[k]; x[k] = x[p]; x[p] = t; } }
  for (int i = 1; i < 20; ++i) { double s = x[i]; for (int j = 0; j < i; ++j) s -= A[i * 20 + j] * x[j]; x[i] = s; }
  for (int i = 19; i >= 0; --i) { double s = x[i]; for (int j = i + 1; j < 20; ++j) s -= A[i * 20 + j] * x[j]; x[i] = s / A[i * 20 + i]; }
}

struct CossRM { int iters; int capped; int singular; };

// return_mapping_VEP + return_mapping_VEP_updateStrain (:516-552, 736-754): hist = [e_eq, dLambda_v, dLambda_p,
// creep path]; Dmat = scale1 K^-1(0:18, 0:18) of the last system
__device__ inline void coss_return_map(const CossMat& c, double Dam, double dt, const double* eps, const double* eplO,
                                       double* epl, double* hist, const double* histO, double* Dmat, double& diss,
                                       double& damdiss, int tight, CossRM& ro) {
  double sol[20], f[20], fOld[20], dsol[20], K[400];
  int piv[20];
  for (int i = 0; i < 18; ++i) sol[i] = eps[i] - epl[i];
  sol[18] = hist[1];
  sol[19] = hist[2];
  coss_getKF(c, sol, eps, eplO, dt, Dam, histO[0], K, f);
  double e0 = 0;
  for (int i = 0; i < 20; ++i) e0 += f[i] * f[i];
  e0 = fmax(e0, 1e-12);
  double eprev = 1e300;
  int it = 0;
  for (;;) {
    it += 1;
    for (int i = 0; i < 20; ++i) dsol[i] = -f[i];
    if (!coss_lu20(K, piv)) { ro.singular = 1; break; }
    coss_lu20_solve(K, piv, dsol);
    for (int i = 0; i < 20; ++i) { sol[i] += dsol[i]; fOld[i] = f[i]; }
    coss_getKF(c, sol, eps, eplO, dt, Dam, histO[0], K, f);
    double ls1 = 0, ls2 = 0;
    for (int i = 0; i < 20; ++i) { ls1 += f[i] * dsol[i]; ls2 += fOld[i] * dsol[i]; }
    double ls = 1.0;
    if ((ls1 - ls2) != 0.0) ls = fmin(fmax(-(ls2) / (ls1 - ls2), 0.01), 1.0);
    for (int i = 0; i < 20; ++i) sol[i] = sol[i] - (1.0 - ls) * dsol[i];
    coss_getKF(c, sol, eps, eplO, dt, Dam, histO[0], K, f);
    double e = 0;
    for (int i = 0; i < 20; ++i) e += f[i] * f[i];
    bool conv = tight ? (e == 0.0 || e >= eprev || e / e0 < 1e-20) : (e < 1.0e-6 || e / e0 < 1.0e-5);
    eprev = e;
    if (it > 500) { conv = true; ro.capped += 1; }
    if (isnan(e) || isnan(e0) || (fabs(e / e0) > 1e6 && it > 25)) conv = true;
    if (conv) break;
  }
  ro.iters += it;
  double S[18], dJ2[18];
  coss_D(c, sol, S);
  for (int i = 0; i < 18; ++i) S[i] *= Dam;
  const double J2 = coss_j2(S, dJ2);
  const double r = 1.0 / sqrt(J2 + kCeps);
  double dv = 0, dp = 0;
  for (int i = 0; i < 18; ++i) {
    const double sv = sol[18] * (0.5 * sqrt(2.0) * r * dJ2[i]), sp = sol[19] * (0.5 * sqrt(3.0) * r * dJ2[i]);
    epl[i] = eplO[i] + sv + sp;
    dv += 1.0 / dt * fabs(sv * S[i]);
    dp += 1.0 / dt * fabs(sp * S[i]);
  }
  hist[0] = histO[0] + sqrt(sol[19] * sol[19]);
  hist[1] = sol[18];
  hist[2] = sol[19];
  hist[3] = histO[3] + sqrt(sol[18] * sol[18]);
  diss = dv + dp;
  damdiss = dp;
  if (!coss_lu20(K, piv)) { ro.singular = 1; for (int i = 0; i < 324; ++i) Dmat[i] = 0.0; return; }
  for (int j = 0; j < 18; ++j) {   // column j of K^-1, rows 0..17
    double x[20];
    for (int i = 0; i < 20; ++i) x[i] = (i == j) ? 1.0 : 0.0;
    coss_lu20_solve(K, piv, x);
    for (int i = 0; i < 18; ++i) Dmat[i * 18 + j] = kCs1 * x[i];
  }
}

}  // namespace ifem
