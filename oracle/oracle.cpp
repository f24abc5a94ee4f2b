// ORACLE — test infrastructure only (used by tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / --impl reference legs; never by the product library).
//
// Plain C++17 restatement of IceFEM's element assembly on the CPU, following the reference
// function by function (file:line cited at each routine, paths relative to the reference repo):
//   PhaseField.cpp:311-768 (Assemble_U / Assemble_Phase / Assemble_T), ThermalModel.cpp:72-135,
//   SolidMaterial.cpp:5-301, PhaseFieldMaterial.cpp:47-117,194-245,356-408, IceMaterial.cpp:49-84,
//   PhaseFieldUtil.cpp:77-348,350-380, B2_2.cpp:16-88, NURBS3_Cube2.cpp:17-115,
//   BaseElemType.cpp:197-221, IPScheme.cpp:9-109, math.cpp:3-61,301-331, DofSpace.cpp:177-1008,
//   physics.cpp:228-304.
//
// PARITY UNPINNED: the reference ships no tests, fixtures or golden vectors, and it cannot be
// compiled here (it needs PETSc, MPI, Eigen3, HighFive/HDF5 and RapidJSON, none installed).
// This restatement is pinned by known-answer tests (partition of unity, integrated volume,
// patch test, rigid-body null space, closed-form material points) and by central finite
// differences, in tests/.
//
// Deliberate deviations, each from an undefined or non-finite reference behaviour:
//   * SetTemperature(T, 0.0): the reference passes porosity 1.0 (PhaseField.cpp:383,598), which
//     makes E = 0 and Gc = 0/0 (IceMaterial.cpp:50-72) and traps under PETSc's FP trap.
//   * With no T DOF the reference reads uninitialised storage for T (PhaseField.cpp:338-341);
//     here T = options.pinned_temperature at every integration point.
//   * Eigen's 7x7 K.inverse() (SolidMaterial.cpp:225,260) is replaced by the closed-form Schur
//     inverse, exact because K(0:5,0:5) == I while ddF is zeroed (SolidMaterial.cpp:289-292).
//   * `abs(ls1-ls2)` (SolidMaterial.cpp:236) is the double overload (libstdc++ exports
//     std::abs(double) through <stdlib.h> and PETSc includes it).
//
// It exports the ifem_* C-ABI of include/icefem_b200.h under the prefix oracle_ so the same test
// harness drives both, plus oracle_assemble_mt (the multi-threaded CPU baseline).

#include "../include/icefem_b200.h"

#include <algorithm>
#include <cfloat>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr double kR = 8.31446261815324;  // BaseMaterial.h:26

struct Err { int code; std::string msg; };

// ----------------------------------------------------------------------------------------
// Small dense helpers
// ----------------------------------------------------------------------------------------
inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }  // math.cpp:101-105

// Inverse by adjugate / determinant (the closed forms Eigen uses for fixed 2x2 and 3x3).
inline double det2(const double J[4]) { return J[0] * J[3] - J[2] * J[1]; }
inline void inv2(const double J[4], double Ji[4]) {
  const double invdet = 1.0 / det2(J);
  Ji[0] = J[3] * invdet; Ji[2] = -J[2] * invdet; Ji[1] = -J[1] * invdet; Ji[3] = J[0] * invdet;
}
// row-major 3x3
inline double det3(const double m[9]) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[3] * (m[1] * m[8] - m[2] * m[7]) +
         m[6] * (m[1] * m[5] - m[2] * m[4]);
}
inline void inv3(const double m[9], double r[9]) {
  const double c00 = m[4] * m[8] - m[5] * m[7];
  const double c10 = m[5] * m[6] - m[3] * m[8];
  const double c20 = m[3] * m[7] - m[4] * m[6];
  const double det = m[0] * c00 + m[1] * c10 + m[2] * c20;
  const double id = 1.0 / det;
  r[0] = c00 * id; r[1] = (m[2] * m[7] - m[1] * m[8]) * id; r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r[3] = c10 * id; r[4] = (m[0] * m[8] - m[2] * m[6]) * id; r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r[6] = c20 * id; r[7] = (m[1] * m[6] - m[0] * m[7]) * id; r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

// Dense LU with partial pivoting, n <= 8 (used for the consistent return-map Jacobian).
bool lu_inverse(int n, const double* A, double* Ainv) {
  double a[64], inv[64];
  int piv[8];
  std::memcpy(a, A, sizeof(double) * n * n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  for (int k = 0; k < n; ++k) {
    int p = k; double best = std::fabs(a[k * n + k]);
    for (int i = k + 1; i < n; ++i) if (std::fabs(a[i * n + k]) > best) { best = std::fabs(a[i * n + k]); p = i; }
    if (best == 0.0) return false;
    if (p != k) { for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[p * n + j]); std::swap(piv[k], piv[p]); }
    for (int i = k + 1; i < n; ++i) {
      a[i * n + k] /= a[k * n + k];
      for (int j = k + 1; j < n; ++j) a[i * n + j] -= a[i * n + k] * a[k * n + j];
    }
  }
  for (int c = 0; c < n; ++c) {
    double x[8];
    for (int i = 0; i < n; ++i) x[i] = (piv[i] == c) ? 1.0 : 0.0;
    for (int i = 0; i < n; ++i) for (int j = 0; j < i; ++j) x[i] -= a[i * n + j] * x[j];
    for (int i = n - 1; i >= 0; --i) { for (int j = i + 1; j < n; ++j) x[i] -= a[i * n + j] * x[j]; x[i] /= a[i * n + i]; }
    for (int i = 0; i < n; ++i) inv[i * n + c] = x[i];
  }
  std::memcpy(Ainv, inv, sizeof(double) * n * n);
  return true;
}

// ----------------------------------------------------------------------------------------
// Gauss rule (IPScheme.cpp:9-109) and Bernstein basis (BaseElemType.cpp:197-221)
// ----------------------------------------------------------------------------------------
int fact(int n) { return (n == 0) || (n == 1) ? 1 : n * fact(n - 1); }

void ip_scheme_1d(int n, std::vector<double>& w, std::vector<double>& c) {
  switch (n) {
    case 1: c = {0}; w = {2.0}; break;
    case 3: c = {-std::sqrt(3.0 / 5.0), 0, std::sqrt(3.0 / 5.0)}; w = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0}; break;
    case 4:
      c = {-std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0)), -std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0)),
           std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0)), std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0))};
      w = {(18.0 - std::sqrt(30.0)) / 36.0, (18.0 + std::sqrt(30.0)) / 36.0, (18.0 + std::sqrt(30.0)) / 36.0,
           (18.0 - std::sqrt(30.0)) / 36.0};
      break;
    default: throw Err{IFEM_ERR_UNSUPPORTED, "ipcount1D must be 1, 3 or 4"};
  }
  for (size_t i = 0; i < w.size(); ++i) { c[i] = (c[i] + 1) / 2; w[i] = w[i] / 2; }
}

void bezier_basis(int p, double x, double* N, double* G) {
  for (int i = 0; i < p + 1; ++i) {
    const double pre = fact(p) / fact(p - i) / fact(i);
    N[i] = pre * std::pow(1.0 - x, std::max(0, p - i)) * std::pow(x, std::max(0, i));
    G[i] = pre * ((i - p) * std::pow(1.0 - x, std::max(0, p - i - 1)) * std::pow(x, std::max(0, i)) +
                  i * std::pow(1.0 - x, p - i) * std::pow(x, std::max(0, i - 1)));
  }
}

// second derivative of the Bernstein basis (BezierBasis, BaseElemType.cpp:209-211)
void bezier_basis2(int p, double x, double* G2) {
  for (int i = 0; i < p + 1; ++i) {
    const double pre = fact(p) / fact(p - i) / fact(i);
    G2[i] = pre * (2 * i * std::pow(x, std::max(0, i - 1)) * (i - p) * std::pow(1.0 - x, std::max(0, p - i - 1)) +
                   i * std::pow(x, std::max(0, i - 2)) * (i - 1) * std::pow(1.0 - x, std::max(0, p - i)) +
                   (i - p + 1) * std::pow(x, std::max(0, i)) * (i - p) * std::pow(1.0 - x, std::max(0, p - i - 2)));
  }
}

// ----------------------------------------------------------------------------------------
// Material point (IceMaterial::SetTemperature, IceMaterial.cpp:49-84; SolidMaterial ctor :5-107)
// ----------------------------------------------------------------------------------------
struct MatPt {
  double E, nu, G, lame, K;  // Young, Poisson, Shear, Lame, Bulk
  double D[36];
  double A, n, Gc, l, visc, phi_visc_lim;
  double ice_eref, ice_creduce, star_gamma;
  double sy, yield_alpha, pot_alpha, hardening, pl_visc;   // VEP (SolidMaterial.cpp:50-65)
  double b_dp;                                              // DruckerPrager split
  int rheology, split, consistent_energy;
};

// Friction-angle factor 6 sin(a) / (3 - sin(a)) of an angle in degrees (SolidMaterial.cpp:59-60)
inline double dp_alpha(double deg) {
  const double a = 3.14159265358979323846 / 180.0 * deg;
  return 6.0 * std::sin(a) / (3.0 - std::sin(a));
}

void set_temperature(const ifem_material& m, double T, MatPt& p) {
  const double dam = 1 - 0.0;  // porosity 0 (see header)
  double TAbs = T + m.t_offset;
  if (TAbs > 273.15) TAbs = 273.15;
  p.E = m.young * dam;
  p.nu = m.poisson;
  p.G = p.E / (2.0 * (1 + p.nu));
  p.lame = p.E * p.nu / ((1.0 + p.nu) * (1.0 - 2.0 * p.nu));
  p.K = p.lame + 2.0 / 3.0 * p.G;
  // D = Lame*i*i^T + 2*Shear*I ; D(3,3)=D(4,4)=D(5,5)=Shear (SolidMaterial.cpp:90-94), built from
  // the constructor's moduli (E0); with porosity 0 the values are identical.
  for (int i = 0; i < 36; ++i) p.D[i] = 0.0;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) p.D[i * 6 + j] = p.lame;
  for (int i = 0; i < 6; ++i) p.D[i * 6 + i] += 2 * p.G;
  p.D[3 * 6 + 3] = p.G; p.D[4 * 6 + 4] = p.G; p.D[5 * 6 + 5] = p.G;
  const double ExpTerm = -m.q_creep / kR * (1 / TAbs - 1 / m.t_ref);
  p.A = m.creep_a * std::exp(ExpTerm);
  p.n = m.creep_n;
  const double ft = dam * (m.ft0 - m.ftdeg * (TAbs - m.t_ref));
  p.l = m.pf_l;
  p.Gc = (m.gc_mode == 1) ? m.gc : 2.0 * ft * ft / p.E * p.l;
  p.visc = m.pf_visc;
  p.phi_visc_lim = m.phi_visc_lim;
  p.star_gamma = m.star_convex_gamma;
  p.ice_eref = m.ice_eref;
  p.ice_creduce = m.ice_creduce;
  if (m.split == IFEM_SPLIT_ICE) {
    p.ice_eref = m.ice_eref + m.ice_ereduce_fact * std::sqrt(std::max(1e-3, -(TAbs - m.t_ref)));
    p.ice_creduce = m.ice_creduce - (TAbs - m.t_ref) * m.ice_creduce_fact;
  }
  p.rheology = m.rheology;
  p.split = m.split;
  p.consistent_energy = m.consistent_energy;
  // plasticity (IceMaterial.cpp:81-82)
  p.sy = dam * (m.vep_sy - m.vep_sydeg * (TAbs - m.t_ref));
  p.yield_alpha = dp_alpha(m.vep_f_deg);
  p.pot_alpha = dp_alpha(m.vep_g_deg);
  p.hardening = m.vep_hardening;
  p.pl_visc = m.vep_pl_visc;
  p.b_dp = m.b_dp;
}

// ----------------------------------------------------------------------------------------
// Degradation and distribution functions (PhaseFieldUtil.cpp:77-221, 282-348)
// ----------------------------------------------------------------------------------------
// PorderDamage exponent (PhaseFieldUtil.cpp:24-25): properties/PhaseField/p, default 2 (0 = default)
double porder(const ifem_options& o) { return o.porder_p != 0.0 ? o.porder_p : 2.0; }

void damage_function(double phi, int f, double k0, double p, double& D, double& dD, double& ddD) {
  double pl = phi;
  if (pl < 0.0) pl = 0.0;
  if (pl > 1.0) pl = 1.0;
  switch (f) {
    case IFEM_DAM_NONE: D = 1.0; dD = 0.0; ddD = 0.0; break;
    case IFEM_DAM_LINEAR: D = (1.0 - k0) * (1.0 - pl) + k0; dD = -1.0 * (1.0 - k0); ddD = 0.0; break;
    case IFEM_DAM_LINEAR_NR: D = (1.0 - pl); dD = -1.0; ddD = 0.0; break;
    case IFEM_DAM_QUADRATIC: D = (1.0 - k0) * std::pow((1.0 - pl), 2) + k0; dD = -2.0 * (1.0 - k0) * (1.0 - phi); ddD = 2.0 * (1.0 - k0); break;
    case IFEM_DAM_QUADRATIC_NR: D = std::pow((1.0 - pl), 2); dD = -2.0 * (1.0 - phi); ddD = 2.0; break;
    case IFEM_DAM_CUBIC: D = (1.0 - k0) * std::pow((1.0 - pl), 3) + k0; dD = -3.0 * (1.0 - k0) * (1.0 - phi) * (1.0 - phi); ddD = 6.0 * (1.0 - k0) * (1.0 - phi); break;
    case IFEM_DAM_CUBIC_NR: D = std::pow((1.0 - pl), 3); dD = -3.0 * (1.0 - phi) * (1.0 - phi); ddD = 6.0 * (1.0 - phi); break;
    case IFEM_DAM_PORDER:
      D = (1.0 - k0) * std::pow((1.0 - pl), p) + k0; dD = -p * (1.0 - k0) * std::pow((1.0 - phi), p - 1);
      ddD = (p > 1) ? p * (p - 1) * (1.0 - k0) * std::pow((1.0 - phi), p - 2) : 0.0; break;
    case IFEM_DAM_CZM:
      D = (1.0 - k0) * (2.0 * std::pow(1 - phi, 2) - 1.0 * std::pow(1 - phi, 3)) + k0;
      dD = (1.0 - k0) * (3.0 * (1 - phi) * (1 - phi) - 4.0 * (1 - phi));
      ddD = (1.0 - k0) * (-6.0 * (1 - phi) + 4.0); break;
    case IFEM_DAM_STEP2: D = phi < 0.2 ? 1.0 : 0.0; dD = 0.0; ddD = 0.0; break;
    case IFEM_DAM_STEP5: D = phi < 0.5 ? 1.0 : 0.0; dD = 0.0; ddD = 0.0; break;
    case IFEM_DAM_STEP8: D = phi < 0.8 ? 1.0 : 0.0; dD = 0.0; ddD = 0.0; break;
    default: throw Err{IFEM_ERR_INVALID, "damage function not defined"};
  }
}

// ----------------------------------------------------------------------------------------
// Energy split (PhaseFieldMaterial.cpp:47-117,194-245,356-408)
// ----------------------------------------------------------------------------------------
const double kI[6] = {1, 1, 1, 0, 0, 0};
const double kVC[6] = {1, 1, 1, 0.5, 0.5, 0.5};    // VoightCorrect
const double kVDD[6] = {1, 1, 1, 2, 2, 2};         // VoightDoubleDot

// Symmetric 3x3 eigen-decomposition by the cyclic Jacobi method (Golub & Van Loan, Matrix Computations,
// sec. 8.5): A is diagonalised in place by plane rotations, their product accumulating in V (columns =
// eigenvectors).  It stands in for Eigen's SelfAdjointEigenSolver (PhaseFieldMaterial.cpp:133); the positive
// part sum_{l_k > 0} l_k v_k v_k^T it feeds is the same for any accurate solver.
void jacobi3(double A[3][3], double V[3][3]) {
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
  static const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 16; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (off == 0.0 || off <= 1e-36 * dia) break;
    for (int k = 0; k < 3; ++k) {
      const int p = P[k], q = Q[k];
      const double apq = A[p][q];
      if (apq == 0.0) continue;
      const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
      const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
      const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
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
}

// SpecStressSplit energy (PhaseFieldMaterial.cpp:118-151): the positive principal part of sigma = D e, with
// the reference's perturbation of near-zero normal and xy components, contracted with the strain
double spec_stress_energy(const MatPt& M, const double e[6]) {
  double S[6];
  for (int i = 0; i < 6; ++i) { double t = 0; for (int j = 0; j < 6; ++j) t += M.D[i * 6 + j] * e[j]; S[i] = t; }
  for (int i = 0; i < 4; ++i) if (S[i] * S[i] < 1.0e-9) S[i] = (i + 1) * 1e-9;
  double A[3][3] = {{S[0], S[3], S[5]}, {S[3], S[1], S[4]}, {S[5], S[4], S[2]}}, V[3][3];
  jacobi3(A, V);
  double Sp[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int k = 0; k < 3; ++k) {
    const double l = A[k][k];
    if (l > 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Sp[i][j] += l * V[i][k] * V[j][k];
  }
  const double v[6] = {Sp[0][0], Sp[1][1], Sp[2][2], 0.5 * (Sp[0][1] + Sp[1][0]), 0.5 * (Sp[1][2] + Sp[2][1]),
                       0.5 * (Sp[0][2] + Sp[2][0])};
  double Energy = 0;
  for (int i = 0; i < 6; ++i) Energy += v[i] * e[i];
  return 0.5 * Energy;
}

// GetEigenValues2D (PhaseFieldMaterial.cpp:408-448): plane-strain principal values of a Voigt tensor with
// tensor shears, s[0] = zz and s[1,2] = (xx + yy -/+ sqrt((xx - yy)^2 + 4 xy^2)) / 2, with first and second
// derivatives.  The derivatives use xx, yy, zz moved to (i+1) 1e-6 when below 1e-6 in magnitude.
void eig2d(const double su[6], double s[3], double ds[3][6], double dds[3][36]) {
  double sn[6];
  for (int i = 0; i < 6; ++i) sn[i] = su[i];
  for (int i = 0; i < 3; ++i) if (std::fabs(sn[i]) < 1.0e-6) sn[i] = (i + 1.0) * 1.0e-6;
  for (int k = 0; k < 3; ++k) { for (int i = 0; i < 6; ++i) ds[k][i] = 0; for (int i = 0; i < 36; ++i) dds[k][i] = 0; }
  s[0] = su[2];
  ds[0][2] = 1.0;
  const double sq = sn[0] * sn[0] + sn[1] * sn[1] - 2.0 * sn[0] * sn[1] + 4 * sn[3] * sn[3];
  const double squ = su[0] * su[0] + su[1] * su[1] - 2.0 * su[0] * su[1] + 4 * su[3] * su[3];
  const double r1 = std::pow(sq + DBL_EPSILON, -0.5), r3 = std::pow(sq + DBL_EPSILON, -1.5);
  const double c1 = 2.0 * sn[3] * (sn[0] - sn[1]) * r3, c2 = 2.0 * sn[3] * sn[3] * r3;
  const double c3 = 2.0 * (sn[0] - sn[1]) * (sn[0] - sn[1]) * r3;
  for (int k = 1; k < 3; ++k) {
    const double sg = 2.0 * k - 3.0;
    s[k] = 0.5 * (su[0] + su[1] + sg * std::pow(squ, 0.5));
    ds[k][0] = 0.5 + 0.5 * sg * (sn[0] - sn[1]) * r1;
    ds[k][1] = 0.5 + 0.5 * sg * (-sn[0] + sn[1]) * r1;
    ds[k][3] = 2.0 * sg * sn[3] * r1;
    double* h = dds[k];
    h[0 * 6 + 0] = sg * c2;  h[0 * 6 + 1] = -sg * c2; h[0 * 6 + 3] = -sg * c1;
    h[1 * 6 + 0] = -sg * c2; h[1 * 6 + 1] = sg * c2;  h[1 * 6 + 3] = sg * c1;
    h[3 * 6 + 0] = -sg * c1; h[3 * 6 + 1] = sg * c1;  h[3 * 6 + 3] = sg * c3;
  }
}

// SpecStrainSplit (PhaseFieldMaterial.cpp:239-290): Lame term on the principal-strain sum, shear terms per
// principal strain, assembled in tensor-shear Voigt form and mapped back; stresses recomputed from the tangents.
double spec_strain_split(const MatPt& M, double Dd[36], double Du[36], double Sd[6], double Su[6], const double e[6]) {
  double ev[6], s[3], ds[3][6], dds[3][36];
  for (int i = 0; i < 6; ++i) ev[i] = kVC[i] * e[i];
  eig2d(ev, s, ds, dds);
  const double p0 = s[0] + s[1] + s[2];
  double p1[6], p2[36];
  for (int i = 0; i < 6; ++i) p1[i] = ds[0][i] + ds[1][i] + ds[2][i];
  for (int i = 0; i < 36; ++i) p2[i] = dds[0][i] + dds[1][i] + dds[2][i];
  double Energy = 0, sd[6] = {0}, su[6] = {0}, dd[36] = {0}, du[36] = {0};
  double* S = p0 >= 0 ? sd : su;
  double* Dm = p0 >= 0 ? dd : du;
  if (p0 >= 0) Energy += 0.5 * M.lame * p0 * p0;
  for (int i = 0; i < 6; ++i) S[i] += M.lame * p0 * p1[i];
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dm[i * 6 + j] += M.lame * (p0 * p2[i * 6 + j] + p1[i] * p1[j]);
  for (int k = 0; k < 3; ++k) {
    double* Sk = s[k] >= 0 ? sd : su;
    double* Dk = s[k] >= 0 ? dd : du;
    if (s[k] >= 0) Energy += M.G * s[k] * s[k];
    for (int i = 0; i < 6; ++i) Sk[i] += M.G * 2 * s[k] * ds[k][i];
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j)
      Dk[i * 6 + j] += M.G * (2 * s[k] * dds[k][i * 6 + j] + 2 * ds[k][i] * ds[k][j]);
  }
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) {
    Dd[i * 6 + j] = kVC[i] * dd[i * 6 + j] * kVC[j];
    Du[i * 6 + j] = kVC[i] * du[i * 6 + j] * kVC[j];
  }
  for (int i = 0; i < 6; ++i) {
    double a = 0, b = 0;
    for (int j = 0; j < 6; ++j) { a += Dd[i * 6 + j] * e[j]; b += Du[i * 6 + j] * e[j]; }
    Sd[i] = a; Su[i] = b;
  }
  return Energy;
}

// DruckerPragerSplit (PhaseFieldMaterial.cpp:292-343): three regimes of I1 against sqrt(J2) of the strain
double drucker_prager_split(const MatPt& M, double Dd[36], double Du[36], double Sd[6], double Su[6], const double e[6]) {
  static const double J2M[6] = {1, 1, 1, 0.5, 0.5, 0.5};   // diagonal of J2Mat_strain; normal block - 1/3 11^T
  auto j2m = [](int i, int j) { return (i == j ? J2M[i] : 0.0) - ((i < 3 && j < 3) ? 1.0 / 3.0 : 0.0); };
  const double B = M.b_dp, K = M.K, G = M.G;
  const double I1 = e[0] + e[1] + e[2];
  double dJ2[6];
  for (int i = 0; i < 6; ++i) { double t = 0; for (int j = 0; j < 6; ++j) t += j2m(i, j) * e[j]; dJ2[i] = t; }
  double J2 = 0; for (int i = 0; i < 6; ++i) J2 += e[i] * dJ2[i];
  J2 *= 0.5;
  const double sq = std::sqrt(J2 + 1.0e-16);
  double dsq[6];
  for (int i = 0; i < 6; ++i) dsq[i] = 0.5 / sq * dJ2[i];
  auto ddsq = [&](int i, int j) { return 0.5 / sq * j2m(i, j) - 0.25 / sq / sq / sq * dJ2[i] * dJ2[j]; };
  for (int i = 0; i < 6; ++i) { Sd[i] = 0; Su[i] = 0; }
  for (int i = 0; i < 36; ++i) { Dd[i] = 0; Du[i] = 0; }
  double Energy = 0;
  if (-6.0 * B * std::sqrt(J2) < I1 || 2 * G * std::sqrt(J2) < 3 * B * K * I1) {
    const bool dam = -6.0 * B * std::sqrt(J2) < I1;
    double* S = dam ? Sd : Su;
    double* Dm = dam ? Dd : Du;
    if (dam) Energy = 0.5 * K * I1 * I1 + 2.0 * G * J2;
    for (int i = 0; i < 6; ++i) S[i] = K * I1 * (i < 3 ? 1.0 : 0.0) + 2.0 * G * dJ2[i];
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dm[i * 6 + j] = K * ((i < 3 && j < 3) ? 1.0 : 0.0) + 2.0 * G * j2m(i, j);
  } else {
    double pre = 1.0 / (18.0 * B * B * K + 2.0 * G);
    double q = -3.0 * B * K * I1 + 2 * G * sq, dq[6];
    for (int i = 0; i < 6; ++i) dq[i] = -3.0 * B * K * (i < 3 ? 1.0 : 0.0) + 2.0 * G * dsq[i];
    Energy = pre * q * q;
    for (int i = 0; i < 6; ++i) Sd[i] = pre * 2.0 * q * dq[i];
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dd[i * 6 + j] = pre * (2.0 * q * 2.0 * G * ddsq(i, j) + 2.0 * dq[i] * dq[j]);
    pre = K * G / (18.0 * B * B * K + 2.0 * G);
    q = I1 + 6 * B * sq;
    for (int i = 0; i < 6; ++i) dq[i] = (i < 3 ? 1.0 : 0.0) + 6 * B * dsq[i];
    for (int i = 0; i < 6; ++i) Su[i] = pre * 2.0 * q * dq[i];
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Du[i * 6 + j] = pre * (2.0 * q * 6 * B * ddsq(i, j) + 2.0 * dq[i] * dq[j]);
  }
  return Energy;
}

double energy_split(const MatPt& M, double Dd[36], double Du[36], double Sd[6], double Su[6], const double e[6]) {
  double Energy = 0;
  for (int i = 0; i < 36; ++i) { Dd[i] = 0; Du[i] = 0; }
  for (int i = 0; i < 6; ++i) { Sd[i] = 0; Su[i] = 0; }
  // P = I - 1/3 i i^T ; its product with diag matrices is formed entrywise
  auto devproj = [](int r, int c) { return (r == c ? 1.0 : 0.0) - ((r < 3 && c < 3) ? 1.0 / 3.0 : 0.0); };
  switch (M.split) {
    case IFEM_SPLIT_NONE: {
      std::memcpy(Dd, M.D, sizeof(double) * 36);
      for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += M.D[i * 6 + j] * e[j]; Sd[i] = s; }
      for (int i = 0; i < 6; ++i) Energy += 0.5 * Sd[i] * e[i];
    } break;
    case IFEM_SPLIT_VOLSTRAINS: {
      const double p = e[0] + e[1] + e[2];
      if (p >= 0) {
        Energy += 0.5 * M.K * p * p;
        for (int i = 0; i < 3; ++i) { Sd[i] += M.K * p; for (int j = 0; j < 3; ++j) Dd[i * 6 + j] += M.K; }
      } else {
        for (int i = 0; i < 3; ++i) { Su[i] += M.K * p; for (int j = 0; j < 3; ++j) Du[i * 6 + j] += M.K; }
      }
      double dev[6];
      for (int i = 0; i < 6; ++i) dev[i] = kVC[i] * e[i] - 1.0 / 3.0 * p * kI[i];
      double ed = 0;
      for (int i = 0; i < 6; ++i) ed += dev[i] * kVDD[i] * dev[i];
      Energy += M.G * ed;
      for (int i = 0; i < 6; ++i) Sd[i] += 2 * M.G * kVC[i] * kVDD[i] * dev[i];
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dd[i * 6 + j] += 2 * M.G * kVC[i] * kVDD[i] * kVC[i] * devproj(i, j);
    } break;
    case IFEM_SPLIT_VOLSTRESS: {
      double S[6];
      for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += M.D[i * 6 + j] * e[j]; S[i] = s; }
      const double p = 1.0 / 3.0 * (S[0] + S[1] + S[2]);
      // 1/3 i i^T D
      double iiD[36];
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j)
        iiD[i * 6 + j] = (i < 3) ? 1.0 / 3.0 * (M.D[0 * 6 + j] + M.D[1 * 6 + j] + M.D[2 * 6 + j]) : 0.0;
      if (p >= 0) { for (int i = 0; i < 6; ++i) Sd[i] += kI[i] * p; for (int k = 0; k < 36; ++k) Dd[k] += iiD[k]; }
      else { for (int i = 0; i < 6; ++i) Su[i] += kI[i] * p; for (int k = 0; k < 36; ++k) Du[k] += iiD[k]; }
      for (int i = 0; i < 6; ++i) Sd[i] += S[i] - kI[i] * p;
      for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) {
        double s = 0; for (int k = 0; k < 6; ++k) s += devproj(i, k) * M.D[k * 6 + j];
        Dd[i * 6 + j] += s;
      }
      for (int i = 0; i < 6; ++i) Energy += 0.5 * Sd[i] * e[i];
    } break;
    case IFEM_SPLIT_STARCONVEX:
    case IFEM_SPLIT_ICE: {
      const double p = e[0] + e[1] + e[2];
      double pplus, pmin, dpplus, dpmin;
      if (p >= 0) { pplus = p; dpplus = 1.0; pmin = 0.0; dpmin = 0.0; }
      else { pplus = 0.0; dpplus = 0.0; pmin = p; dpmin = 1.0; }
      double dev[6];
      for (int i = 0; i < 6; ++i) dev[i] = kVC[i] * e[i] - 1.0 / 3.0 * p * kI[i];
      double ed = 0;
      for (int i = 0; i < 6; ++i) ed += dev[i] * kVDD[i] * dev[i];
      if (M.split == IFEM_SPLIT_STARCONVEX) {
        const double g = M.star_gamma;
        Energy += 0.5 * M.K * (pplus * pplus - g * pmin * pmin);
        for (int i = 0; i < 3; ++i) {
          Sd[i] += M.K * (pplus * dpplus - g * pmin * dpmin);
          Su[i] += (1.0 + g) * M.K * pmin * dpmin;
          for (int j = 0; j < 3; ++j) {
            Dd[i * 6 + j] += M.K * (dpplus * dpplus - g * dpmin * dpmin);
            Du[i * 6 + j] += (1.0 + g) * M.K * dpmin * dpmin;
          }
        }
        Energy += M.G * ed;
        for (int i = 0; i < 6; ++i) Sd[i] += 2 * M.G * kVC[i] * kVDD[i] * dev[i];
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dd[i * 6 + j] += 2 * M.G * kVC[i] * kVDD[i] * kVC[i] * devproj(i, j);
      } else {
        Energy += 0.5 * M.K * pplus * pplus;
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
          Dd[i * 6 + j] += M.K * dpplus * dpplus;
          Du[i * 6 + j] += M.K * dpmin * dpmin;
        }
        Energy += M.G * ed;
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Dd[i * 6 + j] += 2 * M.G * kVC[i] * kVDD[i] * kVC[i] * devproj(i, j);
        Energy += -0.5 * M.K * M.ice_creduce * pmin * pmin / (M.ice_eref * M.ice_eref + pmin * pmin);
        for (int i = 0; i < 6; ++i) {
          double s1 = 0, s2 = 0;
          for (int j = 0; j < 6; ++j) { s1 += Dd[i * 6 + j] * e[j]; s2 += Du[i * 6 + j] * e[j]; }
          Sd[i] = s1; Su[i] = s2;
        }
        if (Energy < 0.0) Energy = 0.0;
        if (Energy > 1.0e12 || std::isnan(Energy)) Energy = 1.0e12;
        if (Energy < -1.0e12) Energy = -1.0e12;
      }
    } break;
    case IFEM_SPLIT_SPECSTRESS:   // energy only; stresses and tangents are D e / D (consistent_energy = 0)
      Energy = spec_stress_energy(M, e);
      break;
    case IFEM_SPLIT_SPECSTRAINS:
      Energy = spec_strain_split(M, Dd, Du, Sd, Su, e);
      break;
    case IFEM_SPLIT_DRUCKERPRAGER:
      Energy = drucker_prager_split(M, Dd, Du, Sd, Su, e);
      break;
    default: throw Err{IFEM_ERR_UNSUPPORTED, "energy split not supported"};
  }
  if (M.consistent_energy == 0) {
    for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += M.D[i * 6 + j] * e[j]; Sd[i] = s; Su[i] = 0; }
    std::memcpy(Dd, M.D, sizeof(double) * 36);
    for (int i = 0; i < 36; ++i) Du[i] = 0;
  }
  return Energy;
}

// ----------------------------------------------------------------------------------------
// Glen viscous return map (SolidMaterial.cpp:123-301, 477-492)
// ----------------------------------------------------------------------------------------
const double kJ2[36] = {2.0 / 3.0, -1.0 / 3.0, -1.0 / 3.0, 0, 0, 0,
                        -1.0 / 3.0, 2.0 / 3.0, -1.0 / 3.0, 0, 0, 0,
                        -1.0 / 3.0, -1.0 / 3.0, 2.0 / 3.0, 0, 0, 0,
                        0, 0, 0, 2.0, 0, 0,
                        0, 0, 0, 0, 2.0, 0,
                        0, 0, 0, 0, 0, 2.0};

struct J2Tab { double m[36]; J2Tab() {
  // Identity - 1/3 i i^T, then shear diagonal 2.0 (SolidMaterial.cpp:96-100)
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) m[i * 6 + j] = (i == j ? 1.0 : 0.0) - ((i < 3 && j < 3) ? 1.0 / 3.0 : 0.0);
  m[21] = 2.0; m[28] = 2.0; m[35] = 2.0; } };
const J2Tab kJ2Mat;

double yield_ve(const double S[6], double dF[6], double* J2out) {
  const double sc = 1.0e6, eps = 1.0e-12;
  double Ss[6], dJ2[6];
  for (int i = 0; i < 6; ++i) Ss[i] = S[i] / sc;
  for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += kJ2Mat.m[i * 6 + j] * Ss[j]; dJ2[i] = s; }
  double J2 = 0; for (int i = 0; i < 6; ++i) J2 += Ss[i] * dJ2[i];
  J2 *= 0.5;
  const double F = sc * std::sqrt(2.0 * J2);
  const double c = 0.5 * std::sqrt(2.0) / std::sqrt(J2 + eps);
  for (int i = 0; i < 6; ++i) dF[i] = c * dJ2[i];
  if (J2out) *J2out = J2;
  return F;
}

struct RMOut { long iters = 0; long capped = 0; };   // Newton iterations and ips that hit the cap

// return_mapping_getKF: f and the two non-trivial blocks of K = [[I, a],[b^T, -1]]
void rm_getKF(const MatPt& M, double f[7], double a[6], double b[6], const double sol[7], const double eps_t[6],
              const double epl_old[6], double damage, double dt) {
  double S[6];
  for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += M.D[i * 6 + j] * sol[j]; S[i] = s; }
  double dF[6];
  const double F = yield_ve(S, dF, nullptr);
  for (int i = 0; i < 6; ++i) f[i] = sol[i] - eps_t[i] + epl_old[i] + sol[6] * dF[i];
  for (int i = 0; i < 6; ++i) a[i] = dF[i];
  const double sc = 1.0e6;
  const double PreFac = M.A * dt * std::pow(sc, M.n);
  f[6] = PreFac * std::pow(F / sc, M.n) - sol[6];
  const double coef = M.n * PreFac / sc * std::pow(F / sc, M.n - 1.0);
  for (int j = 0; j < 6; ++j) { double s = 0; for (int i = 0; i < 6; ++i) s += (damage * dF[i]) * M.D[i * 6 + j]; b[j] = coef * s; }
}

// Consistent Jacobian of the converged local system (exact derivative of rm_getKF's f, no
// damage factor, full d(dF)/dsigma), 7x7 row-major.
void rm_exact_jacobian(const MatPt& M, const double sol[7], double dt, double Kx[49]) {
  const double sc = 1.0e6, eps = 1.0e-12;
  double S[6], Ss[6], dJ2[6];
  for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += M.D[i * 6 + j] * sol[j]; S[i] = s; }
  for (int i = 0; i < 6; ++i) Ss[i] = S[i] / sc;
  for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += kJ2Mat.m[i * 6 + j] * Ss[j]; dJ2[i] = s; }
  double J2 = 0; for (int i = 0; i < 6; ++i) J2 += Ss[i] * dJ2[i];
  J2 *= 0.5;
  const double c = 0.5 * std::sqrt(2.0) / std::sqrt(J2 + eps);
  // d(dF)/dsigma = c/sc * (J2Mat - 1/(2(J2+eps)) dJ2 dJ2^T)
  double H[36];
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) H[i * 6 + j] = c / sc * (kJ2Mat.m[i * 6 + j] - 0.5 / (J2 + eps) * dJ2[i] * dJ2[j]);
  double HD[36];
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) { double s = 0; for (int k = 0; k < 6; ++k) s += H[i * 6 + k] * M.D[k * 6 + j]; HD[i * 6 + j] = s; }
  for (int i = 0; i < 49; ++i) Kx[i] = 0;
  for (int i = 0; i < 6; ++i) {
    for (int j = 0; j < 6; ++j) Kx[i * 7 + j] = (i == j ? 1.0 : 0.0) + sol[6] * HD[i * 6 + j];
    Kx[i * 7 + 6] = c * dJ2[i];
  }
  // f6 = A dt sc^n (F/sc)^n - dl ; dF/dsigma (exact) = dJ2 / sqrt(2 J2)
  const double F = sc * std::sqrt(2.0 * J2);
  const double PreFac = M.A * dt * std::pow(sc, M.n);
  const double coef = (J2 > 0) ? M.n * PreFac / sc * std::pow(F / sc, M.n - 1.0) / std::sqrt(2.0 * J2) : 0.0;
  for (int j = 0; j < 6; ++j) { double s = 0; for (int i = 0; i < 6; ++i) s += dJ2[i] * M.D[i * 6 + j]; Kx[6 * 7 + j] = coef * s; }
  Kx[6 * 7 + 6] = -1.0;
}

// Solve [[I, a],[b^T, -1]] x = f in closed form.
inline void schur_solve(const double a[6], const double b[6], const double f[7], double x[7]) {
  double bf = 0, ba = 0;
  for (int i = 0; i < 6; ++i) { bf += b[i] * f[i]; ba += b[i] * a[i]; }
  x[6] = (bf - f[6]) / (1.0 + ba);
  for (int i = 0; i < 6; ++i) x[i] = f[i] - a[i] * x[6];
}

double return_mapping_viscous(const MatPt& M, double DMat[36], double epl[6], const double eps_t[6],
                              const double epl_old[6], double damage, double dt, double& hist0, int tol_mode,
                              int maxit, int tangent_mode, RMOut& ro) {
  double sol[7], f[7], fOld[7], a[6], b[6], dsol[7];
  for (int i = 0; i < 6; ++i) sol[i] = eps_t[i] - epl[i];
  sol[6] = hist0;
  rm_getKF(M, f, a, b, sol, eps_t, epl_old, damage, dt);
  double e0 = 0; for (int i = 0; i < 7; ++i) e0 += f[i] * f[i];
  e0 = std::max(e0, 1e-12);
  double eprev = 1e300;
  bool conv = false;
  int it = 0;
  while (!conv) {
    it += 1;
    double x[7];
    schur_solve(a, b, f, x);
    for (int i = 0; i < 7; ++i) { dsol[i] = -x[i]; sol[i] += dsol[i]; }
    std::memcpy(fOld, f, sizeof(f));
    rm_getKF(M, f, a, b, sol, eps_t, epl_old, damage, dt);
    double ls1 = 0, ls2 = 0;
    for (int i = 0; i < 7; ++i) { ls1 += f[i] * dsol[i]; ls2 += fOld[i] * dsol[i]; }
    double ls;
    if ((ls1 - ls2) == 0.0) ls = 1.0;
    else { ls = -(ls2) / (std::fabs(ls1 - ls2) + 1e-12) * sgn(ls1 - ls2); ls = std::min(std::max(ls, 0.2), 1.0); }
    for (int i = 0; i < 7; ++i) sol[i] = sol[i] - (1.0 - ls) * dsol[i];
    rm_getKF(M, f, a, b, sol, eps_t, epl_old, damage, dt);
    double e = 0; for (int i = 0; i < 7; ++i) e += f[i] * f[i];
    if (tol_mode == IFEM_RM_REFERENCE) {
      if (e < 1.0e-16 || e / e0 < 1.0e-9) conv = true;
    } else {
      if (e < 1.0e-36 || (it >= 3 && e >= eprev)) conv = true;
    }
    eprev = e;
    if (it > maxit) { conv = true; ++ro.capped; }
  }
  ro.iters += it;
  double S[6], dF[6];
  for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += M.D[i * 6 + j] * sol[j]; S[i] = s; }
  yield_ve(S, dF, nullptr);
  for (int i = 0; i < 6; ++i) epl[i] = epl_old[i] + sol[6] * dF[i];
  if (tangent_mode == IFEM_TANGENT_REFERENCE) {
    // Kinv(0:5,0:5) = I - a b^T / (1 + b.a)
    double ba = 0; for (int i = 0; i < 6; ++i) ba += b[i] * a[i];
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) DMat[i * 6 + j] = (i == j ? 1.0 : 0.0) - a[i] * b[j] / (1.0 + ba);
  } else {
    double Kx[49], Ki[49];
    rm_exact_jacobian(M, sol, dt, Kx);
    if (!lu_inverse(7, Kx, Ki)) throw Err{IFEM_ERR_NUMERIC, "singular return-map Jacobian"};
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) DMat[i * 6 + j] = Ki[i * 7 + j];
  }
  double diss = 0; for (int i = 0; i < 6; ++i) diss += S[i] * (epl[i] - epl_old[i]);
  diss = damage * diss;
  diss = std::fabs(diss) / dt;
  hist0 = sol[6];
  return diss;
}

// ----------------------------------------------------------------------------------------
// Viscoelastic-plastic return map (SolidMaterial.cpp:303-521).  Unknowns x = [eps_e (6), dLambda_v,
// dLambda_p]; stresses are unscaled.  P = I - 1/3 i i^T without a shear correction (SolidMaterial.cpp:86).
// ----------------------------------------------------------------------------------------
inline void dev_P(const double S[6], double out[6]) {
  const double m = (S[0] + S[1] + S[2]) / 3.0;
  for (int i = 0; i < 3; ++i) out[i] = S[i] - m;
  for (int i = 3; i < 6; ++i) out[i] = S[i];
}
inline void mat6_vec(const double* A, const double x[6], double y[6]) {
  for (int i = 0; i < 6; ++i) { double s = 0; for (int j = 0; j < 6; ++j) s += A[i * 6 + j] * x[j]; y[i] = s; }
}

// YieldFunction (SolidMaterial.cpp:447-475): the apex branch is chosen by the trial stress's I1
double vep_yield(const MatPt& M, const double S[6], const double St[6], double dF[6], double ddF[36]) {
  const double I1 = S[0] + S[1] + S[2];
  double dJ2[6];
  mat6_vec(kJ2Mat.m, S, dJ2);
  double J2 = 0; for (int i = 0; i < 6; ++i) J2 += S[i] * dJ2[i];
  J2 *= 0.5;
  bool apex = false;
  if (M.yield_alpha > 0.0) {
    const double I1Apex = M.sy * 3.0 / M.yield_alpha;
    if (St[0] + St[1] + St[2] > I1Apex) apex = true;
  }
  double F;
  if (!apex) {
    F = std::sqrt(3.0 * J2 + 1.0e-6) + M.yield_alpha / 3.0 * I1 - M.sy;
    const double c = 0.5 * std::sqrt(3.0) / std::sqrt(J2 + 1.0e-6);
    const double c2 = 0.25 * std::sqrt(3.0) * std::pow(J2 + 1.0e-6, -1.5);
    for (int i = 0; i < 6; ++i) dF[i] = c * dJ2[i] + (i < 3 ? M.yield_alpha / 3.0 : 0.0);
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) ddF[i * 6 + j] = c * kJ2Mat.m[i * 6 + j] - c2 * dJ2[i] * dJ2[j];
  } else {
    F = M.yield_alpha / 3.0 * I1 - M.sy;
    for (int i = 0; i < 6; ++i) dF[i] = i < 3 ? M.yield_alpha / 3.0 : 0.0;
    for (int i = 0; i < 36; ++i) ddF[i] = 0.0;
  }
  return F;
}

// PotentialFunction (SolidMaterial.cpp:494-521): dG normalised afterwards (Eigen normalize() leaves a zero
// vector unchanged), ddG not
void vep_potential(const MatPt& M, const double S[6], const double St[6], double dG[6], double ddG[36]) {
  double dJ2[6];
  mat6_vec(kJ2Mat.m, S, dJ2);
  double J2 = 0; for (int i = 0; i < 6; ++i) J2 += S[i] * dJ2[i];
  J2 *= 0.5;
  bool apex = false;
  if (M.yield_alpha > 0.0) {
    const double I1Apex = M.sy * 3.0 / M.yield_alpha;
    if (St[0] + St[1] + St[2] > I1Apex) apex = true;
  }
  if (!apex) {
    const double c = 0.5 * std::sqrt(3.0) / std::sqrt(J2 + 1.0e-6);
    const double c2 = 0.25 * std::sqrt(3.0) * std::pow(J2 + 1.0e-6, -1.5);
    for (int i = 0; i < 6; ++i) dG[i] = c * dJ2[i] + (i < 3 ? M.pot_alpha / 3.0 : 0.0);
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) ddG[i * 6 + j] = c * kJ2Mat.m[i * 6 + j] - c2 * dJ2[i] * dJ2[j];
  } else {
    double dS[6], Dinv[36];
    for (int i = 0; i < 6; ++i) dS[i] = St[i] - (i < 3 ? 3.0 * M.sy / M.yield_alpha : 0.0);
    if (!lu_inverse(6, M.D, Dinv)) throw Err{IFEM_ERR_NUMERIC, "singular elasticity matrix"};
    mat6_vec(Dinv, dS, dG);
    for (int i = 0; i < 36; ++i) ddG[i] = 0.0;
  }
  double z = 0; for (int i = 0; i < 6; ++i) z += dG[i] * dG[i];
  if (z > 0.0) { const double nrm = std::sqrt(z); for (int i = 0; i < 6; ++i) dG[i] /= nrm; }
}

// return_mapping_VEP_getKF (SolidMaterial.cpp:358-407): f (8) and K (8x8, row-major)
void vep_getKF(const MatPt& M, double K[64], double f[8], const double x[8], const double eps_t[6],
               const double eplo[6], double dt, double damage, double h_old) {
  for (int i = 0; i < 64; ++i) K[i] = 0.0;
  double S[6], Sd[6], St[6], r[6];
  mat6_vec(M.D, x, S);
  for (int i = 0; i < 6; ++i) S[i] *= damage;
  dev_P(S, Sd);
  for (int i = 0; i < 6; ++i) r[i] = eps_t[i] - eplo[i] - x[6] * Sd[i];
  mat6_vec(M.D, r, St);
  for (int i = 0; i < 6; ++i) St[i] *= damage;
  double dF[6], ddF[36], dG[6], ddG[36];
  const double FTrial = vep_yield(M, St, St, dF, ddF);
  const double F = vep_yield(M, S, St, dF, ddF);
  vep_potential(M, S, St, dG, ddG);
  double h = h_old + M.hardening * std::sqrt(x[7] * x[7]);
  double dh = M.hardening * sgn(x[7]);
  if (h < -0.9 * M.sy) { h = -0.9 * M.sy; dh = -0.0; }
  for (int i = 0; i < 6; ++i) f[i] = x[i] - eps_t[i] + eplo[i] + x[6] * Sd[i] + x[7] * dG[i];
  // K(0:5,0:5) = I + damage x6 P D + damage x7 ddG D
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double pd = 0, gd = 0;
      for (int k = 0; k < 6; ++k) {
        const double Pik = (i == k ? 1.0 : 0.0) - ((i < 3 && k < 3) ? 1.0 / 3.0 : 0.0);
        pd += Pik * M.D[k * 6 + j];
        gd += ddG[i * 6 + k] * M.D[k * 6 + j];
      }
      K[i * 8 + j] = (i == j ? 1.0 : 0.0) + damage * x[6] * pd + damage * x[7] * gd;
    }
  for (int i = 0; i < 6; ++i) { K[i * 8 + 6] = Sd[i]; K[i * 8 + 7] = dG[i]; }
  double ss = 0; for (int i = 0; i < 6; ++i) ss += Sd[i] * Sd[i];
  f[6] = x[6] - M.A * dt * std::pow(ss, (M.n - 1.0) / 2.0);
  K[6 * 8 + 6] = 1.0;
  // K(6,0:5) = -A dt ss^((n-3)/2) (n-1)/2 2 damage SDev^T P D
  double sP[6];
  dev_P(Sd, sP);   // P symmetric: (SDev^T P)^T = P SDev
  const double c6 = -M.A * dt * std::pow(ss, (M.n - 3.0) / 2.0) * (M.n - 1.0) / 2.0 * 2.0 * damage;
  for (int j = 0; j < 6; ++j) { double t = 0; for (int k = 0; k < 6; ++k) t += sP[k] * M.D[k * 6 + j]; K[6 * 8 + j] = c6 * t; }
  if (FTrial - h_old < 0.0) {
    f[7] = -(M.pl_visc + 1.0e0) / dt * x[7];
    K[7 * 8 + 7] = -(M.pl_visc + 1.0e0) / dt;
  } else {
    f[7] = F - h - M.pl_visc / dt * std::sqrt(x[7] * x[7] + 1.0e-12);
    for (int j = 0; j < 6; ++j) { double t = 0; for (int k = 0; k < 6; ++k) t += dF[k] * M.D[k * 6 + j]; K[7 * 8 + j] = damage * t; }
    K[7 * 8 + 7] = -M.pl_visc / dt * sgn(x[7]) - dh;
  }
}

// return_mapping_VEP (SolidMaterial.cpp:303-356) and return_mapping_VEP_updateStrain (:409-445).
// hist: the ip's current MatHist (initial guess x6 = hist[1], x7 = hist[2]; written back), h_old = MatHistOld[0].
// Returns DissRate; damdiss = DamDissRate.  DMat = K^-1(0:5,0:5) of the last evaluated K.
double return_mapping_vep(const MatPt& M, double DMat[36], double epl[6], const double eps_t[6],
                          const double eplo[6], double dt, double damage, double hist[4], double h_old,
                          int tol_mode, int maxit, double& damdiss, RMOut& ro) {
  double x[8], f[8], fOld[8], K[64], Ki[64], dx[8];
  for (int i = 0; i < 6; ++i) x[i] = eps_t[i] - epl[i];
  x[6] = hist[1];
  x[7] = hist[2];
  vep_getKF(M, K, f, x, eps_t, eplo, dt, damage, h_old);
  double e0 = 0; for (int i = 0; i < 8; ++i) e0 += f[i] * f[i];
  e0 = std::max(e0, 1e-12);
  double eprev = 1e300;
  bool conv = false;
  int it = 0;
  while (!conv) {
    it += 1;
    if (!lu_inverse(8, K, Ki)) throw Err{IFEM_ERR_NUMERIC, "singular VEP return-map Jacobian"};
    for (int i = 0; i < 8; ++i) { double s = 0; for (int j = 0; j < 8; ++j) s += Ki[i * 8 + j] * f[j]; dx[i] = -s; x[i] += dx[i]; }
    std::memcpy(fOld, f, sizeof(f));
    vep_getKF(M, K, f, x, eps_t, eplo, dt, damage, h_old);
    double ls1 = 0, ls2 = 0;
    for (int i = 0; i < 8; ++i) { ls1 += f[i] * dx[i]; ls2 += fOld[i] * dx[i]; }
    double ls;
    if ((ls1 - ls2) == 0.0) ls = 1.0;
    else { ls = -(ls2) / (std::fabs(ls1 - ls2) + 1e-12) * sgn(ls1 - ls2); ls = std::min(std::max(ls, 0.2), 1.0); }
    for (int i = 0; i < 8; ++i) x[i] = x[i] - (1.0 - ls) * dx[i];
    vep_getKF(M, K, f, x, eps_t, eplo, dt, damage, h_old);
    double e = 0; for (int i = 0; i < 8; ++i) e += f[i] * f[i];
    if (tol_mode == IFEM_RM_REFERENCE) {
      if (e < 1.0e-16 || e / e0 < 1.0e-8) conv = true;
    } else {
      if (e < 1.0e-36 || (it >= 3 && e >= eprev)) conv = true;
    }
    eprev = e;
    if (it > maxit) { conv = true; ++ro.capped; }
  }
  ro.iters += it;
  // updateStrain
  double S[6], Sd[6], St[6], r[6], dG[6], ddG[36];
  mat6_vec(M.D, x, S);
  for (int i = 0; i < 6; ++i) S[i] *= damage;
  dev_P(S, Sd);
  for (int i = 0; i < 6; ++i) r[i] = eps_t[i] - eplo[i] - x[6] * Sd[i];
  mat6_vec(M.D, r, St);
  for (int i = 0; i < 6; ++i) St[i] *= damage;
  vep_potential(M, S, St, dG, ddG);
  double dissV = 0, dissP = 0;
  for (int i = 0; i < 6; ++i) {
    const double ev = x[6] * Sd[i], ep = x[7] * dG[i];
    epl[i] = eplo[i] + ev + ep;
    dissV += 1.0 / dt * std::fabs(ev * S[i]);
    dissP += 1.0 / dt * std::fabs(ep * S[i]);
  }
  hist[0] = h_old + M.hardening * std::sqrt(x[7] * x[7]);
  hist[1] = x[6];
  hist[2] = x[7];
  if (!lu_inverse(8, K, Ki)) throw Err{IFEM_ERR_NUMERIC, "singular VEP return-map Jacobian"};
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) DMat[i * 6 + j] = Ki[i * 8 + j];
  damdiss = dissP;
  return dissV + dissP;
}

// ----------------------------------------------------------------------------------------
// The oracle context
// ----------------------------------------------------------------------------------------
// Constraints of one staggered step: Constrainer::conDofToVal (Constrainer.h:26) and the reduced system
// of Physics::Constraint (physics.cpp:328-362).
#include "oracle_cosserat.inc"

struct ConsData {
  std::map<int64_t, double> dof_to_val;   // ascending dof: the order of ConMats' columns (Constrainer.cpp:101-109)
  std::vector<int64_t> fmap;              // dof -> free index (>= 0) or -1 - constrained index
  std::vector<int64_t> free_dofs;         // free index -> dof (UnconMats, ascending)
  std::vector<int32_t> rowptr, colidx;    // pattern of K_con = U^T K U
  std::vector<double> cv, f_con, vals;    // C_v, f_con, K_con values
  bool built = false;
};

struct StepData {
  int64_t ndofs = 0;
  std::vector<int32_t> rowptr, colidx;
  std::vector<double> f, vals;
  std::vector<double> state[4];
  ifem_stats stats{};
  ConsData cons;
};

struct ShapeIP { double N[27]; double G[3][27]; double w; };
// getShapeGrads2: N, G and the second gradients G2 (3 or 6 components) at one ip
struct ShapeIP2 { ShapeIP s; double G2[6][27]; };

// TriAxial model (TriAxial.h:44-56): boundary element groups and running state
struct FaceGroup { int64_t nf = 0; std::vector<int64_t> F; std::vector<double> C; };
struct TriAxial {
  bool on = false;
  FaceGroup side, top;
  ifem_triaxial prm{};
  ifem_triaxial_state st{};
};

struct Oracle {
  int dim = 0, etype = 0, nen = 0, nip = 0, ip1d = 0;
  int64_t nn = 0, nel = 0;
  std::vector<double> X, W, C;  // coords, weights, full extraction ops
  std::vector<int64_t> E;
  std::vector<int32_t> emat;
  std::vector<ifem_material> mats;
  ifem_options opt{};
  // reference shapes
  std::vector<double> wip, Nbase, Gbase;  // [nip], [nip][nen], [nip][dim][nen]
  std::vector<double> G2base;             // [nip][3 or 6][nen]: xx, yy, xy (2D); xx, yy, zz, xy, yz, xz (3D)
  int nsteps = 0, step_u = -1, step_ph = -1, step_T = -1;
  bool hasT = false;
  std::vector<int64_t> dofnum[IFEM_N_DOF_KINDS];  // per kind: node -> dof (-1 absent)
  int ncs = 6;                     // strain components per ip: 6, or 18 for the Cosserat model
  std::vector<StepData> steps;
  std::vector<double> EH, EHo, EP, EPo, VD, VDo, DVD, DVDo, MH, MHo;
  int hist_size = 0;
  int nlag = 0;                    // Lagrange multipliers per phase node (irreversibility methods 3-5)
  std::string err;
  std::vector<double> ip_gc_last;  // scratch
  // last adjoint results per step, and the recorded "graph" (a replayable list of assemblies)
  std::vector<std::vector<double>> adj_full, adj_sets;
  std::vector<int> g_steps;
  ifem_time g_tm{};
  int g_adjoint = 0;
  TriAxial tri;
};

thread_local std::string g_create_err;

void build_shapes(Oracle& o) {
  std::vector<double> w1, c1;
  ip_scheme_1d(o.ip1d, w1, c1);
  const int q = o.ip1d;
  o.nip = (o.dim == 2) ? q * q : q * q * q;
  o.wip.assign(o.nip, 0);
  o.Nbase.assign((size_t)o.nip * o.nen, 0);
  o.Gbase.assign((size_t)o.nip * o.dim * o.nen, 0);
  o.G2base.assign((size_t)o.nip * (o.dim == 2 ? 3 : 6) * o.nen, 0);
  int cnt = 0;
  if (o.dim == 2) {
    for (int j = 0; j < q; ++j) for (int i = 0; i < q; ++i) {
      o.wip[cnt] = w1[i] * w1[j];
      double Nx[3], Gx[3], Ny[3], Gy[3], Hx[3], Hy[3];
      bezier_basis(2, c1[i], Nx, Gx);
      bezier_basis(2, c1[j], Ny, Gy);
      bezier_basis2(2, c1[i], Hx);
      bezier_basis2(2, c1[j], Hy);
      for (int b = 0; b < 3; ++b) for (int a = 0; a < 3; ++a) {   // KronProd: result(a + 3 b)
        o.Nbase[cnt * o.nen + a + 3 * b] = Nx[a] * Ny[b];
        o.Gbase[(cnt * 2 + 0) * o.nen + a + 3 * b] = Gx[a] * Ny[b];
        o.Gbase[(cnt * 2 + 1) * o.nen + a + 3 * b] = Nx[a] * Gy[b];
        // B2_2::SetUpBaseShapes (B2_2.cpp:43-49): G2x Ny, Nx G2y, Gx Gy
        o.G2base[(cnt * 3 + 0) * o.nen + a + 3 * b] = Hx[a] * Ny[b];
        o.G2base[(cnt * 3 + 1) * o.nen + a + 3 * b] = Nx[a] * Hy[b];
        o.G2base[(cnt * 3 + 2) * o.nen + a + 3 * b] = Gx[a] * Gy[b];
      }
      ++cnt;
    }
  } else {
    for (int k = 0; k < q; ++k) for (int j = 0; j < q; ++j) for (int i = 0; i < q; ++i) {
      o.wip[cnt] = w1[i] * w1[j] * w1[k];
      double Nx[3], Gx[3], Ny[3], Gy[3], Nz[3], Gz[3], Hx[3], Hy[3], Hz[3];
      bezier_basis(2, c1[i], Nx, Gx);
      bezier_basis(2, c1[j], Ny, Gy);
      bezier_basis(2, c1[k], Nz, Gz);
      bezier_basis2(2, c1[i], Hx);
      bezier_basis2(2, c1[j], Hy);
      bezier_basis2(2, c1[k], Hz);
      int m = 0;
      for (int c = 0; c < 3; ++c) for (int b = 0; b < 3; ++b) for (int a = 0; a < 3; ++a) {
        o.Nbase[cnt * o.nen + m] = Nx[a] * Ny[b] * Nz[c];
        o.Gbase[(cnt * 3 + 0) * o.nen + m] = Gx[a] * Ny[b] * Nz[c];
        o.Gbase[(cnt * 3 + 1) * o.nen + m] = Nx[a] * Gy[b] * Nz[c];
        o.Gbase[(cnt * 3 + 2) * o.nen + m] = Nx[a] * Ny[b] * Gz[c];
        // NURBS3_Cube2::SetUpBaseShapes (NURBS3_Cube2.cpp:45-56): xx, yy, zz, xy, yz, xz
        o.G2base[(cnt * 6 + 0) * o.nen + m] = Hx[a] * Ny[b] * Nz[c];
        o.G2base[(cnt * 6 + 1) * o.nen + m] = Nx[a] * Hy[b] * Nz[c];
        o.G2base[(cnt * 6 + 2) * o.nen + m] = Nx[a] * Ny[b] * Hz[c];
        o.G2base[(cnt * 6 + 3) * o.nen + m] = Gx[a] * Gy[b] * Nz[c];
        o.G2base[(cnt * 6 + 4) * o.nen + m] = Nx[a] * Gy[b] * Gz[c];
        o.G2base[(cnt * 6 + 5) * o.nen + m] = Gx[a] * Ny[b] * Gz[c];
        ++m;
      }
      ++cnt;
    }
  }
}

// Mesh::getShapeGrads -> B2_2::getShapeGrads (B2_2.cpp:72-88) / NURBS3_Cube2::getShapeGrads
// (NURBS3_Cube2.cpp:89-115).
void shape_grads(const Oracle& o, int64_t el, ShapeIP* out) {
  const int nen = o.nen, dim = o.dim;
  const double* C = &o.C[(size_t)el * nen * nen];
  const int64_t* nodes = &o.E[(size_t)el * nen];
  double Xe[27][3];
  double We[27];
  for (int a = 0; a < nen; ++a) {
    for (int d = 0; d < dim; ++d) Xe[a][d] = o.X[nodes[a] * dim + d];
    We[a] = o.W.empty() ? 1.0 : o.W[nodes[a]];
  }
  for (int ip = 0; ip < o.nip; ++ip) {
    const double* Nb = &o.Nbase[(size_t)ip * nen];
    ShapeIP& s = out[ip];
    if (dim == 2) {
      double GB[2][9];
      for (int a = 0; a < nen; ++a) {
        double sN = 0, s0 = 0, s1 = 0;
        for (int k = 0; k < nen; ++k) {
          sN += Nb[k] * C[a * nen + k];
          s0 += o.Gbase[(ip * 2 + 0) * nen + k] * C[a * nen + k];
          s1 += o.Gbase[(ip * 2 + 1) * nen + k] * C[a * nen + k];
        }
        s.N[a] = sN; GB[0][a] = s0; GB[1][a] = s1;
      }
      double J[4] = {0, 0, 0, 0};  // J(d,e) = sum_a GB(d,a) X(a,e), then transposed in place
      for (int d = 0; d < 2; ++d) for (int e = 0; e < 2; ++e) {
        double t = 0; for (int a = 0; a < nen; ++a) t += GB[d][a] * Xe[a][e];
        J[e * 2 + d] = t;
      }
      double Ji[4];
      inv2(J, Ji);
      s.w = o.wip[ip] * std::fabs(det2(J));
      for (int a = 0; a < nen; ++a) {
        s.G[0][a] = Ji[0] * GB[0][a] + Ji[1] * GB[1][a];
        s.G[1][a] = Ji[2] * GB[0][a] + Ji[3] * GB[1][a];
      }
    } else {
      double CB[27], GB[27][3];
      double wFun = 0;
      for (int a = 0; a < nen; ++a) {
        double sN = 0, g0 = 0, g1 = 0, g2 = 0;
        for (int k = 0; k < nen; ++k) {
          const double c = C[a * nen + k];
          sN += c * Nb[k];
          g0 += c * o.Gbase[(ip * 3 + 0) * nen + k];
          g1 += c * o.Gbase[(ip * 3 + 1) * nen + k];
          g2 += c * o.Gbase[(ip * 3 + 2) * nen + k];
        }
        CB[a] = sN; GB[a][0] = g0; GB[a][1] = g1; GB[a][2] = g2;
      }
      for (int a = 0; a < nen; ++a) wFun += CB[a] * We[a];
      for (int a = 0; a < nen; ++a) s.N[a] = We[a] * CB[a] / wFun;
      double dW[3] = {0, 0, 0};
      for (int d = 0; d < 3; ++d) for (int a = 0; a < nen; ++a) dW[d] += GB[a][d] * We[a];
      double GXi[27][3];
      for (int a = 0; a < nen; ++a) for (int d = 0; d < 3; ++d)
        GXi[a][d] = We[a] * (GB[a][d] / wFun - CB[a] * dW[d] / wFun / wFun);
      double J[9];
      for (int d = 0; d < 3; ++d) for (int e = 0; e < 3; ++e) {
        double t = 0; for (int a = 0; a < nen; ++a) t += GXi[a][d] * Xe[a][e];
        J[d * 3 + e] = t;
      }
      double Ji[9];
      inv3(J, Ji);
      s.w = o.wip[ip] * std::fabs(det3(J));
      for (int a = 0; a < nen; ++a) for (int d = 0; d < 3; ++d)
        s.G[d][a] = Ji[d * 3 + 0] * GXi[a][0] + Ji[d * 3 + 1] * GXi[a][1] + Ji[d * 3 + 2] * GXi[a][2];
    }
  }
}

// Mesh::getShapeGrads with second gradients -> B2_2::getShapeGrads2 (B2_2.cpp:90-125) /
// NURBS3_Cube2::getShapeGrads2 (NURBS3_Cube2.cpp:117-216).  As in the reference: in 2D the gradients use
// J^{-1} G_xi with J = G_xi X (getShapeGrads applies the inverse of J^T); the second gradients are
// J2^{-1} (G2_xi - J2Part2 G_xi) with the parametric first gradients, J2Part2 = G2_xi X.
void shape_grads2(const Oracle& o, int64_t el, ShapeIP2* out) {
  const int nen = o.nen, dim = o.dim;
  const double* C = &o.C[(size_t)el * nen * nen];
  const int64_t* nodes = &o.E[(size_t)el * nen];
  double Xe[27][3], We[27];
  for (int a = 0; a < nen; ++a) {
    for (int d = 0; d < dim; ++d) Xe[a][d] = o.X[nodes[a] * dim + d];
    We[a] = o.W.empty() ? 1.0 : o.W[nodes[a]];
  }
  for (int ip = 0; ip < o.nip; ++ip) {
    const double* Nb = &o.Nbase[(size_t)ip * nen];
    ShapeIP2& s2 = out[ip];
    ShapeIP& s = s2.s;
    if (dim == 2) {
      double GB[2][9], G2B[3][9];
      for (int a = 0; a < nen; ++a) {
        double sN = 0, g0 = 0, g1 = 0, h0 = 0, h1 = 0, h2 = 0;
        for (int k = 0; k < nen; ++k) {
          const double c = C[a * nen + k];
          sN += Nb[k] * c;
          g0 += o.Gbase[(ip * 2 + 0) * nen + k] * c;
          g1 += o.Gbase[(ip * 2 + 1) * nen + k] * c;
          h0 += o.G2base[(ip * 3 + 0) * nen + k] * c;
          h1 += o.G2base[(ip * 3 + 1) * nen + k] * c;
          h2 += o.G2base[(ip * 3 + 2) * nen + k] * c;
        }
        s.N[a] = sN; GB[0][a] = g0; GB[1][a] = g1; G2B[0][a] = h0; G2B[1][a] = h1; G2B[2][a] = h2;
      }
      double J[2][2], P[3][2];   // J = GB X, J2Part2 = G2B X
      for (int d = 0; d < 2; ++d) for (int e = 0; e < 2; ++e) {
        double t = 0; for (int a = 0; a < nen; ++a) t += GB[d][a] * Xe[a][e];
        J[d][e] = t;
      }
      for (int r = 0; r < 3; ++r) for (int e = 0; e < 2; ++e) {
        double t = 0; for (int a = 0; a < nen; ++a) t += G2B[r][a] * Xe[a][e];
        P[r][e] = t;
      }
      double J2[9] = {J[0][0] * J[0][0], J[0][1] * J[0][1], 2 * J[0][0] * J[0][1],
                      J[1][0] * J[1][0], J[1][1] * J[1][1], 2 * J[1][0] * J[1][1],
                      J[0][0] * J[1][0], J[0][1] * J[1][1], J[1][0] * J[0][1] + J[1][1] * J[0][0]};
      const double Jm[4] = {J[0][0], J[0][1], J[1][0], J[1][1]};
      double Ji[4], J2i[9];
      inv2(Jm, Ji);
      inv3(J2, J2i);
      s.w = o.wip[ip] * std::fabs(det2(Jm));
      for (int a = 0; a < nen; ++a) {
        s.G[0][a] = Ji[0] * GB[0][a] + Ji[1] * GB[1][a];
        s.G[1][a] = Ji[2] * GB[0][a] + Ji[3] * GB[1][a];
        double v[3];
        for (int r = 0; r < 3; ++r) v[r] = G2B[r][a] - (P[r][0] * GB[0][a] + P[r][1] * GB[1][a]);
        for (int r = 0; r < 3; ++r) s2.G2[r][a] = J2i[r * 3 + 0] * v[0] + J2i[r * 3 + 1] * v[1] + J2i[r * 3 + 2] * v[2];
      }
    } else {
      double CB[27], GB[27][3], G2B[27][6];
      for (int a = 0; a < nen; ++a) {
        double sN = 0, g[3] = {0, 0, 0}, h[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < nen; ++k) {
          const double c = C[a * nen + k];
          sN += c * Nb[k];
          for (int d = 0; d < 3; ++d) g[d] += c * o.Gbase[(ip * 3 + d) * nen + k];
          for (int r = 0; r < 6; ++r) h[r] += c * o.G2base[(ip * 6 + r) * nen + k];
        }
        CB[a] = sN;
        for (int d = 0; d < 3; ++d) GB[a][d] = g[d];
        for (int r = 0; r < 6; ++r) G2B[a][r] = h[r];
      }
      double wFun = 0, dW[3] = {0, 0, 0}, dW2[6] = {0, 0, 0, 0, 0, 0};
      for (int a = 0; a < nen; ++a) {
        wFun += CB[a] * We[a];
        for (int d = 0; d < 3; ++d) dW[d] += GB[a][d] * We[a];
        for (int r = 0; r < 6; ++r) dW2[r] += G2B[a][r] * We[a];
      }
      for (int a = 0; a < nen; ++a) s.N[a] = We[a] * CB[a] / wFun;
      double GXi[27][3], G2Xi[27][6];
      for (int a = 0; a < nen; ++a) for (int d = 0; d < 3; ++d)
        GXi[a][d] = We[a] * (GB[a][d] / wFun - CB[a] * dW[d] / wFun / wFun);
      const int pi[6] = {0, 1, 2, 0, 1, 0}, pj[6] = {0, 1, 2, 1, 2, 2};   // component -> (ii, jj)
      for (int a = 0; a < nen; ++a) for (int r = 0; r < 6; ++r) {
        const int ii = pi[r], jj = pj[r];
        G2Xi[a][r] = We[a] * (G2B[a][r] / wFun - dW[jj] * GB[a][ii] / wFun / wFun - dW[ii] * GB[a][jj] / wFun / wFun -
                              dW2[r] * CB[a] / wFun / wFun + 2 * dW[ii] * dW[jj] * CB[a] / wFun / wFun / wFun);
      }
      double J[3][3], P[6][3];
      for (int d = 0; d < 3; ++d) for (int e = 0; e < 3; ++e) {
        double t = 0; for (int a = 0; a < nen; ++a) t += GXi[a][d] * Xe[a][e];
        J[d][e] = t;
      }
      for (int r = 0; r < 6; ++r) for (int e = 0; e < 3; ++e) {
        double t = 0; for (int a = 0; a < nen; ++a) t += G2Xi[a][r] * Xe[a][e];
        P[r][e] = t;
      }
      double J2[36];
      for (int r = 0; r < 3; ++r) {   // rows xx, yy, zz
        J2[r * 6 + 0] = J[r][0] * J[r][0]; J2[r * 6 + 1] = J[r][1] * J[r][1]; J2[r * 6 + 2] = J[r][2] * J[r][2];
        J2[r * 6 + 3] = 2 * J[r][0] * J[r][1]; J2[r * 6 + 4] = 2 * J[r][1] * J[r][2]; J2[r * 6 + 5] = 2 * J[r][0] * J[r][2];
      }
      const int ra[3] = {0, 1, 0}, rb[3] = {1, 2, 2};   // rows xy, yz, xz pair the Jacobian rows (0,1), (1,2), (0,2)
      for (int t = 0; t < 3; ++t) {
        const int a = ra[t], b = rb[t], r = 3 + t;
        J2[r * 6 + 0] = J[a][0] * J[b][0]; J2[r * 6 + 1] = J[a][1] * J[b][1]; J2[r * 6 + 2] = J[a][2] * J[b][2];
        J2[r * 6 + 3] = J[a][0] * J[b][1] + J[b][0] * J[a][1];
        J2[r * 6 + 4] = J[a][1] * J[b][2] + J[b][1] * J[a][2];
        J2[r * 6 + 5] = J[a][0] * J[b][2] + J[b][0] * J[a][2];
      }
      const double Jm[9] = {J[0][0], J[0][1], J[0][2], J[1][0], J[1][1], J[1][2], J[2][0], J[2][1], J[2][2]};
      double Ji[9], J2i[36];
      inv3(Jm, Ji);
      if (!lu_inverse(6, J2, J2i)) throw Err{IFEM_ERR_NUMERIC, "singular second-derivative Jacobian"};
      s.w = o.wip[ip] * std::fabs(det3(Jm));
      for (int a = 0; a < nen; ++a) {
        for (int d = 0; d < 3; ++d) s.G[d][a] = Ji[d * 3 + 0] * GXi[a][0] + Ji[d * 3 + 1] * GXi[a][1] + Ji[d * 3 + 2] * GXi[a][2];
        double v[6];
        for (int r = 0; r < 6; ++r) v[r] = G2Xi[a][r] - (P[r][0] * GXi[a][0] + P[r][1] * GXi[a][1] + P[r][2] * GXi[a][2]);
        for (int r = 0; r < 6; ++r) {
          double t = 0; for (int k = 0; k < 6; ++k) t += J2i[r * 6 + k] * v[k];
          s2.G2[r][a] = t;
        }
      }
    }
  }
}

// ConstructBMat (math.cpp:3-26): B (6 x dim*nen), row-major
void build_B(const Oracle& o, const ShapeIP& s, double* B) {
  const int nen = o.nen, nU = o.dim * nen;
  std::fill(B, B + 6 * nU, 0.0);
  for (int a = 0; a < nen; ++a) {
    if (o.dim == 2) {
      B[0 * nU + a] = s.G[0][a]; B[3 * nU + a] = s.G[1][a];
      B[1 * nU + nen + a] = s.G[1][a]; B[3 * nU + nen + a] = s.G[0][a];
    } else {
      B[0 * nU + a] = s.G[0][a]; B[3 * nU + a] = s.G[1][a]; B[5 * nU + a] = s.G[2][a];
      B[1 * nU + nen + a] = s.G[1][a]; B[3 * nU + nen + a] = s.G[0][a]; B[4 * nU + nen + a] = s.G[2][a];
      B[2 * nU + 2 * nen + a] = s.G[2][a]; B[4 * nU + 2 * nen + a] = s.G[1][a]; B[5 * nU + 2 * nen + a] = s.G[0][a];
    }
  }
}

const ifem_material& mat_of(const Oracle& o, int64_t el) { return o.mats[o.emat.empty() ? 0 : o.emat[el]]; }

// element DOF lists (DofSpace::getDofForNodes, component-major, DofSpace.cpp:974-1008)
void elem_dofs(const Oracle& o, int64_t el, const std::vector<int>& kinds, int64_t* out) {
  const int64_t* nodes = &o.E[(size_t)el * o.nen];
  for (size_t j = 0; j < kinds.size(); ++j)
    for (int i = 0; i < o.nen; ++i) {
      const int64_t d = o.dofnum[kinds[j]][nodes[i]];
      if (d < 0) throw Err{IFEM_ERR_INVALID, "node not found for DOF type"};
      out[i + j * o.nen] = d;
    }
}

std::vector<int> phase_kinds(const Oracle& o) {
  std::vector<int> k = {IFEM_DOF_PHASE};
  if (o.nlag >= 1) k.push_back(IFEM_DOF_LMULT);
  if (o.nlag == 2) k.push_back(IFEM_DOF_LMULT2);
  return k;
}

std::vector<int> u_kinds(const Oracle& o) {
  if (o.opt.cosserat)   // DofNames_u of CossPhaseField (CossPhaseField.h:15, .cpp:170-180)
    return o.dim == 3 ? std::vector<int>{IFEM_DOF_UX, IFEM_DOF_UY, IFEM_DOF_UZ, IFEM_DOF_OX, IFEM_DOF_OY, IFEM_DOF_OZ}
                      : std::vector<int>{IFEM_DOF_UX, IFEM_DOF_UY, IFEM_DOF_OZ};
  std::vector<int> k = {IFEM_DOF_UX, IFEM_DOF_UY};
  if (o.dim == 3) k.push_back(IFEM_DOF_UZ);
  return k;
}

// Element output: dofs, F, K (column-major like Eigen, rows=cols=ndof_e)
struct ElemOut { int n = 0; int64_t dofs[162]; double F[162]; std::vector<double> K; double lcrack = 0; };

double ip_temperature(const Oracle& o, const ShapeIP& s, const double* Te) {
  if (!o.hasT) return o.opt.pinned_temperature;
  double t = 0; for (int a = 0; a < o.nen; ++a) t += s.N[a] * Te[a];
  return t;
}

void elem_U_coss(Oracle& o, int64_t el, const ifem_time& tm, ElemOut& out, RMOut& ro, bool write_hist);

// PhaseFieldDamage::Assemble_U, one element (PhaseField.cpp:353-482)
void elem_U(Oracle& o, int64_t el, const ifem_time& tm, ElemOut& out, RMOut& ro, bool write_hist) {
  if (o.opt.cosserat) { elem_U_coss(o, el, tm, out, ro, write_hist); return; }
  const int nen = o.nen, nU = o.dim * nen, nip = o.nip;
  const ifem_material& m = mat_of(o, el);
  ShapeIP sh[27];
  shape_grads(o, el, sh);
  out.n = nU;
  elem_dofs(o, el, u_kinds(o), out.dofs);
  int64_t dph[27];
  elem_dofs(o, el, {IFEM_DOF_PHASE}, dph);
  const StepData& su = o.steps[o.step_u];
  const StepData& sp = o.steps[o.step_ph];
  double U[81], UO[81], dU[81], ddU[81], Ph[27], PhO[27], Te[27];
  for (int i = 0; i < nU; ++i) {
    U[i] = su.state[IFEM_STATE_CUR][out.dofs[i]]; UO[i] = su.state[IFEM_STATE_OLD][out.dofs[i]];
    dU[i] = su.state[IFEM_STATE_D][out.dofs[i]]; ddU[i] = su.state[IFEM_STATE_DD][out.dofs[i]];
  }
  for (int i = 0; i < nen; ++i) { Ph[i] = sp.state[IFEM_STATE_CUR][dph[i]]; PhO[i] = sp.state[IFEM_STATE_OLD][dph[i]]; }
  if (o.hasT) {
    int64_t dT[27]; elem_dofs(o, el, {IFEM_DOF_T}, dT);
    for (int i = 0; i < nen; ++i) Te[i] = o.steps[o.step_T].state[IFEM_STATE_CUR][dT[i]];
  }
  std::fill(out.F, out.F + nU, 0.0);
  out.K.assign((size_t)nU * nU, 0.0);
  double WL[27] = {0};
  std::vector<double> B(6 * nU), DtB(6 * nU);
  MatPt M{};
  const double k0 = o.opt.k0;
  for (int ip = 0; ip < nip; ++ip) {
    set_temperature(m, ip_temperature(o, sh[ip], Te), M);
    double phi = 0, phiO = 0;
    for (int a = 0; a < nen; ++a) { phi += sh[ip].N[a] * Ph[a]; phiO += sh[ip].N[a] * PhO[a]; }
    double Dam, dDam, nn_, DamI, dDamI, DamG, dDamG;
    damage_function(phi, o.opt.dam_function, k0, porder(o.opt), Dam, dDam, nn_);
    damage_function(phi, o.opt.density_dam_function, k0, porder(o.opt), DamI, dDamI, nn_);
    damage_function(phi, o.opt.density_dam_function, k0, porder(o.opt), DamG, dDamG, nn_);
    build_B(o, sh[ip], B.data());
    double eps[6], epsO[6];
    for (int r = 0; r < 6; ++r) {
      double s = 0, t = 0;
      for (int c = 0; c < nU; ++c) { s += B[r * nU + c] * U[c]; t += B[r * nU + c] * UO[c]; }
      eps[r] = s; epsO[r] = t;
    }
    const size_t hi = (size_t)el * nip + ip;
    double epl[6], eplO[6];
    for (int r = 0; r < 6; ++r) { epl[r] = o.EP[hi * 6 + r]; eplO[r] = o.EPo[hi * 6 + r]; }
    double DPl[36];
    double diss = 0, damdiss = 0;
    auto ident = [&]() { for (int i = 0; i < 36; ++i) DPl[i] = (i % 7 == 0) ? 1.0 : 0.0; };
    const size_t hs = o.hist_size == 4 ? 4 : 1;    // MatHist values per ip
    double hist0 = o.hist_size > 0 ? o.MH[hi * hs] : 0.0;
    double vh[4] = {0, 0, 0, 0};
    bool vep = false;
    switch (M.rheology) {
      case IFEM_RHEO_LE: ident(); for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplO[r]; break;
      case IFEM_RHEO_VE:
        if (phi > M.phi_visc_lim) { ident(); for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplO[r]; }
        else diss = return_mapping_viscous(M, DPl, epl, eps, eplO, 1.0, tm.dt, hist0, o.opt.rm_tol_mode, o.opt.rm_max_it, o.opt.tangent_mode, ro);
        break;
      case IFEM_RHEO_DVE:
        if (phi > M.phi_visc_lim) { ident(); for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplO[r]; }
        else {
          double dmg, u1, u2;
          damage_function(phi, o.opt.dam_function, k0, porder(o.opt), dmg, u1, u2);
          diss = return_mapping_viscous(M, DPl, epl, eps, eplO, dmg, tm.dt, hist0, o.opt.rm_tol_mode, o.opt.rm_max_it, o.opt.tangent_mode, ro);
        }
        break;
      case IFEM_RHEO_VE_EXPL:
        if (phiO > M.phi_visc_lim) { ident(); for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplO[r]; }
        else { diss = return_mapping_viscous(M, DPl, epl, epsO, eplO, 1.0, tm.dt, hist0, o.opt.rm_tol_mode, o.opt.rm_max_it, o.opt.tangent_mode, ro); ident(); }
        break;
      case IFEM_RHEO_DVE_EXPL:
        if (phiO > M.phi_visc_lim) { ident(); for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplO[r]; }
        else {
          double dmg, u1, u2;
          damage_function(phiO, o.opt.dam_function, k0, porder(o.opt), dmg, u1, u2);
          diss = return_mapping_viscous(M, DPl, epl, epsO, eplO, dmg, tm.dt, hist0, o.opt.rm_tol_mode, o.opt.rm_max_it, o.opt.tangent_mode, ro);
          ident();
        }
        break;
      case IFEM_RHEO_VEP:   // SolidMaterial.cpp:174-182: damage fixed at 1, phiOld against PhiViscLim
        if (phiO > M.phi_visc_lim) { ident(); for (int r = 0; r < 6; ++r) epl[r] = 1.0 * eplO[r]; }
        else {
          for (int k = 0; k < 4; ++k) vh[k] = o.MH[hi * 4 + k];
          diss = return_mapping_vep(M, DPl, epl, eps, eplO, tm.dt, 1.0, vh, o.MHo[hi * 4], o.opt.rm_tol_mode,
                                    o.opt.rm_max_it, damdiss, ro);
          vep = true;
        }
        break;
      default: throw Err{IFEM_ERR_UNSUPPORTED, "rheology not supported"};
    }
    if (write_hist) {
      for (int r = 0; r < 6; ++r) o.EP[hi * 6 + r] = epl[r];
      o.VD[hi] = o.VDo[hi] + diss * tm.dt;
      o.DVD[hi] = o.DVDo[hi] + damdiss * tm.dt;
      if (vep) for (int k = 0; k < 3; ++k) o.MH[hi * 4 + k] = vh[k];
      else if (o.hist_size > 0) o.MH[hi * hs] = hist0;
    }
    double ee[6];
    for (int r = 0; r < 6; ++r) ee[r] = eps[r] - epl[r];
    double Dd[36], Du[36], Sd[6], Su[6];
    energy_split(M, Dd, Du, Sd, Su, ee);
    const double w = sh[ip].w;
    double sig[6];
    for (int r = 0; r < 6; ++r) sig[r] = Dam * Sd[r] + Su[r];
    for (int c = 0; c < nU; ++c) { double s = 0; for (int r = 0; r < 6; ++r) s += B[r * nU + c] * sig[r]; out.F[c] += w * s; }
    // Dt = (Dam*Dd + Du) * DPlast
    double Dt[36];
    for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) {
      double s = 0; for (int k = 0; k < 6; ++k) s += (Dam * Dd[i * 6 + k] + Du[i * 6 + k]) * DPl[k * 6 + j];
      Dt[i * 6 + j] = s;
    }
    for (int r = 0; r < 6; ++r) for (int c = 0; c < nU; ++c) {
      double s = 0; for (int k = 0; k < 6; ++k) s += Dt[r * 6 + k] * B[k * nU + c];
      DtB[r * nU + c] = s;
    }
    for (int c = 0; c < nU; ++c) for (int r = 0; r < nU; ++r) {
      double s = 0; for (int k = 0; k < 6; ++k) s += B[k * nU + r] * DtB[k * nU + c];
      out.K[(size_t)c * nU + r] += w * s;
    }
    for (int a = 0; a < nen; ++a) WL[a] += w * sh[ip].N[a];
  }
  const double g3[3] = {0, o.dim == 3 ? 0 : -9.81, o.dim == 3 ? -9.81 : 0};
  const double gv[3] = {o.opt.gravity ? g3[0] : 0.0, o.opt.gravity ? g3[1] : 0.0, o.opt.gravity ? g3[2] : 0.0};
  const double rho = m.density;
  for (int n = 0; n < nen; ++n) {
    const int ny = n + nen, nz = n + 2 * nen;
    double DamI, dDamI, u;
    if (o.opt.inertia) {
      damage_function(Ph[n], o.opt.density_dam_function, k0, porder(o.opt), DamI, dDamI, u);
      out.F[n] += WL[n] * DamI * rho * ddU[n]; out.K[(size_t)n * nU + n] += WL[n] * DamI * rho * tm.ddu_dt;
      out.F[ny] += WL[n] * DamI * rho * ddU[ny]; out.K[(size_t)ny * nU + ny] += WL[n] * DamI * rho * tm.ddu_dt;
      if (o.dim == 3) { out.F[nz] += WL[n] * DamI * rho * ddU[nz]; out.K[(size_t)nz * nU + nz] += WL[n] * DamI * rho * tm.ddu_dt; }
    }
    if (m.damping > 0.0) {
      out.F[n] += WL[n] * m.damping * dU[n]; out.K[(size_t)n * nU + n] += WL[n] * m.damping * tm.du_dt;
      out.F[ny] += WL[n] * m.damping * dU[ny]; out.K[(size_t)ny * nU + ny] += WL[n] * m.damping * tm.du_dt;
      if (o.dim == 3) { out.F[nz] += WL[n] * m.damping * dU[nz]; out.K[(size_t)nz * nU + nz] += WL[n] * m.damping * tm.du_dt; }
    }
    double DamG, dDamG;
    damage_function(Ph[n], o.opt.density_dam_function, k0, porder(o.opt), DamG, dDamG, u);
    out.F[n] += -WL[n] * DamG * rho * gv[0];
    out.F[ny] += -WL[n] * DamG * rho * gv[1];
    if (o.dim == 3) out.F[nz] += -WL[n] * DamG * rho * gv[2];
  }
}

// PhaseFieldUtility::GetDistributionFunction (PhaseFieldUtil.cpp:185-221)
// ConstructBMatCoss (CossPhaseField.cpp:1168-1223): B [18][nc * nen], columns in DofNames_u order
// (ux, uy, oz in 2D; ux, uy, uz, ox, oy, oz in 3D), strains 0-8 and curvatures 9-17
void coss_B(const Oracle& o, double lc, const ShapeIP& s, double* B) {
  const int nen = o.nen, nc = o.dim == 2 ? 3 : 6, nU = nc * nen;
  std::fill(B, B + 18 * nU, 0.0);
  auto put = [&](int row, int blk, int kind, double f) {   // kind 0..2: G(kind); 3: N
    for (int a = 0; a < nen; ++a) B[row * nU + blk * nen + a] += f * (kind < 3 ? s.G[kind][a] : s.N[a]);
  };
  if (o.dim == 2) {
    put(0, 0, 0, 1.0);
    put(1, 1, 1, 1.0);
    put(3, 1, 0, 1.0); put(3, 2, 3, -1.0);
    put(4, 0, 1, 1.0); put(4, 2, 3, 1.0);
    put(14, 2, 0, lc);
    put(16, 2, 1, lc);
  } else {
    put(0, 0, 0, 1.0); put(1, 1, 1, 1.0); put(2, 2, 2, 1.0);
    put(3, 1, 0, 1.0); put(3, 5, 3, -1.0);
    put(4, 0, 1, 1.0); put(4, 5, 3, 1.0);
    put(5, 2, 1, 1.0); put(5, 3, 3, -1.0);
    put(6, 1, 2, 1.0); put(6, 3, 3, 1.0);
    put(7, 2, 0, 1.0); put(7, 4, 3, -1.0);
    put(8, 0, 2, 1.0); put(8, 4, 3, 1.0);
    put(9, 3, 0, lc); put(10, 4, 1, lc); put(11, 5, 2, lc);
    put(12, 3, 0, lc); put(13, 4, 1, lc);
    put(14, 4, 1, lc); put(15, 5, 2, lc);
    put(16, 3, 0, lc); put(17, 5, 2, lc);
  }
}

// CossPhaseField::Assemble_U, one element (CossPhaseField.cpp:337-534)
void elem_U_coss(Oracle& o, int64_t el, const ifem_time& tm, ElemOut& out, RMOut& ro, bool write_hist) {
  const int nen = o.nen, nc = o.dim == 2 ? 3 : 6, nU = nc * nen, nip = o.nip;
  const ifem_material& m = mat_of(o, el);
  ShapeIP sh[27];
  shape_grads(o, el, sh);
  out.n = nU;
  elem_dofs(o, el, u_kinds(o), out.dofs);
  int64_t dph[27];
  elem_dofs(o, el, {IFEM_DOF_PHASE}, dph);
  const StepData& su = o.steps[o.step_u];
  const StepData& sp = o.steps[o.step_ph];
  double U[162], dU[162], ddU[162], Ph[27], Te[27];
  for (int i = 0; i < nU; ++i) {
    U[i] = su.state[IFEM_STATE_CUR][out.dofs[i]];
    dU[i] = su.state[IFEM_STATE_D][out.dofs[i]]; ddU[i] = su.state[IFEM_STATE_DD][out.dofs[i]];
  }
  for (int i = 0; i < nen; ++i) Ph[i] = sp.state[IFEM_STATE_CUR][dph[i]];
  if (o.hasT) {
    int64_t dT[27]; elem_dofs(o, el, {IFEM_DOF_T}, dT);
    for (int i = 0; i < nen; ++i) Te[i] = o.steps[o.step_T].state[IFEM_STATE_CUR][dT[i]];
  }
  std::fill(out.F, out.F + nU, 0.0);
  out.K.assign((size_t)nU * nU, 0.0);
  double WLI[27] = {0}, WLG[27] = {0};
  std::vector<double> B(18 * nU), DtB(18 * nU);
  MatPt M{};
  CossPt c{};
  const double k0 = o.opt.k0;
  for (int ip = 0; ip < nip; ++ip) {
    set_temperature(m, ip_temperature(o, sh[ip], Te), M);
    coss_point(m, M, c);
    double phi = 0;
    for (int a = 0; a < nen; ++a) phi += sh[ip].N[a] * Ph[a];
    double Dam, dDam, nn_, DamI, dDamI, DamG, dDamG;
    damage_function(phi, o.opt.dam_function, k0, porder(o.opt), Dam, dDam, nn_);
    damage_function(phi, o.opt.density_dam_function, k0, porder(o.opt), DamI, dDamI, nn_);
    damage_function(phi, o.opt.gravity_dam_function, k0, porder(o.opt), DamG, dDamG, nn_);
    coss_B(o, c.l_coss, sh[ip], B.data());
    double eps[18];   // the old total strain is not used by the Cosserat rheologies
    for (int r = 0; r < 18; ++r) { double s = 0; for (int k = 0; k < nU; ++k) s += B[r * nU + k] * U[k]; eps[r] = s; }
    const size_t hi = (size_t)el * nip + ip;
    double epl[18], eplO[18], hist[4] = {0, 0, 0, 0}, histO[4] = {0, 0, 0, 0};
    for (int r = 0; r < 18; ++r) { epl[r] = o.EP[hi * 18 + r]; eplO[r] = o.EPo[hi * 18 + r]; }
    if (o.hist_size == 4) for (int k = 0; k < 4; ++k) { hist[k] = o.MH[hi * 4 + k]; histO[k] = o.MHo[hi * 4 + k]; }
    double DPl[324], diss = 0, damdiss = 0;
    coss_update_plastic(c, M, o.opt, phi, tm.dt, eps, eplO, epl, hist, histO, DPl, diss, damdiss, ro);
    if (write_hist) {
      for (int r = 0; r < 18; ++r) o.EP[hi * 18 + r] = epl[r];
      o.VD[hi] = o.VDo[hi] + diss * tm.dt;
      o.DVD[hi] = o.DVDo[hi] + damdiss * tm.dt;
      if (o.hist_size == 4) for (int k = 0; k < 4; ++k) o.MH[hi * 4 + k] = hist[k];
    }
    double ee[18];
    for (int r = 0; r < 18; ++r) ee[r] = eps[r] - epl[r];
    double Dd[324], Du[324], Sd[18], Su[18];
    coss_energy_split(c, M, ee, Dd, Du, Sd, Su);
    const double w = sh[ip].w;
    double sig[18];
    for (int r = 0; r < 18; ++r) sig[r] = Dam * Sd[r] + Su[r];
    for (int k = 0; k < nU; ++k) { double s = 0; for (int r = 0; r < 18; ++r) s += B[r * nU + k] * sig[r]; out.F[k] += w * s; }
    double Dt[324];
    for (int i = 0; i < 18; ++i) for (int j = 0; j < 18; ++j) {
      double s = 0; for (int k = 0; k < 18; ++k) s += (Dam * Dd[i * 18 + k] + Du[i * 18 + k]) * DPl[k * 18 + j];
      Dt[i * 18 + j] = s;
    }
    for (int r = 0; r < 18; ++r) for (int k = 0; k < nU; ++k) {
      double s = 0; for (int q = 0; q < 18; ++q) s += Dt[r * 18 + q] * B[q * nU + k];
      DtB[r * nU + k] = s;
    }
    for (int cc = 0; cc < nU; ++cc) for (int r = 0; r < nU; ++r) {
      double s = 0; for (int q = 0; q < 18; ++q) s += B[q * nU + r] * DtB[q * nU + cc];
      out.K[(size_t)cc * nU + r] += w * s;
    }
    for (int a = 0; a < nen; ++a) { WLI[a] += w * sh[ip].N[a] * DamI; WLG[a] += w * sh[ip].N[a] * (1.0 - 0.0) * DamG; }
  }
  const double g3[3] = {0, o.dim == 3 ? 0 : -9.81, o.dim == 3 ? -9.81 : 0};
  const double gv[3] = {o.opt.gravity ? g3[0] : 0.0, o.opt.gravity ? g3[1] : 0.0, o.opt.gravity ? g3[2] : 0.0};
  const double rho = m.density, lc = m.l_coss;
  const double rhoCoss = 2 * lc * lc * rho / (1 + m.poisson);
  auto add = [&](int i, double f, double k) { out.F[i] += f; out.K[(size_t)i * nU + i] += k; };
  for (int n = 0; n < nen; ++n) {
    const int ny = n + nen, nz = n + 2 * nen, ox = n + 3 * nen, oy = n + 4 * nen;
    const int oz = o.dim == 2 ? n + 2 * nen : n + 5 * nen;
    if (o.opt.inertia) {
      add(n, WLI[n] * rho * ddU[n], WLI[n] * rho * tm.ddu_dt);
      add(ny, WLI[n] * rho * ddU[ny], WLI[n] * rho * tm.ddu_dt);
      add(oz, WLI[n] * rhoCoss * ddU[oz], WLI[n] * rhoCoss * tm.ddu_dt);
      if (o.dim == 3) {
        add(nz, WLI[n] * rho * ddU[nz], WLI[n] * rho * tm.ddu_dt);
        add(ox, WLI[n] * rhoCoss * ddU[ox], WLI[n] * rho * tm.ddu_dt);   // Density in the tangent, as the reference
        add(oy, WLI[n] * rhoCoss * ddU[oy], WLI[n] * rho * tm.ddu_dt);
      }
    }
    if (m.damping > 0.0) {
      const double dr = 2 * lc * lc * m.damping;
      add(n, WLI[n] * m.damping * dU[n], WLI[n] * m.damping * tm.du_dt);
      add(ny, WLI[n] * m.damping * dU[ny], WLI[n] * m.damping * tm.du_dt);
      add(oz, WLI[n] * dr * dU[oz], WLI[n] * dr * tm.du_dt);
      if (o.dim == 3) {
        add(nz, WLI[n] * m.damping * dU[nz], WLI[n] * m.damping * tm.du_dt);
        add(ox, WLI[n] * dr * dU[ox], WLI[n] * dr * tm.du_dt);
        add(oy, WLI[n] * dr * dU[oy], WLI[n] * dr * tm.du_dt);
      }
    }
    out.F[n] += -WLG[n] * rho * gv[0];
    out.F[ny] += -WLG[n] * rho * gv[1];
    if (o.dim == 3) out.F[nz] += -WLG[n] * rho * gv[2];
  }
}

double distribution(int method, double l, const ShapeIP& s, int nen, int dim, const double* Ph, double* Dist, double* dDist) {
  double phi = 0; for (int a = 0; a < nen; ++a) phi += s.N[a] * Ph[a];
  double dG[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) for (int a = 0; a < nen; ++a) dG[d] += s.G[d][a] * Ph[a];
  double dGdG = 0; for (int d = 0; d < dim; ++d) dGdG += dG[d] * dG[d];
  double c, qphi, lin, grad;  // Dist = c*(qphi*N*phi + lin*N + grad*G^T dG); dDist = c*(qphi*NN + grad*GG)
  double gamma;
  switch (method) {
    case IFEM_DIST_QUADRATIC: c = 1.0 / (2.0 * l); gamma = c * (phi * phi + l * l * dGdG); qphi = 2.0; lin = 0; grad = 2.0 * l * l; break;
    case IFEM_DIST_LINEAR: c = 3.0 / (8.0 * l); gamma = c * (phi + l * l * dGdG); qphi = 0; lin = 1.0; grad = 2.0 * l * l; break;
    case IFEM_DIST_LINEAR2: c = 1.0 / (4.0 * l); gamma = c * (2.0 * phi + l * l * dGdG); qphi = 0; lin = 2.0; grad = 2.0 * l * l; break;
    case IFEM_DIST_LOCAL: c = 1.0 / l; gamma = c * (phi * phi); qphi = 2; lin = 0; grad = 0; break;
    case IFEM_DIST_CZM: {
      c = 1.0 / (3.141592 * l); gamma = c * (2.0 * phi - phi * phi + l * l * dGdG);
      for (int a = 0; a < nen; ++a) {
        double gd = 0; for (int d = 0; d < dim; ++d) gd += s.G[d][a] * dG[d];
        Dist[a] = c * (2.0 * s.N[a] * (1.0 - phi) + 2.0 * l * l * gd);
        for (int b = 0; b < nen; ++b) {
          double gg = 0; for (int d = 0; d < dim; ++d) gg += s.G[d][a] * s.G[d][b];
          dDist[a + b * nen] = c * (-2.0 * s.N[a] * s.N[b] + 2.0 * l * l * gg);
        }
      }
      return gamma;
    }
    default: throw Err{IFEM_ERR_UNSUPPORTED, "distribution function not supported"};
  }
  for (int a = 0; a < nen; ++a) {
    double gd = 0; for (int d = 0; d < dim; ++d) gd += s.G[d][a] * dG[d];
    Dist[a] = c * (qphi * s.N[a] * phi + lin * s.N[a] + grad * gd);
    for (int b = 0; b < nen; ++b) {
      double gg = 0; for (int d = 0; d < dim; ++d) gg += s.G[d][a] * s.G[d][b];
      dDist[a + b * nen] = c * (qphi * s.N[a] * s.N[b] + grad * gg);
    }
  }
  return gamma;
}

bool needs_grad2(int method) {   // PhaseFieldUtil.cpp:17-21
  return method == IFEM_DIST_HO_LINEAR || method == IFEM_DIST_HO_LINEAR2 || method == IFEM_DIST_HO_QUADRATIC ||
         method == IFEM_DIST_HO_CZM || method == IFEM_DIST_CUSTOM;
}

// PhaseFieldUtility::GetDistributionFunction with second gradients (PhaseFieldUtil.cpp:223-280); the other
// methods fall back to the first-order form with the same N and G
double distribution2(int method, double l, const double* coefs, const ShapeIP2& s2, int nen, int dim, const double* Ph,
                     double* Dist, double* dDist) {
  if (!needs_grad2(method)) return distribution(method, l, s2.s, nen, dim, Ph, Dist, dDist);
  const ShapeIP& s = s2.s;
  const int ng = dim == 2 ? 3 : 6;
  double DC[6];                     // DoubleCon: 1 on the normal, 2 on the mixed second derivatives
  for (int r = 0; r < ng; ++r) DC[r] = r < dim ? 1.0 : 2.0;
  double phi = 0; for (int a = 0; a < nen; ++a) phi += s.N[a] * Ph[a];
  double dG[3] = {0, 0, 0}, ddG[6] = {0, 0, 0, 0, 0, 0};
  for (int d = 0; d < dim; ++d) for (int a = 0; a < nen; ++a) dG[d] += s.G[d][a] * Ph[a];
  for (int r = 0; r < ng; ++r) for (int a = 0; a < nen; ++a) ddG[r] += s2.G2[r][a] * Ph[a];
  double dGdG = 0; for (int d = 0; d < dim; ++d) dGdG += dG[d] * dG[d];
  double hh = 0; for (int r = 0; r < ng; ++r) hh += ddG[r] * DC[r] * ddG[r];
  const double l2 = l * l, l4 = l * l * l * l;
  auto gd = [&](int a) { double t = 0; for (int d = 0; d < dim; ++d) t += s.G[d][a] * dG[d]; return t; };
  auto hd = [&](int a) { double t = 0; for (int r = 0; r < ng; ++r) t += s2.G2[r][a] * DC[r] * ddG[r]; return t; };
  auto gg = [&](int a, int b) { double t = 0; for (int d = 0; d < dim; ++d) t += s.G[d][a] * s.G[d][b]; return t; };
  auto hb = [&](int a, int b) { double t = 0; for (int r = 0; r < ng; ++r) t += s2.G2[r][a] * DC[r] * s2.G2[r][b]; return t; };
  double gamma = 0;
  switch (method) {
    case IFEM_DIST_HO_QUADRATIC: {
      const double c = 1.0 / (2.0 * l);
      gamma = c * (phi * phi + 0.5 * l2 * dGdG + l4 / 16.0 * hh);
      for (int a = 0; a < nen; ++a) {
        Dist[a] = c * (2.0 * s.N[a] * phi + l2 * gd(a) + l4 / 8.0 * hd(a));
        for (int b = 0; b < nen; ++b) dDist[a + b * nen] = c * (2.0 * s.N[a] * s.N[b] + l2 * gg(a, b) + l4 / 8.0 * hb(a, b));
      }
    } break;
    case IFEM_DIST_HO_CZM: {
      const double c = 1.0 / (3.020 * l);
      gamma = c * (2.0 * phi - phi * phi + 0.5 * l2 * dGdG + l4 / 16.0 * hh);
      for (int a = 0; a < nen; ++a) {
        Dist[a] = c * (2.0 * s.N[a] * (1.0 - phi) + l2 * gd(a) + l4 / 8.0 * hd(a));
        for (int b = 0; b < nen; ++b) dDist[a + b * nen] = c * (-2.0 * s.N[a] * s.N[b] + l2 * gg(a, b) + l4 / 8.0 * hb(a, b));
      }
    } break;
    case IFEM_DIST_HO_LINEAR: {
      const double c = 1.0 / (19.2 * l);
      gamma = c * (9.0 * phi + l4 * hh);
      for (int a = 0; a < nen; ++a) {
        Dist[a] = c * (9.0 * s.N[a] + 2.0 * l4 * hd(a));
        for (int b = 0; b < nen; ++b) dDist[a + b * nen] = c * (2.0 * l4 * hb(a, b));
      }
    } break;
    case IFEM_DIST_HO_LINEAR2: {
      const double c = 1.0 / (4.0 * l);
      gamma = c * (2.0 * phi + 0.5 * l2 * dGdG + l4 / 16.0 * hh);
      for (int a = 0; a < nen; ++a) {
        Dist[a] = c * (2.0 * s.N[a] + l2 * gd(a) + l4 / 8.0 * hd(a));
        for (int b = 0; b < nen; ++b) dDist[a + b * nen] = c * (l2 * gg(a, b) + l4 / 8.0 * hb(a, b));
      }
    } break;
    default: {   // Custom
      const double c = 1.0 / (coefs[0] * l);
      gamma = c * (coefs[1] * phi + coefs[2] * phi * phi + coefs[3] * l2 * dGdG + coefs[4] * l4 * hh);
      for (int a = 0; a < nen; ++a) {
        Dist[a] = c * (coefs[1] * s.N[a] + 2.0 * coefs[2] * s.N[a] * phi + 2.0 * coefs[3] * l2 * gd(a) +
                       2.0 * coefs[4] * l4 * hd(a));
        for (int b = 0; b < nen; ++b)
          dDist[a + b * nen] = c * (2.0 * coefs[2] * s.N[a] * s.N[b] + 2.0 * coefs[3] * l2 * gg(a, b) + 2.0 * coefs[4] * l4 * hb(a, b));
      }
    } break;
  }
  return gamma;
}

double distribution_gamma(int method, double l, const ShapeIP& s, int nen, int dim, const double* Ph) {
  double Dist[27], dDist[729];
  return distribution(method, l, s, nen, dim, Ph, Dist, dDist);
}

// PhaseFieldUtility::GetCapacityOnly (PhaseFieldUtil.cpp:282-348): lumped parts only
void capacity_lumped(int method, double l, double phi, double& DL, double& dDL, const double* coefs = nullptr) {
  switch (method) {
    case IFEM_DIST_HO_QUADRATIC: DL = 1.0 / (l)*phi; dDL = 1.0 / l; break;
    case IFEM_DIST_HO_CZM: DL = 2.0 / (3.020 * l) * (1 - phi); dDL = -2.0 / (3.020 * l); break;
    case IFEM_DIST_HO_LINEAR: DL = 9.0 / (19.2 * l); dDL = 0.0; break;
    case IFEM_DIST_HO_LINEAR2: DL = 3.0 / (8.0 * l); dDL = 0.0; break;
    case IFEM_DIST_CUSTOM:
      DL = 1.0 / (coefs[0] * l) * (coefs[1] + 2.0 * coefs[2] * phi); dDL = 1.0 / (coefs[0] * l) * 2.0 * coefs[2]; break;
    case IFEM_DIST_QUADRATIC: DL = 1.0 / l * phi; dDL = 1.0 / l; break;
    case IFEM_DIST_CZM: DL = 2.0 / (3.141592 * l) * (1.0 - phi); dDL = -2.0 / (3.141592 * l); break;
    case IFEM_DIST_LINEAR: DL = 3.0 / (8.0 * l); dDL = 0.0; break;
    case IFEM_DIST_LINEAR2: DL = 1.0 / (4.0 * l); dDL = 0.0; break;
    case IFEM_DIST_LOCAL: DL = 2.0 / (l)*phi; dDL = 2.0 / l; break;
    default: throw Err{IFEM_ERR_UNSUPPORTED, "distribution"};
  }
}
void capacity_full(int method, double l, const ShapeIP& s, int nen, double phi, double* D, double* dD,
                   const double* coefs = nullptr) {
  for (int a = 0; a < nen; ++a) {
    double v = 0;
    switch (method) {
      case IFEM_DIST_HO_QUADRATIC: v = 1.0 / (2.0 * l) * (2.0 * s.N[a] * phi); break;
      case IFEM_DIST_HO_CZM: v = 1.0 / (3.020 * l) * (2.0 * s.N[a] * (1.0 - phi)); break;
      case IFEM_DIST_HO_LINEAR: v = 1.0 / (19.2 * l) * (9.0 * s.N[a]); break;
      case IFEM_DIST_HO_LINEAR2: v = 3.0 / (8.0 * l) * s.N[a]; break;
      case IFEM_DIST_CUSTOM: v = 1.0 / (coefs[0] * l) * (coefs[1] * s.N[a] + 2.0 * coefs[2] * s.N[a] * phi); break;
      case IFEM_DIST_QUADRATIC: v = 1.0 / (2.0 * l) * (2.0 * s.N[a] * phi); break;
      case IFEM_DIST_CZM: v = 1.0 / (3.141592 * l) * (2.0 * s.N[a] * (1.0 - phi)); break;
      case IFEM_DIST_LINEAR: v = 3.0 / (8.0 * l) * (s.N[a]); break;
      case IFEM_DIST_LINEAR2: v = 1.0 / (4.0 * l) * (2.0 * s.N[a]); break;
      case IFEM_DIST_LOCAL: v = 1.0 / (l) * (2 * s.N[a] * phi); break;
    }
    D[a] = v;
    for (int b = 0; b < nen; ++b) {
      double k = 0;
      switch (method) {
        case IFEM_DIST_HO_QUADRATIC: k = 1.0 / (2.0 * l) * (2.0 * s.N[a] * s.N[b]); break;
        case IFEM_DIST_HO_CZM: k = 1.0 / (3.020 * l) * (-2.0 * s.N[a] * s.N[b]); break;
        case IFEM_DIST_CUSTOM: k = 1.0 / (coefs[0] * l) * (2.0 * coefs[2] * s.N[a] * s.N[b]); break;
        case IFEM_DIST_QUADRATIC: k = 1.0 / (2.0 * l) * (2.0 * s.N[a] * s.N[b]); break;
        case IFEM_DIST_CZM: k = 1.0 / (3.141592 * l) * (-2.0 * s.N[a] * s.N[b]); break;
        case IFEM_DIST_LOCAL: k = 1.0 / (l) * (2 * s.N[a] * s.N[b]); break;
        default: k = 0.0;
      }
      dD[a + b * nen] = k;
    }
  }
}

// PhaseFieldDamage::Assemble_Phase, one element (PhaseField.cpp:541-730)
void lagrange_terms(const Oracle& o, int64_t el, const ifem_material& m, const double* Ph, const double* PhO,
                    const double* WL, ElemOut& out);

void elem_phase(Oracle& o, int64_t el, const ifem_time& tm, ElemOut& out, bool write_hist) {
  const bool coss = o.opt.cosserat != 0;
  const int nen = o.nen, nU = (coss ? (o.dim == 2 ? 3 : 6) : o.dim) * nen, nip = o.nip;
  // the Cosserat phase step has no lumped driving or lumped capacity (CossPhaseField.cpp:536-769)
  const bool lumped_drive = o.opt.lumped_drive && !coss, lumped_cap = o.opt.lumped_cap && !coss;
  const ifem_material& m = mat_of(o, el);
  ShapeIP sh[27];
  shape_grads(o, el, sh);
  // the phase group's shape functions with second gradients when the distribution needs them (PhaseField.cpp:546-550)
  const bool ho = needs_grad2(o.opt.distribution);
  std::vector<ShapeIP2> sh2(ho ? nip : 0);
  if (ho) shape_grads2(o, el, sh2.data());
  out.n = nen;
  int64_t du[162];
  elem_dofs(o, el, u_kinds(o), du);
  elem_dofs(o, el, {IFEM_DOF_PHASE}, out.dofs);
  const StepData& su = o.steps[o.step_u];
  const StepData& sp = o.steps[o.step_ph];
  double U[162], dU[162], Ph[27], PhO[27], Te[27];
  for (int i = 0; i < nU; ++i) { U[i] = su.state[IFEM_STATE_CUR][du[i]]; dU[i] = su.state[IFEM_STATE_D][du[i]]; }
  for (int i = 0; i < nen; ++i) { Ph[i] = sp.state[IFEM_STATE_CUR][out.dofs[i]]; PhO[i] = sp.state[IFEM_STATE_OLD][out.dofs[i]]; }
  if (o.hasT) {
    if (o.opt.ref_compat_phase_t) {
      for (int i = 0; i < nen; ++i) Te[i] = o.steps[o.step_T].state[IFEM_STATE_CUR][0];
    } else {
      int64_t dT[27]; elem_dofs(o, el, {IFEM_DOF_T}, dT);
      for (int i = 0; i < nen; ++i) Te[i] = o.steps[o.step_T].state[IFEM_STATE_CUR][dT[i]];
    }
  }
  std::fill(out.F, out.F + nen, 0.0);
  out.K.assign((size_t)nen * nen, 0.0);
  double WL[27] = {0}, LD[27] = {0};
  std::vector<double> B((coss ? 18 : 6) * nU);
  double Dist[27], dDist[729], DC[27], dDC[729];
  MatPt M{};
  const double k0 = o.opt.k0;
  const double g3[3] = {0, o.dim == 3 ? 0 : -9.81, o.dim == 3 ? -9.81 : 0};
  const double gv[3] = {o.opt.gravity ? g3[0] : 0.0, o.opt.gravity ? g3[1] : 0.0, o.opt.gravity ? g3[2] : 0.0};
  out.lcrack = 0;
  for (int ip = 0; ip < nip; ++ip) {
    set_temperature(m, ip_temperature(o, sh[ip], Te), M);
    double phi = 0; for (int a = 0; a < nen; ++a) phi += sh[ip].N[a] * Ph[a];
    double Dam, dDam, ddDam, DamI, dDamI, ddDamI, DamG, dDamG, ddDamG;
    damage_function(phi, o.opt.dam_function, k0, porder(o.opt), Dam, dDam, ddDam);
    damage_function(phi, o.opt.density_dam_function, k0, porder(o.opt), DamI, dDamI, ddDamI);
    damage_function(phi, coss ? o.opt.gravity_dam_function : o.opt.density_dam_function, k0, porder(o.opt), DamG,
                    dDamG, ddDamG);
    const size_t hi = (size_t)el * nip + ip;
    double Energy;
    if (coss) {   // CossPhaseField.cpp:676-686: Cosserat split of B U - plastic strain, zero before t = 0
      CossPt c{};
      coss_point(m, M, c);
      coss_B(o, c.l_coss, sh[ip], B.data());
      double ee[18];
      for (int r = 0; r < 18; ++r) { double s = 0; for (int k = 0; k < nU; ++k) s += B[r * nU + k] * U[k]; ee[r] = s - o.EP[hi * 18 + r]; }
      std::vector<double> Dd(324), Du(324);
      double Sd[18], Su[18];
      Energy = coss_energy_split(c, M, ee, Dd.data(), Du.data(), Sd, Su);
      if (tm.t < 0.0) Energy = 0.0;
    } else {
      build_B(o, sh[ip], B.data());
      double ee[6];
      for (int r = 0; r < 6; ++r) { double s = 0; for (int c = 0; c < nU; ++c) s += B[r * nU + c] * U[c]; ee[r] = s - o.EP[hi * 6 + r]; }
      double Dd[36], Du[36], Sd[6], Su[6];
      Energy = energy_split(M, Dd, Du, Sd, Su, ee);
    }
    if (o.opt.irreversible == IFEM_IRR_HIST) {
      if (o.EHo[hi] > Energy) { if (write_hist) o.EH[hi] = o.EHo[hi]; Energy = o.EHo[hi]; }
      else if (write_hist) o.EH[hi] = Energy;
    } else if (write_hist) o.EH[hi] = Energy;
    const double gamma = ho ? distribution2(o.opt.distribution, M.l, o.opt.dist_coefs, sh2[ip], nen, o.dim, Ph, Dist, dDist)
                            : distribution(o.opt.distribution, M.l, sh[ip], nen, o.dim, Ph, Dist, dDist);
    if (lumped_cap) capacity_full(o.opt.distribution, M.l, sh[ip], nen, phi, DC, dDC, o.opt.dist_coefs);
    else { std::fill(DC, DC + nen, 0.0); std::fill(dDC, dDC + nen * nen, 0.0); }
    const double w = sh[ip].w;
    out.lcrack += gamma * w;
    for (int a = 0; a < nen; ++a) out.F[a] += w * M.Gc * (Dist[a] - DC[a]);
    for (int k = 0; k < nen * nen; ++k) out.K[k] += w * M.Gc * (dDist[k] - dDC[k]);
    if (!lumped_drive) {
      for (int a = 0; a < nen; ++a) out.F[a] += w * dDam * sh[ip].N[a] * Energy;
      for (int b = 0; b < nen; ++b) for (int a = 0; a < nen; ++a) out.K[a + b * nen] += w * ddDam * sh[ip].N[a] * sh[ip].N[b] * Energy;
    } else {
      for (int a = 0; a < nen; ++a) LD[a] += w * sh[ip].N[a] * Energy;
    }
    if (o.opt.visco_driving_factor > 1.0e-9) {
      double DamV, dDamV, ddDamV;
      const double PD = o.opt.visco_driving_factor * o.DVD[hi];
      damage_function(phi, o.opt.visco_dam_function, k0, porder(o.opt), DamV, dDamV, ddDamV);
      for (int a = 0; a < nen; ++a) out.F[a] += w * dDamV * sh[ip].N[a] * PD;
      for (int b = 0; b < nen; ++b) for (int a = 0; a < nen; ++a) out.K[a + b * nen] += w * ddDamV * sh[ip].N[a] * sh[ip].N[b] * PD;
    }
    if (o.opt.inertia && o.opt.consistent_degradation) {
      double v2 = 0;
      // N_uu dU: the translations, and in the Cosserat model the micro-rotations (ConstructNMatCoss)
      for (int d = 0; d < nU / nen; ++d) { double v = 0; for (int a = 0; a < nen; ++a) v += sh[ip].N[a] * dU[d * nen + a]; v2 += v * v; }
      for (int a = 0; a < nen; ++a) out.F[a] += -w * 0.5 * m.density * v2 * sh[ip].N[a] * dDamI;
      for (int b = 0; b < nen; ++b) for (int a = 0; a < nen; ++a) out.K[a + b * nen] += -w * 0.5 * m.density * v2 * sh[ip].N[a] * sh[ip].N[b] * ddDamI;
    }
    if (o.opt.consistent_degradation) {
      double gu = 0;
      for (int d = 0; d < o.dim; ++d) { double v = 0; for (int a = 0; a < nen; ++a) v += sh[ip].N[a] * U[d * nen + a]; gu += gv[d] * v; }
      for (int a = 0; a < nen; ++a) out.F[a] += -w * m.density * gu * sh[ip].N[a] * dDamG;
      for (int b = 0; b < nen; ++b) for (int a = 0; a < nen; ++a) out.K[a + b * nen] += -w * m.density * gu * sh[ip].N[a] * sh[ip].N[b] * ddDamG;
    }
    for (int a = 0; a < nen; ++a) WL[a] += w * sh[ip].N[a];
  }
  // nodal terms use the material state of the last integration point (PhaseField.cpp:693-711)
  for (int n = 0; n < nen; ++n) {
    if (lumped_drive) {
      double D, dD, ddD;
      damage_function(Ph[n], o.opt.dam_function, k0, porder(o.opt), D, dD, ddD);
      out.F[n] += LD[n] * dD; out.K[n + n * nen] += LD[n] * ddD;
    }
    if (lumped_cap) {
      double DL, dDL;
      capacity_lumped(o.opt.distribution, M.l, Ph[n], DL, dDL, o.opt.dist_coefs);
      out.F[n] += WL[n] * M.Gc * DL; out.K[n + n * nen] += WL[n] * M.Gc * dDL;
    }
    out.F[n] += WL[n] * M.visc / tm.dt * (Ph[n] - PhO[n]);
    const double stab = (o.opt.tangent_mode == IFEM_TANGENT_CONSISTENT) ? 0.0 : o.opt.visc_num * M.Gc / M.l;
    out.K[n + n * nen] += WL[n] * (M.visc / tm.dt + stab);
  }
  if (o.opt.irreversible == IFEM_IRR_PENALTY) {  // PhaseFieldUtil.cpp:350-380, utility's own JSON Gc
    for (int n = 0; n < nen; ++n) {
      const double lim0 = std::min(1.0 - 1.0e-3, std::max(0.0, PhO[n])), lim1 = 1.0 + 1e-1;
      if (Ph[n] < lim0) { out.F[n] += WL[n] * m.gc * o.opt.penalty_factor * (Ph[n] - lim0); out.K[n + n * nen] += WL[n] * m.gc * o.opt.penalty_factor; }
      if (Ph[n] > lim1) { out.F[n] += WL[n] * m.gc * o.opt.penalty_factor * (Ph[n] - lim1); out.K[n + n * nen] += WL[n] * m.gc * o.opt.penalty_factor; }
    }
  }
  if (o.nlag > 0) lagrange_terms(o, el, m, Ph, PhO, WL, out);
}

// EnforceIrreversible with the Lagrange-multiplier methods (PhaseFieldUtil.cpp:350-484, PhaseField.cpp:712-729):
// the phase element grows to the [Phase, L(, L2)] x nodes system; every coupling is nodal (diagonal blocks), and
// the terms come after all other phase terms, node by node, as in the reference.  The utility's own Gc and l
// (the JSON values) scale the augmented methods.
void lagrange_terms(const Oracle& o, int64_t el, const ifem_material& m, const double* Ph, const double* PhO,
                    const double* WL, ElemOut& out) {
  const int nen = o.nen, nc = 1 + o.nlag, n = nc * nen;
  std::vector<double> K((size_t)n * n, 0.0);   // column-major, rows/cols [Phase nodes, L nodes, L2 nodes]
  for (int b = 0; b < nen; ++b) for (int a = 0; a < nen; ++a) K[a + (size_t)b * n] = out.K[a + (size_t)b * nen];
  for (int i = nen; i < n; ++i) out.F[i] = 0.0;
  int64_t dl[81];
  elem_dofs(o, el, phase_kinds(o), dl);
  const StepData& sp = o.steps[o.step_ph];
  const double LF = o.opt.lag_fact, Gc = m.gc, l = m.pf_l;
  auto k = [&](int r, int c) -> double& { return K[r + (size_t)c * n]; };
  for (int a = 0; a < nen; ++a) {
    const double W = WL[a];
    const double L = sp.state[IFEM_STATE_CUR][dl[nen + a]];
    const double L2 = o.nlag == 2 ? sp.state[IFEM_STATE_CUR][dl[2 * nen + a]] : 0.0;
    const double lim0 = std::min(1.0 - 1.0e-3, std::max(0.0, PhO[a])), lim1 = 1.0 + 1e-1;
    const int p = a, q = nen + a, q2 = 2 * nen + a;
    double& FPh = out.F[p];
    double& FL = out.F[q];
    switch (o.opt.irreversible) {
      case IFEM_IRR_LAGRANGE:   // LagrMultIrr (:383-399)
        FPh += W * L; k(p, q) += W;
        if (Ph[a] >= 1.0) { FL += W * (Ph[a] - lim1); k(q, p) += W; }
        else if (Ph[a] < PhO[a]) { FL += W * (Ph[a] - lim0); k(q, p) += W; }
        else { FL += W * L; k(q, q) += W; }
        break;
      case IFEM_IRR_AUGLAG: {   // AugLagrIrr (:401-441)
        const double sc = Gc / l / LF, d = LF;
        FL += -W * sc * L * (1.0 + 1.0e-10); k(q, q) += -W * sc * (1.0 + 1.0e-10);
        const double pre = L + LF * (Ph[a] - lim0);
        FPh += W * sc * L * d; k(p, q) += W * sc * d;
        if (pre <= 0) {
          FPh += W * sc * (pre - L) * d; k(p, p) += W * sc * d * d;
          FL += W * sc * pre; k(q, q) += W * sc; k(q, p) += W * sc * d;
        }
      } break;
      case IFEM_IRR_AUGLAG2: {  // AugLagrIrr2 (:444-484)
        const double c = Gc / l / LF, d = LF;
        double& FL2 = out.F[q2];
        FL += -W * c * L * (1.0 - 1.0e-8); k(q, q) += -W * c * (1.0 - 1.0e-8);
        FL2 += -W * c * L2 * (1.0 - 1.0e-8); k(q2, q2) += -W * c * (1.0 - 1.0e-8);
        FPh += W * c * L * d; k(p, q) += W * c * d;
        FPh += W * c * L2 * d; k(p, q2) += W * c * d;
        const double pre = L + LF * (Ph[a] - lim0);
        if (pre <= 0) {
          FPh += W * c * (pre - L) * d; k(p, p) += W * c * d * d;
          FL += W * c * pre; k(q, q) += W * c; k(q, p) += W * c * d;
        }
        const double pre2 = L2 + LF * (Ph[a] - lim1);
        if (pre2 >= 0) {
          FPh += W * c * (pre2 - L2) * d; k(p, p) += W * c * d * d;
          FL2 += W * c * pre2; k(q2, q2) += W * c; k(q2, p) += W * c * d;
        }
      } break;
    }
  }
  out.n = n;
  std::copy(dl, dl + n, out.dofs);
  out.K.swap(K);
}

// OceanBCModel::Assemble_U, one element (OceanBC.cpp:96-150, 2D): the water pressure rho g (hw - y) of each
// node, zero above the water level, on its ux row, weighted by the phase-field lumped integral
// W(n) = sum_q w_q (N_q . Phase) N_q,n.  Residual only.
void elem_ocean_u(Oracle& o, int64_t el, ElemOut& out) {
  const int nen = o.nen, nip = o.nip;
  ShapeIP sh[27];
  shape_grads(o, el, sh);
  const std::vector<int> kinds = u_kinds(o);
  out.n = (int)kinds.size() * nen;
  elem_dofs(o, el, kinds, out.dofs);
  std::fill(out.F, out.F + out.n, 0.0);
  out.K.clear();
  int64_t dp[27];
  elem_dofs(o, el, {IFEM_DOF_PHASE}, dp);
  const StepData& sp = o.steps[o.step_ph];
  double Ph[27], WL[27];
  for (int a = 0; a < nen; ++a) { Ph[a] = sp.state[IFEM_STATE_CUR][dp[a]]; WL[a] = 0.0; }
  for (int ip = 0; ip < nip; ++ip) {
    double phi = 0;
    for (int a = 0; a < nen; ++a) phi += sh[ip].N[a] * Ph[a];
    for (int a = 0; a < nen; ++a) WL[a] += sh[ip].w * phi * sh[ip].N[a];
  }
  const double g = 9.81;   // OceanBC.h:43
  for (int n = 0; n < nen; ++n) {
    const int64_t node = o.E[(size_t)el * nen + n];
    const double hIP = o.opt.ocean_hw - o.X[(size_t)node * o.dim + 1];
    const double pTarget = hIP < 0.0 ? 0.0 : g * o.opt.ocean_density * hIP;
    out.F[n] += WL[n] * pTarget;
  }
}

// PhaseFieldDamage::Assemble_T, one element (PhaseField.cpp:748-767): residual only
void elem_visc_heat(Oracle& o, int64_t el, const ifem_time& tm, ElemOut& out) {
  const int nen = o.nen, nip = o.nip;
  ShapeIP sh[27];
  shape_grads(o, el, sh);
  out.n = nen;
  elem_dofs(o, el, {IFEM_DOF_T}, out.dofs);
  std::fill(out.F, out.F + nen, 0.0);
  out.K.clear();
  for (int ip = 0; ip < nip; ++ip) {
    const size_t hi = (size_t)el * nip + ip;
    const double rate = (o.VD[hi] - o.VDo[hi]) / tm.dt;
    for (int a = 0; a < nen; ++a) out.F[a] += -sh[ip].w * sh[ip].N[a] * rate;
  }
}

// ThermalModel::Assemble, one element (ThermalModel.cpp:94-133)
void elem_thermal(Oracle& o, int64_t el, const ifem_time& tm, ElemOut& out) {
  const int nen = o.nen, nip = o.nip;
  const ifem_material& m = mat_of(o, el);
  ShapeIP sh[27];
  shape_grads(o, el, sh);
  out.n = nen;
  elem_dofs(o, el, {IFEM_DOF_T}, out.dofs);
  const StepData& st = o.steps[o.step_T];
  double T[27], dT[27];
  for (int i = 0; i < nen; ++i) { T[i] = st.state[IFEM_STATE_CUR][out.dofs[i]]; dT[i] = st.state[IFEM_STATE_D][out.dofs[i]]; }
  std::fill(out.F, out.F + nen, 0.0);
  out.K.assign((size_t)nen * nen, 0.0);
  double WL[27] = {0};
  for (int ip = 0; ip < nip; ++ip) {
    const double w = sh[ip].w;
    double gT[3] = {0, 0, 0};
    for (int d = 0; d < o.dim; ++d) for (int a = 0; a < nen; ++a) gT[d] += sh[ip].G[d][a] * T[a];
    for (int a = 0; a < nen; ++a) {
      double s = 0; for (int d = 0; d < o.dim; ++d) s += sh[ip].G[d][a] * gT[d];
      out.F[a] += w * m.k_thermal * s;
    }
    for (int b = 0; b < nen; ++b) for (int a = 0; a < nen; ++a) {
      double s = 0; for (int d = 0; d < o.dim; ++d) s += sh[ip].G[d][a] * sh[ip].G[d][b];
      out.K[a + b * nen] += w * m.k_thermal * s;
    }
    for (int a = 0; a < nen; ++a) WL[a] += w * sh[ip].N[a];
  }
  for (int i = 0; i < nen; ++i) {
    out.F[i] += WL[i] * m.density * m.cp * dT[i];
    out.K[i + i * nen] += WL[i] * m.density * m.cp * tm.du_dt;
  }
}

// CSR position of (row, col): binary search in the row (columns ascending)
inline int64_t csr_pos(const StepData& s, int64_t r, int64_t c) {
  const int32_t* b = s.colidx.data() + s.rowptr[r];
  const int32_t* e = s.colidx.data() + s.rowptr[r + 1];
  const int32_t* p = std::lower_bound(b, e, (int32_t)c);
  if (p == e || *p != c) return -1;
  return p - s.colidx.data();
}

// VecAdd / MatAdd with ADD_VALUES (math.cpp:301-331)
// ----------------------------------------------------------------------------------------
// Boundary element groups: B1_2 lines (B1_2.cpp:55-105) and NURBS3_Plane2 faces (NURBS3_Plane2.cpp,
// getShapeGrads and getNormals), and the TriAxial loads on them (TriAxial.cpp:124-276)
// ----------------------------------------------------------------------------------------
struct FaceIP { double N[9]; double w; double n[3]; };

// shape values, weights and outward normals of face f of group g at the face's Gauss points
int face_shapes(const Oracle& o, const FaceGroup& g, int64_t f, FaceIP* out) {
  std::vector<double> w1, c1;
  ip_scheme_1d(o.ip1d, w1, c1);
  const int q = o.ip1d, dim = o.dim, nfn = dim == 2 ? 3 : 9;
  const int64_t* nodes = &g.F[(size_t)f * nfn];
  const double* C = &g.C[(size_t)f * nfn * nfn];
  double X[9][3] = {}, Wn[9];
  for (int a = 0; a < nfn; ++a) {
    for (int d = 0; d < dim; ++d) X[a][d] = o.X[nodes[a] * dim + d];
    Wn[a] = o.W.empty() ? 1.0 : o.W[nodes[a]];
  }
  int cnt = 0;
  auto outward = [](const double P[3], double n[3]) {   // getNormals: "ensure outwards Normal"
    const double d1 = std::sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
    double Q[3];
    for (int d = 0; d < 3; ++d) Q[d] = P[d] + n[d] * d1 * 1e-3;
    const double d2 = std::sqrt(Q[0] * Q[0] + Q[1] * Q[1] + Q[2] * Q[2]);
    if (d1 > d2) for (int d = 0; d < 3; ++d) n[d] = -n[d];
  };
  if (dim == 2) {
    for (int i = 0; i < q; ++i) {
      double Nb[3], Gb[3];
      bezier_basis(2, c1[i], Nb, Gb);
      FaceIP& s = out[cnt++];
      double GB[3], J[2] = {0, 0}, P[3] = {0, 0, 0};
      for (int a = 0; a < 3; ++a) {
        s.N[a] = 0; GB[a] = 0;
        for (int k = 0; k < 3; ++k) { s.N[a] += Nb[k] * C[a * 3 + k]; GB[a] += Gb[k] * C[a * 3 + k]; }
      }
      for (int a = 0; a < 3; ++a) for (int d = 0; d < 2; ++d) { J[d] += GB[a] * X[a][d]; P[d] += s.N[a] * X[a][d]; }
      const double len = std::sqrt(J[0] * J[0] + J[1] * J[1]);
      const double t0 = J[0] / len, t1 = J[1] / len;
      s.w = w1[i] * std::fabs(t0 * J[0] + t1 * J[1]);
      const double nl = std::sqrt(t1 * t1 + t0 * t0);
      s.n[0] = t1 / nl; s.n[1] = -t0 / nl; s.n[2] = 0;
      outward(P, s.n);
    }
  } else {
    for (int j = 0; j < q; ++j) for (int i = 0; i < q; ++i) {
      double Nx[3], Gx[3], Ny[3], Gy[3];
      bezier_basis(2, c1[i], Nx, Gx);
      bezier_basis(2, c1[j], Ny, Gy);
      double Nb[9], Gb0[9], Gb1[9];
      for (int b = 0; b < 3; ++b) for (int a = 0; a < 3; ++a) {   // KronProd(Nx, Ny): index a + 3 b
        Nb[a + 3 * b] = Nx[a] * Ny[b]; Gb0[a + 3 * b] = Gx[a] * Ny[b]; Gb1[a + 3 * b] = Nx[a] * Gy[b];
      }
      FaceIP& s = out[cnt++];
      double CB[9], GB[9][2], wFun = 0, dW[2] = {0, 0};
      for (int a = 0; a < 9; ++a) {
        CB[a] = GB[a][0] = GB[a][1] = 0;
        for (int k = 0; k < 9; ++k) {
          CB[a] += C[a * 9 + k] * Nb[k]; GB[a][0] += C[a * 9 + k] * Gb0[k]; GB[a][1] += C[a * 9 + k] * Gb1[k];
        }
      }
      for (int a = 0; a < 9; ++a) wFun += CB[a] * Wn[a];
      for (int a = 0; a < 9; ++a) { dW[0] += GB[a][0] * Wn[a]; dW[1] += GB[a][1] * Wn[a]; }
      double J[2][3] = {}, P[3] = {0, 0, 0};
      for (int a = 0; a < 9; ++a) {
        s.N[a] = Wn[a] * CB[a] / wFun;
        for (int d = 0; d < 2; ++d) {
          const double gx = Wn[a] * (GB[a][d] / wFun - CB[a] * dW[d] / wFun / wFun);
          for (int e = 0; e < 3; ++e) J[d][e] += gx * X[a][e];
        }
        for (int e = 0; e < 3; ++e) P[e] += s.N[a] * X[a][e];
      }
      const double nv[3] = {J[0][1] * J[1][2] - J[0][2] * J[1][1], J[0][2] * J[1][0] - J[0][0] * J[1][2],
                            J[0][0] * J[1][1] - J[0][1] * J[1][0]};
      const double nn = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
      s.w = w1[i] * w1[j] * std::fabs(nn);
      for (int d = 0; d < 3; ++d) s.n[d] = nv[d] / nn;
      outward(P, s.n);
    }
  }
  return cnt;
}

void scatter(StepData& s, const ElemOut& eo, bool with_K);

// TriAxialModel::Assemble (TriAxial.cpp:124-276) on the displacement step: the side pressure, then the top
// pressure (t + dt < 0) or displacement penalty (t + dt >= 0), face by face
void triaxial_u(Oracle& o, const ifem_time& tm, StepData& s) {
  TriAxial& T = o.tri;
  const double t = tm.t + tm.dt;
  if (T.st.t_break > 0.0) T.st.p0 = 0.0;
  const int dim = o.dim, nfn = dim == 2 ? 3 : 9, ctop = dim - 1;
  FaceIP ips[9];
  ElemOut eo;
  eo.n = dim * nfn;
  for (int64_t f = 0; f < T.side.nf; ++f) {
    const int nq = face_shapes(o, T.side, f, ips);
    const int64_t* nodes = &T.side.F[(size_t)f * nfn];
    for (int c = 0; c < dim; ++c) for (int a = 0; a < nfn; ++a) {
      eo.dofs[c * nfn + a] = o.dofnum[IFEM_DOF_UX + c][nodes[a]];
      eo.F[c * nfn + a] = 0.0;
    }
    for (int ip = 0; ip < nq; ++ip) {
      double Dam = 1.0;
      if (T.prm.damaged_forces) {
        double phi = 0;
        const std::vector<double>& ph = o.steps[o.step_ph].state[0];
        for (int a = 0; a < nfn; ++a) phi += ips[ip].N[a] * ph[o.dofnum[IFEM_DOF_PHASE][nodes[a]]];
        double u2, u3;
        damage_function(phi, IFEM_DAM_QUADRATIC_NR, 0.0, 2.0, Dam, u2, u3);
      }
      for (int c = 0; c < dim; ++c) for (int a = 0; a < nfn; ++a)
        eo.F[c * nfn + a] += Dam * ips[ip].w * (ips[ip].N[a] * ips[ip].n[c]) * T.st.p0;
    }
    scatter(s, eo, false);
  }
  T.st.uz_sum = 0.0; T.st.f_ext = 0.0; T.st.area = 0.0;
  const std::vector<double>& U = o.steps[o.step_u].state[0];
  for (int64_t f = 0; f < T.top.nf; ++f) {
    const int nq = face_shapes(o, T.top, f, ips);
    const int64_t* nodes = &T.top.F[(size_t)f * nfn];
    double Ut[9];
    for (int c = 0; c < dim; ++c) for (int a = 0; a < nfn; ++a) {
      eo.dofs[c * nfn + a] = o.dofnum[IFEM_DOF_UX + c][nodes[a]];
      eo.F[c * nfn + a] = 0.0;
    }
    for (int a = 0; a < nfn; ++a) Ut[a] = U[eo.dofs[ctop * nfn + a]];
    eo.K.assign((size_t)eo.n * eo.n, 0.0);
    for (int ip = 0; ip < nq; ++ip) {
      const FaceIP& p = ips[ip];
      double ut = 0;
      for (int a = 0; a < nfn; ++a) ut += p.N[a] * Ut[a];
      if (t < 0.0) {
        for (int a = 0; a < nfn; ++a) eo.F[ctop * nfn + a] += p.w * p.N[a] * T.st.p0;
        T.st.f_ext += -p.w * T.st.p0;
      } else {
        const double uTarget = T.st.u0 + t * T.prm.du;
        const double pExt = T.prm.penalty * (ut - uTarget);
        for (int a = 0; a < nfn; ++a) {
          eo.F[ctop * nfn + a] += p.w * p.N[a] * pExt;
          for (int b = 0; b < nfn; ++b)   // K[(col) * n + (row)], as ElemOut stores it
            eo.K[(size_t)(ctop * nfn + b) * eo.n + ctop * nfn + a] += p.w * T.prm.penalty * p.N[a] * p.N[b];
        }
        T.st.f_ext += -p.w * pExt;
      }
      T.st.area += p.w;
      T.st.uz_sum += p.w * ut;
    }
    scatter(s, eo, true);
  }
}

void scatter(StepData& s, const ElemOut& eo, bool with_K) {
  for (int i = 0; i < eo.n; ++i) s.f[eo.dofs[i]] += eo.F[i];
  if (!with_K) return;
  for (int j = 0; j < eo.n; ++j) for (int i = 0; i < eo.n; ++i) {
    const int64_t p = csr_pos(s, eo.dofs[i], eo.dofs[j]);
    s.vals[p] += eo.K[(size_t)j * eo.n + i];
  }
}

void setup(Oracle& o, const ifem_mesh_desc* mesh, const ifem_material* mats, int n_mats, const ifem_options* opts) {
  if (!mesh || !mats || !opts || n_mats < 1) throw Err{IFEM_ERR_INVALID, "null argument"};
  o.dim = mesh->dim; o.etype = mesh->elem_type; o.ip1d = mesh->ipcount1d;
  if (o.etype == IFEM_ELEM_B2_2 && o.dim == 2) o.nen = 9;
  else if (o.etype == IFEM_ELEM_NURBS3_CUBE2 && o.dim == 3) o.nen = 27;
  else throw Err{IFEM_ERR_UNSUPPORTED, "element type / dim"};
  o.nn = mesh->n_nodes; o.nel = mesh->n_elems;
  o.X.assign(mesh->coords, mesh->coords + o.nn * o.dim);
  if (mesh->node_weights && o.dim == 3) o.W.assign(mesh->node_weights, mesh->node_weights + o.nn);
  o.E.assign(mesh->elems, mesh->elems + o.nel * o.nen);
  for (int64_t v : o.E) if (v < 0 || v >= o.nn) throw Err{IFEM_ERR_INVALID, "element node out of range"};
  const size_t csz = (size_t)o.nen * o.nen;
  o.C.resize((size_t)o.nel * csz);
  if (mesh->elem_data) {
    std::memcpy(o.C.data(), mesh->elem_data, sizeof(double) * o.C.size());
  } else if (mesh->elem_kron) {
    // C = kron(Cz, kron(Cy, Cx)) (bezierExtraction3D.m / bezierExtraction2D.m)
    for (int64_t e = 0; e < o.nel; ++e) {
      const double* k = mesh->elem_kron + (size_t)e * o.dim * 9;
      double* Ce = &o.C[(size_t)e * csz];
      if (o.dim == 2) {
        for (int iy = 0; iy < 3; ++iy) for (int ix = 0; ix < 3; ++ix)
          for (int jy = 0; jy < 3; ++jy) for (int jx = 0; jx < 3; ++jx)
            Ce[(ix + 3 * iy) * 9 + jx + 3 * jy] = k[9 + iy * 3 + jy] * k[ix * 3 + jx];
      } else {
        for (int iz = 0; iz < 3; ++iz) for (int iy = 0; iy < 3; ++iy) for (int ix = 0; ix < 3; ++ix)
          for (int jz = 0; jz < 3; ++jz) for (int jy = 0; jy < 3; ++jy) for (int jx = 0; jx < 3; ++jx)
            Ce[(ix + 3 * iy + 9 * iz) * 27 + jx + 3 * jy + 9 * jz] = k[18 + iz * 3 + jz] * (k[9 + iy * 3 + jy] * k[ix * 3 + jx]);
      }
    }
  } else throw Err{IFEM_ERR_INVALID, "mesh needs elem_data or elem_kron"};
  if (mesh->elem_mat) {
    o.emat.assign(mesh->elem_mat, mesh->elem_mat + o.nel);
    for (int32_t v : o.emat) if (v < 0 || v >= n_mats) throw Err{IFEM_ERR_INVALID, "elem_mat out of range"};
  }
  o.mats.assign(mats, mats + n_mats);
  o.opt = *opts;
  if (o.opt.distribution == IFEM_DIST_CUSTOM && !(o.opt.dist_coefs[0] != 0.0))
    throw Err{IFEM_ERR_INVALID, "the Custom distribution needs Coefs[0] != 0"};
  if (o.opt.rm_max_it <= 0) o.opt.rm_max_it = 250;
  build_shapes(o);
  // DOF steps
  int maxstep = -1;
  bool has[IFEM_N_DOF_KINDS] = {};
  int kstep[IFEM_N_DOF_KINDS];
  std::fill(kstep, kstep + IFEM_N_DOF_KINDS, -1);
  if (o.opt.n_dofs < 1 || o.opt.n_dofs > IFEM_N_DOF_KINDS) throw Err{IFEM_ERR_INVALID, "n_dofs"};
  for (int i = 0; i < o.opt.n_dofs; ++i) {
    const int k = o.opt.dof_kind[i];
    if (k < 0 || k >= IFEM_N_DOF_KINDS || has[k]) throw Err{IFEM_ERR_INVALID, "dof kinds"};
    has[k] = true; kstep[k] = o.opt.dof_step[i];
    maxstep = std::max(maxstep, o.opt.dof_step[i]);
  }
  if (!has[IFEM_DOF_UX] || !has[IFEM_DOF_UY] || (o.dim == 3 && !has[IFEM_DOF_UZ]) || !has[IFEM_DOF_PHASE])
    throw Err{IFEM_ERR_INVALID, "Dof of type ux/uy(/uz)/phase is not defined"};
  if (kstep[IFEM_DOF_UX] != kstep[IFEM_DOF_UY] || (o.dim == 3 && kstep[IFEM_DOF_UZ] != kstep[IFEM_DOF_UX]))
    throw Err{IFEM_ERR_INVALID, "displacements must share a solver step"};
  o.step_u = kstep[IFEM_DOF_UX]; o.step_ph = kstep[IFEM_DOF_PHASE];
  // micro-rotations: oz in 2D, ox oy oz in 3D, in the displacement step (CossPhaseField.cpp:170-219)
  if (o.opt.cosserat) {
    const bool ok = has[IFEM_DOF_OZ] && kstep[IFEM_DOF_OZ] == o.step_u &&
                    (o.dim == 3 ? (has[IFEM_DOF_OX] && has[IFEM_DOF_OY] && kstep[IFEM_DOF_OX] == o.step_u &&
                                   kstep[IFEM_DOF_OY] == o.step_u)
                                : (!has[IFEM_DOF_OX] && !has[IFEM_DOF_OY]));
    if (!ok) throw Err{IFEM_ERR_INVALID, "the Cosserat model needs oz (2D) or ox, oy, oz (3D) in the displacement step"};
    o.ncs = 18;
  } else if (has[IFEM_DOF_OX] || has[IFEM_DOF_OY] || has[IFEM_DOF_OZ]) {
    throw Err{IFEM_ERR_INVALID, "micro-rotation dofs need the Cosserat model"};
  }
  // Lagrange-multiplier irreversibility: its multipliers are DOFs of the phase step (PhaseField.cpp:95-101,
  // 270-280); other methods have none
  o.nlag = o.opt.irreversible == IFEM_IRR_AUGLAG2 ? 2
         : (o.opt.irreversible == IFEM_IRR_LAGRANGE || o.opt.irreversible == IFEM_IRR_AUGLAG) ? 1 : 0;
  if (o.opt.irreversible < IFEM_IRR_NONE || o.opt.irreversible > IFEM_IRR_AUGLAG2)
    throw Err{IFEM_ERR_UNSUPPORTED, "irreversibility method"};
  if (has[IFEM_DOF_LMULT] != (o.nlag >= 1) || has[IFEM_DOF_LMULT2] != (o.nlag == 2))
    throw Err{IFEM_ERR_INVALID, "lMult_pf / lMult_pf2 DOFs must match the irreversibility method"};
  if ((o.nlag >= 1 && kstep[IFEM_DOF_LMULT] != o.step_ph) || (o.nlag == 2 && kstep[IFEM_DOF_LMULT2] != o.step_ph))
    throw Err{IFEM_ERR_INVALID, "the Lagrange multipliers must be in the phase-field solver step"};
  o.hasT = has[IFEM_DOF_T];
  o.step_T = o.hasT ? kstep[IFEM_DOF_T] : -1;
  if (o.opt.ocean_bc && o.dim != 2) throw Err{IFEM_ERR_UNSUPPORTED, "OceanBC is a 2D model"};
  if (o.step_u == o.step_ph || (o.hasT && (o.step_T == o.step_u || o.step_T == o.step_ph)))
    throw Err{IFEM_ERR_UNSUPPORTED, "u, phase and T must be solved in distinct staggered steps"};
  o.nsteps = maxstep + 1;
  // DofSpace::AddDofs on the unique nodes of the group + SyncDofs numbering (DofSpace.cpp:486-513)
  std::vector<int64_t> uniq(o.E);
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  for (int k = 0; k < IFEM_N_DOF_KINDS; ++k) o.dofnum[k].assign(o.nn, -1);
  o.steps.assign(o.nsteps, StepData{});
  for (int s = 0; s < o.nsteps; ++s) {
    int64_t counter = 0;
    for (int i = 0; i < o.opt.n_dofs; ++i) {
      if (o.opt.dof_step[i] != s) continue;
      const int k = o.opt.dof_kind[i];
      if (k == IFEM_DOF_UZ && o.dim != 3) continue;
      for (int64_t nd : uniq) o.dofnum[k][nd] = counter++;
    }
    o.steps[s].ndofs = counter;
    for (int q = 0; q < 4; ++q) o.steps[s].state[q].assign(counter, 0.0);
    o.steps[s].f.assign(counter, 0.0);
  }
  // AIJ pattern: union of the element DOF pairs each step inserts (math.cpp:301-304)
  for (int s = 0; s < o.nsteps; ++s) {
    std::vector<int> kinds;
    if (s == o.step_u) kinds = u_kinds(o);
    else if (s == o.step_ph) kinds = phase_kinds(o);
    else if (o.hasT && s == o.step_T && o.opt.thermal_model) kinds = {IFEM_DOF_T};
    StepData& sd = o.steps[s];
    std::vector<std::vector<int32_t>> rows(sd.ndofs);
    if (!kinds.empty()) {
      std::vector<int64_t> d(kinds.size() * o.nen);
      for (int64_t e = 0; e < o.nel; ++e) {
        elem_dofs(o, e, kinds, d.data());
        for (int64_t r : d) for (int64_t c : d) rows[r].push_back((int32_t)c);
      }
    }
    sd.rowptr.assign(sd.ndofs + 1, 0);
    for (int64_t r = 0; r < sd.ndofs; ++r) {
      auto& v = rows[r];
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      sd.rowptr[r + 1] = sd.rowptr[r] + (int32_t)v.size();
    }
    sd.colidx.resize(sd.rowptr[sd.ndofs]);
    for (int64_t r = 0; r < sd.ndofs; ++r) std::copy(rows[r].begin(), rows[r].end(), sd.colidx.begin() + sd.rowptr[r]);
    sd.vals.assign(sd.colidx.size(), 0.0);
  }
  const size_t nh = (size_t)o.nel * o.nip;
  o.EH.assign(nh, 0); o.EHo.assign(nh, 0); o.EP.assign(nh * o.ncs, 0); o.EPo.assign(nh * o.ncs, 0);
  o.VD.assign(nh, 0); o.VDo.assign(nh, 0); o.DVD.assign(nh, 0); o.DVDo.assign(nh, 0);
  o.hist_size = 0;
  for (const auto& m : o.mats) {
    if (m.split < IFEM_SPLIT_NONE || m.split > IFEM_SPLIT_STARCONVEX) throw Err{IFEM_ERR_UNSUPPORTED, "energy split not supported"};
    if (m.split == IFEM_SPLIT_SPECSTRESS && m.consistent_energy && !o.opt.cosserat)   // PhaseFieldMaterial.cpp:148-150
      throw Err{IFEM_ERR_UNSUPPORTED, "Spectral Stress split not implemented when using a consistent split"};
    if (o.opt.cosserat) {   // CosseratMaterial.cpp:107-154, 450-514
      if (m.rheology != IFEM_RHEO_LE && m.rheology != IFEM_RHEO_VEP && m.rheology != IFEM_RHEO_DVEP)
        throw Err{IFEM_ERR_UNSUPPORTED, "Rheology type not defined in CosseratMaterial.cpp"};
      if (m.split != IFEM_SPLIT_NONE && m.split != IFEM_SPLIT_SPECSTRESS && m.split != IFEM_SPLIT_DRUCKERPRAGER &&
          m.split != IFEM_SPLIT_STARCONVEX)
        throw Err{IFEM_ERR_UNSUPPORTED, "Stress split function type not defined for a Cosserat Material"};
      if (m.rheology != IFEM_RHEO_LE) {
        if (!(m.hard_e_ref != 0.0)) throw Err{IFEM_ERR_INVALID, "the Cosserat return map needs hard_eRef != 0"};
        o.hist_size = 4;
      }
      continue;
    }
    if (m.rheology == IFEM_RHEO_DVEP)   // UpdatePlasticStrains has no case for it (SolidMaterial.cpp:185-188)
      throw Err{IFEM_ERR_UNSUPPORTED, "Rheology type not defined: DamViscoElasticPlastic has no return map"};
    if (m.rheology != IFEM_RHEO_LE && o.hist_size == 0) o.hist_size = 1;
    if (m.rheology == IFEM_RHEO_VEP) o.hist_size = 4;   // SolidMaterial.cpp:50-51
  }
  o.MH.assign(nh * (o.hist_size == 4 ? 4 : 1), 0); o.MHo.assign(nh * (o.hist_size == 4 ? 4 : 1), 0);
}

// Physics::Assemble(step) restricted to this model (+ thermal) (physics.cpp:255-304)
void assemble(Oracle& o, int step, const ifem_time& tm, bool write_hist) {
  if (step < 0 || step >= o.nsteps) throw Err{IFEM_ERR_INVALID, "step"};
  StepData& s = o.steps[step];
  std::fill(s.f.begin(), s.f.end(), 0.0);
  std::fill(s.vals.begin(), s.vals.end(), 0.0);
  s.stats = ifem_stats{};
  ElemOut eo;
  RMOut ro;
  auto t0 = std::chrono::steady_clock::now();
  if (step == o.step_u) {
    for (int64_t e = 0; e < o.nel; ++e) { elem_U(o, e, tm, eo, ro, write_hist); scatter(s, eo, true); }
    if (o.opt.ocean_bc) for (int64_t e = 0; e < o.nel; ++e) { elem_ocean_u(o, e, eo); scatter(s, eo, false); }
    if (o.tri.on) triaxial_u(o, tm, s);
  }
  if (step == o.step_ph) {
    double lc = 0;
    for (int64_t e = 0; e < o.nel; ++e) { elem_phase(o, e, tm, eo, write_hist); lc += eo.lcrack; scatter(s, eo, true); }
    s.stats.crack_length = lc;
  }
  if (o.hasT && step == o.step_T) {
    if (o.opt.viscous_heating) for (int64_t e = 0; e < o.nel; ++e) { elem_visc_heat(o, e, tm, eo); scatter(s, eo, false); }
    if (o.opt.thermal_model) for (int64_t e = 0; e < o.nel; ++e) { elem_thermal(o, e, tm, eo); scatter(s, eo, true); }
  }
  s.stats.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  s.stats.rm_iterations = ro.iters;
  s.stats.rm_capped = ro.capped;
}

std::vector<double>* hist_ptr(Oracle& o, int field, int old) {
  switch (field) {
    case IFEM_HIST_ENERGY: return old ? &o.EHo : &o.EH;
    case IFEM_HIST_PLASTIC_STRAIN: return old ? &o.EPo : &o.EP;
    case IFEM_HIST_VISC_DISS: return old ? &o.VDo : &o.VD;
    case IFEM_HIST_DAM_VISC_DISS: return old ? &o.DVDo : &o.DVD;
    case IFEM_HIST_MAT: return old ? &o.MHo : &o.MH;
  }
  return nullptr;
}

template <class F>
int guarded(Oracle* o, F&& fn) {
  try { fn(); return IFEM_OK; }
  catch (const Err& e) { if (o) o->err = e.msg; else g_create_err = e.msg; return e.code; }
  catch (const std::exception& e) { if (o) o->err = e.what(); else g_create_err = e.what(); return IFEM_ERR_INVALID; }
}

}  // namespace

struct ifem_ctx;  // opaque in the header; the oracle casts its own type

extern "C" {

int oracle_abi_version(void) { return IFEM_ABI_VERSION; }

int oracle_ctx_create(const ifem_mesh_desc* mesh, const ifem_material* mats, int32_t n_mats,
                      const ifem_options* opts, int32_t /*device*/, ifem_ctx** out) {
  if (!out) return IFEM_ERR_INVALID;
  Oracle* o = new Oracle();
  const int rc = guarded(nullptr, [&] { setup(*o, mesh, mats, n_mats, opts); });
  if (rc != IFEM_OK) { delete o; *out = nullptr; return rc; }
  *out = reinterpret_cast<ifem_ctx*>(o);
  return IFEM_OK;
}

int oracle_ctx_destroy(ifem_ctx* ctx) { delete reinterpret_cast<Oracle*>(ctx); return IFEM_OK; }

int oracle_last_error(const ifem_ctx* ctx, char* buf, size_t len) {
  const std::string& m = ctx ? reinterpret_cast<const Oracle*>(ctx)->err : g_create_err;
  if (buf && len) { std::strncpy(buf, m.c_str(), len - 1); buf[len - 1] = 0; }
  return IFEM_OK;
}

int oracle_step_info(const ifem_ctx* ctx, int32_t step, int64_t* n_dofs, int64_t* nnz) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  if (n_dofs) *n_dofs = o->steps[step].ndofs;
  if (nnz) *nnz = (int64_t)o->steps[step].colidx.size();
  return IFEM_OK;
}

int oracle_get_dof_numbers(const ifem_ctx* ctx, int32_t kind, int64_t* out) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || kind < 0 || kind >= IFEM_N_DOF_KINDS || !out) return IFEM_ERR_INVALID;
  std::copy(o->dofnum[kind].begin(), o->dofnum[kind].end(), out);
  return IFEM_OK;
}

int oracle_build_pattern(const ifem_ctx* ctx, int32_t step, int32_t* row_ptr, int32_t* col_idx) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  const StepData& s = o->steps[step];
  if (row_ptr) std::copy(s.rowptr.begin(), s.rowptr.end(), row_ptr);
  if (col_idx) std::copy(s.colidx.begin(), s.colidx.end(), col_idx);
  return IFEM_OK;
}

int oracle_set_state(ifem_ctx* ctx, int32_t step, int32_t kind, const double* src, int64_t n) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps || kind < 0 || kind > 3 || n != o->steps[step].ndofs) return IFEM_ERR_INVALID;
  std::copy(src, src + n, o->steps[step].state[kind].begin());
  return IFEM_OK;
}

int oracle_get_state(const ifem_ctx* ctx, int32_t step, int32_t kind, double* dst, int64_t n) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps || kind < 0 || kind > 3 || n != o->steps[step].ndofs) return IFEM_ERR_INVALID;
  std::copy(o->steps[step].state[kind].begin(), o->steps[step].state[kind].end(), dst);
  return IFEM_OK;
}

int oracle_assemble(ifem_ctx* ctx, int32_t step, const ifem_time* tm) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !tm) return IFEM_ERR_INVALID;
  return guarded(o, [&] { assemble(*o, step, *tm, true); });
}

int oracle_assemble_async(ifem_ctx* ctx, int32_t step, const ifem_time* tm) { return oracle_assemble(ctx, step, tm); }
int oracle_sync(ifem_ctx* ctx, int32_t step) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  return (!o || step < 0 || step >= o->nsteps) ? IFEM_ERR_INVALID : IFEM_OK;
}
int oracle_get_stream(const ifem_ctx* ctx, void** stream) {
  if (!ctx || !stream) return IFEM_ERR_INVALID;
  *stream = nullptr;
  return IFEM_OK;
}

// Residual-only evaluation that leaves history untouched (finite-difference checks).
int oracle_assemble_nohist(ifem_ctx* ctx, int32_t step, const ifem_time* tm) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !tm) return IFEM_ERR_INVALID;
  return guarded(o, [&] { assemble(*o, step, *tm, false); });
}

int oracle_get_residual(const ifem_ctx* ctx, int32_t step, double* dst, int64_t n) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps || n != o->steps[step].ndofs) return IFEM_ERR_INVALID;
  std::copy(o->steps[step].f.begin(), o->steps[step].f.end(), dst);
  return IFEM_OK;
}

int oracle_get_matrix(const ifem_ctx* ctx, int32_t step, void* dst, int64_t nnz, int32_t dtype) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps || nnz != (int64_t)o->steps[step].vals.size()) return IFEM_ERR_INVALID;
  const auto& v = o->steps[step].vals;
  if (dtype == IFEM_F64) std::copy(v.begin(), v.end(), (double*)dst);
  else if (dtype == IFEM_F32) for (size_t i = 0; i < v.size(); ++i) ((float*)dst)[i] = (float)v[i];
  else return IFEM_ERR_INVALID;
  return IFEM_OK;
}

int oracle_commit(ifem_ctx* ctx, int32_t type) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o) return IFEM_ERR_INVALID;
  if (type == IFEM_COMMIT_TIMEDEP) {  // PhaseField.cpp:123-145
    o->EHo = o->EH; o->EPo = o->EP; o->VDo = o->VD; o->DVDo = o->DVD;
    if (o->hist_size > 0) o->MHo = o->MH;
  }
  return IFEM_OK;
}

int oracle_reset_step(ifem_ctx* ctx) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o) return IFEM_ERR_INVALID;
  o->EH = o->EHo; o->EP = o->EPo; o->VD = o->VDo; o->DVD = o->DVDo;
  if (o->hist_size > 0) o->MH = o->MHo;
  return IFEM_OK;
}

int oracle_get_history(const ifem_ctx* ctx, int32_t field, int32_t old, double* dst, int64_t n) {
  Oracle* o = const_cast<Oracle*>(reinterpret_cast<const Oracle*>(ctx));
  std::vector<double>* v = o ? hist_ptr(*o, field, old) : nullptr;
  if (!v || n != (int64_t)v->size()) return IFEM_ERR_INVALID;
  std::copy(v->begin(), v->end(), dst);
  return IFEM_OK;
}

int oracle_set_history(ifem_ctx* ctx, int32_t field, int32_t old, const double* src, int64_t n) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  std::vector<double>* v = o ? hist_ptr(*o, field, old) : nullptr;
  if (!v || n != (int64_t)v->size()) return IFEM_ERR_INVALID;
  std::copy(src, src + n, v->begin());
  return IFEM_OK;
}

int oracle_set_tangent(ifem_ctx* ctx, int32_t mode, int32_t prec) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o) return IFEM_ERR_INVALID;
  o->opt.tangent_mode = mode; o->opt.tangent_precision = prec;
  return IFEM_OK;
}

// The oracle assembles serially into host memory: there is no read-back to overlap, so the slab count only
// gets the same argument checks as the product library's.
int oracle_set_readback_slabs(ifem_ctx* ctx, int32_t n_slabs) {
  if (!ctx || n_slabs < 1 || n_slabs > 16) return IFEM_ERR_INVALID;
  return IFEM_OK;
}

int oracle_set_options(ifem_ctx* ctx, const ifem_options* opts) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !opts) return IFEM_ERR_INVALID;
  o->opt = *opts;
  if (o->opt.rm_max_it <= 0) o->opt.rm_max_it = 250;
  return IFEM_OK;
}

int oracle_get_stats(const ifem_ctx* ctx, int32_t step, ifem_stats* out) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps || !out) return IFEM_ERR_INVALID;
  *out = o->steps[step].stats;
  return IFEM_OK;
}

int oracle_set_param(ifem_ctx* ctx, int32_t mat, int32_t theta, double value) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || mat < 0 || mat >= (int)o->mats.size()) return IFEM_ERR_INVALID;
  ifem_material& m = o->mats[mat];
  switch (theta) {
    case 0: m.gc = value; break;
    case 1: m.pf_l = value; break;
    case 2: m.creep_a = value; break;
    case 3: m.creep_n = value; break;
    default: return IFEM_ERR_INVALID;
  }
  return IFEM_OK;
}

// Per-element integration-point shape data (tests: partition of unity, volume, gradients).
int oracle_shape(const ifem_ctx* ctx, int64_t el, double* N, double* G, double* w) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || el < 0 || el >= o->nel) return IFEM_ERR_INVALID;
  ShapeIP sh[27];
  shape_grads(*o, el, sh);
  for (int ip = 0; ip < o->nip; ++ip) {
    if (w) w[ip] = sh[ip].w;
    for (int a = 0; a < o->nen; ++a) {
      if (N) N[ip * o->nen + a] = sh[ip].N[a];
      if (G) for (int d = 0; d < o->dim; ++d) G[(ip * o->dim + d) * o->nen + a] = sh[ip].G[d][a];
    }
  }
  return IFEM_OK;
}

// Per-element shape data with second gradients, getShapeGrads2 (tests: a quadratic field's Hessian is exact).
// G2 is [nip][3 or 6][nen].
int oracle_shape2(const ifem_ctx* ctx, int64_t el, double* N, double* G, double* G2, double* w) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || el < 0 || el >= o->nel) return IFEM_ERR_INVALID;
  try {
    std::vector<ShapeIP2> sh(o->nip);
    shape_grads2(*o, el, sh.data());
    const int ng = o->dim == 2 ? 3 : 6;
    for (int ip = 0; ip < o->nip; ++ip) {
      if (w) w[ip] = sh[ip].s.w;
      for (int a = 0; a < o->nen; ++a) {
        if (N) N[ip * o->nen + a] = sh[ip].s.N[a];
        if (G) for (int d = 0; d < o->dim; ++d) G[(ip * o->dim + d) * o->nen + a] = sh[ip].s.G[d][a];
        if (G2) for (int r = 0; r < ng; ++r) G2[(ip * ng + r) * o->nen + a] = sh[ip].G2[r][a];
      }
    }
    return IFEM_OK;
  } catch (const Err& e) { return e.code; }
}

// The oracle checks assembly, not linear solves: the library's device solve is checked against a direct
// sparse solve of the same constrained system.
int oracle_solve_constrained(ifem_ctx*, int32_t, double, int32_t, int32_t, double*, int32_t*, double*) {
  return IFEM_ERR_UNSUPPORTED;
}
int oracle_set_preconditioner(ifem_ctx*, int32_t, int32_t) { return IFEM_ERR_UNSUPPORTED; }
int oracle_set_multigrid(ifem_ctx*, int32_t, double, int32_t) { return IFEM_ERR_UNSUPPORTED; }
int oracle_multigrid_plan(int64_t, const int64_t*, const int32_t*, const double*, const int32_t*, int64_t, int32_t,
                          const double*, double, int32_t, int32_t*, int64_t*, int64_t*) {
  return IFEM_ERR_UNSUPPORTED;
}
int oracle_preconditioner_info(const ifem_ctx*, int32_t, int32_t*, int64_t*, double*) { return IFEM_ERR_UNSUPPORTED; }

// Single material-point return map (tests: closed-form checks).  Returns dissipation rate.
int oracle_return_map(const ifem_material* m, double T, const double* eps, const double* epl_old,
                      double* epl_inout, double* hist0_inout, double damage, double dt, int32_t tol_mode,
                      int32_t tangent_mode, double* DMat, int64_t* iters, double* diss) {
  try {
    MatPt M{};
    set_temperature(*m, T, M);
    RMOut ro;
    double h = *hist0_inout;
    const double d = return_mapping_viscous(M, DMat, epl_inout, eps, epl_old, damage, dt, h, tol_mode, 250, tangent_mode, ro);
    *hist0_inout = h;
    if (iters) *iters = ro.iters;
    if (diss) *diss = d;
    return IFEM_OK;
  } catch (const Err& e) { return e.code; }
}

// Single material-point VEP return map (tests).  hist_inout [4]: the ip's current MatHist; h_old = MatHistOld[0].
// Also returns the local residual f (8) and Jacobian K (8x8) re-evaluated at the converged unknowns.
int oracle_return_map_vep(const ifem_material* m, double T, const double* eps, const double* epl_old,
                          double* epl_inout, double* hist_inout, double h_old, double dt, int32_t tol_mode,
                          double* DMat, int64_t* iters, double* diss, double* damdiss, double* f_out, double* K_out) {
  try {
    MatPt M{};
    set_temperature(*m, T, M);
    RMOut ro;
    double dd = 0;
    const double d = return_mapping_vep(M, DMat, epl_inout, eps, epl_old, dt, 1.0, hist_inout, h_old, tol_mode, 250,
                                        dd, ro);
    if (f_out || K_out) {
      double x[8], f[8], K[64];
      for (int i = 0; i < 6; ++i) x[i] = eps[i] - epl_inout[i];
      x[6] = hist_inout[1]; x[7] = hist_inout[2];
      vep_getKF(M, K, f, x, eps, epl_old, dt, 1.0, h_old);
      if (f_out) std::memcpy(f_out, f, sizeof(f));
      if (K_out) std::memcpy(K_out, K, sizeof(K));
    }
    if (iters) *iters = ro.iters;
    if (diss) *diss = d;
    if (damdiss) *damdiss = dd;
    return IFEM_OK;
  } catch (const Err& e) { return e.code; }
}

int oracle_energy_split(const ifem_material* m, double T, const double* e, double* Dd, double* Du, double* Sd,
                        double* Su, double* energy) {
  try {
    MatPt M{};
    set_temperature(*m, T, M);
    *energy = energy_split(M, Dd, Du, Sd, Su, e);
    return IFEM_OK;
  } catch (const Err& er) { return er.code; }
}

// Multi-threaded CPU baseline of one assembly over elements [0, n_sample): contiguous element
// ranges per thread (one per MPI rank in the reference), private element buffers, then an
// ordered merge into the step's CSR and residual.  Writes history like the serial path.
// Returns wall time in ms through ms_out.
int oracle_assemble_mt(ifem_ctx* ctx, int32_t step, const ifem_time* tm, int32_t nthreads, int64_t n_sample,
                       double* ms_out) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !tm || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  if (n_sample <= 0 || n_sample > o->nel) n_sample = o->nel;
  if (nthreads < 1) nthreads = 1;
  return guarded(o, [&] {
    StepData& s = o->steps[step];
    auto t0 = std::chrono::steady_clock::now();
    std::fill(s.f.begin(), s.f.end(), 0.0);
    std::fill(s.vals.begin(), s.vals.end(), 0.0);
    s.stats = ifem_stats{};
    const int kinds = (step == o->step_u) ? 0 : (step == o->step_ph ? 1 : 2);
    // the T step: viscous heating is residual-only and cheap; it comes first, as in the serial path
    if (kinds == 2 && o->hasT && o->opt.viscous_heating) {
      ElemOut eo;
      for (int64_t e = 0; e < n_sample; ++e) { elem_visc_heat(*o, e, *tm, eo); scatter(s, eo, false); }
    }
    const bool threaded = kinds != 2 || (o->hasT && o->opt.thermal_model);
    std::vector<std::vector<ElemOut>> outs(nthreads);
    std::vector<RMOut> ros(nthreads);
    std::vector<std::thread> th;
    std::atomic<int> failed{0};
    for (int t = 0; t < nthreads && threaded; ++t) {
      const int64_t b = n_sample * t / nthreads, e = n_sample * (t + 1) / nthreads;
      outs[t].resize(e - b);
      th.emplace_back([&, t, b, e] {
        try {
          for (int64_t el = b; el < e; ++el) {
            ElemOut& eo = outs[t][el - b];
            if (kinds == 0) elem_U(*o, el, *tm, eo, ros[t], true);
            else if (kinds == 1) elem_phase(*o, el, *tm, eo, true);
            else elem_thermal(*o, el, *tm, eo);
          }
        } catch (...) { failed = 1; }
      });
    }
    for (auto& x : th) x.join();
    if (failed) throw Err{IFEM_ERR_NUMERIC, "thread failed"};
    double lc = 0;   // crack length in element order, as the serial path sums it
    for (int t = 0; t < nthreads; ++t) {
      for (auto& eo : outs[t]) {
        lc += eo.lcrack;
        scatter(s, eo, true);
      }
      s.stats.rm_iterations += ros[t].iters;
      s.stats.rm_capped += ros[t].capped;
    }
    if (kinds == 1) s.stats.crack_length = lc;
    if (kinds == 0 && o->opt.ocean_bc) {     // OceanBC after the phase-field model, as the serial path
      ElemOut eo;
      for (int64_t e = 0; e < n_sample; ++e) { elem_ocean_u(*o, e, eo); scatter(s, eo, false); }
    }
    if (kinds == 0 && o->tri.on) triaxial_u(*o, *tm, s);
    if (ms_out) *ms_out = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  });
}


// Host pointers of the residual / CSR values (the oracle has no device memory).
int oracle_device_outputs(const ifem_ctx* ctx, int32_t step, const double** f_dev, const void** vals_dev,
                          int32_t* dtype_out) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  if (f_dev) *f_dev = o->steps[step].f.data();
  if (vals_dev) *vals_dev = o->steps[step].vals.data();
  if (dtype_out) *dtype_out = IFEM_F64;
  return IFEM_OK;
}

// dR/dtheta by central finite differences of the residual (relative step 1e-6), evaluated at the
// stored state and start-of-assembly history, which are restored afterwards.  This is the
// finite-difference reference of the analytic adjoint kernel.  lam_dr has 4*n_mats entries
// (derivative w.r.t. each material set's parameters); dr_dtheta is the derivative w.r.t. a
// parameter shared by all sets.
int oracle_adjoint(ifem_ctx* ctx, int32_t step, const ifem_time* tm, const double* lambda, double* dr_dtheta,
                   double* lam_dr) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !tm || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  return guarded(o, [&] {
    StepData& s = o->steps[step];
    const int64_t n = s.ndofs;
    const int nm = (int)o->mats.size();
    auto param = [](ifem_material& m, int k) -> double& {
      return k == 0 ? m.gc : (k == 1 ? m.pf_l : (k == 2 ? m.creep_a : m.creep_n));
    };
    std::vector<double> fp(n), fm(n), all(4 * (size_t)n, 0.0);
    for (int k = 0; k < 4; ++k) {
      for (int mi = -1; mi < nm; ++mi) {   // -1: all sets together (dr_dtheta)
        if (mi == -1 && !dr_dtheta) continue;
        if (mi >= 0 && !lam_dr) continue;
        const std::vector<ifem_material> saved = o->mats;
        double h = 0;
        for (int j = 0; j < nm; ++j) if (mi < 0 || j == mi) h = std::max(h, 1e-6 * std::fabs(param(o->mats[j], k)));
        if (h == 0) h = 1e-6;
        for (int sign = 0; sign < 2; ++sign) {
          o->mats = saved;
          for (int j = 0; j < nm; ++j) if (mi < 0 || j == mi) param(o->mats[j], k) += (sign == 0 ? h : -h);
          assemble(*o, step, *tm, false);
          (sign == 0 ? fp : fm) = s.f;
        }
        o->mats = saved;
        if (mi < 0) for (int64_t i = 0; i < n; ++i) all[k * n + i] = (fp[i] - fm[i]) / (2 * h);
        else {
          double acc = 0;
          for (int64_t i = 0; i < n; ++i) acc += (lambda ? lambda[i] : 1.0) * (fp[i] - fm[i]) / (2 * h);
          lam_dr[mi * 4 + k] = acc;
        }
      }
    }
    if (dr_dtheta) std::copy(all.begin(), all.end(), dr_dtheta);
    assemble(*o, step, *tm, false);
    o->adj_full.resize(o->nsteps);
    o->adj_sets.resize(o->nsteps);
    if (dr_dtheta) o->adj_full[step] = all;
    if (lam_dr) o->adj_sets[step].assign(lam_dr, lam_dr + 4 * (size_t)nm);
  });
}

// The oracle evaluates every derivative by central finite differences in FP64: the adjoint's arithmetic choice
// has nothing to act on here.
int oracle_set_adjoint_precision(ifem_ctx* ctx, int32_t dtype) {
  if (!ctx || (dtype != IFEM_F64 && dtype != IFEM_F32)) return IFEM_ERR_INVALID;
  return IFEM_OK;
}

// dR_step/dT . dT by central finite differences of the residual, at the stored state and start-of-assembly
// history (restored afterwards): the temperature state moves by +-h dT (h = 1e-3 K over max |dT|), or the pinned
// temperature by +-1e-3 K when the context has no T DOF.  The reference of the analytic temperature sensitivity.
int oracle_temperature_sensitivity(ifem_ctx* ctx, int32_t step, const ifem_time* tm, const double* dT, double* dr_out) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !tm || step < 0 || step >= o->nsteps || !dr_out) return IFEM_ERR_INVALID;
  if (o->hasT != (dT != nullptr)) return IFEM_ERR_INVALID;
  if (o->hasT && step == o->step_T) return IFEM_ERR_INVALID;
  return guarded(o, [&] {
    StepData& s = o->steps[step];
    const int64_t n = s.ndofs;
    std::vector<double> fp(n), fm(n);
    if (o->hasT) {
      std::vector<double>& T = o->steps[o->step_T].state[IFEM_STATE_CUR];
      const std::vector<double> T0 = T;
      double dmax = 0;
      for (size_t i = 0; i < T.size(); ++i) dmax = std::max(dmax, std::fabs(dT[i]));
      const double h = dmax > 0 ? 1e-3 / dmax : 1e-3;
      for (int sign = 0; sign < 2; ++sign) {
        for (size_t i = 0; i < T.size(); ++i) T[i] = T0[i] + (sign == 0 ? h : -h) * dT[i];
        assemble(*o, step, *tm, false);
        (sign == 0 ? fp : fm) = s.f;
      }
      T = T0;
      for (int64_t i = 0; i < n; ++i) dr_out[i] = (fp[i] - fm[i]) / (2 * h);
    } else {
      const double T0 = o->opt.pinned_temperature, h = 1e-3;
      for (int sign = 0; sign < 2; ++sign) {
        o->opt.pinned_temperature = T0 + (sign == 0 ? h : -h);
        assemble(*o, step, *tm, false);
        (sign == 0 ? fp : fm) = s.f;
      }
      o->opt.pinned_temperature = T0;
      for (int64_t i = 0; i < n; ++i) dr_out[i] = (fp[i] - fm[i]) / (2 * h);
    }
    assemble(*o, step, *tm, false);
  });
}

int oracle_adjoint_results(const ifem_ctx* ctx, int32_t step, double* dr_dtheta, double* lam_dr) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  if ((size_t)step >= o->adj_full.size()) return IFEM_ERR_STATE;
  if (dr_dtheta) {
    if (o->adj_full[step].empty()) return IFEM_ERR_STATE;
    std::copy(o->adj_full[step].begin(), o->adj_full[step].end(), dr_dtheta);
  }
  if (lam_dr) {
    if (o->adj_sets[step].empty()) return IFEM_ERR_STATE;
    std::copy(o->adj_sets[step].begin(), o->adj_sets[step].end(), lam_dr);
  }
  return IFEM_OK;
}

// The CPU side has no graphs: "capture" records the sequence and "launch" runs it.
int oracle_graph_capture(ifem_ctx* ctx, int32_t n_steps, const int32_t* steps, const ifem_time* tm,
                         int32_t with_adjoint) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !tm || n_steps <= 0 || !steps) return IFEM_ERR_INVALID;
  for (int i = 0; i < n_steps; ++i) if (steps[i] < 0 || steps[i] >= o->nsteps) return IFEM_ERR_INVALID;
  o->g_steps.assign(steps, steps + n_steps);
  o->g_tm = *tm;
  o->g_adjoint = with_adjoint;
  return IFEM_OK;
}

int oracle_graph_launch(ifem_ctx* ctx) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o) return IFEM_ERR_INVALID;
  if (o->g_steps.empty()) return IFEM_ERR_STATE;
  for (int s : o->g_steps) {
    int rc = oracle_assemble(ctx, s, &o->g_tm);
    if (rc != IFEM_OK) return rc;
    if (o->g_adjoint) {
      std::vector<double> full(4 * (size_t)o->steps[s].ndofs), sets(4 * o->mats.size());
      rc = oracle_adjoint(ctx, s, &o->g_tm, nullptr, full.data(), sets.data());
      if (rc != IFEM_OK) return rc;
    }
  }
  return IFEM_OK;
}


// ---- Constraints (Constrainer.cpp:38-126, physics.cpp:314-362, 408-419) ----

// Constrainer::SetZero + AddConstraint (Constrainer.cpp:38-64); the free/constrained numbering of
// Constrainer::Assemble (:91-109) and the symbolic PtAP pattern of Physics::Constraint (:332-339).
int oracle_set_constraints(ifem_ctx* ctx, int32_t step, int64_t n, const int64_t* dofs, const double* values) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps || n < 0 || (n > 0 && (!dofs || !values))) return IFEM_ERR_INVALID;
  return guarded(o, [&] {
    StepData& s = o->steps[step];
    std::map<int64_t, double> m;
    for (int64_t i = 0; i < n; ++i) {
      if (dofs[i] < 0 || dofs[i] >= s.ndofs) throw Err{IFEM_ERR_INVALID, "constrained dof out of range"};
      auto it = m.find(dofs[i]);
      if (it != m.end()) {
        if (it->second != values[i]) throw Err{IFEM_ERR_INVALID, "dof doubly constrained with different values"};
      } else {
        m.insert({dofs[i], values[i]});
      }
    }
    ConsData& c = s.cons;
    c.dof_to_val = m;
    c.fmap.assign(s.ndofs, 0);
    c.free_dofs.clear();
    int64_t ci = 0;
    for (int64_t d = 0; d < s.ndofs; ++d) {
      if (m.count(d)) c.fmap[d] = -1 - ci++;
      else { c.fmap[d] = (int64_t)c.free_dofs.size(); c.free_dofs.push_back(d); }
    }
    const int64_t nf = (int64_t)c.free_dofs.size();
    c.rowptr.assign(nf + 1, 0);
    c.colidx.clear();
    if (!s.colidx.empty())
      for (int64_t i = 0; i < nf; ++i) {
        const int64_t r = c.free_dofs[i];
        for (int32_t j = s.rowptr[r]; j < s.rowptr[r + 1]; ++j)
          if (c.fmap[s.colidx[j]] >= 0) c.colidx.push_back((int32_t)c.fmap[s.colidx[j]]);
        c.rowptr[i + 1] = (int32_t)c.colidx.size();
      }
    c.cv.assign(m.size(), 0.0);
    c.f_con.assign(nf, 0.0);
    c.vals.assign(c.colidx.size(), 0.0);
    c.built = false;
  });
}

int oracle_constrained_info(const ifem_ctx* ctx, int32_t step, int64_t* n_free, int64_t* nnz) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  const StepData& s = o->steps[step];
  const bool any = !s.cons.fmap.empty();
  if (n_free) *n_free = any ? (int64_t)s.cons.free_dofs.size() : s.ndofs;
  if (nnz) *nnz = any ? (int64_t)s.cons.colidx.size() : (int64_t)s.colidx.size();
  return IFEM_OK;
}

int oracle_build_constrained_pattern(const ifem_ctx* ctx, int32_t step, int32_t* row_ptr, int32_t* col_idx) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  const ConsData& c = o->steps[step].cons;
  if (c.fmap.empty()) return IFEM_ERR_STATE;
  if (row_ptr) std::copy(c.rowptr.begin(), c.rowptr.end(), row_ptr);
  if (col_idx) std::copy(c.colidx.begin(), c.colidx.end(), col_idx);
  return IFEM_OK;
}

// Constrainer::Assemble's C_v = value - State(dof) (Constrainer.cpp:112-118), then
//   CForceVec = -C C_v; CForceVec2 = K CForceVec + f (MatMultAdd: f_r, then the row's products in column order);
//   fCon = -(U^T CForceVec2); K_con = U^T K U                                  (physics.cpp:341-347, 332-339)
int oracle_constrain(ifem_ctx* ctx, int32_t step, int32_t want_matrix) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  return guarded(o, [&] {
    StepData& s = o->steps[step];
    ConsData& c = s.cons;
    if (c.fmap.empty()) throw Err{IFEM_ERR_STATE, "no constraints set for this step"};
    const std::vector<double>& u = s.state[IFEM_STATE_CUR];
    int64_t k = 0;
    for (const auto& dv : c.dof_to_val) c.cv[k++] = dv.second - u[dv.first];
    std::vector<double> x(s.ndofs, 0.0);
    k = 0;
    for (const auto& dv : c.dof_to_val) x[dv.first] = -c.cv[k++];
    const int64_t nf = (int64_t)c.free_dofs.size();
    int64_t o_nz = 0;
    for (int64_t i = 0; i < nf; ++i) {
      const int64_t r = c.free_dofs[i];
      double sum = s.f[r];
      if (!s.colidx.empty())
        for (int32_t j = s.rowptr[r]; j < s.rowptr[r + 1]; ++j) {
          sum += s.vals[j] * x[s.colidx[j]];
          if (want_matrix && c.fmap[s.colidx[j]] >= 0) c.vals[o_nz++] = s.vals[j];
        }
      c.f_con[i] = -sum;
    }
    c.built = true;
  });
}

int oracle_get_constrained(const ifem_ctx* ctx, int32_t step, double* f_con, void* vals, int64_t nnz, int32_t dtype) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  const ConsData& c = o->steps[step].cons;
  if (!c.built) return IFEM_ERR_STATE;
  if (f_con) std::copy(c.f_con.begin(), c.f_con.end(), f_con);
  if (vals) {
    if (nnz != (int64_t)c.vals.size()) return IFEM_ERR_INVALID;
    if (dtype == IFEM_F64) std::copy(c.vals.begin(), c.vals.end(), static_cast<double*>(vals));
    else for (int64_t i = 0; i < nnz; ++i) static_cast<float*>(vals)[i] = (float)c.vals[i];
  }
  return IFEM_OK;
}

int oracle_device_constrained(const ifem_ctx* ctx, int32_t step, const double** f_con, const void** vals,
                              int32_t* dtype_out) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps) return IFEM_ERR_INVALID;
  const ConsData& c = o->steps[step].cons;
  if (!c.built) return IFEM_ERR_STATE;
  if (f_con) *f_con = c.f_con.data();
  if (vals) *vals = c.vals.data();
  if (dtype_out) *dtype_out = IFEM_F64;
  return IFEM_OK;
}

// Physics::UpdateState: u += U dx (MatMultAdd, free dofs), then u += C C_v (constrained dofs)
int oracle_update_state(ifem_ctx* ctx, int32_t step, const double* dx) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || step < 0 || step >= o->nsteps || !dx) return IFEM_ERR_INVALID;
  StepData& s = o->steps[step];
  ConsData& c = s.cons;
  if (!c.built) return IFEM_ERR_STATE;
  std::vector<double>& u = s.state[IFEM_STATE_CUR];
  for (int64_t d = 0; d < s.ndofs; ++d) {
    const int64_t m = c.fmap[d];
    if (m >= 0) u[d] = u[d] + dx[m];
    else u[d] = u[d] + c.cv[-1 - m];
  }
  return IFEM_OK;
}

// Crack length of a node-ordered phase field (host pointers): sum_e sum_ip gamma * w
// (PhaseField.cpp:650, PhaseFieldUtil.cpp:185-221), element by element in order.
// TriAxialModel::init / Setup (TriAxial.cpp:22-71)
int oracle_set_triaxial(ifem_ctx* ctx, const ifem_face_group* side, const ifem_face_group* top, const ifem_triaxial* prm) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !side || !top || !prm) return IFEM_ERR_INVALID;
  return guarded(o, [&] {
    if (o->step_u < 0) throw Err{IFEM_ERR_INVALID, "TriAxial needs displacement dofs"};
    if (prm->damaged_forces && o->step_ph < 0) throw Err{IFEM_ERR_INVALID, "DamagedForces needs a phase field"};
    const int nfn = o->dim == 2 ? 3 : 9;
    FaceGroup* dst[2] = {&o->tri.side, &o->tri.top};
    const ifem_face_group* g[2] = {side, top};
    for (int k = 0; k < 2; ++k) {
      if (g[k]->n_faces < 1 || !g[k]->faces || !g[k]->face_data) throw Err{IFEM_ERR_INVALID, "empty face group"};
      for (int64_t i = 0; i < g[k]->n_faces * nfn; ++i) {
        const int64_t nd = g[k]->faces[i];
        if (nd < 0 || nd >= o->nn || o->dofnum[IFEM_DOF_UX][nd] < 0)
          throw Err{IFEM_ERR_INVALID, "face node without displacement dofs"};
      }
      dst[k]->nf = g[k]->n_faces;
      dst[k]->F.assign(g[k]->faces, g[k]->faces + g[k]->n_faces * nfn);
      dst[k]->C.assign(g[k]->face_data, g[k]->face_data + g[k]->n_faces * nfn * nfn);
    }
    o->tri.prm = *prm;
    ifem_triaxial_state st{};
    st.area = 1.0; st.u0 = -1.0e8; st.max_load = -1e9; st.p0 = prm->p0;   // TriAxial.cpp:63-70
    o->tri.st = st;
    o->tri.on = true;
  });
}

// TriAxialModel::Commit (TriAxial.cpp:75-122)
int oracle_triaxial_commit(ifem_ctx* ctx, int32_t commit_type, double time, double* max_time) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o) return IFEM_ERR_INVALID;
  if (!o->tri.on) return IFEM_ERR_STATE;
  if (commit_type != IFEM_COMMIT_TIMEDEP) return IFEM_OK;
  ifem_triaxial_state& S = o->tri.st;
  const double uRate = o->tri.prm.du, p0 = o->tri.prm.p0;
  const int sg = (0.0 < uRate) - (uRate < 0.0);
  S.max_load = std::max(S.max_load, S.f_ext / S.area * sg);
  if (sg < 0) {
    if (!S.min_load_passed && (S.f_ext / S.area) * sg > std::max(1.0e3, std::fabs(p0)) && time > 0.0)
      S.min_load_passed = 1;
    const double MinLoad = std::max(0.05 * std::fabs(p0), 0.05 * S.max_load);
    if (S.min_load_passed && std::fabs(S.f_ext / S.area) < MinLoad && S.t_break < 1e-8) {
      S.t_break = time;
      if (max_time) *max_time = S.t_break + o->tri.prm.t_post_fail;
    }
  } else {
    const double MinLoad = std::max(0.0, 0.25 * S.max_load);
    if (S.min_load_passed && std::fabs(S.f_ext / S.area) < MinLoad && S.t_break < 1e-8) {
      S.t_break = time;
      if (max_time) *max_time = S.t_break + o->tri.prm.t_post_fail;
    }
    if (!S.min_load_passed && (S.f_ext / S.area) * sg > 0.0 && time > 0.0) S.min_load_passed = 1;
  }
  if (time < 0.0) S.u0 = S.uz_sum / S.area;
  return IFEM_OK;
}

int oracle_triaxial_get_state(const ifem_ctx* ctx, ifem_triaxial_state* out) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || !out) return IFEM_ERR_INVALID;
  if (!o->tri.on) return IFEM_ERR_STATE;
  *out = o->tri.st;
  return IFEM_OK;
}

int oracle_triaxial_set_state(ifem_ctx* ctx, const ifem_triaxial_state* in) {
  Oracle* o = reinterpret_cast<Oracle*>(ctx);
  if (!o || !in) return IFEM_ERR_INVALID;
  if (!o->tri.on) return IFEM_ERR_STATE;
  o->tri.st = *in;
  return IFEM_OK;
}

// shape values, weights and normals of one face of a TriAxial group (0 side, 1 top): N [nq][nfn], w [nq], n [nq][3]
int oracle_face_shapes(const ifem_ctx* ctx, int32_t group, int64_t face, double* N, double* w, double* n) {
  const Oracle* o = reinterpret_cast<const Oracle*>(ctx);
  if (!o || !o->tri.on || group < 0 || group > 1) return IFEM_ERR_INVALID;
  const FaceGroup& g = group ? o->tri.top : o->tri.side;
  if (face < 0 || face >= g.nf) return IFEM_ERR_INVALID;
  FaceIP ips[9];
  const int nq = face_shapes(*o, g, face, ips), nfn = o->dim == 2 ? 3 : 9;
  for (int q = 0; q < nq; ++q) {
    for (int a = 0; a < nfn; ++a) N[q * nfn + a] = ips[q].N[a];
    w[q] = ips[q].w;
    for (int d = 0; d < 3; ++d) n[q * 3 + d] = ips[q].n[d];
  }
  return IFEM_OK;
}

int oracle_crack_length_noalloc(int32_t dim, int64_t n_elems, const double* coords, const double* node_weights,
                                const int32_t* elems, const double* elem_kron, const double* phase,
                                double length_scale, int32_t distribution, double* length_out, void* /*stream*/) {
  if ((dim != 2 && dim != 3) || n_elems < 0 || !coords || !elems || !elem_kron || !phase || !length_out) return IFEM_ERR_INVALID;
  try {
    Oracle o;
    o.dim = dim; o.nen = dim == 2 ? 9 : 27; o.ip1d = 3; o.nel = n_elems;
    int64_t nn = 0;
    for (int64_t i = 0; i < n_elems * o.nen; ++i) nn = std::max<int64_t>(nn, (int64_t)elems[i] + 1);
    o.nn = nn;
    o.X.assign(coords, coords + nn * dim);
    if (dim == 3 && node_weights) o.W.assign(node_weights, node_weights + nn);
    o.E.assign(elems, elems + n_elems * o.nen);
    build_shapes(o);
    o.C.assign((size_t)o.nen * o.nen, 0.0);
    double total = 0;
    Oracle one = o;                 // one-element view: element 0 of `one` is element e of the mesh
    one.nel = 1;
    one.E.assign(o.nen, 0);
    for (int64_t e = 0; e < n_elems; ++e) {
      const double* k = elem_kron + (size_t)e * dim * 9;   // C = kron(Cz, kron(Cy, Cx))
      for (int j = 0; j < o.nen; ++j)
        for (int c = 0; c < o.nen; ++c) {
          const int ix = j % 3, iy = (j / 3) % 3, iz = j / 9, jx = c % 3, jy = (c / 3) % 3, jz = c / 9;
          double v = k[9 + iy * 3 + jy] * k[ix * 3 + jx];
          if (dim == 3) v = k[18 + iz * 3 + jz] * v;
          one.C[j * o.nen + c] = v;
        }
      for (int a = 0; a < o.nen; ++a) one.E[a] = elems[e * o.nen + a];
      ShapeIP sh[27];
      shape_grads(one, 0, sh);
      double Ph[27];
      for (int a = 0; a < o.nen; ++a) Ph[a] = phase[one.E[a]];
      double el_sum = 0;
      for (int ip = 0; ip < o.nip; ++ip)
        el_sum += distribution_gamma(distribution, length_scale, sh[ip], o.nen, dim, Ph) * sh[ip].w;
      total += el_sum;
    }
    *length_out = total;
    return IFEM_OK;
  } catch (const Err& er) { return er.code; }
}

}  // extern "C"
