// Phase step with the second-gradient crack-density functions HO_Linear, HO_Linear2, HO_CZM, HO_Quadratic and
// Custom (PhaseFieldUtil.cpp:223-280), which integrate second derivatives of the phase field.
//
// The phase group's shape functions come from getShapeGrads2 (B2_2.cpp:90-125, NURBS3_Cube2.cpp:117-216):
//   2D:  G = J^{-1} G_xi with J = G_xi X (the first-order path inverts J^T instead; the two agree on axis-aligned
//        elements), G2 = J2^{-1} (G2_xi - J2Part2 G_xi), J2Part2 = G2_xi X, J2 the 3x3 second-order Jacobian;
//   3D:  the rational basis R = W CB / w, its parametric first and second derivatives by the quotient rule,
//        G = J^{-1} G_xi and G2 = J2^{-1} (G2_xi - J2Part2 G_xi) with the 6x6 J2,
// second derivatives ordered xx, yy, xy (2D) and xx, yy, zz, xy, yz, xz (3D), contracted with DoubleCon =
// diag(1, .., 2, ..).  The displacement strain keeps the first-order gradients (Assemble_Phase calls
// getShapeGrads for the u group).
//
// Every distribution of this family has the form
//   gamma = c (g0 phi + g1 phi^2 + g2 l^2 |grad phi|^2 + g3 l^4 ddphi^T DC ddphi)
//   Dist  = c (N (g0 + 2 g1 phi) + 2 g2 l^2 G^T grad phi + 2 g3 l^4 G2^T DC ddphi)
//   dDist = c (2 g1 N N^T + 2 g2 l^2 G^T G + 2 g3 l^4 G2^T DC G2)
// with (c, g0, g1, g2, g3) = (1/2l, 0, 1, 1/2, 1/16) HO_Quadratic, (1/(3.020 l), 2, -1, 1/2, 1/16) HO_CZM,
// (1/(19.2 l), 9, 0, 0, 1) HO_Linear, (1/4l, 2, 0, 1/2, 1/16) HO_Linear2 and (1/(C0 l), C1, C2, C3, C4) Custom.
// The lumped capacities are those of GetCapacityOnly (PhaseFieldUtil.cpp:282-348).
//
// One warp per element (lanes = ips, then nodes), FP64 arithmetic; the tangent is stored in the element
// matrices' precision.  Every other term is the one of the general phase kernel.

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

__device__ __forceinline__ int ho_mat(const Geo& g, int64_t el) { return g.emat ? g.emat[el] : 0; }
__device__ __forceinline__ int ho_dof(const DofMap& dm, int kind, int node) { return dm.base[kind] + dm.node_rank[node]; }

template <int DIM>
struct HoGeo {
  static constexpr int NG = DIM == 2 ? 3 : 6;
  double Ji[DIM * DIM];       // inverse Jacobian of the parametric map (row-major)
  double J2i[NG * NG];        // inverse second-order Jacobian
  double P[NG][DIM];          // J2Part2 = G2_xi X
  double rw, dW[3], dW2[6];   // 3D: 1 / w, dw / dxi, d2w / dxi2 of the rational weight function
};

template <int DIM, bool KRON>
struct HoSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN, NG = DIM == 2 ? 3 : 6, NT = 1 + DIM + NG;
  ElemSm<DIM, KRON> e;
  double HX[DIM][3][3];       // KRON: extraction applied to the second derivatives of the 1-D basis
  double U[DIM][NEN], dU[DIM][NEN];
  double Ph[NEN], PhO[NEN], Tn[NEN];
  IpGeo<DIM> g[NEN];          // first-order geometry (the strain)
  HoGeo<DIM> hg[NEN];         // second-order geometry (the distribution)
  double kNF[NEN], kGF[NEN], kHF[NEN], kNN[NEN], kLD[NEN];
  double dG[NEN][DIM], hG[NEN][NG];   // per ip: grad phi and DC ddphi
  double lc[NEN];
  double tab[NEN][NT];        // (N, G, G2) of every node at the ip being summed
  double last_Gc, last_l, last_visc;
};

// Gauss-Jordan inverse with partial pivoting (n x n, row-major); false when singular
template <int N>
__device__ inline bool invn(double* A, double* Ai) {
  for (int i = 0; i < N * N; ++i) Ai[i] = (i % (N + 1) == 0) ? 1.0 : 0.0;
  for (int k = 0; k < N; ++k) {
    int p = k;
    double best = fabs(A[k * N + k]);
    for (int i = k + 1; i < N; ++i) if (fabs(A[i * N + k]) > best) { best = fabs(A[i * N + k]); p = i; }
    if (best == 0.0) return false;
    if (p != k)
      for (int j = 0; j < N; ++j) {
        double t = A[k * N + j]; A[k * N + j] = A[p * N + j]; A[p * N + j] = t;
        t = Ai[k * N + j]; Ai[k * N + j] = Ai[p * N + j]; Ai[p * N + j] = t;
      }
    const double ip = 1.0 / A[k * N + k];
    for (int j = 0; j < N; ++j) { A[k * N + j] *= ip; Ai[k * N + j] *= ip; }
    for (int i = 0; i < N; ++i) {
      if (i == k) continue;
      const double f = A[i * N + k];
      if (f == 0.0) continue;
      for (int j = 0; j < N; ++j) { A[i * N + j] -= f * A[k * N + j]; Ai[i * N + j] -= f * Ai[k * N + j]; }
    }
  }
  return true;
}

// parametric values of node a at ip q: CB, its first derivatives GB and second derivatives G2B (extraction applied)
template <int DIM, bool KRON>
__device__ inline void ho_bern(const HoSm<DIM, KRON>& s, const Rule& R, int q, int a, double& CB, double GB[DIM],
                               double G2B[DIM == 2 ? 3 : 6]) {
  const ElemSm<DIM, KRON>& e = s.e;
  if (DIM == 2) {
    const int qx = q % 3, qy = q / 3;
    if (KRON) {
      const int ia = a % 3, ja = a / 3;
      const double nx = e.NX[0][qx][ia], ny = e.NX[1][qy][ja], gx = e.GX[0][qx][ia], gy = e.GX[1][qy][ja];
      const double hx = s.HX[0][qx][ia], hy = s.HX[1][qy][ja];
      CB = nx * ny; GB[0] = gx * ny; GB[1] = nx * gy;
      G2B[0] = hx * ny; G2B[1] = nx * hy; G2B[2] = gx * gy;
    } else {
      CB = 0; GB[0] = GB[1] = 0; G2B[0] = G2B[1] = G2B[2] = 0;
      for (int k = 0; k < 9; ++k) {
        const int kx = k % 3, ky = k / 3;
        const double c = e.C[a * 9 + k];
        CB += c * (R.B[qx][kx] * R.B[qy][ky]);
        GB[0] += c * (R.dB[qx][kx] * R.B[qy][ky]);
        GB[1] += c * (R.B[qx][kx] * R.dB[qy][ky]);
        G2B[0] += c * (R.d2B[qx][kx] * R.B[qy][ky]);
        G2B[1] += c * (R.B[qx][kx] * R.d2B[qy][ky]);
        G2B[2] += c * (R.dB[qx][kx] * R.dB[qy][ky]);
      }
    }
  } else {
    const int qx = q % 3, qy = (q / 3) % 3, qz = q / 9;
    if (KRON) {
      const int ia = a % 3, ja = (a / 3) % 3, ka = a / 9;
      const double nx = e.NX[0][qx][ia], ny = e.NX[1][qy][ja], nz = e.NX[2 % DIM][qz][ka];
      const double gx = e.GX[0][qx][ia], gy = e.GX[1][qy][ja], gz = e.GX[2 % DIM][qz][ka];
      const double hx = s.HX[0][qx][ia], hy = s.HX[1][qy][ja], hz = s.HX[2 % DIM][qz][ka];
      CB = nx * ny * nz;
      GB[0] = gx * ny * nz; GB[1] = nx * gy * nz; GB[DIM - 1] = nx * ny * gz;
      G2B[0] = hx * ny * nz; G2B[1] = nx * hy * nz; G2B[2 % (DIM == 2 ? 3 : 6)] = nx * ny * hz;
      G2B[3 % (DIM == 2 ? 3 : 6)] = gx * gy * nz; G2B[4 % (DIM == 2 ? 3 : 6)] = nx * gy * gz;
      G2B[5 % (DIM == 2 ? 3 : 6)] = gx * ny * gz;
    } else {
      CB = 0;
      for (int d = 0; d < DIM; ++d) GB[d] = 0;
      for (int r = 0; r < (DIM == 2 ? 3 : 6); ++r) G2B[r] = 0;
      for (int k = 0; k < 27; ++k) {
        const int kx = k % 3, ky = (k / 3) % 3, kz = k / 9;
        const double c = e.C[a * 27 + k];
        const double bx = R.B[qx][kx], by = R.B[qy][ky], bz = R.B[qz][kz];
        const double dx = R.dB[qx][kx], dy = R.dB[qy][ky], dz = R.dB[qz][kz];
        CB += c * (bx * by * bz);
        GB[0] += c * (dx * by * bz); GB[1] += c * (bx * dy * bz); GB[DIM - 1] += c * (bx * by * dz);
        double h[6] = {R.d2B[qx][kx] * by * bz, bx * R.d2B[qy][ky] * bz, bx * by * R.d2B[qz][kz],
                       dx * dy * bz, bx * dy * dz, dx * by * dz};
        for (int r = 0; r < (DIM == 2 ? 3 : 6); ++r) G2B[r] += c * h[r];
      }
    }
  }
}

// component r of the 3D second derivatives pairs the parametric directions (ii, jj)
__device__ __forceinline__ int ho_pi(int r) { return r < 3 ? r : (r == 3 ? 0 : (r == 4 ? 1 : 0)); }
__device__ __forceinline__ int ho_pj(int r) { return r < 3 ? r : (r == 3 ? 1 : 2); }

// rational parametric first and second derivatives of node a (3D; 2D: the polynomial ones)
template <int DIM, bool KRON>
__device__ inline void ho_param(const HoSm<DIM, KRON>& s, const Rule& R, const HoGeo<DIM>& hg, int q, int a, double& N,
                                double GXi[DIM], double G2Xi[DIM == 2 ? 3 : 6]) {
  constexpr int NG = DIM == 2 ? 3 : 6;
  double CB, GB[DIM], G2B[NG];
  ho_bern<DIM, KRON>(s, R, q, a, CB, GB, G2B);
  if (DIM == 2) {
    N = CB;
    for (int d = 0; d < DIM; ++d) GXi[d] = GB[d];
    for (int r = 0; r < NG; ++r) G2Xi[r] = G2B[r];
  } else {
    const double W = s.e.W[a], rw = hg.rw, rw2 = rw * rw, rw3 = rw2 * rw;
    N = W * CB * rw;
    for (int d = 0; d < DIM; ++d) GXi[d] = W * (GB[d] * rw - CB * hg.dW[d] * rw2);
    for (int r = 0; r < NG; ++r) {
      const int ii = ho_pi(r), jj = ho_pj(r);
      G2Xi[r] = W * (G2B[r] * rw - hg.dW[jj] * GB[ii % DIM] * rw2 - hg.dW[ii] * GB[jj % DIM] * rw2 - hg.dW2[r] * CB * rw2 +
                     2.0 * hg.dW[ii] * hg.dW[jj] * CB * rw3);
    }
  }
}

// physical N, G and G2 of node a at ip q
template <int DIM, bool KRON>
__device__ inline void ho_node(const HoSm<DIM, KRON>& s, const Rule& R, const HoGeo<DIM>& hg, int q, int a, double& N,
                               double G[DIM], double G2[DIM == 2 ? 3 : 6]) {
  constexpr int NG = DIM == 2 ? 3 : 6;
  double GXi[DIM], G2Xi[NG];
  ho_param<DIM, KRON>(s, R, hg, q, a, N, GXi, G2Xi);
  for (int d = 0; d < DIM; ++d) {
    double t = 0;
    for (int c = 0; c < DIM; ++c) t += hg.Ji[d * DIM + c] * GXi[c];
    G[d] = t;
  }
  double v[NG];
  for (int r = 0; r < NG; ++r) {
    double t = G2Xi[r];
    for (int c = 0; c < DIM; ++c) t -= hg.P[r][c] * GXi[c];
    v[r] = t;
  }
  for (int r = 0; r < NG; ++r) {
    double t = 0;
    for (int k = 0; k < NG; ++k) t += hg.J2i[r * NG + k] * v[k];
    G2[r] = t;
  }
}

// second-order geometry of ip q
template <int DIM, bool KRON>
__device__ inline bool ho_geometry(const HoSm<DIM, KRON>& s, const Rule& R, int q, HoGeo<DIM>& hg) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NG = DIM == 2 ? 3 : 6;
  hg.rw = 1.0;
  for (int d = 0; d < 3; ++d) hg.dW[d] = 0;
  for (int r = 0; r < 6; ++r) hg.dW2[r] = 0;
  if (DIM == 3) {
    double wf = 0;
    for (int a = 0; a < NEN; ++a) {
      double CB, GB[DIM], G2B[NG];
      ho_bern<DIM, KRON>(s, R, q, a, CB, GB, G2B);
      const double W = s.e.W[a];
      wf += CB * W;
      for (int d = 0; d < DIM; ++d) hg.dW[d] += GB[d] * W;
      for (int r = 0; r < NG; ++r) hg.dW2[r] += G2B[r] * W;
    }
    hg.rw = 1.0 / wf;
  }
  double J[DIM * DIM], P[NG * DIM];
  for (int i = 0; i < DIM * DIM; ++i) J[i] = 0;
  for (int i = 0; i < NG * DIM; ++i) P[i] = 0;
  for (int a = 0; a < NEN; ++a) {
    double N, GXi[DIM], G2Xi[NG];
    ho_param<DIM, KRON>(s, R, hg, q, a, N, GXi, G2Xi);
    for (int d = 0; d < DIM; ++d)
      for (int c = 0; c < DIM; ++c) J[d * DIM + c] += GXi[d] * s.e.X[a][c];
    for (int r = 0; r < NG; ++r)
      for (int c = 0; c < DIM; ++c) P[r * DIM + c] += G2Xi[r] * s.e.X[a][c];
  }
  for (int r = 0; r < NG; ++r)
    for (int c = 0; c < DIM; ++c) hg.P[r][c] = P[r * DIM + c];
  double J2[NG * NG];
  if (DIM == 2) {
    const double j00 = J[0], j01 = J[1], j10 = J[DIM], j11 = J[DIM + 1];
    const double v[9] = {j00 * j00, j01 * j01, 2 * j00 * j01, j10 * j10, j11 * j11, 2 * j10 * j11,
                         j00 * j10, j01 * j11, j10 * j01 + j11 * j00};
    for (int i = 0; i < 9; ++i) J2[i % (NG * NG)] = v[i];
  } else {
    auto j = [&](int r, int c) { return J[r * DIM + c % DIM]; };
    for (int r = 0; r < 3; ++r) {
      J2[(r * 6 + 0) % (NG * NG)] = j(r, 0) * j(r, 0); J2[(r * 6 + 1) % (NG * NG)] = j(r, 1) * j(r, 1);
      J2[(r * 6 + 2) % (NG * NG)] = j(r, 2) * j(r, 2); J2[(r * 6 + 3) % (NG * NG)] = 2 * j(r, 0) * j(r, 1);
      J2[(r * 6 + 4) % (NG * NG)] = 2 * j(r, 1) * j(r, 2); J2[(r * 6 + 5) % (NG * NG)] = 2 * j(r, 0) * j(r, 2);
    }
    const int ra[3] = {0, 1, 0}, rb[3] = {1, 2, 2};
    for (int t = 0; t < 3; ++t) {
      const int a = ra[t], b = rb[t], r = 3 + t;
      J2[(r * 6 + 0) % (NG * NG)] = j(a, 0) * j(b, 0); J2[(r * 6 + 1) % (NG * NG)] = j(a, 1) * j(b, 1);
      J2[(r * 6 + 2) % (NG * NG)] = j(a, 2) * j(b, 2);
      J2[(r * 6 + 3) % (NG * NG)] = j(a, 0) * j(b, 1) + j(b, 0) * j(a, 1);
      J2[(r * 6 + 4) % (NG * NG)] = j(a, 1) * j(b, 2) + j(b, 1) * j(a, 2);
      J2[(r * 6 + 5) % (NG * NG)] = j(a, 0) * j(b, 2) + j(b, 0) * j(a, 2);
    }
  }
  bool ok = invn<DIM>(J, hg.Ji);
  ok = invn<NG>(J2, hg.J2i) && ok;
  return ok;
}

// (c, g0, g1, g2, g3) of the distribution; lumped-capacity coefficients capF (of N), capK (of N N^T)
__device__ inline void ho_coefs(int dist, double l, const double* C, double& c, double& g0, double& g1, double& g2,
                                double& g3) {
  switch (dist) {
    case IFEM_DIST_HO_QUADRATIC: c = 1.0 / (2.0 * l); g0 = 0.0; g1 = 1.0; g2 = 0.5; g3 = 1.0 / 16.0; break;
    case IFEM_DIST_HO_CZM: c = 1.0 / (3.020 * l); g0 = 2.0; g1 = -1.0; g2 = 0.5; g3 = 1.0 / 16.0; break;
    case IFEM_DIST_HO_LINEAR: c = 1.0 / (19.2 * l); g0 = 9.0; g1 = 0.0; g2 = 0.0; g3 = 1.0; break;
    case IFEM_DIST_HO_LINEAR2: c = 1.0 / (4.0 * l); g0 = 2.0; g1 = 0.0; g2 = 0.5; g3 = 1.0 / 16.0; break;
    default: c = 1.0 / (C[0] * l); g0 = C[1]; g1 = C[2]; g2 = C[3]; g3 = C[4]; break;   // Custom
  }
}

__device__ inline void ho_capacity(int dist, double l, const double* C, double phi, double& capF, double& capK) {
  switch (dist) {
    case IFEM_DIST_HO_QUADRATIC: capF = 1.0 / (2.0 * l) * (2.0 * phi); capK = 1.0 / (2.0 * l) * 2.0; break;
    case IFEM_DIST_HO_CZM: capF = 1.0 / (3.020 * l) * (2.0 * (1.0 - phi)); capK = 1.0 / (3.020 * l) * -2.0; break;
    case IFEM_DIST_HO_LINEAR: capF = 1.0 / (19.2 * l) * 9.0; capK = 0.0; break;
    case IFEM_DIST_HO_LINEAR2: capF = 3.0 / (8.0 * l); capK = 0.0; break;
    default: capF = 1.0 / (C[0] * l) * (C[1] + 2.0 * C[2] * phi); capK = 1.0 / (C[0] * l) * (2.0 * C[2]); break;
  }
}

__device__ inline void ho_capacity_lumped(int dist, double l, const double* C, double ph, double& DL, double& dDL) {
  switch (dist) {
    case IFEM_DIST_HO_QUADRATIC: DL = 1.0 / l * ph; dDL = 1.0 / l; break;
    case IFEM_DIST_HO_CZM: DL = 2.0 / (3.020 * l) * (1 - ph); dDL = -2.0 / (3.020 * l); break;
    case IFEM_DIST_HO_LINEAR: DL = 9.0 / (19.2 * l); dDL = 0.0; break;
    case IFEM_DIST_HO_LINEAR2: DL = 3.0 / (8.0 * l); dDL = 0.0; break;
    default: DL = 1.0 / (C[0] * l) * (C[1] + 2.0 * C[2] * ph); dDL = 1.0 / (C[0] * l) * 2.0 * C[2]; break;
  }
}

constexpr int kHoWarps = 2;

template <int DIM, bool KRON, typename T>
__global__ void __launch_bounds__(32 * kHoWarps) k_phase_ho(const PParams p) {
  using S = HoSm<DIM, KRON>;
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, NG = S::NG;
  extern __shared__ __align__(16) unsigned char smraw[];
  S* sm = reinterpret_cast<S*>(smraw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t el = (int64_t)blockIdx.x * kHoWarps + warp;
  const Geo& geo = p.geo;
  if (el >= geo.nel) return;                      // whole warp; no CTA-wide barrier in this kernel
  S& s = sm[warp];
  const int64_t nh = geo.nel * NIP;
  const DofMap& dm = p.dm;
  const ModelOpts& mo = p.mo;
  const bool act = lane < NEN;
  const int q = lane;
  unsigned bad = 0;
  const double DCv[6] = {1.0, 1.0, DIM == 2 ? 2.0 : 1.0, 2.0, 2.0, 2.0};   // DoubleCon

  fill_elem<DIM, KRON>(s.e, geo, p.rule, el, lane, 32);
  if (KRON)
    for (int i = lane; i < DIM * 9; i += 32) {
      const int ax = i / 9, pt = (i / 3) % 3, fn = i % 3;
      const double* Ce = geo.ext + (el * DIM + ax) * 9;
      double h = 0;
      for (int k = 0; k < 3; ++k) h += Ce[fn * 3 + k] * p.rule.d2B[pt][k];
      s.HX[ax][pt][fn] = h;
    }
  if (act) {
    const int a = lane;
    const int node = geo.conn[el * NEN + a];
    for (int b = 0; b < DIM; ++b) {
      const int d = ho_dof(dm, IFEM_DOF_UX + b, node);
      s.U[b][a] = p.su.cur[d];
      s.dU[b][a] = p.su.d[d];
    }
    const int dph = ho_dof(dm, IFEM_DOF_PHASE, node);
    s.Ph[a] = p.sp.cur[dph];
    s.PhO[a] = p.sp.old[dph];
    if (mo.hasT) s.Tn[a] = mo.ref_compat_T ? p.sT.cur[0] : p.sT.cur[ho_dof(dm, IFEM_DOF_T, node)];
    else s.Tn[a] = 0.0;
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, KRON>(s.e, p.rule, q, g);
    s.g[q] = g;
    HoGeo<DIM> hg;
    if (!ho_geometry<DIM, KRON>(s, p.rule, q, hg)) bad = 1;
    s.hg[q] = hg;
    double phi = 0, Tip = 0, eps[6] = {0, 0, 0, 0, 0, 0}, uip[DIM], vip[DIM], dG[DIM], ddG[NG];
    for (int d = 0; d < DIM; ++d) { uip[d] = 0; vip[d] = 0; dG[d] = 0; }
    for (int r = 0; r < NG; ++r) ddG[r] = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, KRON>(s.e, p.rule, g, q, a, N, G);   // first-order gradients: the strain
      for (int d = 0; d < DIM; ++d) { uip[d] += N * s.U[d][a]; vip[d] += N * s.dU[d][a]; }
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
      double Nh, Gh[DIM], G2[NG];
      ho_node<DIM, KRON>(s, p.rule, hg, q, a, Nh, Gh, G2);   // the phase group's gradients
      for (int d = 0; d < DIM; ++d) dG[d] += Gh[d] * s.Ph[a];
      for (int r = 0; r < NG; ++r) ddG[r] += G2[r] * s.Ph[a];
    }
    const MatDev& m = geo.mats[ho_mat(geo, el)];
    PtMat M;
    set_temperature(m, !mo.hasT, mo.hasT ? Tip : mo.pinned_T, M);
    double Dam, dDam, ddDam, DamI, dDamI, ddDamI, DamG, dDamG, ddDamG;
    damage_function(phi, mo.dam_f, mo.k0, mo.porder_p, Dam, dDam, ddDam);
    damage_function(phi, mo.dens_f, mo.k0, mo.porder_p, DamI, dDamI, ddDamI);
    damage_function(phi, mo.grav_f, mo.k0, mo.porder_p, DamG, dDamG, ddDamG);
    const int64_t hi = el * NIP + q;
    double ee[6];
    for (int r = 0; r < 6; ++r) ee[r] = eps[r] - p.h.EP[r * nh + hi];
    double Sd[6], Su[6];
    double Energy;
    if (p.e_in) {   // Cosserat model: split, initialisation period and history applied by k_coss_energy
      Energy = p.e_in[hi];
    } else {
      Energy = energy_split<true, true>(M, ee, Sd, Su, nullptr, nullptr, false);
      if (mo.irr == IFEM_IRR_HIST) {
        const double Eo = p.h.EHo[hi];
        if (Eo > Energy) { if (p.write_hist) p.h.EH[hi] = Eo; Energy = Eo; }
        else if (p.write_hist) p.h.EH[hi] = Energy;
      } else if (p.write_hist) p.h.EH[hi] = Energy;
    }
    const double l = M.l, l2 = l * l, l4 = l2 * l2;
    double c, g0, g1, g2, g3;
    ho_coefs(mo.dist, l, mo.dist_coefs, c, g0, g1, g2, g3);
    double dGdG = 0, hh = 0;
    for (int d = 0; d < DIM; ++d) dGdG += dG[d] * dG[d];
    for (int r = 0; r < NG; ++r) hh += ddG[r] * DCv[r] * ddG[r];
    const double gamma = c * (g0 * phi + g1 * phi * phi + g2 * l2 * dGdG + g3 * l4 * hh);
    double capF = 0, capK = 0;
    if (mo.lumped_cap) ho_capacity(mo.dist, l, mo.dist_coefs, phi, capF, capK);
    const double w = g.w;
    double kNF = w * M.Gc * (c * (g0 + 2.0 * g1 * phi) - capF);
    double kNN = w * M.Gc * (c * 2.0 * g1 - capK);
    const double kG = w * M.Gc * c * 2.0 * g2 * l2;
    const double kH = w * M.Gc * c * 2.0 * g3 * l4;
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
      for (int d = 0; d < DIM; ++d) gu += mo.g[d] * uip[d];
      kNF += -w * m.density * gu * dDamG; kNN += -w * m.density * gu * ddDamG;
    }
    s.kNF[q] = kNF; s.kGF[q] = kG; s.kHF[q] = kH; s.kNN[q] = kNN; s.kLD[q] = kLD;
    for (int d = 0; d < DIM; ++d) s.dG[q][d] = dG[d];
    for (int r = 0; r < NG; ++r) s.hG[q][r] = DCv[r] * ddG[r];
    s.lc[q] = gamma * w;
    if (q == NIP - 1) { s.last_Gc = M.Gc; s.last_l = M.l; s.last_visc = M.visc; }
  }
  __syncwarp();
  // residual and tangent column b (lane = node b); the ips in order, every node's (N, G, G2) tabulated per ip
  double F = 0, WL = 0, LD = 0, acc[NEN];
  for (int a = 0; a < NEN; ++a) acc[a] = 0.0;
  for (int qq = 0; qq < NIP; ++qq) {
    if (act) {
      double N, G[DIM], G2[NG];
      ho_node<DIM, KRON>(s, p.rule, s.hg[qq], qq, lane, N, G, G2);
      s.tab[lane][0] = N;
      for (int d = 0; d < DIM; ++d) s.tab[lane][1 + d] = G[d];
      for (int r = 0; r < NG; ++r) s.tab[lane][1 + DIM + r] = G2[r];
    }
    __syncwarp();
    if (act) {
      const int b = lane;
      const double* tb = s.tab[b];
      double gd = 0, hd = 0;
      for (int d = 0; d < DIM; ++d) gd += tb[1 + d] * s.dG[qq][d];
      for (int r = 0; r < NG; ++r) hd += tb[1 + DIM + r] * s.hG[qq][r];
      F += s.kNF[qq] * tb[0] + s.kGF[qq] * gd + s.kHF[qq] * hd;
      WL += s.g[qq].w * tb[0];
      LD += s.kLD[qq] * tb[0];
      const double cn = s.kNN[qq] * tb[0], cg = s.kGF[qq], ch = s.kHF[qq];
      for (int a = 0; a < NEN; ++a) {
        const double* ta = s.tab[a];
        double gg = 0, h2 = 0;
        for (int d = 0; d < DIM; ++d) gg += ta[1 + d] * tb[1 + d];
        for (int r = 0; r < NG; ++r) h2 += ta[1 + DIM + r] * DCv[r] * tb[1 + DIM + r];
        acc[a] += cn * ta[0] + cg * gg + ch * h2;
      }
    }
    __syncwarp();
  }
  if (act) {
    const int b = lane;
    const double Gc = s.last_Gc, l = s.last_l, visc = s.last_visc;
    const MatDev& m = geo.mats[ho_mat(geo, el)];
    double diag = 0;
    if (mo.lumped_drive) {
      double D, dD, ddD;
      damage_function(s.Ph[b], mo.dam_f, mo.k0, mo.porder_p, D, dD, ddD);
      F += LD * dD; diag += LD * ddD;
    }
    if (mo.lumped_cap) {
      double DL, dDL;
      ho_capacity_lumped(mo.dist, l, mo.dist_coefs, s.Ph[b], DL, dDL);
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
    constexpr int KB = ke_block(1, NEN);
    T* Ke = reinterpret_cast<T*>(p.Ke) + el * NEN * KB;
    for (int a = 0; a < NEN; ++a) Ke[a * KB + b] = (T)(a == b ? acc[a] + diag : acc[a]);
    if (b == 0) {
      double lc = 0;
      for (int qq = 0; qq < NIP; ++qq) lc += s.lc[qq];
      p.lcrack_el[el] = lc;
    }
  }
  const unsigned tot_bad = __reduce_add_sync(0xffffffffu, bad);
  if (lane == 0 && tot_bad) atomicAdd(&p.stats[2], (unsigned long long)tot_bad);
}

template <int DIM, bool KRON, typename T>
void phase_ho_go(const PParams& p, cudaStream_t s) {
  const size_t smem = sizeof(HoSm<DIM, KRON>) * kHoWarps;
  auto k = k_phase_ho<DIM, KRON, T>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned blocks = (unsigned)((p.geo.nel + kHoWarps - 1) / kHoWarps);
  k<<<blocks, 32 * kHoWarps, smem, s>>>(p);
}

}  // namespace

void launch_phase_ho(const PParams& p, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  if (p.geo.dim == 2) {
    if (p.geo.kron) { if (p.ke_f32) phase_ho_go<2, true, float>(p, s); else phase_ho_go<2, true, double>(p, s); }
    else { if (p.ke_f32) phase_ho_go<2, false, float>(p, s); else phase_ho_go<2, false, double>(p, s); }
  } else {
    if (p.geo.kron) { if (p.ke_f32) phase_ho_go<3, true, float>(p, s); else phase_ho_go<3, true, double>(p, s); }
    else { if (p.ke_f32) phase_ho_go<3, false, float>(p, s); else phase_ho_go<3, false, double>(p, s); }
  }
}

}  // namespace ifem
