// TriAxial boundary loads (Models/ExternalForce/TriAxial.cpp:124-276) on boundary element groups.
//
// The groups are small next to the volume mesh (the faces of its boundary), so one thread integrates one face:
// its shape functions at the face's Gauss points, the outward normal, and the face residual (and, for the top
// group, the penalty matrix).  A second kernel adds the face terms into the u-step's residual and CSR values,
// one thread per face node, over the node's faces in group order (side, then top) and face order: the order of
// the reference's VecAdd / MatAdd calls, after every phase-field term.
//
// Face shapes:
//   B1_2 (2D lines, mesh/ElementTypes/Bezier/B1_2.cpp:55-105): N = Nbase ElemData^T, J = G X, tangent t = J/|J|,
//     w = w_q |t . J|, normal (t_y, -t_x);
//   NURBS3_Plane2 (3D faces, NURBS3_Plane2.cpp getShapeGrads / getNormals): rational N = W CB / wFun with
//     CB = ElemData Nbase, G_xi by the quotient rule, J = G_xi^T X (2x3), normal t1 x t2, w = w_q |t1 x t2|.
// getNormals flips a normal when a step of 1e-3 |x| along it brings the point closer to the origin.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {
namespace {

struct FaceIp {
  double N[9];
  double w;
  double n[3];
  double Xip[3];
};

// Shape values, weight and normal of face f at face ip (i, j) (j = 0 for 2D lines).
__device__ void face_ip(const FaceParams& p, const double (*Xf)[3], const double* Wf, const double* C, int i, int j,
                        FaceIp& o) {
  const Rule& R = p.rule;
  if (p.dim == 2) {
    double GB[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double sN = 0, sG = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) { sN += R.B[i][k] * C[a * 3 + k]; sG += R.dB[i][k] * C[a * 3 + k]; }
      o.N[a] = sN; GB[a] = sG;
    }
    double J0 = 0, J1 = 0, P0 = 0, P1 = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      J0 += GB[a] * Xf[a][0]; J1 += GB[a] * Xf[a][1];
      P0 += o.N[a] * Xf[a][0]; P1 += o.N[a] * Xf[a][1];
    }
    const double len = sqrt(J0 * J0 + J1 * J1);
    const double t0 = J0 / len, t1 = J1 / len;
    o.w = R.w1[i] * fabs(t0 * J0 + t1 * J1);
    const double nl = sqrt(t1 * t1 + t0 * t0);
    o.n[0] = t1 / nl; o.n[1] = -t0 / nl; o.n[2] = 0;
    o.Xip[0] = P0; o.Xip[1] = P1; o.Xip[2] = 0;
  } else {
    double CB[9], GB[9][2];
    double wFun = 0, dW0 = 0, dW1 = 0;
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      double sN = 0, s0 = 0, s1 = 0;
#pragma unroll
      for (int k = 0; k < 9; ++k) {   // Nbase(k = kx + 3 ky) = B(x) B(y) (KronProd, x fastest)
        const int kx = k % 3, ky = k / 3;
        const double c = C[a * 9 + k];
        sN += c * (R.B[i][kx] * R.B[j][ky]);
        s0 += c * (R.dB[i][kx] * R.B[j][ky]);
        s1 += c * (R.B[i][kx] * R.dB[j][ky]);
      }
      CB[a] = sN; GB[a][0] = s0; GB[a][1] = s1;
      wFun += sN * Wf[a];
    }
#pragma unroll
    for (int a = 0; a < 9; ++a) { dW0 += GB[a][0] * Wf[a]; dW1 += GB[a][1] * Wf[a]; }
    double J[2][3] = {{0, 0, 0}, {0, 0, 0}}, P[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      o.N[a] = Wf[a] * CB[a] / wFun;
      const double g0 = Wf[a] * (GB[a][0] / wFun - CB[a] * dW0 / wFun / wFun);
      const double g1 = Wf[a] * (GB[a][1] / wFun - CB[a] * dW1 / wFun / wFun);
#pragma unroll
      for (int e = 0; e < 3; ++e) { J[0][e] += g0 * Xf[a][e]; J[1][e] += g1 * Xf[a][e]; P[e] += o.N[a] * Xf[a][e]; }
    }
    const double c0 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    const double c1 = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    const double c2 = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const double nn = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    o.w = R.w1[i] * R.w1[j] * nn;
    o.n[0] = c0 / nn; o.n[1] = c1 / nn; o.n[2] = c2 / nn;
    o.Xip[0] = P[0]; o.Xip[1] = P[1]; o.Xip[2] = P[2];
  }
  // outward normal (getNormals): flip when a small step along it moves the point toward the origin
  const double d1 = sqrt(o.Xip[0] * o.Xip[0] + o.Xip[1] * o.Xip[1] + o.Xip[2] * o.Xip[2]);
  const double s = d1 * 1e-3;
  const double q0 = o.Xip[0] + o.n[0] * s, q1 = o.Xip[1] + o.n[1] * s, q2 = o.Xip[2] + o.n[2] * s;
  const double d2 = sqrt(q0 * q0 + q1 * q1 + q2 * q2);
  if (d1 > d2) { o.n[0] = -o.n[0]; o.n[1] = -o.n[1]; o.n[2] = -o.n[2]; }
}

__device__ __forceinline__ int64_t dof_at(const DofMap& dm, int kind, int32_t node) {
  return (int64_t)dm.base[kind] + dm.node_rank[node];
}

__global__ void __launch_bounds__(128) k_face_loads(const FaceParams p) {
  const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f >= p.nside + p.ntop) return;
  const int nfn = p.nfn, dim = p.dim, nq1 = 3, nq2 = (dim == 2) ? 1 : 3;
  const bool top = f >= p.nside;
  const int32_t* nodes = p.faces + f * nfn;
  const double* C = p.C + f * nfn * nfn;
  double Xf[9][3], Wf[9], Uf[9], Pf[9];
  const int ctop = dim - 1;
  for (int a = 0; a < nfn; ++a) {
    const int32_t nd = nodes[a];
    for (int e = 0; e < 3; ++e) Xf[a][e] = (e < dim) ? p.X[(int64_t)nd * dim + e] : 0.0;
    Wf[a] = p.W ? p.W[nd] : 1.0;
    Uf[a] = top ? p.ucur[dof_at(p.dm, IFEM_DOF_UX + ctop, nd)] : 0.0;
    Pf[a] = (!top && p.phase) ? p.phase[dof_at(p.dm, IFEM_DOF_PHASE, nd)] : 0.0;
  }
  double F[3][9];
  for (int c = 0; c < 3; ++c) for (int a = 0; a < 9; ++a) F[c][a] = 0.0;
  double* K = top ? p.K + (f - p.nside) * nfn * nfn : nullptr;
  if (top) for (int i = 0; i < nfn * nfn; ++i) K[i] = 0.0;
  double area = 0, fext = 0, uz = 0;
  const bool pressure = p.t < 0.0;
  const double uTarget = p.u0 + p.t * p.du;
  for (int j = 0; j < nq2; ++j) for (int i = 0; i < nq1; ++i) {
    FaceIp ip;
    face_ip(p, Xf, Wf, C, i, j, ip);
    if (!top) {
      double Dam = 1.0;
      if (p.phase) {   // GenericDamageFunction(QuadraticDamageNR)
        double phi = 0;
        for (int a = 0; a < nfn; ++a) phi += ip.N[a] * Pf[a];
        double d1, d2;
        damage_function(phi, IFEM_DAM_QUADRATIC_NR, 0.0, 2.0, Dam, d1, d2);
      }
      const double sc = Dam * ip.w;
      for (int c = 0; c < dim; ++c)
        for (int a = 0; a < nfn; ++a) F[c][a] += sc * (ip.N[a] * ip.n[c]) * p.p0;
    } else {
      double ut = 0;
      for (int a = 0; a < nfn; ++a) ut += ip.N[a] * Uf[a];
      if (pressure) {
        for (int a = 0; a < nfn; ++a) F[ctop][a] += ip.w * ip.N[a] * p.p0;
        fext += -ip.w * p.p0;
      } else {
        const double pExt = p.penalty * (ut - uTarget);
        const double wk = ip.w * p.penalty;
        for (int a = 0; a < nfn; ++a) {
          F[ctop][a] += ip.w * ip.N[a] * pExt;
          for (int b = 0; b < nfn; ++b) K[a * nfn + b] += wk * ip.N[a] * ip.N[b];
        }
        fext += -ip.w * pExt;
      }
      area += ip.w;
      uz += ip.w * ut;
    }
  }
  double* Fo = p.F + f * dim * nfn;
  for (int c = 0; c < dim; ++c) for (int a = 0; a < nfn; ++a) Fo[c * nfn + a] = F[c][a];
  if (top) {
    const int64_t t = f - p.nside;
    p.sums[t] = area;
    p.sums[p.ntop + t] = fext;
    p.sums[2 * p.ntop + t] = uz;
  }
}

// CSR positions of the top faces' (u_top a, u_top b) pairs, by binary search in each row's sorted columns.
__global__ void k_face_kpos(const FaceParams p, int64_t* kpos) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int nfn = p.nfn;
  if (i >= p.ntop * nfn * nfn) return;
  const int64_t t = i / (nfn * nfn);
  const int a = (int)(i / nfn % nfn), b = (int)(i % nfn);
  const int32_t* nodes = p.faces + (p.nside + t) * nfn;
  const int kind = IFEM_DOF_UX + p.dim - 1;
  const int64_t row = dof_at(p.dm, kind, nodes[a]);
  const int32_t col = (int32_t)dof_at(p.dm, kind, nodes[b]);
  int64_t lo = p.rowptr[row], hi = p.rowptr[row + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (p.colidx[mid] < col) lo = mid + 1; else hi = mid;
  }
  if (lo < p.rowptr[row + 1] && p.colidx[lo] == col) {
    kpos[i] = lo;
  } else {
    kpos[i] = -1;
    atomicAdd(p.err, 1ull);
  }
}

template <typename VT>
__global__ void __launch_bounds__(128) k_face_gather(const FaceParams p) {
  const int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (u >= p.nnodes) return;
  const int32_t nd = p.node[u];
  const int nfn = p.nfn, dim = p.dim;
  const int ctop = dim - 1;
  VT* vals = reinterpret_cast<VT*>(p.vals);
  for (int i = p.inc_ptr[u]; i < p.inc_ptr[u + 1]; ++i) {
    const int e = p.inc[i];
    const int64_t f = e / nfn;
    const int a = e % nfn;
    const double* Fo = p.F + f * dim * nfn;
    for (int c = 0; c < dim; ++c) p.f[dof_at(p.dm, IFEM_DOF_UX + c, nd)] += Fo[c * nfn + a];
    if (f >= p.nside && !(p.t < 0.0)) {
      const int64_t t = f - p.nside;
      const double* K = p.K + t * nfn * nfn + a * nfn;
      const int64_t* pos = p.kpos + t * nfn * nfn + a * nfn;
      for (int b = 0; b < nfn; ++b) vals[pos[b]] = (VT)((double)vals[pos[b]] + K[b]);
    }
  }
  (void)ctop;
}

}  // namespace

void launch_face_kpos(const FaceParams& p, int64_t* kpos, cudaStream_t s) {
  const int64_t n = p.ntop * p.nfn * p.nfn;
  if (n > 0) k_face_kpos<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(p, kpos);
}

void launch_face_loads(const FaceParams& p, cudaStream_t s) {
  const int64_t n = p.nside + p.ntop;
  if (n > 0) k_face_loads<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(p);
}

void launch_face_gather(const FaceParams& p, cudaStream_t s) {
  if (p.nnodes <= 0) return;
  const unsigned g = (unsigned)((p.nnodes + 127) / 128);
  if (p.vals_f32) k_face_gather<float><<<g, 128, 0, s>>>(p);
  else k_face_gather<double><<<g, 128, 0, s>>>(p);
}

}  // namespace ifem
