// Building blocks of the device Krylov solve of the constrained system K_con dx = f_con (restarted GMRES with a
// node-block Jacobi preconditioner; the iteration itself runs on the host side of this library, in host.cu).
//
// All reductions are deterministic: each dot product is one CTA's fixed-order tree over a fixed grid-stride
// partition, so a solve repeated on the same inputs gives the same iterates bit for bit.

#include <cuda_runtime.h>
#include <cstdint>

#include "icefem_internal.h"

namespace ifem {

namespace {

constexpr int kRedThreads = 512;

// y = K x, one warp per row; values in the matrix's precision, vectors and sums in FP64
template <typename VT>
__global__ void __launch_bounds__(256) k_spmv(int64_t n, const int64_t* rp, const int32_t* ci, const VT* v,
                                              const double* x, double* y) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int64_t k = rp[row] + lane; k < rp[row + 1]; k += 32) s += (double)v[k] * x[ci[k]];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

// dinv = 1 / diag(K) (1 where the diagonal is zero or absent)
template <typename VT>
__global__ void k_diag_inv(int64_t n, const int64_t* rp, const int32_t* ci, const VT* v, double* dinv) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  double d = 0.0;
  for (int64_t k = rp[row]; k < rp[row + 1]; ++k)
    if (ci[k] == row) d = (double)v[k];
  dinv[row] = d != 0.0 ? 1.0 / d : 1.0;
}

// out[j] = V_j . w for j < k (V column j at V + j * ld), one CTA per j; a CTA with j = k (launched when the
// caller asks for it) gives out[k] = w . w
__global__ void __launch_bounds__(kRedThreads) k_dots(int64_t n, const double* V, int64_t ld, int k, const double* w,
                                                      double* out) {
  __shared__ double red[kRedThreads / 32];
  const double* vj = (int)blockIdx.x < k ? V + (int64_t)blockIdx.x * ld : w;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kRedThreads) s += vj[i] * w[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kRedThreads / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) out[blockIdx.x] = t;
  }
}

// w += a * sum_{j<k} c_j V_j   (c in device memory)
__global__ void k_comb(int64_t n, const double* V, int64_t ld, const double* c, int k, double a, double* w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < k; ++j) s += c[j] * V[(int64_t)j * ld + i];
  w[i] += a * s;
}

// y = a * x * d (d may be null: y = a x)
__global__ void k_scale(int64_t n, double a, const double* x, const double* d, double* y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = a * x[i] * (d ? d[i] : 1.0);
}

// r = b - y
__global__ void k_sub(int64_t n, const double* b, const double* y, double* r) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  r[i] = b[i] - y[i];
}

// node-block Jacobi: the free rows of one node (its components) form a block of at most 3 x 3.  tbl[r * nc + c] =
// free row of component c of node rank r, or -1 (constrained)
__global__ void k_block_table(int64_t nfree, const int32_t* row_src, int64_t nu, int nc, int32_t* tbl) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nfree) return;
  const int64_t dof = row_src[i];
  tbl[(dof % nu) * nc + dof / nu] = (int32_t)i;
}

// Binv[r] = inverse of the node block (rows/cols in component order, unused ones 0); a singular block falls back
// to the inverse of its diagonal (1 where that is zero)
template <typename VT>
__global__ void k_block_inv(int64_t nu, int nc, const int32_t* tbl, const int64_t* rp, const int32_t* ci,
                            const VT* v, double* Binv) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nu) return;
  int idx[3] = {-1, -1, -1};
  for (int c = 0; c < nc; ++c) idx[c] = tbl[r * nc + c];
  double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, I[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int a = 0; a < nc; ++a) {
    if (idx[a] < 0) { A[a][a] = 1.0; continue; }
    for (int64_t k = rp[idx[a]]; k < rp[idx[a] + 1]; ++k)
      for (int b = 0; b < nc; ++b)
        if (idx[b] >= 0 && ci[k] == idx[b]) A[a][b] = (double)v[k];
  }
  double D[3] = {A[0][0], A[1][1], A[2][2]};
  bool ok = true;
  for (int k = 0; k < nc && ok; ++k) {               // Gauss-Jordan with partial pivoting
    int p = k;
    for (int i = k + 1; i < nc; ++i) if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
    if (A[p][k] == 0.0) { ok = false; break; }
    if (p != k) for (int j = 0; j < 3; ++j) {
      double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t;
      t = I[k][j]; I[k][j] = I[p][j]; I[p][j] = t;
    }
    const double ip = 1.0 / A[k][k];
    for (int j = 0; j < 3; ++j) { A[k][j] *= ip; I[k][j] *= ip; }
    for (int i = 0; i < nc; ++i) {
      if (i == k) continue;
      const double f = A[i][k];
      for (int j = 0; j < 3; ++j) { A[i][j] -= f * A[k][j]; I[i][j] -= f * I[k][j]; }
    }
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      Binv[r * 9 + a * 3 + b] = ok ? I[a][b] : (a == b && a < nc ? (D[a] != 0.0 ? 1.0 / D[a] : 1.0) : 0.0);
}

// y = Binv x per node (y may be x)
__global__ void k_block_apply(int64_t nu, int nc, const int32_t* tbl, const double* Binv, const double* x, double* y) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nu) return;
  int idx[3] = {-1, -1, -1};
  double in[3] = {0, 0, 0};
  for (int c = 0; c < nc; ++c) { idx[c] = tbl[r * nc + c]; if (idx[c] >= 0) in[c] = x[idx[c]]; }
  for (int a = 0; a < nc; ++a) {
    if (idx[a] < 0) continue;
    double s = 0.0;
    for (int b = 0; b < nc; ++b) s += Binv[r * 9 + a * 3 + b] * in[b];
    y[idx[a]] = s;
  }
}

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_spmv(int64_t n, const int64_t* rp, const int32_t* ci, const void* v, int f32, const double* x, double* y,
                 cudaStream_t s) {
  if (n == 0) return;
  if (f32) k_spmv<float><<<blocks_for(n * 32, 256), 256, 0, s>>>(n, rp, ci, (const float*)v, x, y);
  else k_spmv<double><<<blocks_for(n * 32, 256), 256, 0, s>>>(n, rp, ci, (const double*)v, x, y);
}

void launch_diag_inv(int64_t n, const int64_t* rp, const int32_t* ci, const void* v, int f32, double* dinv,
                     cudaStream_t s) {
  if (n == 0) return;
  if (f32) k_diag_inv<float><<<blocks_for(n, 256), 256, 0, s>>>(n, rp, ci, (const float*)v, dinv);
  else k_diag_inv<double><<<blocks_for(n, 256), 256, 0, s>>>(n, rp, ci, (const double*)v, dinv);
}

void launch_dots(int64_t n, const double* V, int64_t ld, int k, const double* w, double* out, cudaStream_t s,
                 bool with_norm) {
  const int blocks = k + (with_norm ? 1 : 0);
  if (blocks > 0) k_dots<<<(unsigned)blocks, kRedThreads, 0, s>>>(n, V, ld, k, w, out);
}

void launch_comb(int64_t n, const double* V, int64_t ld, const double* c, int k, double a, double* w, cudaStream_t s) {
  if (n > 0 && k > 0) k_comb<<<blocks_for(n, 256), 256, 0, s>>>(n, V, ld, c, k, a, w);
}

void launch_scale(int64_t n, double a, const double* x, const double* d, double* y, cudaStream_t s) {
  if (n > 0) k_scale<<<blocks_for(n, 256), 256, 0, s>>>(n, a, x, d, y);
}

void launch_block_setup(int64_t nfree, const int32_t* row_src, int64_t nu, int nc, int32_t* tbl, const int64_t* rp,
                        const int32_t* ci, const void* v, int f32, double* Binv, cudaStream_t s) {
  if (nu == 0) return;
  cudaMemsetAsync(tbl, 0xff, (size_t)nu * nc * sizeof(int32_t), s);   // -1: constrained
  if (nfree > 0) k_block_table<<<blocks_for(nfree, 256), 256, 0, s>>>(nfree, row_src, nu, nc, tbl);
  if (f32) k_block_inv<float><<<blocks_for(nu, 128), 128, 0, s>>>(nu, nc, tbl, rp, ci, (const float*)v, Binv);
  else k_block_inv<double><<<blocks_for(nu, 128), 128, 0, s>>>(nu, nc, tbl, rp, ci, (const double*)v, Binv);
}

void launch_block_apply(int64_t nu, int nc, const int32_t* tbl, const double* Binv, const double* x, double* y,
                        cudaStream_t s) {
  if (nu > 0) k_block_apply<<<blocks_for(nu, 256), 256, 0, s>>>(nu, nc, tbl, Binv, x, y);
}

void launch_sub(int64_t n, const double* b, const double* y, double* r, cudaStream_t s) {
  if (n > 0) k_sub<<<blocks_for(n, 256), 256, 0, s>>>(n, b, y, r);
}

}  // namespace ifem
