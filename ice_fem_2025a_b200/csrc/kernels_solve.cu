// Building blocks of the device Krylov solve of the constrained system K_con dx = f_con (restarted GMRES with a
// diagonal preconditioner; the iteration itself runs on the host side of this library, in host.cu).
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

// out[j] = V_j . w for j < k (V column j at V + j * ld), one CTA per j
__global__ void __launch_bounds__(kRedThreads) k_dots(int64_t n, const double* V, int64_t ld, const double* w,
                                                      double* out) {
  __shared__ double red[kRedThreads / 32];
  const double* vj = V + (int64_t)blockIdx.x * ld;
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

void launch_dots(int64_t n, const double* V, int64_t ld, int k, const double* w, double* out, cudaStream_t s) {
  if (k > 0) k_dots<<<(unsigned)k, kRedThreads, 0, s>>>(n, V, ld, w, out);
}

void launch_comb(int64_t n, const double* V, int64_t ld, const double* c, int k, double a, double* w, cudaStream_t s) {
  if (n > 0 && k > 0) k_comb<<<blocks_for(n, 256), 256, 0, s>>>(n, V, ld, c, k, a, w);
}

void launch_scale(int64_t n, double a, const double* x, const double* d, double* y, cudaStream_t s) {
  if (n > 0) k_scale<<<blocks_for(n, 256), 256, 0, s>>>(n, a, x, d, y);
}

void launch_sub(int64_t n, const double* b, const double* y, double* r, cudaStream_t s) {
  if (n > 0) k_sub<<<blocks_for(n, 256), 256, 0, s>>>(n, b, y, r);
}

}  // namespace ifem
