// Constraint application on the device CSR (Physics::Constraint, physics.cpp:314-362) and the state update
// (Physics::UpdateState, physics.cpp:408-419).
//
//   k_cons_cv     C_v = value - state(dof) for the constrained dofs (Constrainer.cpp:112-118).
//   k_constrain   one warp per free row: compacts the row's free columns into K_con = U^T K U (ballot +
//                 popc gives each kept entry its position) and forms f_con = -(f_r + sum_j K_rj x_j) with
//                 x = -C C_v, adding the products of the constrained columns in column order.  The free
//                 columns contribute K_rj * 0 to the reference's MatMultAdd, which leaves the sum unchanged,
//                 so they are skipped.  Products and sums are rounded separately (no FMA contraction),
//                 as in a compiled MatMultAdd without contraction.
//   k_update      u += dx (free dofs) or u += C_v (constrained dofs), one thread per dof.
// The kernels stream K once (HBM-bound); nothing is accumulated across warps, so results are deterministic.

#include <cuda_runtime.h>
#include <cstdint>

#include "icefem_internal.h"

namespace ifem {

namespace {

__global__ void k_cons_cv(const int64_t* con_dof, const double* con_val, int64_t n, const double* u, double* cv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cv[i] = con_val[i] - u[con_dof[i]];
}

constexpr int kCWarps = 8;

template <typename VT>
__global__ void __launch_bounds__(256) k_constrain(const ConsParams p) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * kCWarps + (threadIdx.x >> 5);
  if (i >= p.n_free) return;
  const int64_t r = p.row_src[i];
  double s = p.f[r];
  if (p.vals) {
    const VT* vals = reinterpret_cast<const VT*>(p.vals);
    VT* out_vals = reinterpret_cast<VT*>(p.vals_con);
    const int64_t b = p.rowptr[r], e = p.rowptr[r + 1];
    int64_t out = p.rowptr_con[i];
    for (int64_t j0 = b; j0 < e; j0 += 32) {
      const int64_t j = j0 + lane;
      const bool in = j < e;
      int m = 0;
      VT v = VT(0);
      if (in) { m = p.fmap[p.colidx[j]]; v = vals[j]; }
      const unsigned fr = __ballot_sync(0xffffffffu, in && m >= 0);
      const unsigned cn = __ballot_sync(0xffffffffu, in && m < 0);
      if (p.want_matrix && in && m >= 0) out_vals[out + __popc(fr & ((1u << lane) - 1u))] = v;
      out += __popc(fr);
      const double prod = (in && m < 0) ? __dmul_rn((double)v, -p.cv[-1 - m]) : 0.0;
      unsigned mask = cn;
      while (mask) {                      // constrained columns of this chunk, in column order
        const int src = __ffs(mask) - 1;
        s = __dadd_rn(s, __shfl_sync(0xffffffffu, prod, src));
        mask &= mask - 1u;
      }
    }
  }
  if (lane == 0) p.f_con[i] = -s;
}

__global__ void k_update(const int32_t* fmap, int64_t n, const double* dx, const double* cv, double* u) {
  const int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  const int m = fmap[d];
  u[d] = __dadd_rn(u[d], m >= 0 ? dx[m] : cv[-1 - m]);
}

}  // namespace

void launch_cons_cv(const int64_t* con_dof, const double* con_val, int64_t n, const double* u, double* cv,
                    cudaStream_t s) {
  if (n > 0) k_cons_cv<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(con_dof, con_val, n, u, cv);
}

void launch_constrain(const ConsParams& p, cudaStream_t s) {
  if (p.n_free == 0) return;
  const unsigned blocks = (unsigned)((p.n_free + kCWarps - 1) / kCWarps);
  if (p.vals_f32) k_constrain<float><<<blocks, 32 * kCWarps, 0, s>>>(p);
  else k_constrain<double><<<blocks, 32 * kCWarps, 0, s>>>(p);
}

void launch_update_state(const int32_t* fmap, int64_t n, const double* dx, const double* cv, double* u,
                         cudaStream_t s) {
  if (n > 0) k_update<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(fmap, n, dx, cv, u);
}

}  // namespace ifem
