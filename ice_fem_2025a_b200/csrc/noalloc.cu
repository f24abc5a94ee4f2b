// Crack length of a phase field without any allocation by the library.
//
// Who needs this: a caller whose device memory is owned by someone else cannot let a library call
// cudaMalloc.  Examples are a host solver that hands out all device memory from its own pool
// (PETSc-style memory management, or a process that fixes its footprint at start-up), and a
// monitoring loop between time steps.  For the monitoring loop, a cudaMalloc/cudaFree pair would add a
// device-wide synchronisation.  The caller passes every input and the output as device pointers.
// The per-element partial sums go into a fixed array in this file; the library holds it for as long
// as it is loaded.
//
// It computes the same quantity as the phase-step assembly's crack length (LCrack += gamma * w,
// PhaseField.cpp:540,650, crack density of PhaseFieldUtil.cpp:185-221).  Per element, the ip
// contributions are summed in ip order; the element sums are then reduced in a fixed order.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

// 2^21 element partial sums (16 MiB): the largest mesh this entry point accepts.
constexpr int64_t kNoAllocMaxElems = int64_t(1) << 21;
static __device__ __align__(256) double g_crack_scratch[kNoAllocMaxElems];

namespace {

constexpr int kCWarps = 4;

template <int DIM>
struct CSm {
  static constexpr int NEN = ElemTraits<DIM>::NEN;
  ElemSm<DIM, true> e;
  double Ph[NEN];
  double lc[NEN];
};

template <int DIM>
__global__ void __launch_bounds__(128) k_crack_length_elems(Geo geo, Rule rule, const double* phase, double l,
                                                            int dist, double* partial) {
  constexpr int NEN = ElemTraits<DIM>::NEN, NIP = NEN, EPW = (DIM == 2) ? 3 : 1;
  __shared__ CSm<DIM> sm[kCWarps * EPW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / NIP;
  const int q = lane - sub * NIP;
  const int64_t el = ((int64_t)blockIdx.x * kCWarps + warp) * EPW + sub;
  const bool act = (sub < EPW) && (el < geo.nel);
  CSm<DIM>& s = sm[warp * EPW + (sub < EPW ? sub : 0)];
  if (act) {
    fill_elem<DIM, true>(s.e, geo, rule, el, q, NIP);
    s.Ph[q] = phase[geo.conn[el * NEN + q]];
  }
  __syncwarp();
  if (act) {
    IpGeo<DIM> g;
    ip_geometry<DIM, true>(s.e, rule, q, g);
    double phi = 0, gphi[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) gphi[d] = 0;
    for (int a = 0; a < NEN; ++a) {
      double N, G[DIM];
      shape_at<DIM, true>(s.e, rule, g, q, a, N, G);
      phi += N * s.Ph[a];
#pragma unroll
      for (int d = 0; d < DIM; ++d) gphi[d] += G[d] * s.Ph[a];
    }
    double dGdG = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) dGdG += gphi[d] * gphi[d];
    double gamma = 0;
    switch (dist) {
      case IFEM_DIST_QUADRATIC: gamma = 1.0 / (2.0 * l) * (phi * phi + l * l * dGdG); break;
      case IFEM_DIST_LINEAR: gamma = 3.0 / (8.0 * l) * (phi + l * l * dGdG); break;
      case IFEM_DIST_LINEAR2: gamma = 1.0 / (4.0 * l) * (2.0 * phi + l * l * dGdG); break;
      case IFEM_DIST_LOCAL: gamma = 1.0 / l * (phi * phi); break;
      case IFEM_DIST_CZM: gamma = 1.0 / (3.141592 * l) * (2.0 * phi - phi * phi + l * l * dGdG); break;
      default: break;
    }
    s.lc[q] = gamma * g.w;
  }
  __syncwarp();
  if (act && q == 0) {
    double sum = 0;
    for (int qq = 0; qq < NIP; ++qq) sum += s.lc[qq];
    partial[el] = sum;
  }
}

std::mutex g_scratch_mutex;
void* g_scratch_ptr[64] = {};

}  // namespace
}  // namespace ifem

extern "C" int ifem_crack_length_noalloc(int32_t dim, int64_t n_elems, const double* coords,
                                         const double* node_weights, const int32_t* elems,
                                         const double* elem_kron, const double* phase, double length_scale,
                                         int32_t distribution, double* length_out, void* stream) {
  using namespace ifem;
  if ((dim != 2 && dim != 3) || n_elems < 0 || !coords || !elems || !elem_kron || !phase || !length_out)
    return IFEM_ERR_INVALID;
  if (!(length_scale > 0)) return IFEM_ERR_INVALID;
  if (!(distribution == IFEM_DIST_QUADRATIC || distribution == IFEM_DIST_LINEAR || distribution == IFEM_DIST_LINEAR2 ||
        distribution == IFEM_DIST_LOCAL || distribution == IFEM_DIST_CZM))
    return IFEM_ERR_UNSUPPORTED;
  if (n_elems > kNoAllocMaxElems) return IFEM_ERR_CAPACITY;   // the fixed scratch holds 2^21 elements
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return IFEM_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &capture) != cudaSuccess) return IFEM_ERR_CUDA;
  void* scratch = nullptr;
  {
    // The array's device address, looked up with this device current.  Outside stream capture every call
    // looks it up again (a cheap query, no allocation), so a cudaDeviceReset or a new context on this
    // ordinal, which reloads the module and may move the array, never leaves a stale address behind.  A call
    // inside a stream capture uses the address of the last lookup on this device; a capture before any
    // lookup on the device is refused.
    std::lock_guard<std::mutex> lk(g_scratch_mutex);
    if (capture == cudaStreamCaptureStatusNone) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_crack_scratch) != cudaSuccess || !p) return IFEM_ERR_CUDA;
      g_scratch_ptr[dev] = p;
    } else if (!g_scratch_ptr[dev]) {
      return IFEM_ERR_STATE;
    }
    scratch = g_scratch_ptr[dev];
  }
  Geo geo{};
  geo.dim = dim; geo.nen = dim == 2 ? 9 : 27; geo.nip = geo.nen; geo.kron = 1;
  geo.nel = n_elems; geo.nn = 0;
  geo.X = coords; geo.W = dim == 3 ? node_weights : nullptr; geo.conn = elems; geo.ext = elem_kron;
  geo.emat = nullptr; geo.mats = nullptr;
  Rule rule;
  build_rule(3, dim, rule);
  double* partial = static_cast<double*>(scratch);
  if (n_elems > 0) {
    const int64_t per_block = (int64_t)kCWarps * (dim == 2 ? 3 : 1);
    const unsigned blocks = (unsigned)((n_elems + per_block - 1) / per_block);
    if (dim == 2) k_crack_length_elems<2><<<blocks, 128, 0, s>>>(geo, rule, phase, length_scale, distribution, partial);
    else k_crack_length_elems<3><<<blocks, 128, 0, s>>>(geo, rule, phase, length_scale, distribution, partial);
  }
  launch_reduce_sum(partial, n_elems, length_out, s);
  return cudaGetLastError() == cudaSuccess ? IFEM_OK : IFEM_ERR_CUDA;
}
