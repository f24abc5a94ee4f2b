// One-component row gather (phase and thermal steps), a translation unit of its own so that it compiles as
// whole-program device code (the multi-component gathers stay relocatable; see build.py).

#include <cuda_runtime.h>
#include <cstdint>

#include "icefem_internal.h"

namespace ifem {

namespace {

// One-component rows (phase and thermal steps): the row blocks are short (NEN values, 112 B for the FP32 hex), so
// instead of one bulk copy per incidence the warp stages all of a node's row blocks with coalesced 16-byte loads,
// every lane several independent ones, and then adds them into the shared accumulator in ascending element order
// (the same order and precision as the bulk-copy kernel, so the results are identical).
constexpr int kGDWarps = 4;

template <int NEN, typename KT, typename MT>
struct GDLayout {
  static constexpr int KB = ke_block(1, NEN);
  static constexpr int V16 = KB * (int)sizeof(KT) / 16;            // 16-byte pieces per row block
  static_assert(KB * (int)sizeof(KT) % 16 == 0, "row blocks are whole 16-byte pieces");
  static constexpr int STAGE = 32 * KB * (int)sizeof(KT);          // up to 32 incidences
  static constexpr int EMB = 32 * 32 * (int)sizeof(MT);
  __host__ __device__ static size_t warp_bytes(int acc_stride) {
    return (((size_t)STAGE + EMB + (size_t)acc_stride * sizeof(KT)) + 127) / 128 * 128;
  }
};

template <int NEN, typename KT, typename VT, typename MT>
__global__ void __launch_bounds__(kGDWarps * 32) k_gather_direct1(const GParams p) {
  using L = GDLayout<NEN, KT, MT>;
  constexpr int KB = L::KB, V16 = L::V16;
  constexpr int PER = (32 * V16 + 31) / 32;                        // pieces per lane for 32 incidences
  extern __shared__ __align__(128) unsigned char gsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = p.node0 + (int64_t)blockIdx.x * kGDWarps + warp;
  if (r >= p.n_nodes) return;                                       // whole warp; no CTA-wide barrier below
  const int k0 = p.inc_ptr[r], nk = p.inc_ptr[r + 1] - k0;          // nk <= 32 (checked on the host)
  if (nk == 0) return;
  unsigned char* wb = gsm + (size_t)warp * L::warp_bytes(p.acc_stride);
  float4* stage = reinterpret_cast<float4*>(wb);
  MT* em_s = reinterpret_cast<MT*>(wb + L::STAGE);
  KT* acc = reinterpret_cast<KT*>(wb + L::STAGE + L::EMB);
  const int deg = p.nbr_ptr[r + 1] - p.nbr_ptr[r];
  const int my_el = lane < nk ? p.inc_el[k0 + lane] : 0;
  const int my_loc = lane < nk ? (int)p.inc_loc[k0 + lane] : 0;
  const float4* Ke = reinterpret_cast<const float4*>(p.Ke);
  // every lane issues its loads before any use: the incidence's row block and the position rows
  float4 v[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int i = lane + 32 * j, k = i / V16, c = i - k * V16;
    const int el = __shfl_sync(0xffffffffu, my_el, k < 32 ? k : 0);
    const int a1 = __shfl_sync(0xffffffffu, my_loc, k < 32 ? k : 0);
    v[j] = k < nk ? __ldg(Ke + ((int64_t)el * NEN + a1) * V16 + c) : make_float4(0, 0, 0, 0);
  }
  const MT* em_g = reinterpret_cast<const MT*>(p.inc_em) + (size_t)k0 * 32;
  for (int i = lane; i < nk * 32; i += 32) em_s[i] = em_g[i];
  for (int i = lane; i < deg; i += 32) acc[i] = (KT)0;
  // residual: element-order sums of the incident elements' entries (lane k loads incidence k)
  const double fv = lane < nk ? p.Fe1[(int64_t)my_el * NEN + my_loc] : 0.0;
  const double fv2 = (p.Fe2 && lane < nk) ? p.Fe2[(int64_t)my_el * NEN + my_loc] : 0.0;
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int i = lane + 32 * j;
    if (i < nk * V16) stage[i] = v[j];
  }
  __syncwarp();
  const KT* blk = reinterpret_cast<const KT*>(stage);
  for (int k = 0; k < nk; ++k) {                                    // ascending element order
    if (lane < NEN) acc[(int)em_s[k * 32 + lane]] += blk[k * KB + lane];
    __syncwarp();
  }
  VT* vals = reinterpret_cast<VT*>(p.vals);
  const int64_t off = p.rowptr[p.row_base[0] + r];
  for (int i = lane; i < deg; i += 32) vals[off + i] = (VT)acc[i];
  double sum = 0.0;
  for (int k = 0; k < nk; ++k) sum += __shfl_sync(0xffffffffu, fv, k);
  if (p.Fe2)
    for (int k = 0; k < nk; ++k) sum += __shfl_sync(0xffffffffu, fv2, k);
  if (lane == 0) p.f[p.row_base[0] + r] = sum;
}

template <int NEN, typename KT, typename VT>
bool gather_direct1(const GParams& p, cudaStream_t s) {
  const size_t per_warp = p.emap16 ? GDLayout<NEN, KT, uint16_t>::warp_bytes(p.acc_stride)
                                   : GDLayout<NEN, KT, uint8_t>::warp_bytes(p.acc_stride);
  const size_t smem = per_warp * kGDWarps;
  if (smem > 200 * 1024) return false;
  void (*k)(const GParams) = p.emap16 ? k_gather_direct1<NEN, KT, VT, uint16_t> : k_gather_direct1<NEN, KT, VT, uint8_t>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned blocks = (unsigned)((p.n_nodes - p.node0 + kGDWarps - 1) / kGDWarps);
  k<<<blocks, kGDWarps * 32, smem, s>>>(p);
  return true;
}

}  // namespace

// false when the layout does not qualify (the caller then uses another gather)
bool launch_gather_direct1(const GParams& p, cudaStream_t s) {
  if (p.nc != 1) return false;
  if (p.nen == 9)
    return p.ke_f32 ? (p.vals_f32 ? gather_direct1<9, float, float>(p, s) : gather_direct1<9, float, double>(p, s))
                    : (p.vals_f32 ? gather_direct1<9, double, float>(p, s) : gather_direct1<9, double, double>(p, s));
  return p.ke_f32 ? (p.vals_f32 ? gather_direct1<27, float, float>(p, s) : gather_direct1<27, float, double>(p, s))
                  : (p.vals_f32 ? gather_direct1<27, double, float>(p, s) : gather_direct1<27, double, double>(p, s));
}

}  // namespace ifem
