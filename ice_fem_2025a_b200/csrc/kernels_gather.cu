// Deterministic node-row gather of element matrices into the device CSR, fed by bulk asynchronous copies.
//
// One warp owns the CSR rows of one mesh node (all its components) and adds the row blocks of the node's
// incident elements in ascending element order, the order in which serial MatSetValues(ADD_VALUES)
// accumulates them (math.cpp:301-331).  Sums are taken in the element matrices' precision: FP64 element
// matrices give the same result, bit for bit, as a serial element-order sum in FP64; FP32 ones (the FP32 and
// tensor-core tangents) are summed in FP32 in the same order, so the result stays deterministic, and the 27
// or fewer additions per entry add about 1e-7 relative to an FP32-accurate tangent, without one conversion
// per value.
//
// Data movement.  A row block (node a1 of element e: NC x NC x NEN values, padded to a multiple of 16
// bytes) is contiguous in the element-matrix scratch, so lane 0 of the warp fetches it with one
// cp.async.bulk (global -> shared, completion counted on an mbarrier) into a ring of S slots.  The warp
// keeps S blocks in flight and refills a slot as soon as it has added the block it held.  The in-row
// positions of the block's columns come from an incidence-ordered copy of the element position map (one
// 32-entry row per incidence, fetched for all of the node's incidences by one bulk copy).
//
// Every mbarrier wait is bounded: on time-out the warp records an error word, stops adding, waits
// (bounded) for the copies it has in flight and leaves its rows unwritten.

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "icefem_internal.h"

namespace ifem {

namespace {

constexpr int kGBWarps = 4;                  // warps (nodes) per CTA
constexpr long long kGBWaitLimit = 1LL << 24;

template <int NC, int NEN, typename KT, typename MT>
struct GBLayout {
  static constexpr int KB = ke_block(NC, NEN);                      // values per padded row block
  static constexpr int BLKB = KB * (int)sizeof(KT);                 // bytes per row block (multiple of 16)
  static constexpr int S = (int)(32 / sizeof(KT));                  // ring slots: 8 (FP32) or 4 (FP64)
  static constexpr int EMROW = 32 * (int)sizeof(MT);                // bytes per incidence position row
  static constexpr int MAXINC = 32;                                 // incidences per node (one lane each)
  static constexpr int RING = S * BLKB;
  static constexpr int EMB = MAXINC * EMROW;
  static constexpr int BARS = 8 * (S + 1);
  __host__ __device__ static size_t warp_bytes(int acc_stride) {   // rounded to 128 B: rings stay 16-B aligned
    return (((size_t)RING + EMB + BARS + (size_t)acc_stride * 8) + 127) / 128 * 128;
  }
};

__device__ __forceinline__ uint32_t sm_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kGBWaitLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

template <int NC, int NEN, typename KT, typename VT, typename MT>
__global__ void __launch_bounds__(kGBWarps * 32) k_gather_bulk(const GParams p) {
  using L = GBLayout<NC, NEN, KT, MT>;
  constexpr int KB = L::KB, S = L::S, BLK = NC * NC * NEN;
  constexpr int PERV = (BLK + 31) / 32;
  extern __shared__ __align__(128) unsigned char gsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = p.node0 + (int64_t)blockIdx.x * kGBWarps + warp;
  if (r >= p.n_nodes) return;                                       // whole warp; no CTA-wide barrier below
  if (p.inc_ptr[r + 1] == p.inc_ptr[r]) return;                     // a node without elements has no entries
  unsigned char* wb = gsm + (size_t)warp * L::warp_bytes(p.acc_stride);
  KT* ring = reinterpret_cast<KT*>(wb);
  const MT* em_s = reinterpret_cast<const MT*>(wb + L::RING);
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(wb + L::RING + L::EMB);
  KT* acc = reinterpret_cast<KT*>(wb + L::RING + L::EMB + L::BARS);   // sums in the element matrices' precision
  const uint32_t ring_a = sm_addr(ring), em_a = sm_addr(em_s), bar0 = sm_addr(bars);
  const uint32_t em_bar = bar0 + 8 * S;

  const int deg = p.nbr_ptr[r + 1] - p.nbr_ptr[r];
  const int rowlen = NC * deg;
  const int k0 = p.inc_ptr[r], nk = p.inc_ptr[r + 1] - k0;          // nk <= 32 (checked on the host)
  const int my_el = lane < nk ? p.inc_el[k0 + lane] : 0;
  const int my_loc = lane < nk ? (int)p.inc_loc[k0 + lane] : 0;
  const KT* Ke = reinterpret_cast<const KT*>(p.Ke);

  if (lane == 0) {
#pragma unroll
    for (int s = 0; s <= S; ++s) bar_init(bar0 + 8 * s);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // barrier init visible to the copy engine
    bar_expect(em_bar, (uint32_t)(nk * L::EMROW));
    bulk_g2s(em_a, reinterpret_cast<const unsigned char*>(p.inc_em) + (size_t)k0 * L::EMROW, (uint32_t)(nk * L::EMROW),
             em_bar);
  }
  // first S row blocks
  for (int s = 0; s < S; ++s) {
    const int el = __shfl_sync(0xffffffffu, my_el, s < nk ? s : 0);
    const int a1 = __shfl_sync(0xffffffffu, my_loc, s < nk ? s : 0);
    if (lane == 0 && s < nk) {
      bar_expect(bar0 + 8 * s, (uint32_t)L::BLKB);
      bulk_g2s(ring_a + s * L::BLKB, Ke + ((int64_t)el * NEN + a1) * KB, (uint32_t)L::BLKB, bar0 + 8 * s);
    }
  }
  for (int i = lane; i < NC * rowlen; i += 32) acc[i] = (KT)0;
  // per-lane slots of a row block (independent of the element)
  int sb[PERV], sa[PERV];
#pragma unroll
  for (int jj = 0; jj < PERV; ++jj) {
    const int i = lane + 32 * jj;
    const int b1 = i / (NC * NEN), rem = i - b1 * (NC * NEN), b2 = rem / NEN, a2 = rem - b2 * NEN;
    sb[jj] = (i < BLK) ? b1 * rowlen + p.blk_pos[b2 < NC ? b2 : 0] * deg : -1;
    sa[jj] = a2;
  }
  // residual: element-order sums of the incident elements' entries (lane k loads incidence k)
  double fv[NC], fv2[NC];
#pragma unroll
  for (int b = 0; b < NC; ++b) {
    fv[b] = lane < nk ? p.Fe1[(int64_t)my_el * (NC * NEN) + b * NEN + my_loc] : 0.0;
    fv2[b] = (p.Fe2 && lane < nk) ? p.Fe2[(int64_t)my_el * (NC * NEN) + b * NEN + my_loc] : 0.0;
  }
  double fa[NC];
#pragma unroll
  for (int b = 0; b < NC; ++b) {
    double sum = 0.0;
    for (int k = 0; k < nk; ++k) sum += __shfl_sync(0xffffffffu, fv[b], k);
    if (p.Fe2)
      for (int k = 0; k < nk; ++k) sum += __shfl_sync(0xffffffffu, fv2[b], k);
    fa[b] = sum;
  }
  __syncwarp();
  bool ok = __all_sync(0xffffffffu, bar_wait(em_bar, 0));     // warp-uniform decisions only
  int issued = nk < S ? nk : S, consumed = 0;
  for (int k = 0; k < nk && ok; ++k) {
    const int s = k % S;
    ok = __all_sync(0xffffffffu, bar_wait(bar0 + 8 * s, (uint32_t)((k / S) & 1)));
    if (!ok) break;
    consumed = k + 1;
    const KT* blk = ring + s * KB;
    const MT* em = em_s + k * 32;
#pragma unroll
    for (int jj = 0; jj < PERV; ++jj)
      if (sb[jj] >= 0) acc[sb[jj] + (int)em[sa[jj]]] += blk[lane + 32 * jj];
    __syncwarp();
    const int kn = k + S;
    const int el = __shfl_sync(0xffffffffu, my_el, kn < nk ? kn : 0);
    const int a1 = __shfl_sync(0xffffffffu, my_loc, kn < nk ? kn : 0);
    if (kn < nk) {
      if (lane == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // this slot's reads before the refill
        bar_expect(bar0 + 8 * s, (uint32_t)L::BLKB);
        bulk_g2s(ring_a + s * L::BLKB, Ke + ((int64_t)el * NEN + a1) * KB, (uint32_t)L::BLKB, bar0 + 8 * s);
      }
      ++issued;
    }
  }
  if (!ok) {
    if (lane == 0) atomicExch(p.err, 1ull);
    for (int k = consumed; k < issued; ++k) bar_wait(bar0 + 8 * (k % S), (uint32_t)((k / S) & 1));
    return;
  }
  __syncwarp();
  VT* vals = reinterpret_cast<VT*>(p.vals);
#pragma unroll
  for (int b1 = 0; b1 < NC; ++b1) {
    const int64_t off = p.rowptr[p.row_base[b1] + r];
    for (int i = lane; i < rowlen; i += 32) vals[off + i] = (VT)acc[b1 * rowlen + i];
  }
#pragma unroll
  for (int b = 0; b < NC; ++b)
    if (lane == b) p.f[p.row_base[b] + r] = fa[b];
}

// Register-accumulator variant (nodes with at most 32 NPL neighbours).  Lane l owns neighbour columns
// n = l + 32 i (i < NPL) of all NC x NC component pairs and keeps their sums in registers.  For each
// incident element, the lanes of its 27 (or 9) nodes write their local index into a per-warp inverse
// table at the node's neighbour position (tagged with the incidence number, so the table is never
// cleared); each lane then reads the table at its own neighbours and adds the matching row-block entries.
// No shared-memory read-modify-write, so no bank-conflicted accumulator traffic.  Same element order and
// accumulator precision as the shared-accumulator kernel: identical results.
template <int NC, int NEN, typename KT, typename MT, int NPL>
struct GRLayout {
  static constexpr int KB = ke_block(NC, NEN);
  static constexpr int BLKB = KB * (int)sizeof(KT);
  // ring slots: FP32 6 (29 KB per CTA of 4 warps, 7 CTAs per SM; measured 0.46 ms at 65,536 hex elements against
  // 0.49 with 8 slots and 6 CTAs, 0.48 with 5 slots and 8 CTAs at 64 registers), FP64 4
  static constexpr int S = sizeof(KT) == 4 ? 6 : 4;
  static constexpr int EMROW = 32 * (int)sizeof(MT);
  static constexpr int RING = S * BLKB;
  static constexpr int EMB = 32 * EMROW;
  static constexpr int INV = 32 * NPL * 2;                        // uint16 inverse table
  static constexpr int BARS = 8 * (S + 1);
  static constexpr size_t WARP = ((size_t)RING + EMB + INV + BARS + 127) / 128 * 128;
};

template <int NC, int NEN, typename KT, typename VT, typename MT, int NPL>
__global__ void __launch_bounds__(kGBWarps * 32) k_gather_bulk_reg(const GParams p) {
  using L = GRLayout<NC, NEN, KT, MT, NPL>;
  constexpr int KB = L::KB, S = L::S;
  extern __shared__ __align__(128) unsigned char gsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = p.node0 + (int64_t)blockIdx.x * kGBWarps + warp;
  if (r >= p.n_nodes) return;
  if (p.inc_ptr[r + 1] == p.inc_ptr[r]) return;
  unsigned char* wb = gsm + (size_t)warp * L::WARP;
  KT* ring = reinterpret_cast<KT*>(wb);
  const MT* em_s = reinterpret_cast<const MT*>(wb + L::RING);
  uint16_t* inv = reinterpret_cast<uint16_t*>(wb + L::RING + L::EMB);
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(wb + L::RING + L::EMB + L::INV);
  const uint32_t ring_a = sm_addr(ring), em_a = sm_addr(em_s), bar0 = sm_addr(bars);
  const uint32_t em_bar = bar0 + 8 * S;

  const int deg = p.nbr_ptr[r + 1] - p.nbr_ptr[r];                 // <= 32 NPL (checked on the host)
  const int k0 = p.inc_ptr[r], nk = p.inc_ptr[r + 1] - k0;
  const int my_el = lane < nk ? p.inc_el[k0 + lane] : 0;
  const int my_loc = lane < nk ? (int)p.inc_loc[k0 + lane] : 0;
  const KT* Ke = reinterpret_cast<const KT*>(p.Ke);

  if (lane == 0) {
#pragma unroll
    for (int s = 0; s <= S; ++s) bar_init(bar0 + 8 * s);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    bar_expect(em_bar, (uint32_t)(nk * L::EMROW));
    bulk_g2s(em_a, reinterpret_cast<const unsigned char*>(p.inc_em) + (size_t)k0 * L::EMROW, (uint32_t)(nk * L::EMROW),
             em_bar);
  }
  for (int s = 0; s < S; ++s) {
    const int el = __shfl_sync(0xffffffffu, my_el, s < nk ? s : 0);
    const int a1 = __shfl_sync(0xffffffffu, my_loc, s < nk ? s : 0);
    if (lane == 0 && s < nk) {
      bar_expect(bar0 + 8 * s, (uint32_t)L::BLKB);
      bulk_g2s(ring_a + s * L::BLKB, Ke + ((int64_t)el * NEN + a1) * KB, (uint32_t)L::BLKB, bar0 + 8 * s);
    }
  }
#pragma unroll
  for (int i = 0; i < NPL; ++i) inv[lane + 32 * i] = 0xFFFFu;
  // sums in the element matrices' precision (FP32 values are added without a conversion per value)
  using AT = KT;
  AT acc[NPL][NC * NC];
#pragma unroll
  for (int i = 0; i < NPL; ++i)
#pragma unroll
    for (int c = 0; c < NC * NC; ++c) acc[i][c] = (AT)0;
  // residual (element-order sums, as the shared-accumulator kernel)
  double fv[NC], fv2[NC];
#pragma unroll
  for (int b = 0; b < NC; ++b) {
    fv[b] = lane < nk ? p.Fe1[(int64_t)my_el * (NC * NEN) + b * NEN + my_loc] : 0.0;
    fv2[b] = (p.Fe2 && lane < nk) ? p.Fe2[(int64_t)my_el * (NC * NEN) + b * NEN + my_loc] : 0.0;
  }
  double fa[NC];
#pragma unroll
  for (int b = 0; b < NC; ++b) {
    double sum = 0.0;
    for (int k = 0; k < nk; ++k) sum += __shfl_sync(0xffffffffu, fv[b], k);
    if (p.Fe2)
      for (int k = 0; k < nk; ++k) sum += __shfl_sync(0xffffffffu, fv2[b], k);
    fa[b] = sum;
  }
  __syncwarp();
  bool ok = __all_sync(0xffffffffu, bar_wait(em_bar, 0));
  int issued = nk < S ? nk : S, consumed = 0;
  for (int k = 0; k < nk && ok; ++k) {
    const int s = k % S;
    ok = __all_sync(0xffffffffu, bar_wait(bar0 + 8 * s, (uint32_t)((k / S) & 1)));
    if (!ok) break;
    consumed = k + 1;
    const KT* blk = ring + s * KB;
    if (lane < NEN) inv[(int)em_s[k * 32 + lane]] = (uint16_t)((k << 8) | lane);   // node lane -> its column
    __syncwarp();
#pragma unroll
    for (int i = 0; i < NPL; ++i) {
      const uint32_t v = inv[lane + 32 * i];
      if ((int)(v >> 8) == k && lane + 32 * i < deg) {
        const int a2 = (int)(v & 0xFFu);
#pragma unroll
        for (int b1 = 0; b1 < NC; ++b1)
#pragma unroll
          for (int b2 = 0; b2 < NC; ++b2) acc[i][b1 * NC + b2] += blk[(b1 * NC + b2) * NEN + a2];
      }
    }
    __syncwarp();
    const int kn = k + S;
    const int el = __shfl_sync(0xffffffffu, my_el, kn < nk ? kn : 0);
    const int a1 = __shfl_sync(0xffffffffu, my_loc, kn < nk ? kn : 0);
    if (kn < nk) {
      if (lane == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        bar_expect(bar0 + 8 * s, (uint32_t)L::BLKB);
        bulk_g2s(ring_a + s * L::BLKB, Ke + ((int64_t)el * NEN + a1) * KB, (uint32_t)L::BLKB, bar0 + 8 * s);
      }
      ++issued;
    }
  }
  if (!ok) {
    if (lane == 0) atomicExch(p.err, 1ull);
    for (int k = consumed; k < issued; ++k) bar_wait(bar0 + 8 * (k % S), (uint32_t)((k / S) & 1));
    return;
  }
  VT* vals = reinterpret_cast<VT*>(p.vals);
  const int rowlen = NC * deg;
#pragma unroll
  for (int b1 = 0; b1 < NC; ++b1) {
    const int64_t off = p.rowptr[p.row_base[b1] + r];
#pragma unroll
    for (int b2 = 0; b2 < NC; ++b2) {
      const int64_t o2 = off + (int64_t)p.blk_pos[b2] * deg;
#pragma unroll
      for (int i = 0; i < NPL; ++i) {
        const int n = lane + 32 * i;
        if (n < deg) vals[o2 + n] = (VT)acc[i][b1 * NC + b2];
      }
    }
  }
  (void)rowlen;
#pragma unroll
  for (int b = 0; b < NC; ++b)
    if (lane == b) p.f[p.row_base[b] + r] = fa[b];
}

template <int NC, int NEN, typename KT, typename VT, int NPL>
void gather_reg3(const GParams& p, cudaStream_t s) {
  const size_t smem = (p.emap16 ? GRLayout<NC, NEN, KT, uint16_t, NPL>::WARP : GRLayout<NC, NEN, KT, uint8_t, NPL>::WARP) *
                      kGBWarps;
  void (*k)(const GParams) =
      p.emap16 ? k_gather_bulk_reg<NC, NEN, KT, VT, uint16_t, NPL> : k_gather_bulk_reg<NC, NEN, KT, VT, uint8_t, NPL>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned blocks = (unsigned)((p.n_nodes - p.node0 + kGBWarps - 1) / kGBWarps);
  k<<<blocks, kGBWarps * 32, smem, s>>>(p);
}

// register accumulators when every node has at most 128 neighbours and rows have several components (with
// one component the shared accumulator has no bank conflicts to avoid and is faster)
template <int NC, int NEN, typename KT, typename VT>
bool gather_reg2(const GParams& p, cudaStream_t s) {
  if (NC == 1) return false;
  const int npl = (p.max_deg + 31) / 32;
  switch (npl) {
    case 1: gather_reg3<NC, NEN, KT, VT, 1>(p, s); return true;
    case 2: gather_reg3<NC, NEN, KT, VT, 2>(p, s); return true;
    case 3: gather_reg3<NC, NEN, KT, VT, 3>(p, s); return true;
    case 4: gather_reg3<NC, NEN, KT, VT, 4>(p, s); return true;
    default: return false;
  }
}

template <int NC, int NEN, typename KT, typename VT>
bool gather_bulk2(const GParams& p, cudaStream_t s) {
  using L8 = GBLayout<NC, NEN, KT, uint8_t>;
  using L16 = GBLayout<NC, NEN, KT, uint16_t>;
  if (NC == 1 && launch_gather_direct1(p, s)) return true;
  if (gather_reg2<NC, NEN, KT, VT>(p, s)) return true;
  const size_t per_warp = p.emap16 ? L16::warp_bytes(p.acc_stride) : L8::warp_bytes(p.acc_stride);
  const size_t smem = per_warp * kGBWarps;
  if (smem > 200 * 1024) return false;
  void (*k)(const GParams) = p.emap16 ? k_gather_bulk<NC, NEN, KT, VT, uint16_t> : k_gather_bulk<NC, NEN, KT, VT, uint8_t>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned blocks = (unsigned)((p.n_nodes - p.node0 + kGBWarps - 1) / kGBWarps);
  k<<<blocks, kGBWarps * 32, smem, s>>>(p);
  return true;
}

template <int NC, int NEN>
bool gather_bulk1(const GParams& p, cudaStream_t s) {
  if (p.ke_f32) return p.vals_f32 ? gather_bulk2<NC, NEN, float, float>(p, s) : gather_bulk2<NC, NEN, float, double>(p, s);
  return p.vals_f32 ? gather_bulk2<NC, NEN, double, float>(p, s) : gather_bulk2<NC, NEN, double, double>(p, s);
}

}  // namespace

// Matrix-and-residual gathers through the bulk-copy kernel; false when the layout does not qualify (the
// caller then uses the register-staged gather).
bool launch_gather_bulk(const GParams& p, cudaStream_t s) {
  if (p.n_nodes <= p.node0 || !p.Ke || !p.inc_em || !p.err || p.max_inc > 32) return false;
  if (p.nen == 9) return p.nc == 1 ? gather_bulk1<1, 9>(p, s) : (p.nc == 2 ? gather_bulk1<2, 9>(p, s) : gather_bulk1<3, 9>(p, s));
  return p.nc == 1 ? gather_bulk1<1, 27>(p, s) : (p.nc == 2 ? gather_bulk1<2, 27>(p, s) : gather_bulk1<3, 27>(p, s));
}

}  // namespace ifem
