// U-step element tangent of the 3D quadratic hex on the 5th-generation tensor cores (tcgen05).
//
// K_e (81x81) = sum_q B_q^T C_q B_q  (PhaseField.cpp:422).  Written per displacement-component
// block (a,b) with the physical shape gradients G_p(i;q):
//     K[(a,i),(b,j)] = sum_{q,p} G_p(i;q) * Z^{ab}[(q,p), j],
//     Z^{ab}[(q,p), j] = sum_r C_q[v(a,p), v(b,r)] G_r(j;q)       (v = Voigt index of (comp, dir))
// i.e. one GEMM per element  D[m=(a,b,j), n=i] = sum_k A[m,k] B[n,k]  with M = 243 (two M=128
// MMAs), N = 27 (padded to 32), K = (q,p) = 81 (padded to 88).  For an FP32-accurate tangent each
// operand is split x = hi + lo into TF32 parts and D = Ahi*Bhi + Ahi*Blo + Alo*Bhi (FP32
// accumulate), so the error is O(2^-22) instead of TF32's 2^-11.  Bhi and Blo sit side by side as one
// N = 64 operand, so Ahi*[Bhi; Blo] is one MMA and Alo*Bhi (N = 32) a second one per k-step and tile.
//
// Operand placement.  A (= Z, 2 x 243 x 88 values per element) never touches shared memory: the thread
// that owns TMEM lane m builds row m = (a,b,j) in registers from the per-ip material tangents and the
// shape gradients and writes it into tensor memory with tcgen05.st; the MMAs read A from TMEM.  B (= G,
// 27 rows) is staged in shared memory in the no-swizzle K-major canonical layout, double-buffered so that
// the next element's B can be built while the current element's MMAs run.  TMEM columns:
//     [0, 128)     accumulators of the two M tiles (64 columns each: Ahi Bhi + Alo Bhi, then Ahi Blo)
//     [128, 512)   A regions of 96 columns: tile 0 hi, tile 0 lo, tile 1 hi, tile 1 lo (88 used each)
//
// Schedule (one persistent CTA per SM: 16 builder warps, one MMA warp, 4 epilogue warps):
//   builders:  inputs of e landed (four bulk copies, issued one element ahead) -> tables, B(e), G table ->
//              wait for the MMAs of e-1 (A is reused) -> build A(e) in TMEM -> arrive "A ready";
//   MMA warp:  "A ready"(e) and "accumulator free"(e-1) -> 44 MMAs of e -> commit to "done";
//   epilogue:  "done"(e) -> accumulator to registers -> arrive "accumulator free" -> staging (+ lumped
//              diagonal) -> one bulk copy of the element matrix.
//   The MMAs of e and the read-out of e run while the builders prepare e+1.
//
// Builder warp w owns TMEM lane quarter w % 4 of M tile (w / 4) % 2; warps w < 8 build k-columns [0, 42) of
// their rows (ips 0..13), warps 8..15 build k-columns [42, 88) (ips 14..26 and the K padding).  Epilogue warp
// w reads lane quarter w % 4 of both tiles.
//
// Every wait on the MMA-completion mbarrier is bounded; on time-out the kernel records an error word,
// waits (bounded) once more, releases its TMEM and returns.

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

constexpr int TC_THREADS = 512;
constexpr int TC_KB = 244;                  // padded (node, comp, comp, node) row-block stride of K_e
constexpr int TC_K = 88;                    // K padded to a multiple of 8 (tf32 k-step)
constexpr int TC_KCH = TC_K / 4;            // 16-byte chunks per row
constexpr int TC_SBO = TC_KCH * 128;        // bytes between 8-row core-matrix groups
constexpr int TC_BROWS = 32;
constexpr int TC_BBYTES = TC_BROWS / 8 * TC_SBO;   // 11264
constexpr uint32_t TC_TMEM_COLS = 512;
constexpr uint32_t TC_COL_A = 128;          // A region r (= 2 tile + lo) starts at TC_COL_A + 96 r
constexpr uint32_t TC_AREG = 96;
constexpr long long kWaitLimit = 1LL << 26;

// per-element inputs, double-buffered and filled one element ahead by four bulk copies of the
// element-major blocks the points kernel writes (same layouts as in HBM)
struct alignas(16) TcStage {
  float C[36][27];          // w * (g D+ + D-) DPlast per ip
  float geo[13][27];        // Jinv (9), 1/wFun, dW/wFun^2 (3) per ip
  float geo_pad[kTcGeo - 13 * 27];
  float nx[2][3][3][3];     // 1-D basis tables [value / derivative][axis][ip coordinate][function]
  float W[27];              // nodal NURBS weights
  float nx_pad[kTcNx - 81];
  double Kd[kTcKd];         // lumped diagonal terms per node (inertia / damping), padding
};
constexpr uint32_t kStageTx = (uint32_t)(sizeof(float) * (kTcCq + kTcGeo + kTcNx) + sizeof(double) * kTcKd);
static_assert(sizeof(TcStage) == kStageTx, "stage layout differs from the HBM blocks");
static_assert(offsetof(TcStage, geo) % 16 == 0 && offsetof(TcStage, nx) % 16 == 0 && offsetof(TcStage, Kd) % 16 == 0,
              "bulk-copy destinations must be 16-byte aligned");

struct TcSm {
  // B operand per buffer: rows 0..31 = G hi, rows 32..63 = G lo (one N = 64 operand, or its first 32 rows)
  alignas(128) unsigned char B[2][2 * TC_BBYTES];
  TcStage st[2];
  float4 G[27][27];        // G[q][j] = (G_0, G_1, G_2, 0)(j; q), FP32
  float4 Cb[27][3][6];     // Cb[q][b][s] = (C_q[s][v(b,0)], C_q[s][v(b,1)], C_q[s][v(b,2)], 0)
  double kd[2][27];        // lumped diagonal, by stage
  alignas(128) float stage[27 * TC_KB];   // one element matrix, written back by one bulk copy
  unsigned long long mb_in[2];          // inputs of a stage landed (transaction count of the bulk copies)
  unsigned long long mb_afull;          // A and B of an element ready (one arrival per builder warp)
  unsigned long long mb_done;           // the element's MMAs completed (tcgen05.commit)
  unsigned long long mb_accfree;        // the accumulator has been read out (one arrival per epilogue warp)
  uint32_t tmem_base;
  int abort_flag;
};

// global -> shared bulk copy completing on an mbarrier (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          (uint32_t)__cvta_generic_to_shared(dst)),
      "l"(src), "r"(bytes), "r"(mbar)
      : "memory");
}

// one thread: element `el`'s inputs into a staging buffer, completion counted on `mbar`
__device__ __forceinline__ void tc_prefetch(TcStage& st, const TParams& p, int64_t el, uint32_t mbar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(kStageTx) : "memory");
  bulk_g2s(st.C, reinterpret_cast<const float*>(p.Cq) + el * kTcCq, sizeof(float) * kTcCq, mbar);
  bulk_g2s(st.geo, p.geoq + el * kTcGeo, sizeof(float) * kTcGeo, mbar);
  bulk_g2s(st.nx, p.nxq + el * kTcNx, sizeof(float) * kTcNx, mbar);
  bulk_g2s(st.Kd, p.Kd + el * kTcKd, sizeof(double) * kTcKd, mbar);
}

// byte offset of element (row, k) in a no-swizzle K-major operand
__device__ __forceinline__ uint32_t kmajor_off(int row, int k) {
  return (uint32_t)((row >> 3) * TC_SBO + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  // start address >> 4 [0,14), LBO = 128 B [16,30), SBO [32,46), version 1 [46,48), no swizzle
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)((uint32_t)TC_SBO >> 4) << 32) | (1ull << 46);
}

// kind::tf32, D f32, A/B tf32 K-major, N = 32, M = 128
constexpr uint32_t kIdesc32 = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
// the same with N = 64 (B rows hi and lo side by side)
constexpr uint32_t kIdesc64 = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// D[tmem] (+)= A[tmem] * B[smem]^T
__device__ __forceinline__ void mma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar_addr) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_addr)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar_addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar_addr), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar_addr, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(mbar_addr, parity)) return true;
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// X consecutive TMEM columns of this thread's lane
template <int X>
__device__ __forceinline__ void tmem_stx(uint32_t taddr, const float* v) {
  if constexpr (X == 8) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
        ::"r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
          "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
          "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
        : "memory");
  } else if constexpr (X == 4) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};"
                 ::"r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                   "r"(__float_as_uint(v[3]))
                 : "memory");
  } else if constexpr (X == 2) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1,%2};"
                 ::"r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1]))
                 : "memory");
  } else {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(__float_as_uint(v[0]))
                 : "memory");
  }
}

// columns [C0, C0 + N) of this lane, as naturally aligned x8 / x4 / x2 / x1 pieces
template <int C0, int N>
__device__ __forceinline__ void tmem_st_cols(uint32_t base, const float* v) {
  if constexpr (N > 0) {
    constexpr int X = (C0 % 8 == 0 && N >= 8) ? 8 : (C0 % 4 == 0 && N >= 4) ? 4 : (C0 % 2 == 0 && N >= 2) ? 2 : 1;
    tmem_stx<X>(base + C0, v);
    tmem_st_cols<C0 + X, N - X>(base, v + X);
  }
}

// Row (a,b,j) of A over NQ ips from q0 (k-columns 3 q + p relative to 3 q0), split into TF32 hi / lo.
// NV >= 3 NQ values; the ones beyond 3 NQ are zero (K padding).
template <int NQ, int NV>
__device__ __forceinline__ void build_a_cols(const TcSm& s, bool row_ok, int a, int b, int j, int q0,
                                             float hi[NV], float lo[NV]) {
#pragma unroll
  for (int qq = 0; qq < NQ; ++qq) {
    float y[3] = {0.0f, 0.0f, 0.0f};
    if (row_ok) {
      const int q = q0 + qq;
      const float4 g = s.G[q][j];
#pragma unroll
      for (int pp = 0; pp < 3; ++pp) {
        const float4 c = s.Cb[q][b][voigt_idx(a, pp)];
        y[pp] = c.x * g.x + c.y * g.y + c.z * g.z;
      }
    }
#pragma unroll
    for (int pp = 0; pp < 3; ++pp) {
      const float h = tf32_rna(y[pp]);
      hi[3 * qq + pp] = h;
      lo[3 * qq + pp] = y[pp] - h;   // exact; the MMA reads its TF32 part (truncation error ~2^-21 |y|)
    }
  }
#pragma unroll
  for (int k = 3 * NQ; k < NV; ++k) { hi[k] = 0.0f; lo[k] = 0.0f; }
}

constexpr int TC_EPI = 4;                                   // epilogue warps (one per TMEM lane quarter)
constexpr int TC_ALL = TC_THREADS + 32 + 32 * TC_EPI;       // builders, MMA warp, epilogue warps

// builder barrier that also returns the OR of `x` over all builder threads (a CTA-uniform decision)
__device__ __forceinline__ bool bar_builders_or(bool x) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, 1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)x), "n"(TC_THREADS)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void bar_epilogue() { asm volatile("bar.sync 2, %0;" ::"n"(32 * TC_EPI) : "memory"); }

__device__ __forceinline__ void mbar_arrive(uint32_t mbar_addr) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar_addr) : "memory");
}

__global__ void __launch_bounds__(TC_ALL, 1) k_u_tangent_tc(const TParams p, unsigned long long* err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcSm& s = *reinterpret_cast<TcSm*>(smraw);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const bool mma_warp = warp == TC_THREADS / 32;
  const bool epi_warp = warp > TC_THREADS / 32;
  const Geo& geo = p.geo;
  // the row of A this (builder) thread owns; epilogue warps own TMEM lane quarter warp % 4 of both tiles
  const int quarter = warp & 3, tile = (warp >> 2) & 1, half = (warp >> 3) & 1;
  const int m = tile * 128 + quarter * 32 + lane;
  const bool row_ok = !mma_warp && !epi_warp && m < 243;
  const int ab = row_ok ? m / 27 : 0, j = row_ok ? m % 27 : 0, a = ab / 3, b = ab % 3;

  // zero the B operands and the staging row padding once: they are never written afterwards
  for (int i = t; i < 4 * TC_BBYTES / 16; i += TC_ALL)
    reinterpret_cast<float4*>(&s.B[0][0])[i] = make_float4(0, 0, 0, 0);
  if (t < 27) s.stage[t * TC_KB + 243] = 0.0f;
  if (t == 0) {
    s.abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s.mb_afull)), "n"(TC_THREADS / 32) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mb_done)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s.mb_accfree)), "n"(TC_EPI) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mb_in[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mb_in[1])) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_base)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem_base;
  const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
  const uint32_t mb_afull = smem_u32(&s.mb_afull), mb_done = smem_u32(&s.mb_done), mb_accfree = smem_u32(&s.mb_accfree);

  if (mma_warp) {
    // ---- MMA issuer: A(e), B(e) ready and the accumulator read out -> 44 MMAs -> commit ----
    int cur = 0;
    uint32_t par_a = 0, par_f = 0;
    for (int64_t el = blockIdx.x; el < geo.nel; el += gridDim.x, cur ^= 1) {
      bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(mb_afull, par_a));
      par_a ^= 1u;
      if (ok && el != (int64_t)blockIdx.x) {
        ok = __all_sync(0xffffffffu, mbar_wait_bounded(mb_accfree, par_f));
        par_f ^= 1u;
      }
      if (!ok) {
        if (lane == 0) atomicExch(&s.abort_flag, 1);
        break;
      }
      tc_fence_after();
      if (lane == 0) {
        const uint64_t db = smem_desc(smem_u32(s.B[cur]));
#pragma unroll
        for (int ks = 0; ks < TC_K / 8; ++ks) {      // k-step ks: +8 TMEM columns of A, +256 B (16 desc units) of B
          const uint64_t ko = (uint64_t)(ks * 16);
#pragma unroll
          for (int tl = 0; tl < 2; ++tl) {           // the two M tiles alternate: independent chains
            // accumulator of tile tl: columns [64 tl, 64 tl + 32) = Ahi Bhi + Alo Bhi, [64 tl + 32, 64 tl + 64) = Ahi Blo
            const uint32_t dt = tmem + (uint32_t)(tl * 64);
            const uint32_t ahi = tmem + TC_COL_A + (uint32_t)(2 * tl) * TC_AREG + (uint32_t)(8 * ks);
            mma_tf32_ts(dt, ahi, db + ko, kIdesc64, ks > 0 ? 1u : 0u);
            mma_tf32_ts(dt, ahi + TC_AREG, db + ko, kIdesc32, 1u);
          }
        }
        mma_commit(mb_done);
      }
      __syncwarp();
    }
  } else if (epi_warp) {
    // ---- epilogue: accumulator -> registers (signal "free") -> staging -> one bulk copy per element ----
    const int te = t - TC_THREADS - 32;             // 0 .. 127
    int cur = 0;
    uint32_t par = 0;
    for (int64_t el = blockIdx.x; el < geo.nel; el += gridDim.x, cur ^= 1) {
      const bool ok = mbar_wait_bounded(mb_done, par);
      par ^= 1u;
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicExch(&s.abort_flag, 1);
        break;
      }
      tc_fence_after();
      if (te == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");   // staging free again
      bar_epilogue();
#pragma unroll 1
      for (int tl = 0; tl < 2; ++tl) {
        float v[27], x[16], y[16];
        tmem_ld16(tmem + lane_off + (uint32_t)(tl * 64), x);
        tmem_ld16(tmem + lane_off + (uint32_t)(tl * 64 + 32), y);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = x[i] + y[i];          // (Ahi + Alo) Bhi + Ahi Blo
        tmem_ld16(tmem + lane_off + (uint32_t)(tl * 64 + 16), x);
        tmem_ld16(tmem + lane_off + (uint32_t)(tl * 64 + 48), y);
#pragma unroll
        for (int i = 0; i < 11; ++i) v[16 + i] = x[i] + y[i];
        const int mm = tl * 128 + quarter * 32 + lane;
        if (mm < 243) {
          const int abm = mm / 27, jm = mm % 27;
          const double kd = (abm / 3 == abm % 3) ? s.kd[cur][jm] : 0.0;   // diagonal lumped terms
          // static register indices only (a dynamic v[i] would put v in local memory)
#pragma unroll
          for (int col = 0; col < 27; ++col)
            s.stage[col * TC_KB + mm] = (col == jm && kd != 0.0) ? (float)((double)v[col] + kd) : v[col];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(mb_accfree);        // the MMAs of the next element may overwrite it
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // staging writes -> bulk copy
      bar_epilogue();
      if (te == 0) {
        float* dst = reinterpret_cast<float*>(p.Ke) + el * (27 * TC_KB);
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                     "r"(smem_u32(s.stage)), "n"(27 * TC_KB * 4)
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      }
    }
    if (te == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");   // the last element's store landed
  } else {
    // ---- builders ----
    int cur = 0;
    uint32_t par = 0;
    uint32_t par_in = 0;      // bit x: parity of stage x's next completion
    uint32_t pending = 0;     // bit x: a copy into stage x is in flight (issued by thread 0)
    bool first = true;
    const uint32_t mb_in0 = smem_u32(&s.mb_in[0]), mb_in1 = smem_u32(&s.mb_in[1]);
    if ((int64_t)blockIdx.x < geo.nel && t == 0) {
      tc_prefetch(s.st[0], p, blockIdx.x, mb_in0);
      pending = 1u;
    }
    for (int64_t el = blockIdx.x; el < geo.nel; el += gridDim.x, cur ^= 1) {
      const bool in_ok = mbar_wait_bounded(cur ? mb_in1 : mb_in0, (par_in >> cur) & 1u);
      if (in_ok) { par_in ^= 1u << cur; pending &= ~(1u << cur); }
      else atomicExch(&s.abort_flag, 1);
      // stage `cur` landed; the previous element's A build is done
      if (bar_builders_or(!in_ok || *reinterpret_cast<volatile int*>(&s.abort_flag) != 0)) break;
      if (el + gridDim.x < geo.nel && t == 0) {
        tc_prefetch(s.st[cur ^ 1], p, el + gridDim.x, cur ? mb_in0 : mb_in1);
        pending |= 1u << (cur ^ 1);
      }
      const TcStage& st = s.st[cur];
      // ---- per-element table Cb ----
      for (int i = t; i < 27 * 3 * 6; i += TC_THREADS) {
        const int q = i % 27, rest = i / 27, bb = rest % 3, sv = rest / 3;
        s.Cb[q][bb][sv] = make_float4(st.C[sv * 6 + voigt_idx(bb, 0)][q], st.C[sv * 6 + voigt_idx(bb, 1)][q],
                                      st.C[sv * 6 + voigt_idx(bb, 2)][q], 0.0f);
      }
      // ---- B operand (buffer cur) and G table: rows = nodes, k = 3q + d (NURBS3_Cube2.cpp:97-114) ----
      for (int task = t; task < 27 * 27; task += TC_THREADS) {
        const int nd = task % 27, q = task / 27;
        const int ia = nd % 3, ja = (nd / 3) % 3, ka = nd / 9;
        const int qx = q % 3, qy = (q / 3) % 3, qz = q / 9;
        const float nx = st.nx[0][0][qx][ia], ny = st.nx[0][1][qy][ja], nz = st.nx[0][2][qz][ka];
        const float CB = nx * ny * nz;
        const float GB0 = st.nx[1][0][qx][ia] * ny * nz, GB1 = nx * st.nx[1][1][qy][ja] * nz, GB2 = nx * ny * st.nx[1][2][qz][ka];
        const float rw = st.geo[9][q], Wn = st.W[nd];
        const float g0 = Wn * (GB0 * rw - CB * st.geo[10][q]);
        const float g1 = Wn * (GB1 * rw - CB * st.geo[11][q]);
        const float g2 = Wn * (GB2 * rw - CB * st.geo[12][q]);
        float v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          v[d] = st.geo[d * 3 + 0][q] * g0 + st.geo[d * 3 + 1][q] * g1 + st.geo[d * 3 + 2][q] * g2;
        s.G[q][nd] = make_float4(v[0], v[1], v[2], 0.0f);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float h = tf32_rna(v[d]);
          const uint32_t off = kmajor_off(nd, 3 * q + d);
          *reinterpret_cast<float*>(s.B[cur] + off) = h;
          *reinterpret_cast<float*>(s.B[cur] + TC_BBYTES + off) = v[d] - h;   // exact remainder
        }
      }
      // ---- the previous element's MMAs have to complete before its A is overwritten ----
      if (!first) {
        const bool ok = mbar_wait_bounded(mb_done, par);
        par ^= 1u;
        if (!ok && lane == 0) atomicExch(&s.abort_flag, 1);
        tc_fence_after();
      }
      first = false;
      // lumped diagonal for the epilogue; the epilogue read kd[cur] of element e - 2 before it released the
      // accumulator the MMAs of e - 1 (now complete) wrote into
      if (t >= 480 && t < 480 + 27) s.kd[cur][t - 480] = st.Kd[t - 480];
      // also publishes this element's B and G tables and kd
      if (bar_builders_or(*reinterpret_cast<volatile int*>(&s.abort_flag) != 0)) break;
      // ---- A operand of this element into TMEM ----
      {
        const uint32_t base_hi = tmem + lane_off + TC_COL_A + (uint32_t)(2 * tile) * TC_AREG;
        const uint32_t base_lo = base_hi + TC_AREG;
        if (half == 0) {                     // ips 0..13 -> k-columns [0, 42)
          {
            float hi[24], lo[24];
            build_a_cols<8, 24>(s, row_ok, a, b, j, 0, hi, lo);
            tmem_st_cols<0, 24>(base_hi, hi);
            tmem_st_cols<0, 24>(base_lo, lo);
          }
          float hi[18], lo[18];
          build_a_cols<6, 18>(s, row_ok, a, b, j, 8, hi, lo);
          tmem_st_cols<24, 18>(base_hi, hi);
          tmem_st_cols<24, 18>(base_lo, lo);
        } else {                             // ips 14..26 and the K padding -> k-columns [42, 88)
          {
            float hi[24], lo[24];
            build_a_cols<8, 24>(s, row_ok, a, b, j, 14, hi, lo);
            tmem_st_cols<42, 24>(base_hi, hi);
            tmem_st_cols<42, 24>(base_lo, lo);
          }
          float hi[22], lo[22];
          build_a_cols<5, 22>(s, row_ok, a, b, j, 22, hi, lo);
          tmem_st_cols<66, 22>(base_hi, hi);
          tmem_st_cols<66, 22>(base_lo, lo);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      }
      tc_fence_before();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // B was written by generic stores
      __syncwarp();
      if (lane == 0) mbar_arrive(mb_afull);     // one arrival per builder warp
    }
    // only after an abort: let input copies still in flight land before the CTA exits (bounded)
    if (pending & 1u) mbar_wait_bounded(mb_in0, par_in & 1u);
    if (pending & 2u) mbar_wait_bounded(mb_in1, (par_in >> 1) & 1u);
  }
  __syncthreads();
  if (s.abort_flag) {
    if (t == 0) atomicExch(err, 1ull);
    mbar_wait_bounded(mb_done, 0);             // let MMAs in flight finish (bounded; the parity may be stale)
    mbar_wait_bounded(mb_done, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
}

}  // namespace

size_t tc_smem_bytes() { return sizeof(TcSm); }

void launch_u_tangent_tc(const TParams& p, unsigned long long* err, int n_sm, cudaStream_t s) {
  if (p.geo.nel == 0) return;
  const size_t smem = sizeof(TcSm);
  cudaFuncSetAttribute(k_u_tangent_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int64_t grid = p.geo.nel < n_sm ? p.geo.nel : n_sm;
  k_u_tangent_tc<<<(unsigned)grid, TC_ALL, smem, s>>>(p, err);
}

}  // namespace ifem
