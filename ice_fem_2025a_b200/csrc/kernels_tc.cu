// U-step element tangent of the 3D quadratic hex on the 5th-generation tensor cores (tcgen05).
//
// K_e (81x81) = sum_q B_q^T C_q B_q  (PhaseField.cpp:422).  Written per displacement-component
// block (a,b) with the physical shape gradients G_p(i;q):
//     K[(a,i),(b,j)] = sum_{q,p} G_p(i;q) * Z^{ab}[(q,p), j],
//     Z^{ab}[(q,p), j] = sum_r C_q[v(a,p), v(b,r)] G_r(j;q)       (v = Voigt index of (comp, dir))
// i.e. one GEMM per element  D[m=(a,b,j), n=i] = sum_k A[m,k] B[n,k]  with M = 243 (two M=128
// MMAs), N = 27 (padded to 32), K = (q,p) = 81 (padded to 96).
//
// Precision.  The operands go to the tensor cores as FP16 pairs x = hi + lo (kind::f16, FP32 accumulate)
// after an exact power-of-two scaling per element that keeps the largest possible |A| and |B| below 2^15
// (bounds recorded by the points kernel): D = Ahi*Bhi + Ahi*Blo + Alo*Bhi carries about 22 significant bits
// of the largest products (the dropped Alo*Blo is 2^-22 of them), and the FP16 range spans 28 octaves below
// the largest entry.  Bhi and Blo sit side by side as one N = 64 operand, so Ahi*[Bhi; Blo] is one MMA and
// Alo*Bhi (N = 32) a second one per k-step (K = 16) and tile: 24 MMAs per element.  A tcgen05.mma with
// M = 128 takes the same time for any N up to 192 (about 110 cycles for kind::f16 with A in TMEM, about 85
// for kind::tf32 with K = 8, measured), so the instruction count, not the arithmetic, sets the tensor-core
// time, and K = 16 per instruction halves it against TF32.  Within an ip pair (q, q') = (2 h, 2 h + 1) the
// K values are ordered 6 h + 2 p + o (ip 2 h + o, direction p), in A and in B alike.
//
// Operand placement.  A (= Z, 2 x 243 x 96 FP16 values per element) never touches shared memory: the
// thread that owns TMEM lane m builds row m = (a,b,j) in registers from the per-ip material tangents and
// the shape gradients and writes it into tensor memory with tcgen05.st (two K values per 32-bit column,
// the even one in the low half); the MMAs read A from TMEM.  B (= G, 27 rows) is staged in shared memory
// in the no-swizzle K-major canonical layout.  TMEM columns:
//     [0, 128)     accumulators of the two M tiles (64 columns each: Ahi Bhi + Alo Bhi, then Ahi Blo)
//     [128, 512)   A, double-buffered by element: buffer y, tile t, part (hi 0 / lo 1) at
//                  128 + 192 y + 48 (2 t + part)
//
// Schedule (one persistent CTA per SM; 16 builder warps, one MMA warp, 7 prep warps, 4 epilogue warps; the
// element counter n is CTA-local; inputs and A are double-buffered (x = n % 2), the tables and B
// triple-buffered (xb = n % 3)):
//   prep:      inputs of n landed (three bulk copies, issued one element ahead), the builders released the
//              tables of n-3 and the MMAs of n-3 completed -> gradient table and B(n) (5 warps, of which
//              126 threads have a task) and the material table (2 warps), scaled by the bounds the points
//              kernel recorded -> arrive
//              "tables full"(n) and "scale"(n);
//   builders:  "tables full"(n) and the MMAs of n-2 on their tile completed (A buffer x is reused) ->
//              A(n) of the tile in TMEM -> arrive "A ready"(n) and "tables free"(n);
//   MMA warp:  "A ready"(n) and "tables full"(n); per tile "accumulator free"(tile, n-1) -> 12 MMAs ->
//              commit to "done"(tile, n) (and "B free" after tile 1);
//   epilogue:  per tile "done"(tile, n) -> accumulator to registers -> arrive "accumulator free"(tile) ->
//              unscale (+ lumped diagonal) -> stores of the element matrix, coalesced across rows.
//   The builders run up to one element ahead of the MMAs, the tables of n+1 and n+2 can be built while A(n)
//   is, and the MMAs of tile 0 of n+1 start while tile 1 of n is read out.  No mbarrier can complete a
//   phase beyond the one its slowest waiter is waiting for, so the parity waits are unambiguous.
//
// Builder warp w owns TMEM lane quarter w % 4 of M tile (w / 4) % 2; warps w < 8 build K values [0, 42)
// of their rows (ips 0..13), warps 8..15 build [42, 96) (ips 14..26 and the K padding).  Epilogue warp w
// reads lane quarter w % 4 of both tiles.
//
// Every mbarrier wait is bounded; on time-out the kernel records an error word, lets its own MMAs and copies
// in flight finish (bounded), releases its TMEM and returns.

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

constexpr int TC_BUILD = 16;                // A-builder warps
constexpr int TC_PREP = 7;                  // table / B-operand warps (28 warps in all: 7 per scheduler)
constexpr int TC_PREP_G = 5;                // prep warps on the gradient table and B; the others build the
                                            // material table
constexpr int TC_EPI = 4;                   // epilogue warps (one per TMEM lane quarter)
constexpr int TC_W_MMA = TC_BUILD, TC_W_PREP = TC_BUILD + 1, TC_W_EPI = TC_W_PREP + TC_PREP;
constexpr int TC_ALL = 32 * (TC_W_EPI + TC_EPI);   // 896 threads
constexpr int TC_NT = 3;                    // table / B-operand buffers
constexpr int TC_KB = 244;                  // padded (node, comp, comp, node) row-block stride of K_e
constexpr int TC_K = 96;                    // K padded to a multiple of 16 (f16 k-step)
constexpr int TC_KCH = TC_K / 8;            // 16-byte chunks (8 FP16) per operand row
constexpr int TC_SBO = TC_KCH * 128;        // bytes between 8-row core-matrix groups (1536)
constexpr int TC_BROWS = 32;
constexpr int TC_BBYTES = TC_BROWS / 8 * TC_SBO;   // one 32-row operand (6144)
constexpr uint32_t TC_TMEM_COLS = 512;
constexpr uint32_t TC_COL_A = 128;          // A buffer y, region r (= 2 tile + lo) at TC_COL_A + 192 y + 48 r
constexpr uint32_t TC_AREG = 48;
constexpr uint32_t TC_ABUF = 4 * TC_AREG;
constexpr long long kWaitLimit = 1LL << 26;
constexpr float kTarget = 32768.0f;        // scaled operands stay below 2^15 (FP16 max 65504)

// per-element inputs, double-buffered and filled one element ahead by three bulk copies of the
// element-major blocks the points kernel writes (same layouts as in HBM)
struct alignas(16) TcStage {
  float C[36][27];          // w * (g D+ + D-) DPlast per ip
  float geo[13][27];        // Jinv (9), 1/wFun, dW/wFun^2 (3) per ip
  float geo_pad[kTcGeo - 13 * 27];
  float nx[2][3][3][3];     // 1-D basis tables [value / derivative][axis][ip coordinate][function]
  float W[27];              // nodal NURBS weights
  float cmax;               // max |C_q| of the element
  float gmax;               // an upper bound of max |G| of the element
  float nx_pad[kTcNx - 83];
};
constexpr uint32_t kStageTx = (uint32_t)(sizeof(float) * (kTcCq + kTcGeo + kTcNx));
static_assert(sizeof(TcStage) == kStageTx, "stage layout differs from the HBM blocks");
static_assert(offsetof(TcStage, geo) % 16 == 0 && offsetof(TcStage, nx) % 16 == 0,
              "bulk-copy destinations must be 16-byte aligned");

// A-build tables of one element over ip pairs (q, q') = (2 h, 2 h + 1), h < 14; the pad ip q' = 27 holds zeros
struct TcTables {
  float4 Gxy[14][27];      // (G_0(j;q), G_0(j;q'), G_1(j;q), G_1(j;q')), FP32, unscaled
  float2 Gz[14][27];       // (G_2(j;q), G_2(j;q'))
  float4 Cxy[14][3][6];    // 2^sA (C_q[s][v(b,0)], C_q'[s][v(b,0)], C_q[s][v(b,1)], C_q'[s][v(b,1)]) at [h][b][s]
  float2 Cz[14][3][6];     // 2^sA (C_q[s][v(b,2)], C_q'[s][v(b,2)])
};

struct TcSm {
  // B operand per buffer: rows 0..31 = 2^sB G hi, rows 32..63 = lo (one N = 64 operand, or its first 32 rows)
  alignas(128) unsigned char B[TC_NT][2 * TC_BBYTES];
  TcStage st[2];
  TcTables tb[TC_NT];
  float unscale[4];                     // 2^-(sA + sB) of element n, at n % 4
  unsigned long long mb_in[2];          // inputs of a stage landed (transaction count of the bulk copies)
  unsigned long long mb_tfull[TC_NT];   // tables and B of an element ready (one arrival per prep warp)
  unsigned long long mb_tfree[TC_NT];   // the builders are done with a table buffer (one arrival per builder warp)
  unsigned long long mb_bfree[TC_NT];   // the MMAs are done with a B buffer (tcgen05.commit)
  unsigned long long mb_afull[2];       // A of an element in TMEM buffer x (one arrival per builder warp)
  unsigned long long mb_done[2][2];     // [tile][n % 2]: the MMAs of the tile (and all before) completed
  unsigned long long mb_accfree[2];     // [tile]: accumulator read out (one arrival per epilogue warp)
  unsigned long long mb_scale[4];       // unscale[n % 4] written (prep thread 0)
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
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  // start address >> 4 [0,14), LBO = 128 B [16,30), SBO [32,46), version 1 [46,48), no swizzle
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)((uint32_t)TC_SBO >> 4) << 32) | (1ull << 46);
}

// kind::f16, D f32, A/B f16 K-major, M = 128, N = 32 or 64
constexpr uint32_t kIdesc32 = (1u << 4) | (0u << 7) | (0u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kIdesc64 = (1u << 4) | (0u << 7) | (0u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// D[tmem] (+)= A[tmem] * B[smem]^T
__device__ __forceinline__ void mma_f16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                           uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate));
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

__device__ __forceinline__ void mbar_arrive(uint32_t mbar_addr) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar_addr) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar_addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar_addr), "r"(count) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive TMEM columns of this thread's lane (no wait)
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t r[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// X consecutive TMEM columns of this thread's lane
template <int X>
__device__ __forceinline__ void tmem_stx(uint32_t taddr, const uint32_t* v) {
  if constexpr (X == 8) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]),
                 "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
  } else if constexpr (X == 4) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr), "r"(v[0]), "r"(v[1]),
                 "r"(v[2]), "r"(v[3])
                 : "memory");
  } else if constexpr (X == 2) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1,%2};" ::"r"(taddr), "r"(v[0]), "r"(v[1]) : "memory");
  } else {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(v[0]) : "memory");
  }
}

// columns [C0, C0 + N) of this lane, as naturally aligned x8 / x4 / x2 / x1 pieces
template <int C0, int N>
__device__ __forceinline__ void tmem_st_cols(uint32_t base, const uint32_t* v) {
  if constexpr (N > 0) {
    constexpr int X = (C0 % 8 == 0 && N >= 8) ? 8 : (C0 % 4 == 0 && N >= 4) ? 4 : (C0 % 2 == 0 && N >= 2) ? 2 : 1;
    tmem_stx<X>(base + C0, v);
    tmem_st_cols<C0 + X, N - X>(base, v + X);
  }
}

// two consecutive K values (even, odd) = (y.x, y.y) split into FP16 hi and lo, packed two per 32-bit word
// (even K in the low half): hi = rn(y), lo = rn(y - hi), with y - hi exact in FP32
__device__ __forceinline__ void split_f16x2(float2 y, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __floats2half2_rn(y.x, y.y);
  const float2 r = __ffma2_rn(__half22float2(h), make_float2(-1.0f, -1.0f), y);
  const __half2 l = __floats2half2_rn(r.x, r.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Row (a,b,j) of A over NH ip pairs from pair h0, split into FP16 hi / lo and packed into NC >= 3 NH
// columns; the columns beyond 3 NH are zero (K padding).  Within pair h the K values are ordered
// 6 h + 2 p + o for ip q = 2 h + o and direction p, so a column holds the two ips of one p: the packed FP32x2
// result of one dot product.  The material table carries the element's scale 2^sA.
template <int NH, int NC>
__device__ __forceinline__ void build_a_cols(const TcTables& s, bool row_ok, int a, int b, int j, int h0,
                                             uint32_t hi[NC], uint32_t lo[NC]) {
  const int s0 = voigt_idx(a, 0), s1 = voigt_idx(a, 1), s2 = voigt_idx(a, 2);
#pragma unroll
  for (int hh = 0; hh < NH; ++hh) {
    float2 y[3] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
    if (row_ok) {
      const int h = h0 + hh;
      const float4 gxy = s.Gxy[h][j];
      const float2 gz = s.Gz[h][j];
      const float2 g0 = make_float2(gxy.x, gxy.y), g1 = make_float2(gxy.z, gxy.w);
#pragma unroll
      for (int pp = 0; pp < 3; ++pp) {
        const int sv = pp == 0 ? s0 : pp == 1 ? s1 : s2;
        const float4 cxy = s.Cxy[h][b][sv];
        const float2 cz = s.Cz[h][b][sv];
        float2 acc = __fmul2_rn(make_float2(cxy.x, cxy.y), g0);
        acc = __ffma2_rn(make_float2(cxy.z, cxy.w), g1, acc);
        y[pp] = __ffma2_rn(cz, gz, acc);
      }
    }
    // K values 6 h .. 6 h + 5 = (q, p0) (q', p0) (q, p1) (q', p1) (q, p2) (q', p2)
#pragma unroll
    for (int pp = 0; pp < 3; ++pp) split_f16x2(y[pp], hi[3 * hh + pp], lo[3 * hh + pp]);
  }
#pragma unroll
  for (int c = 3 * NH; c < NC; ++c) { hi[c] = 0u; lo[c] = 0u; }
}

// named barrier over `NT` threads that also returns the OR of `x` over them (a group-uniform decision)
template <int ID, int NT>
__device__ __forceinline__ bool bar_or(bool x) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)x), "n"(ID), "n"(NT)
      : "memory");
  return r != 0;
}
constexpr int kBarPrep = 1, kBarEpi = 2;

__device__ __forceinline__ bool abort_seen(const TcSm& s) {
  return *reinterpret_cast<const volatile int*>(&s.abort_flag) != 0;
}

// Gradient table (FP32) and B operand (FP16 hi / lo rows, scaled by 2^sB) of one element, sum-factorised
// (NURBS3_Cube2.cpp:97-114): task (ip pair h, node row r = ja + 3 ka) keeps the ip geometry in registers and
// forms the three nodes ia = 0..2 of the row from shared y / z products.  Each node's B row gets the K values
// 6 h + 2 d + o (ip 2 h + o, direction d, the order of the A columns) as three 32-bit words; within a warp
// the words of one store fall in distinct banks except for rows r = 0 and 8 of one pair.  K values 84..95 and rows 27..31 of B stay zero from the initial clear.
__device__ __forceinline__ void build_g_and_b(TcTables& tb, unsigned char* B, const TcStage& st, float scale, int tp,
                                              int nt) {
  for (int task = tp; task < 14 * 9; task += nt) {
    const int r = task % 9, h = task / 9, ja = r % 3, ka = r / 3;
    float v[2][3][3];                                  // [ip of the pair][node ia][direction]
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      const int q = 2 * h + o;
      if (q < 27) {
        const int qx = q % 3, qy = (q / 3) % 3, qz = q / 9;
        const float ny = st.nx[0][1][qy][ja], nz = st.nx[0][2][qz][ka];
        const float nyz = ny * nz, dy = st.nx[1][1][qy][ja] * nz, dz = ny * st.nx[1][2][qz][ka];
        float J[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) J[i] = st.geo[i][q];
        const float rw = st.geo[9][q], w0 = st.geo[10][q], w1 = st.geo[11][q], w2 = st.geo[12][q];
#pragma unroll
        for (int ia = 0; ia < 3; ++ia) {
          const float nx = st.nx[0][0][qx][ia], dx = st.nx[1][0][qx][ia];
          const float Wn = st.W[ia + 3 * r];
          const float CB = nx * nyz;
          const float g0 = Wn * (dx * nyz * rw - CB * w0);
          const float g1 = Wn * (nx * dy * rw - CB * w1);
          const float g2 = Wn * (nx * dz * rw - CB * w2);
#pragma unroll
          for (int d = 0; d < 3; ++d) v[o][ia][d] = J[3 * d] * g0 + J[3 * d + 1] * g1 + J[3 * d + 2] * g2;
        }
      } else {
#pragma unroll
        for (int ia = 0; ia < 3; ++ia)
#pragma unroll
          for (int d = 0; d < 3; ++d) v[o][ia][d] = 0.0f;
      }
    }
#pragma unroll
    for (int ia = 0; ia < 3; ++ia) {
      const int nd = ia + 3 * r;
      tb.Gxy[h][nd] = make_float4(v[0][ia][0], v[1][ia][0], v[0][ia][1], v[1][ia][1]);
      tb.Gz[h][nd] = make_float2(v[0][ia][2], v[1][ia][2]);
#pragma unroll
      for (int wd = 0; wd < 3; ++wd) {               // direction d = wd: K values 6 h + 2 d, 6 h + 2 d + 1
        uint32_t hi, lo;
        split_f16x2(make_float2(scale * v[0][ia][wd], scale * v[1][ia][wd]), hi, lo);
        const int word = 3 * h + wd;                   // 32-bit word of the row: K values 2 word, 2 word + 1
        const uint32_t off = (uint32_t)((nd >> 3) * TC_SBO + (word >> 2) * 128 + (nd & 7) * 16 + (word & 3) * 4);
        *reinterpret_cast<uint32_t*>(B + off) = hi;
        *reinterpret_cast<uint32_t*>(B + TC_BBYTES + off) = lo;
      }
    }
  }
}

// material table of one element over ip pairs, scaled by 2^sA: C of ips 2h, 2h+1 side by side
__device__ __forceinline__ void build_c_table(TcTables& tb, const TcStage& st, float scale, int tp, int nt) {
  for (int i = tp; i < 14 * 3 * 6; i += nt) {
    const int h = i / 18, bb = (i / 6) % 3, sv = i % 6;
    const int q = 2 * h;
    float c0[3], c1[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int row = sv * 6 + voigt_idx(bb, r);
      c0[r] = scale * st.C[row][q];
      c1[r] = q + 1 < 27 ? scale * st.C[row][q + 1] : 0.0f;
    }
    tb.Cxy[h][bb][sv] = make_float4(c0[0], c1[0], c0[1], c1[1]);
    tb.Cz[h][bb][sv] = make_float2(c0[2], c1[2]);
  }
}

// 2^e for the integer e with m 2^e <= kTarget < 2 m 2^e (1 for m = 0 or a non-finite m)
__device__ __forceinline__ float pow2_scale(float m) {
  if (!(m > 0.0f) || !(m < 3.0e38f)) return 1.0f;
  int e;
  frexpf(kTarget / m, &e);        // kTarget / m = f 2^e, f in [0.5, 1)
  e -= 1;
  e = e < -126 ? -126 : (e > 127 ? 127 : e);
  return __int_as_float((127 + e) << 23);
}

__global__ void __launch_bounds__(TC_ALL, 1) k_u_tangent_tc(const TParams p, unsigned long long* err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcSm& s = *reinterpret_cast<TcSm*>(smraw);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const Geo& geo = p.geo;
  // TMEM lane quarter this warp may access
  const int quarter = warp & 3;
  const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;

  // zero the B operands once: their padding rows and K values are never written afterwards
  for (int i = t; i < TC_NT * 2 * TC_BBYTES / 16; i += TC_ALL)
    reinterpret_cast<float4*>(&s.B[0][0])[i] = make_float4(0, 0, 0, 0);
  if (t == 0) {
    s.abort_flag = 0;
    for (int x = 0; x < TC_NT; ++x) {
      mbar_init(smem_u32(&s.mb_tfull[x]), TC_PREP);
      mbar_init(smem_u32(&s.mb_tfree[x]), TC_BUILD);
      mbar_init(smem_u32(&s.mb_bfree[x]), 1);
    }
    for (int x = 0; x < 2; ++x) {
      mbar_init(smem_u32(&s.mb_in[x]), 1);
      mbar_init(smem_u32(&s.mb_afull[x]), TC_BUILD);
      mbar_init(smem_u32(&s.mb_done[0][x]), 1);
      mbar_init(smem_u32(&s.mb_done[1][x]), 1);
      mbar_init(smem_u32(&s.mb_accfree[x]), TC_EPI);
    }
    for (int i = 0; i < 4; ++i) mbar_init(smem_u32(&s.mb_scale[i]), 1);
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
  // shared addresses of the mbarrier arrays (consecutive 8-byte words)
  const uint32_t mb_in = smem_u32(&s.mb_in[0]), mb_tfull = smem_u32(&s.mb_tfull[0]);
  const uint32_t mb_tfree = smem_u32(&s.mb_tfree[0]), mb_afull = smem_u32(&s.mb_afull[0]);
  const uint32_t mb_bfree = smem_u32(&s.mb_bfree[0]);
  const uint32_t mb_done = smem_u32(&s.mb_done[0][0]);      // tile t, buffer x at +16 t + 8 x
  const uint32_t mb_accfree = smem_u32(&s.mb_accfree[0]);   // tile t at +8 t
  const uint32_t mb_scale = smem_u32(&s.mb_scale[0]);       // slot n % 4 at +8 (n % 4)

  if (warp < TC_BUILD) {
    // ---- builders: A(n) = rows (a,b,j) of this warp's lane quarter and K half, into TMEM buffer n % 2 ----
    const int tile = (warp >> 2) & 1, half = (warp >> 3) & 1;
    const int m = tile * 128 + quarter * 32 + lane;
    const bool row_ok = m < 243;
    const int ab = row_ok ? m / 27 : 0, j = row_ok ? m % 27 : 0, a = ab / 3, b = ab % 3;
    int n = 0, xb = 0, nb = 0;     // table buffer n % 3 and its use count n / 3
    for (int64_t el = geo.el0 + blockIdx.x; el < geo.el1; el += gridDim.x, ++n, xb = xb == TC_NT - 1 ? 0 : xb + 1,
                 nb += xb == 0) {
      const int x = n & 1;
      bool ok = mbar_wait_bounded(mb_tfull + 8 * xb, (uint32_t)nb & 1u);
      if (ok && n > 1)      // A buffer x is reused: the tile's MMAs of n-2 must have completed
        ok = mbar_wait_bounded(mb_done + 16 * tile + 8 * x, (uint32_t)((n >> 1) - 1) & 1u);
      if (__any_sync(0xffffffffu, !ok || abort_seen(s))) {
        if (lane == 0) atomicExch(&s.abort_flag, 1);
        break;
      }
      tc_fence_after();
      const TcTables& tb = s.tb[xb];
      const uint32_t base_hi = tmem + lane_off + TC_COL_A + (uint32_t)x * TC_ABUF + (uint32_t)(2 * tile) * TC_AREG;
      const uint32_t base_lo = base_hi + TC_AREG;
      if (half == 0) {                     // ip pairs 0..6 (ips 0..13) -> K [0, 42) = columns [0, 21)
        {
          uint32_t hi[12], lo[12];
          build_a_cols<4, 12>(tb, row_ok, a, b, j, 0, hi, lo);
          tmem_st_cols<0, 12>(base_hi, hi);
          tmem_st_cols<0, 12>(base_lo, lo);
        }
        uint32_t hi[9], lo[9];
        build_a_cols<3, 9>(tb, row_ok, a, b, j, 4, hi, lo);
        tmem_st_cols<12, 9>(base_hi, hi);
        tmem_st_cols<12, 9>(base_lo, lo);
      } else {                             // ip pairs 7..13 (ips 14..26, the zero pad ip) and the K padding
        {                                  // -> K [42, 96) = columns [21, 48)
          uint32_t hi[12], lo[12];
          build_a_cols<4, 12>(tb, row_ok, a, b, j, 7, hi, lo);
          tmem_st_cols<21, 12>(base_hi, hi);
          tmem_st_cols<21, 12>(base_lo, lo);
        }
        uint32_t hi[15], lo[15];
        build_a_cols<3, 15>(tb, row_ok, a, b, j, 11, hi, lo);
        tmem_st_cols<33, 15>(base_hi, hi);
        tmem_st_cols<33, 15>(base_lo, lo);
      }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(mb_afull + 8 * x);
        mbar_arrive(mb_tfree + 8 * xb);
      }
    }
  } else if (warp == TC_W_MMA) {
    // ---- MMA issuer: A(n), B(n) ready; per M tile the accumulator read out -> 12 MMAs -> commit ----
    int n = 0, xb = 0, nb = 0;
    int last = -1;             // 2 n + tile of the last commit issued (lane 0)
    bool ok = true;
    for (int64_t el = geo.el0 + blockIdx.x; el < geo.el1 && ok; el += gridDim.x, ++n, xb = xb == TC_NT - 1 ? 0 : xb + 1,
                 nb += xb == 0) {
      const int x = n & 1;
      ok = mbar_wait_bounded(mb_afull + 8 * x, (uint32_t)(n >> 1) & 1u);
      if (ok) ok = mbar_wait_bounded(mb_tfull + 8 * xb, (uint32_t)nb & 1u);
      const uint64_t db = smem_desc(smem_u32(s.B[xb]));
#pragma unroll 1
      for (int tl = 0; tl < 2 && ok; ++tl) {
        if (n > 0) ok = mbar_wait_bounded(mb_accfree + 8 * tl, (uint32_t)(n - 1) & 1u);
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        tc_fence_after();
        if (lane == 0) {
          // accumulator of tile tl: columns [64 tl, 64 tl + 32) = Ahi Bhi + Alo Bhi, [64 tl + 32, 64 tl + 64) = Ahi Blo
          const uint32_t dt = tmem + (uint32_t)(64 * tl);
          const uint32_t ahi = tmem + TC_COL_A + (uint32_t)x * TC_ABUF + (uint32_t)(2 * tl) * TC_AREG;
#pragma unroll
          for (int ks = 0; ks < TC_K / 16; ++ks) {   // k-step ks: +8 TMEM columns of A, +256 B (16 desc units) of B
            const uint64_t ko = (uint64_t)(ks * 16);
            mma_f16_ts(dt, ahi + (uint32_t)(8 * ks), db + ko, kIdesc64, ks > 0 ? 1u : 0u);
            mma_f16_ts(dt, ahi + TC_AREG + (uint32_t)(8 * ks), db + ko, kIdesc32, 1u);
          }
          mma_commit(mb_done + 16 * tl + 8 * x);
          if (tl == 1) mma_commit(mb_bfree + 8 * xb);     // B buffer xb may be rebuilt
          last = 2 * n + tl;
        }
        __syncwarp();
      }
      ok = __all_sync(0xffffffffu, ok);
      if (!ok && lane == 0) atomicExch(&s.abort_flag, 1);
    }
    // the CTA must not release TMEM under MMAs still running (only matters after an abort); the last
    // commit issued covers every MMA before it
    if (lane == 0 && last >= 0) {
      const int nl = last >> 1, tl = last & 1;
      mbar_wait_bounded(mb_done + 16 * tl + 8 * (nl & 1), (uint32_t)(nl >> 1) & 1u);
    }
    __syncwarp();
  } else if (warp < TC_W_EPI) {
    // ---- prep: inputs of n -> gradient table and B(n), material table ----
    const int tp = t - 32 * TC_W_PREP;
    constexpr int NT = 32 * TC_PREP;
    uint32_t pending = 0;     // bit x: a copy into stage x is in flight (issued by tp == 0)
    if (geo.el0 + (int64_t)blockIdx.x < geo.el1 && tp == 0) {
      tc_prefetch(s.st[0], p, geo.el0 + blockIdx.x, mb_in);
      pending = 1u;
    }
    int n = 0, xb = 0, nb = 0;
    for (int64_t el = geo.el0 + blockIdx.x; el < geo.el1; el += gridDim.x, ++n, xb = xb == TC_NT - 1 ? 0 : xb + 1,
                 nb += xb == 0) {
      const int x = n & 1;
      bool ok = mbar_wait_bounded(mb_in + 8 * x, (uint32_t)(n >> 1) & 1u);
      if (ok) pending &= ~(1u << x);
      if (ok && nb > 0) ok = mbar_wait_bounded(mb_tfree + 8 * xb, (uint32_t)(nb - 1) & 1u);   // A(n-3) built
      if (ok && nb > 0) ok = mbar_wait_bounded(mb_bfree + 8 * xb, (uint32_t)(nb - 1) & 1u);   // B(n-3) read
      if (!ok) atomicExch(&s.abort_flag, 1);
      // every prep thread is past element n-1, so its stage buffer can take element n+1
      if (bar_or<kBarPrep, NT>(!ok || abort_seen(s))) break;
      if (el + gridDim.x < geo.el1 && tp == 0) {
        tc_prefetch(s.st[x ^ 1], p, el + gridDim.x, mb_in + 8 * (x ^ 1));
        pending |= 1u << (x ^ 1);
      }
      const TcStage& st = s.st[x];
      TcTables& tb = s.tb[xb];
      // operand scales from the points kernel's bounds, exact powers of two: |B| <= max|G|,
      // |A| <= 3 max|C| max|G|
      const float sB = pow2_scale(st.gmax), sA = pow2_scale(3.0f * st.cmax * st.gmax);
      if (tp < 32 * TC_PREP_G)
        build_g_and_b(tb, s.B[xb], st, sB, tp, 32 * TC_PREP_G);
      else
        build_c_table(tb, st, sA, tp - 32 * TC_PREP_G, NT - 32 * TC_PREP_G);
      if (tp == 0) {
        s.unscale[n & 3] = (float)(1.0 / ((double)sA * (double)sB));
        mbar_arrive(mb_scale + 8 * (n & 3));
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // B is read by the MMAs
      __syncwarp();
      if (lane == 0) mbar_arrive(mb_tfull + 8 * xb);
    }
    // only after an abort: let input copies still in flight land before the CTA exits (bounded); stage y
    // holds element n or n + 1, whichever has parity y
#pragma unroll
    for (int y = 0; y < 2; ++y)
      if (pending & (1u << y)) mbar_wait_bounded(mb_in + 8 * y, (uint32_t)((((n & 1) == y ? n : n + 1)) >> 1) & 1u);
  } else {
    // ---- epilogue: per tile accumulator -> registers (signal "free") -> unscale -> stores ----
    constexpr int NT = 32 * TC_EPI;
    int n = 0;
    for (int64_t el = geo.el0 + blockIdx.x; el < geo.el1; el += gridDim.x, ++n) {
      const int x = n & 1;
      float* ke = reinterpret_cast<float*>(p.Ke) + el * (27 * TC_KB);
      bool ok = mbar_wait_bounded(mb_scale + 8 * (n & 3), (uint32_t)(n >> 2) & 1u);
      const float us = s.unscale[n & 3];
#pragma unroll 1
      for (int tl = 0; tl < 2; ++tl) {
        const int mm = tl * 128 + quarter * 32 + lane;
        const int abm = mm / 27, jm = mm % 27;
        // lumped diagonal term of this row (inertia / damping), read ahead of the wait
        const double kd = (mm < 243 && abm / 3 == abm % 3) ? __ldg(p.Kd + el * kTcKd + jm) : 0.0;
        if (ok) ok = mbar_wait_bounded(mb_done + 16 * tl + 8 * x, (uint32_t)(n >> 1) & 1u);
        if (!ok) atomicExch(&s.abort_flag, 1);
        if (bar_or<kBarEpi, NT>(!ok || abort_seen(s))) {
          ok = false;
          break;
        }
        tc_fence_after();
        // the row's 27 columns: (Ahi + Alo) Bhi + Ahi Blo, summed and unscaled in registers; the accumulator
        // is released before the stores, and the stores of one column of the element matrix are coalesced
        // across the lanes (rows)
        float v[27];
        {
          uint32_t xv[16], yv[16];
          tmem_ld16_nowait(tmem + lane_off + (uint32_t)(64 * tl), xv);
          tmem_ld16_nowait(tmem + lane_off + (uint32_t)(64 * tl + 32), yv);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] = (__uint_as_float(xv[i]) + __uint_as_float(yv[i])) * us;
        }
        {
          uint32_t xv[16], yv[16];
          tmem_ld16_nowait(tmem + lane_off + (uint32_t)(64 * tl + 16), xv);
          tmem_ld16_nowait(tmem + lane_off + (uint32_t)(64 * tl + 48), yv);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 11; ++i) v[16 + i] = (__uint_as_float(xv[i]) + __uint_as_float(yv[i])) * us;
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(mb_accfree + 8 * tl);   // the next element's MMAs may overwrite it
        if (mm < 243) {
          float vd = 0.0f;
#pragma unroll
          for (int col = 0; col < 27; ++col) {
            ke[col * TC_KB + mm] = v[col];
            vd = col == jm ? v[col] : vd;
          }
          // diagonal blocks: the lumped inertia / damping term on the node's own column (rewritten)
          if (kd != 0.0) ke[jm * TC_KB + mm] = (float)((double)vd + kd);
        } else if (mm == 243) {              // the row-block padding entry
#pragma unroll
          for (int col = 0; col < 27; ++col) ke[col * TC_KB + mm] = 0.0f;
        }
      }
      if (!ok) break;
    }
  }
  __syncthreads();
  if (s.abort_flag && t == 0) atomicExch(err, 1ull);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
}

}  // namespace

size_t tc_smem_bytes() { return sizeof(TcSm); }

void launch_u_tangent_tc(const TParams& p, unsigned long long* err, int n_sm, cudaStream_t s) {
  const int64_t nel = p.geo.el1 - p.geo.el0;
  if (nel <= 0) return;
  const size_t smem = sizeof(TcSm);
  cudaFuncSetAttribute(k_u_tangent_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int64_t grid = nel < n_sm ? nel : n_sm;
  k_u_tangent_tc<<<(unsigned)grid, TC_ALL, smem, s>>>(p, err);
}

}  // namespace ifem
