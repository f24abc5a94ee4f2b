// U-step element tangent of the 3D quadratic hex on the 5th-generation tensor cores (tcgen05).
//
// K_e (81x81) = sum_q B_q^T C_q B_q  (PhaseField.cpp:422).  Written per displacement-component
// block (a,b) with the physical shape gradients G_p(i;q):
//     K[(a,i),(b,j)] = sum_{q,p} G_p(i;q) * Z^{ab}[(q,p), j],
//     Z^{ab}[(q,p), j] = sum_r C_q[v(a,p), v(b,r)] G_r(j;q)       (v = Voigt index of (comp, dir))
// i.e. one GEMM per element  D[m=(a,b,j), n=i] = sum_k A[m,k] B[n,k]  with M = 243 (two M=128
// MMAs), N = 27 (padded to 32), K = (q,p) = 81 (padded to 88).  A (= Z, built on CUDA cores from
// the per-ip material tangents) and B (= G) are staged in shared memory in the no-swizzle
// K-major canonical layout; the accumulator lives in TMEM.  For an FP32-accurate tangent each
// operand is split x = hi + lo into TF32 parts and D = Ahi*Bhi + Ahi*Blo + Alo*Bhi (FP32
// accumulate), so the error is O(2^-22) instead of TF32's 2^-11.
//
// TMEM lane m of tile t holds row m = 128 t + lane; a warp reads its lane quarter with
// tcgen05.ld, and since D[(a,b,j), i] is K_e[i][a][b][j] (the node-row-major layout the gather
// consumes) the 27 columns of a thread go to addresses i*243 + m: consecutive threads write
// consecutive words.
//
// One persistent CTA of 256 threads per SM walks the elements.  Every wait on the MMA-completion
// mbarrier is bounded; on time-out the kernel records an error word, waits (bounded) once more,
// releases its TMEM and returns.

#include <cuda_runtime.h>
#include <cstdint>

#include "device_common.cuh"
#include "icefem_internal.h"

namespace ifem {

namespace {

constexpr int TC_THREADS = 256;
constexpr int TC_KB = 244;                  // padded (node, comp, comp, node) row-block stride of K_e
constexpr int TC_K = 88;                    // K padded to a multiple of 8 (tf32 k-step)
constexpr int TC_KCH = TC_K / 4;            // 16-byte chunks per row
constexpr int TC_SBO = TC_KCH * 128;        // bytes between 8-row core-matrix groups
constexpr int TC_AROWS = 256;
constexpr int TC_BROWS = 32;
constexpr int TC_ABYTES = TC_AROWS / 8 * TC_SBO;   // 90112
constexpr int TC_BBYTES = TC_BROWS / 8 * TC_SBO;   // 11264
constexpr uint32_t TC_TMEM_COLS = 64;
constexpr long long kWaitLimit = 1LL << 26;

// per-element inputs, double-buffered and filled by cp.async one element ahead
struct TcStage {
  float geo[13][27];       // Jinv (9), 1/wFun, dW/wFun^2 (3) per ip (same [k][q] order as in HBM)
  float C[36][27];         // w * (g D+ + D-) DPlast per ip
  double ext[27];          // 1-D extraction factors [axis][3][3]
  double WL[27];           // lumped weights (diagonal inertia / damping terms)
  int conn[27];
};

struct TcSm {
  alignas(128) unsigned char Ahi[TC_ABYTES];
  alignas(128) unsigned char Alo[TC_ABYTES];
  alignas(128) unsigned char Bhi[TC_BBYTES];
  alignas(128) unsigned char Blo[TC_BBYTES];
  TcStage st[2];
  float4 Cb[27][3][6];     // Cb[q][b][s] = (C_q[s][v(b,0)], C_q[s][v(b,1)], C_q[s][v(b,2)], 0)
  float NX[3][3][3], GX[3][3][3];
  float W[27];
  unsigned long long mbar;
  uint32_t tmem_base;
  int abort_flag;
};

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// enqueue the copies of element `el`'s inputs into a staging buffer
__device__ __forceinline__ void tc_prefetch(TcStage& st, const TParams& p, int64_t el, int t) {
  const float* Cq = reinterpret_cast<const float*>(p.Cq);
  const int64_t nh = p.nh;
  for (int i = t; i < 13 * 27; i += TC_THREADS) {
    const int k = i / 27, q = i % 27;
    cp_async4(&st.geo[k][q], p.geoq + (int64_t)k * nh + el * 27 + q);
  }
  for (int i = t; i < 36 * 27; i += TC_THREADS) {
    const int k = i / 27, q = i % 27;
    cp_async4(&st.C[k][q], Cq + (int64_t)k * nh + el * 27 + q);
  }
  if (t < 27) {
    cp_async8(&st.ext[t], p.geo.ext + el * 27 + t);
    cp_async8(&st.WL[t], p.WLe + el * 27 + t);
    cp_async4(&st.conn[t], p.geo.conn + el * 27 + t);
  }
  cp_async_commit();
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
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
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

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_u_tangent_tc(const TParams p, unsigned long long* err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcSm& s = *reinterpret_cast<TcSm*>(smraw);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const Geo& geo = p.geo;

  // zero the operands once: padding rows / k columns stay zero for every element
  for (int i = t; i < TC_ABYTES / 16; i += TC_THREADS) {
    reinterpret_cast<float4*>(s.Ahi)[i] = make_float4(0, 0, 0, 0);
    reinterpret_cast<float4*>(s.Alo)[i] = make_float4(0, 0, 0, 0);
  }
  for (int i = t; i < TC_BBYTES / 16; i += TC_THREADS) {
    reinterpret_cast<float4*>(s.Bhi)[i] = make_float4(0, 0, 0, 0);
    reinterpret_cast<float4*>(s.Blo)[i] = make_float4(0, 0, 0, 0);
  }
  if (t == 0) {
    s.abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mbar)) : "memory");
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
  const uint32_t mbar = smem_u32(&s.mbar);
  uint32_t parity = 0;
  const uint32_t aHi = smem_u32(s.Ahi), aLo = smem_u32(s.Alo), bHi = smem_u32(s.Bhi), bLo = smem_u32(s.Blo);

  int cur = 0;
  if ((int64_t)blockIdx.x < geo.nel) tc_prefetch(s.st[0], p, blockIdx.x, t);
  for (int64_t el = blockIdx.x; el < geo.nel; el += gridDim.x, cur ^= 1) {
    cp_async_wait_all();
    __syncthreads();                      // stage `cur` landed; the previous element is finished
    if (el + gridDim.x < geo.nel) tc_prefetch(s.st[cur ^ 1], p, el + gridDim.x, t);
    TcStage& st = s.st[cur];
    // ---- per-element tables: Cb, 1-D factors, NURBS weights ----
    for (int i = t; i < 27 * 3 * 6; i += TC_THREADS) {
      const int q = i % 27, rest = i / 27, b = rest % 3, sv = rest / 3;
      s.Cb[q][b][sv] = make_float4(st.C[sv * 6 + voigt_idx(b, 0)][q], st.C[sv * 6 + voigt_idx(b, 1)][q],
                                   st.C[sv * 6 + voigt_idx(b, 2)][q], 0.0f);
    }
    if (t >= 224 && t < 224 + 27) {
      const int i = t - 224, ax = i / 9, pt = (i / 3) % 3, fn = i % 3;
      double sN = 0, sG = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) { sN += st.ext[ax * 9 + fn * 3 + k] * p.rule.B[pt][k]; sG += st.ext[ax * 9 + fn * 3 + k] * p.rule.dB[pt][k]; }
      s.NX[ax][pt][fn] = (float)sN;
      s.GX[ax][pt][fn] = (float)sG;
    } else if (t >= 192 && t < 192 + 27) {
      s.W[t - 192] = geo.W ? (float)geo.W[st.conn[t - 192]] : 1.0f;
    }
    __syncthreads();
    // ---- B operand: rows = nodes a, k = 3q + d (G_d(a;q), NURBS3_Cube2.cpp:97-114), 4 ips per task ----
    if (t < 27 * 7) {
      const int a = t % 27, qg = t / 27;
      const int ia = a % 3, ja = (a / 3) % 3, ka = a / 9;
      float v[12];
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        const int q = qg * 4 + qq;
        if (q < 27) {
          const int qx = q % 3, qy = (q / 3) % 3, qz = q / 9;
          const float nx = s.NX[0][qx][ia], ny = s.NX[1][qy][ja], nz = s.NX[2][qz][ka];
          const float CB = nx * ny * nz;
          const float GB0 = s.GX[0][qx][ia] * ny * nz, GB1 = nx * s.GX[1][qy][ja] * nz, GB2 = nx * ny * s.GX[2][qz][ka];
          const float rw = st.geo[9][q];
          const float g0 = s.W[a] * (GB0 * rw - CB * st.geo[10][q]);
          const float g1 = s.W[a] * (GB1 * rw - CB * st.geo[11][q]);
          const float g2 = s.W[a] * (GB2 * rw - CB * st.geo[12][q]);
#pragma unroll
          for (int d = 0; d < 3; ++d)
            v[qq * 3 + d] = st.geo[d * 3 + 0][q] * g0 + st.geo[d * 3 + 1][q] * g1 + st.geo[d * 3 + 2][q] * g2;
        } else {
#pragma unroll
          for (int d = 0; d < 3; ++d) v[qq * 3 + d] = 0.0f;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float4 h, l;
        h.x = tf32_rna(v[4 * c + 0]); l.x = tf32_rna(v[4 * c + 0] - h.x);
        h.y = tf32_rna(v[4 * c + 1]); l.y = tf32_rna(v[4 * c + 1] - h.y);
        h.z = tf32_rna(v[4 * c + 2]); l.z = tf32_rna(v[4 * c + 2] - h.z);
        h.w = tf32_rna(v[4 * c + 3]); l.w = tf32_rna(v[4 * c + 3] - h.w);
        const uint32_t off = kmajor_off(a, 12 * qg + 4 * c);
        *reinterpret_cast<float4*>(s.Bhi + off) = h;
        *reinterpret_cast<float4*>(s.Blo + off) = l;
      }
    }
    __syncthreads();
    // ---- A operand: A[(a,b,j)][3q+p] = y_{v(a,p)},  y_s = sum_r C_q[s][v(b,r)] G_r(j;q), 4 ips per task ----
    for (int task = t; task < 27 * 3 * 7; task += TC_THREADS) {
      const int j = task % 27, rest = task / 27, b = rest % 3, qg = rest / 3;
      float g[12];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const uint32_t off = kmajor_off(j, 12 * qg + 4 * c);
        const float4 h = *reinterpret_cast<const float4*>(s.Bhi + off);
        const float4 l = *reinterpret_cast<const float4*>(s.Blo + off);
        g[4 * c + 0] = h.x + l.x; g[4 * c + 1] = h.y + l.y; g[4 * c + 2] = h.z + l.z; g[4 * c + 3] = h.w + l.w;
      }
      float y[4][6];
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        const int q = qg * 4 + qq;
#pragma unroll
        for (int sv = 0; sv < 6; ++sv) {
          if (q < 27) {
            const float4 c4 = s.Cb[q][b][sv];
            y[qq][sv] = c4.x * g[3 * qq] + c4.y * g[3 * qq + 1] + c4.z * g[3 * qq + 2];
          } else {
            y[qq][sv] = 0.0f;
          }
        }
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float v[12];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq)
#pragma unroll
          for (int pp = 0; pp < 3; ++pp) v[3 * qq + pp] = y[qq][voigt_idx(a, pp)];
        const int m = (a * 3 + b) * 27 + j;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float4 h, l;
          h.x = tf32_rna(v[4 * c + 0]); l.x = tf32_rna(v[4 * c + 0] - h.x);
          h.y = tf32_rna(v[4 * c + 1]); l.y = tf32_rna(v[4 * c + 1] - h.y);
          h.z = tf32_rna(v[4 * c + 2]); l.z = tf32_rna(v[4 * c + 2] - h.z);
          h.w = tf32_rna(v[4 * c + 3]); l.w = tf32_rna(v[4 * c + 3] - h.w);
          const uint32_t off = kmajor_off(m, 12 * qg + 4 * c);
          *reinterpret_cast<float4*>(s.Ahi + off) = h;
          *reinterpret_cast<float4*>(s.Alo + off) = l;
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
#pragma unroll 1
      for (int ks = 0; ks < TC_K / 8; ++ks) {      // the two M tiles alternate: independent chains
        const uint32_t ko = (uint32_t)(ks * 256);
#pragma unroll
        for (int tile = 0; tile < 2; ++tile) {
          const uint32_t dt = tmem + (uint32_t)(tile * 32);
          const uint32_t aoff = (uint32_t)(tile * 16 * TC_SBO);
          mma_tf32(dt, smem_desc(aHi + aoff + ko), smem_desc(bHi + ko), ks > 0 ? 1u : 0u);
          mma_tf32(dt, smem_desc(aHi + aoff + ko), smem_desc(bLo + ko), 1u);
          mma_tf32(dt, smem_desc(aLo + aoff + ko), smem_desc(bHi + ko), 1u);
        }
      }
      mma_commit(mbar);
    }
    __syncwarp();
    const bool ok = mbar_wait_bounded(mbar, parity);
    parity ^= 1u;
    if (!ok) {
      if (lane == 0) atomicExch(&s.abort_flag, 1);
    }
    tc_fence_after();
    __syncthreads();
    if (s.abort_flag) break;
    // read the accumulator: warp w -> TMEM lanes 32 (w%4).., tile w/4
    {
      const int quarter = warp & 3, tile = warp >> 2;
      const int m = tile * 128 + quarter * 32 + lane;
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(tile * 32), v);
      if (m < 243) {
        const int ab = m / 27, j = m % 27, a = ab / 3, b = ab % 3;
        double add = 0;   // diagonal lumped terms (PhaseField.cpp:441-468), added after the ip sum
        if (a == b) {
          const MatDev& mat = geo.mats[geo.emat ? geo.emat[el] : 0];
          const TcStage& st = s.st[cur];
          if (p.mo.inertia) {
            double DamI, d1, d2;
            const double ph = p.phase_cur[p.dm.base[IFEM_DOF_PHASE] + p.dm.node_rank[st.conn[j]]];
            damage_function(ph, p.mo.dens_f, p.mo.k0, DamI, d1, d2);
            add += st.WL[j] * DamI * mat.density * p.ddu_dt;
          }
          if (mat.damping > 0.0) add += st.WL[j] * mat.damping * p.du_dt;
        }
        float* Ke = reinterpret_cast<float*>(p.Ke) + el * (27 * TC_KB);
        // static register indices only (a dynamic v[j] would put v in local memory)
#pragma unroll
        for (int i = 0; i < 27; ++i) Ke[i * TC_KB + m] = (i == j && add != 0.0) ? (float)((double)v[i] + add) : v[i];
      }
    }
    tc_fence_before();
  }
  cp_async_wait_all();
  __syncthreads();
  if (s.abort_flag) {
    if (t == 0) atomicExch(err, 1ull);
    mbar_wait_bounded(mbar, parity ^ 1u);   // the MMAs of the failed wait, once more, bounded
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
  k_u_tangent_tc<<<(unsigned)grid, TC_THREADS, smem, s>>>(p, err);
}

}  // namespace ifem
