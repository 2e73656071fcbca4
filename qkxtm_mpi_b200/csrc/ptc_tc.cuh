// ptc_tc.cuh -- tensor-core (tcgen05) form of the 16 -> 16 channel PTC layer
// of ptc.cuh, used for inference (the solver's preconditioner applications).
//
// The layer is a GEMM per colour a: D_a[site][n] = sum_k A_a[site][k] B[k][n]
// with k = (path p, input channel c', re/im) and n = (output channel c, re/im):
//   A_a[site][p, c', re/im] = (T_p in)(site)[c'][a]   (transported, BF16)
//   B[p, c', .][c, .] = the real 2x2 block [[Re W, -Im W], [Im W, Re W]] of W[p][c][c']
// One CTA owns 128 consecutive sites of one parity (the 128 rows of an
// M = 128, N = 32 MMA) and walks the 9 paths as K chunks of 32:
//   * every thread transports its site's 16 channels along path p and writes
//     them, rounded to BF16, into a shared-memory A chunk (no-swizzle K-major
//     canonical layout: 8-row x 16-byte core matrices, 128 B apart along K,
//     512 B apart along M), two chunks in flight;
//   * thread 0 issues, per colour, two kind::f16 MMAs (K = 16 each) into a
//     TMEM accumulator of 32 FP32 columns and commits them to the chunk's
//     mbarrier, so the next chunk's transport overlaps the MMAs;
//   * after the last chunk each warp reads its 32 lanes (sites) back with
//     tcgen05.ld and stores the output activation.
// Waits on an mbarrier are bounded: on timeout the kernel records an error
// code, still waits (bounded) for its MMAs, frees its TMEM and returns.
#pragma once
#include <cuda_bf16.h>

#include "ptc.cuh"

namespace qkx {

constexpr int TC_M = 128;                 // sites per CTA (MMA rows)
constexpr int TC_K = 32;                  // K per path chunk: 16 channels x (re, im)
constexpr int TC_N = 32;                  // N: 16 channels x (re, im)
constexpr int TC_ACHUNK = TC_M * TC_K;    // BF16 per colour per chunk (8 KB)
constexpr int TC_BPATH = TC_N * TC_K;     // BF16 per path of B (2 KB)
constexpr uint32_t TC_LBO = 128;          // bytes between K-adjacent core matrices
constexpr uint32_t TC_SBO = 512;          // bytes between M-adjacent core matrices (4 along K)
constexpr unsigned long long TC_WAIT_NS = 100000000ull;  // an mbarrier wait gives up after 100 ms

// byte offset of element (row, k) in a [rows][32] K-major no-swizzle canonical tile
__device__ __forceinline__ uint32_t tc_off(int row, int k) {
  return (uint32_t)((row >> 3) * TC_SBO + (k >> 3) * TC_LBO + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((TC_LBO >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((TC_SBO >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: F32 accumulate, BF16 A and B, both K-major, N = 32, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// device clock in nanoseconds
__device__ __forceinline__ unsigned long long tc_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait for phase `parity` of the barrier; false once TC_WAIT_NS of wall time have
// passed without it (a try_wait may itself suspend, so the bound is on time, not polls)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const unsigned long long t0 = tc_clock_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (tc_clock_ns() - t0 > TC_WAIT_NS) return false;
  }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
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
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

struct __align__(16) TcSmem {
  __nv_bfloat16 A[2][3][TC_ACHUNK];  // two path chunks x 3 colours, 48 KB
  __nv_bfloat16 B[9][TC_BPATH];      // the real-block weights of all paths, 18 KB
  uint64_t bar[2];
  uint32_t tmem;
};

// One 16 -> 16 PTC layer on the tensor cores, BF16 activations in and out.  Blocks
// alternate parities when npar = 2 (npar = 1: parity par0 only); 128 threads (4
// warps) per block, one site each.  err (if not null) receives a non-zero code
// when a wait timed out.
__global__ void __launch_bounds__(TC_M) k_ptc_layer_tc(PtcField in, PtcField out, const __nv_bfloat162* __restrict__ w,
                                                       GaugeF32x12 u, Geom g, int par0, int npar, int* err) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int par = npar == 2 ? (blockIdx.x & 1) : par0;
  const int cb = (npar == 2 ? (blockIdx.x >> 1) : blockIdx.x) * TC_M + tid;
  const bool valid = cb < g.Vh;

  // B: real 2x2 blocks of W[p][c][c'] at (n = 2c + i, k = 2c' + j), canonical K-major
  for (int e = tid; e < 9 * 16 * 16; e += TC_M) {
    const int p = e / 256, c = (e / 16) % 16, cp = e % 16;
    const __nv_bfloat162 wv = w[e];
    unsigned char* base = reinterpret_cast<unsigned char*>(sm.B[p]);
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c, 2 * cp)) = wv.x;
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c, 2 * cp + 1)) = __hneg(wv.y);
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c + 1, 2 * cp)) = wv.y;
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c + 1, 2 * cp + 1)) = wv.x;
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem;

  int x[4] = {0, 0, 0, 0};
  int s = 0;
  if (valid) {
    cb_coords(g, cb, par, x);
    s = x[0] + g.L[0] * (x[1] + g.L[1] * (x[2] + g.L[2] * x[3]));
  }
  bool ok = true;
  for (int p = 0; p < 9; p++) {
    const int b = p & 1;
    // the chunk written two paths ago must have been consumed by its MMAs
    if (p >= 2 && !mbar_wait(&sm.bar[b], ((p - 2) >> 1) & 1)) ok = false;
    unsigned char* Abase = reinterpret_cast<unsigned char*>(sm.A[b][0]);
    Link<float> U;
    PtcHop h{par, cb};
    if (valid) h = ptc_hop(u, g, par, valid ? cb : 0, x, s, p, U);
#pragma unroll 1
    for (int c4 = 0; c4 < 16; c4 += 4) {  // four channels = one 16-byte K group
      float2 t[4][3];
      if (valid) {
        float2 v[4][3];
        ptc_load4<false>(in, g.Vh, h.npar, h.n, c4 / 4, v);
#pragma unroll
        for (int cl = 0; cl < 4; cl++) {
          if (p == 0) {
#pragma unroll
            for (int a = 0; a < 3; a++) t[cl][a] = v[cl][a];
          } else {
            ptc_mv(U, v[cl], t[cl]);
          }
        }
      } else {
#pragma unroll
        for (int cl = 0; cl < 4; cl++)
#pragma unroll
          for (int a = 0; a < 3; a++) t[cl][a] = make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int a = 0; a < 3; a++) {
        __nv_bfloat162 q0 = __floats2bfloat162_rn(t[0][a].x, t[0][a].y);
        __nv_bfloat162 q1 = __floats2bfloat162_rn(t[1][a].x, t[1][a].y);
        __nv_bfloat162 q2 = __floats2bfloat162_rn(t[2][a].x, t[2][a].y);
        __nv_bfloat162 q3 = __floats2bfloat162_rn(t[3][a].x, t[3][a].y);
        uint4 pk;
        pk.x = *reinterpret_cast<uint32_t*>(&q0);
        pk.y = *reinterpret_cast<uint32_t*>(&q1);
        pk.z = *reinterpret_cast<uint32_t*>(&q2);
        pk.w = *reinterpret_cast<uint32_t*>(&q3);
        *reinterpret_cast<uint4*>(Abase + a * TC_ACHUNK * 2 + tc_off(tid, 2 * c4)) = pk;
      }
    }
    // make the chunk visible to the tensor cores, then one thread issues its MMAs
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sm.A[b][0]);
      const uint32_t b0 = smem_u32(sm.B[p]);
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
          tc_mma(tmem + a * TC_N, tc_desc(a0 + a * TC_ACHUNK * 2 + kk * 2 * TC_LBO), tc_desc(b0 + kk * 2 * TC_LBO),
                 (p > 0 || kk > 0) ? 1u : 0u);
      tc_commit(&sm.bar[b]);
    }
  }
  // completions: bar[0] at p = 0, 2, 4, 6, 8 (5th has parity 0); bar[1] at p = 1, 3, 5, 7 (4th, parity 1)
  if (!mbar_wait(&sm.bar[0], 0)) ok = false;
  if (!mbar_wait(&sm.bar[1], 1)) ok = false;
  tc_fence_after();
  if (ok) {
    float d[3][32];
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int a = 0; a < 3; a++) tc_ld32(lane_base + a * TC_N, d[a]);
    if (valid) {
      // BF16 layout: group q of four channels, word wd holds complex k = 4 wd + j (channel
      // 4q + k/3, colour k%3) in slot j
      uint4* o = static_cast<uint4*>(out.p[par]) + cb;
#pragma unroll
      for (int q = 0; q < 4; q++)
#pragma unroll
        for (int wd = 0; wd < 3; wd++) {
          uint32_t e[4];
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const int k = 4 * wd + j, ch = 4 * q + k / 3, col = k % 3;
            e[j] = ptc_f2bf(make_float2(d[col][2 * ch], d[col][2 * ch + 1]));
          }
          o[(size_t)(3 * q + wd) * g.Vh] = make_uint4(e[0], e[1], e[2], e[3]);
        }
    }
  } else if (err && tid == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

}  // namespace qkx
