// ptc_tc.cuh -- tensor-core (tcgen05) form of the PTC layers of ptc.cuh with 16
// channels on one side (4 -> 16, 16 -> 16, 16 -> 4), used in training and in the
// solver's preconditioner applications.
//
// The layer is a GEMM per colour a: D_a[site][n] = sum_k A_a[site][k] B[k][n]
// with k = (path p, input channel c', re/im) and n = (output channel c, re/im):
//   A_a[site][p, c', re/im] = (T_p in)(site)[c'][a]   (transported, BF16)
//   B[p, c', .][c, .] = the real 2x2 block [[Re W, -Im W], [Im W, Re W]] of W[p][c][c']
// One CTA owns 128 consecutive sites of one parity (the 128 rows of an
// M = 128, N = 2 CO (at least 16) MMA) and walks the 9 paths as K chunks of 32
// (one path of 16 input channels, or four paths of 4):
//   * every thread transports its site's input channels along the paths with packed
//     BF16 complex FMAs (the link rounded to BF16; the A operand is BF16 in any
//     case) and writes them into a shared-memory A chunk (no-swizzle K-major
//     canonical layout: 8-row x 16-byte core matrices, 128 B apart along K,
//     512 B apart along M), one chunk buffer;
//   * thread 0 issues, per colour, two kind::f16 MMAs (K = 16 each) into a
//     TMEM accumulator of N FP32 columns and commits them to the chunk's
//     mbarrier; the next chunk's loads and transport run before the wait for
//     those MMAs;
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
constexpr int TC_N = 32;                  // N: up to 16 output channels x (re, im)
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

// instruction descriptor: F32 accumulate, BF16 A and B, both K-major, N columns, M = 128
template <int N>
constexpr uint32_t tc_idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <int N>
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(tc_idesc<N>()), "r"(accumulate));
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

// One A chunk (24 KB) rather than two: with 42 KB of shared memory a block, four blocks fit
// an SM (the register bound) and L1 keeps ~90 KB for the neighbour loads.  A chunk is
// rewritten only after the MMAs that read it completed; they take a small fraction of the
// time the next path's loads and transport take, and those run before the wait.
struct __align__(16) TcSmem {
  __nv_bfloat16 A[3][TC_ACHUNK];  // one path chunk x 3 colours, 24 KB
  __nv_bfloat16 B[9][TC_BPATH];   // the real-block weights of all paths, 18 KB
  uint64_t bar;
  uint32_t tmem;
};

// One CI -> CO PTC layer on the tensor cores.  CI = 16 takes BF16 activations; CI = 4 takes
// BF16 or, for IN32, the FP32 4-channel spinor layout.  CO = 16 gives BF16; CO = 4 gives
// BF16 or, for OUT32, the FP32 spinor layout, with N = 16 MMA columns of which the upper
// half multiplies zero weights.  A K chunk of 32 holds the 2 CI reals of PPC = 32 / (2 CI)
// paths: one path for CI = 16 (9 chunks), four for CI = 4 (3 chunks, the last with one
// path and three zero slots).  Blocks alternate parities when npar = 2 (npar = 1: parity
// par0 only); 128 threads (4 warps) per block, one site each.  err (if not null) receives a
// non-zero code when a wait timed out.
template <int CI, int CO, bool IN32, bool OUT32>
__global__ void __launch_bounds__(TC_M, 5) k_ptc_layer_tc(PtcField in, PtcField out, const __nv_bfloat162* __restrict__ w,
                                                       GaugeF32x12 u, Geom g, int par0, int npar, int* err) {
  static_assert((CI == 16 && !IN32) || CI == 4, "input width");
  static_assert((CO == 16 && !OUT32) || CO == 4, "output width");
  constexpr int N = 2 * CO < 16 ? 16 : 2 * CO;  // MMA columns (M = 128 takes N >= 16)
  constexpr int PPC = TC_K / (2 * CI);          // paths per K chunk
  constexpr int NCH = (9 + PPC - 1) / PPC;      // K chunks
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int par = npar == 2 ? (blockIdx.x & 1) : par0;
  const int cb = (npar == 2 ? (blockIdx.x >> 1) : blockIdx.x) * TC_M + tid;
  const bool valid = cb < g.Vh;

  // B of chunk ch: the real 2x2 blocks of W[p][c][c'], p = ch PPC + j, at rows n = 2c + i and
  // K index k = 2 CI j + 2c' + jj, canonical K-major; zero elsewhere (rows from 2 CO, slots
  // of paths past the ninth)
  for (int e = tid; e < NCH * N * TC_K; e += TC_M) {
    const int ch = e / (N * TC_K), n = (e / TC_K) % N, k = e % TC_K;
    *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(sm.B[ch]) + tc_off(n, k)) =
        __float2bfloat16(0.f);
  }
  __syncthreads();
  for (int e = tid; e < 9 * CO * CI; e += TC_M) {
    const int p = e / (CO * CI), c = (e / CI) % CO, cp = e % CI;
    const int k0 = 2 * CI * (p % PPC) + 2 * cp;
    const __nv_bfloat162 wv = w[e];
    unsigned char* base = reinterpret_cast<unsigned char*>(sm.B[p / PPC]);
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c, k0)) = wv.x;
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c, k0 + 1)) = __hneg(wv.y);
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c + 1, k0)) = wv.y;
    *reinterpret_cast<__nv_bfloat16*>(base + tc_off(2 * c + 1, k0 + 1)) = wv.x;
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.bar)));
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
  unsigned char* Abase = reinterpret_cast<unsigned char*>(sm.A[0]);
  bool ok = true;
  for (int ch = 0; ch < NCH; ch++) {
#pragma unroll 1
    for (int j = 0; j < PPC; j++) {
      const int p = ch * PPC + j;
      const bool first = j == 0;  // the chunk's first write waits for the previous chunk's MMAs
      if (p >= 9) {  // an empty slot of the last chunk (CI = 4): zeros
#pragma unroll
        for (int a = 0; a < 3; a++)
          *reinterpret_cast<uint4*>(Abase + a * TC_ACHUNK * 2 + tc_off(tid, 2 * CI * j)) = make_uint4(0u, 0u, 0u, 0u);
        continue;
      }
      Link<float> U;
      PtcHop h{par, cb};
      if (valid) h = ptc_hop(u, g, par, valid ? cb : 0, x, s, p, U);
      // the link as BF16 pairs for the packed complex multiply: (re, re) and (-im, im)
      __nv_bfloat162 ur[3][3], ui[3][3];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
          ur[i][jj] = __floats2bfloat162_rn(U.m[i][jj].re, U.m[i][jj].re);
          ui[i][jj] = __floats2bfloat162_rn(-U.m[i][jj].im, U.m[i][jj].im);
        }
      // the neighbour's CI channels, all loads in flight at once: per group of four channels
      // 12 BF16 (re, im) words, channel cl, colour b at word cl*3 + b
      uint32_t wd[CI / 4][12];
      if constexpr (IN32) {
        float4 f[6];
#pragma unroll
        for (int q = 0; q < 6; q++)
          f[q] = valid ? __ldg(static_cast<const float4*>(in.p[h.npar]) + (size_t)q * g.Vh + h.n)
                       : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 6; q++) {
          wd[0][2 * q] = ptc_f2bf(make_float2(f[q].x, f[q].y));
          wd[0][2 * q + 1] = ptc_f2bf(make_float2(f[q].z, f[q].w));
        }
      } else {
        uint4 raw[CI / 4][3];
#pragma unroll
        for (int q = 0; q < CI / 4; q++)
#pragma unroll
          for (int k = 0; k < 3; k++)
            raw[q][k] = valid ? __ldg(static_cast<const uint4*>(in.p[h.npar]) + (size_t)(3 * q + k) * g.Vh + h.n)
                              : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
        for (int q = 0; q < CI / 4; q++)
#pragma unroll
          for (int k = 0; k < 3; k++) {
            wd[q][4 * k] = raw[q][k].x;
            wd[q][4 * k + 1] = raw[q][k].y;
            wd[q][4 * k + 2] = raw[q][k].z;
            wd[q][4 * k + 3] = raw[q][k].w;
          }
      }
#pragma unroll
      for (int q = 0; q < CI / 4; q++) {
        // transported (T_p in)[channel][colour a] as BF16 pairs: the identity path as stored,
        // the others as the row-a complex dot of the link with the colour vector, in packed
        // BF16 FMAs (the A operand is BF16 in any case)
        uint32_t o[3][4];
#pragma unroll
        for (int cl = 0; cl < 4; cl++)
#pragma unroll
          for (int a = 0; a < 3; a++) {
            if (p == 0) {
              o[a][cl] = wd[q][cl * 3 + a];
            } else {
              __nv_bfloat162 acc = __floats2bfloat162_rn(0.f, 0.f);
#pragma unroll
              for (int b = 0; b < 3; b++) {
                const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&wd[q][cl * 3 + b]);
                acc = __hfma2(ur[a][b], v, acc);
                acc = __hfma2(ui[a][b], __lowhigh2highlow(v), acc);
              }
              o[a][cl] = *reinterpret_cast<uint32_t*>(&acc);
            }
          }
        // the previous chunk's MMAs (completion ch - 1 of the barrier) must have read the buffer
        if (first && q == 0 && ch >= 1 && !mbar_wait(&sm.bar, (uint32_t)((ch - 1) & 1))) ok = false;
#pragma unroll
        for (int a = 0; a < 3; a++)
          *reinterpret_cast<uint4*>(Abase + a * TC_ACHUNK * 2 + tc_off(tid, 2 * CI * j + 8 * q)) =
              make_uint4(o[a][0], o[a][1], o[a][2], o[a][3]);
      }
    }
    // make the chunk visible to the tensor cores, then one thread issues its MMAs
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sm.A[0]);
      const uint32_t b0 = smem_u32(sm.B[ch]);
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
          tc_mma<N>(tmem + a * N, tc_desc(a0 + a * TC_ACHUNK * 2 + kk * 2 * TC_LBO), tc_desc(b0 + kk * 2 * TC_LBO),
                    (ch > 0 || kk > 0) ? 1u : 0u);
      tc_commit(&sm.bar);
    }
  }
  // one completion a chunk: the last has index NCH - 1
  if (!mbar_wait(&sm.bar, (uint32_t)((NCH - 1) & 1))) ok = false;
  tc_fence_after();
  if (ok) {
    float d[3][32];
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int a = 0; a < 3; a++) tc_ld32(lane_base + a * N, d[a]);  // columns a N .. a N + 31 (of 128)
    if (valid && OUT32) {
      // FP32 spinor layout: word wd holds complex 2 wd and 2 wd + 1 (channel k/3, colour k%3)
      float4* o = static_cast<float4*>(out.p[par]) + cb;
#pragma unroll
      for (int q = 0; q < 6; q++) {
        const int k0 = 2 * q, k1 = 2 * q + 1;
        o[(size_t)q * g.Vh] = make_float4(d[k0 % 3][2 * (k0 / 3)], d[k0 % 3][2 * (k0 / 3) + 1],
                                          d[k1 % 3][2 * (k1 / 3)], d[k1 % 3][2 * (k1 / 3) + 1]);
      }
    } else if (valid) {
      // BF16 layout: group q of four channels, word k4 holds complex k = 4 k4 + jj (channel
      // 4q + k/3, colour k%3) in slot jj
      uint4* o = static_cast<uint4*>(out.p[par]) + cb;
#pragma unroll
      for (int q = 0; q < CO / 4; q++)
#pragma unroll
        for (int k4 = 0; k4 < 3; k4++) {
          uint32_t e[4];
#pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            const int k = 4 * k4 + jj, c = 4 * q + k / 3, col = k % 3;
            e[jj] = ptc_f2bf(make_float2(d[col][2 * c], d[col][2 * c + 1]));
          }
          o[(size_t)(3 * q + k4) * g.Vh] = make_uint4(e[0], e[1], e[2], e[3]);
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
