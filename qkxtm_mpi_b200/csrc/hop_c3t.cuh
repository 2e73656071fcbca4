// hop_c3t.cuh -- the FP64 hopping term on row tiles that TMA stages in shared
// memory.
//
// Same operator, colour split and epilogues as hop_c3_kernel (reference
// Vector::applyDslash / applyDslashDag, lib/lattice_util.cpp:1158-1213,
// 1643-1699; 18-real links as given), different data movement.  The direct
// kernel issues, per colour thread and neighbour term, fifteen 16-byte global
// loads at computed 64-bit addresses; half of its instructions are those loads
// and their address arithmetic, and each neighbour spinor is fetched from L2 by
// up to eight sites.  Here a block owns a tile of C3T_ROWS consecutive lattice
// rows (fixed z, t, one output parity): W = L0/2 sites a row, 4W sites, three
// colour threads each.  Every input the tile needs is a few contiguous site
// ranges of the other parity, so one thread stages them with 2D TMA boxes of
// [components][sites] (cp.async.bulk.tensor, no multicast, this GPU's own
// memory only):
//   spinor, per right-hand side     own rows (the +-x neighbours), the rows
//                                   y0-1 and y0+4 (+-y halo), the same rows in
//                                   planes z+-1 and t+-1: 22W sites
//   links, once for all right-hand  forward links of the tile's sites (4 x 4W),
//   sides                           backward links at the -mu neighbours (4 x 4W)
// A lattice row of one parity is W consecutive checkerboard indices and the
// C3T_ROWS rows of a tile are consecutive as well (y is the index after x), so
// each range is one box; rows are never split because Ly % C3T_ROWS == 0.  The
// block then walks the batch's right-hand sides with two spinor buffers: the
// next right-hand side's boxes load while the current one is computed.
// Neighbours are found in shared memory by their position in the tile, so the
// hop itself needs no global address arithmetic.
//
// Every wait on an mbarrier is bounded by C3T_WAIT_NS of device clock; a wait
// that gives up records code 1 in *err, then the block waits (bounded again)
// for its copies still in flight and returns.
//
// On B200 this kernel is slower than the direct one and is opt-in
// (QKX_FP64_TILED=1): at W = 16 a tile holds 209 KB of shared memory, so one
// block (six warps) runs on an SM.  Those six warps cannot hide the latency of
// the FP64 arithmetic and shared-memory reads, and with one right-hand side
// nothing overlaps a tile's staging with its compute (32^3x64 tm: 1.11 ms
// against 0.61 ms a launch; the 12-RHS reliable-update hops lose too).
#pragma once
#include <cuda.h>

#include "hop_c3.cuh"

namespace qkx {

constexpr int C3T_ROWS = 4;                                // lattice rows of one tile
constexpr unsigned long long C3T_WAIT_NS = 200000000ull;  // 200 ms

// the TMA descriptors of one launch: input spinor fields of each parity with boxes of
// 4W and W sites (12 components), links with boxes of 4W, W and 3W sites (9 components)
struct C3tMaps {
  CUtensorMap in4[2];
  CUtensorMap in1[2];
  CUtensorMap l4, l1, l3;
};

// byte layout of the dynamic shared memory of a tile with W sites a row
struct C3tLayout {
  int W = 0;
  int link_off[9] = {};     // F0..F3, B0, B1a, B1b, B2, B3
  int link_sites[9] = {};
  int spin_off[7] = {};     // R0..R6 of the first buffer; the second follows at spin_stride
  int spin_stride = 0;
  int spin_sites[7] = {};
  int bar_off = 0;  // three mbarriers, then six doubles for the block reduction
  int red_off = 0;
  int bytes = 0;    // from the 128-byte aligned base; allocate bytes + 128
  int link_bytes = 0, spin_bytes = 0;

  __host__ __device__ static int up128(int b) { return (b + 127) & ~127; }
  __host__ __device__ explicit C3tLayout(int w) : W(w) {
    const int n4 = C3T_ROWS * w;
    const int ls[9] = {n4, n4, n4, n4, n4, w, (C3T_ROWS - 1) * w, n4, n4};
    const int ss[7] = {n4, w, w, n4, n4, n4, n4};
    int off = 0;
    for (int i = 0; i < 9; i++) {
      link_sites[i] = ls[i];
      link_off[i] = off;
      off = up128(off + 9 * ls[i] * 16);
      link_bytes += 9 * ls[i] * 16;
    }
    for (int i = 0; i < 7; i++) spin_sites[i] = ss[i];
    const int first = off;
    for (int i = 0; i < 7; i++) {
      spin_off[i] = off;
      off = up128(off + 12 * ss[i] * 16);
      spin_bytes += 12 * ss[i] * 16;
    }
    spin_stride = off - first;
    off += spin_stride;  // the second buffer
    bar_off = off;
    red_off = off + 3 * 8;
    bytes = red_off + 8 * 8;
  }
};

__device__ __forceinline__ unsigned long long c3t_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t c3t_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void c3t_bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(c3t_smem(bar)) : "memory");
}

__device__ __forceinline__ void c3t_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(c3t_smem(bar)), "r"(bytes) : "memory");
}

// 2D TMA box load into shared memory, completing on the barrier
__device__ __forceinline__ void c3t_load(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          c3t_smem(dst)),
      "l"(map), "r"(x), "r"(y), "r"(c3t_smem(bar))
      : "memory");
}

// wait for phase `parity` of the barrier, giving up after C3T_WAIT_NS
__device__ __forceinline__ bool c3t_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = c3t_smem(bar);
  const unsigned long long t0 = c3t_clock_ns();
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
    if (c3t_clock_ns() - t0 > C3T_WAIT_NS) return false;
  }
}

// one neighbour term of colour a: the neighbour spinor and link read from the staged
// boxes (component k of site j of a box with n sites at base[k * n + j])
template <int B, bool DAG, int MU, bool FW>
__device__ __forceinline__ void hop_side_c3t(const double2* nb, int nn, int ns, const double2* lb, int ln, int lsite,
                                             bool flip, int a, Spin4<double>& acc) {
  constexpr int SF = DAG ? +1 : -1;
  using P = Proj<B, MU, FW ? SF : -SF>;
  Spinor<double> v;
  if constexpr (P::diag) {
#pragma unroll
    for (int sp = 0; sp < 2; sp++)
#pragma unroll
      for (int b = 0; b < 3; b++) {
        const double2 d = nb[((P::drow + sp) * 3 + b) * nn + ns];
        v.c[P::drow + sp][b] = {d.x, d.y};
      }
  } else {
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const double2 d = nb[k * nn + ns];
      v.c[k / 3][k % 3] = {d.x, d.y};
    }
  }
  HalfSpinor<double> h;
  P::project(v, h);
  // row a of U_mu(x) (forward) or of U_mu(x-mu)^+ (backward)
  Cx<double> u[3];
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const double2 d = FW ? lb[(a * 3 + b) * ln + lsite] : lb[(b * 3 + a) * ln + lsite];
    u[b] = FW ? Cx<double>{d.x, d.y} : Cx<double>{d.x, -d.y};
  }
  Cx<double> t0 = cmul(u[0], h.c[0][0]) + cmul(u[1], h.c[0][1]) + cmul(u[2], h.c[0][2]);
  Cx<double> t1 = cmul(u[0], h.c[1][0]) + cmul(u[1], h.c[1][1]) + cmul(u[2], h.c[1][2]);
  if (flip) {
    t0 = -1.0 * t0;
    t1 = -1.0 * t1;
  }
  P::reconstruct1(acc, t0, t1);
}

// blockIdx.x: tile (x 2 parities, interleaved, when out_parity < 0); block (4W, 3)
template <int B, bool DAG, int EPI>
__global__ void __launch_bounds__(192) hop_c3t_kernel(HopArgs<SpinorF64, GaugeF64x18> A, HopRes Rz,
                                                      const __grid_constant__ C3tMaps M, int W, int* err) {
  extern __shared__ __align__(128) unsigned char sm_raw[];
  // TMA destinations must start on 128-byte boundaries: align the base at run time
  unsigned char* sm = sm_raw + ((128u - (c3t_smem(sm_raw) & 127u)) & 127u);
  const C3tLayout lay(W);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + lay.bar_off);
  double* red = reinterpret_cast<double*>(sm + lay.red_off);
  const int blk = blockIdx.x;
  const int par = A.out_parity < 0 ? (blk & 1) : A.out_parity;
  const int tile = A.out_parity < 0 ? (blk >> 1) : blk;
  const int q = 1 - par;  // the parity of the neighbours
  const Geom& g = A.g;
  const int Ly = g.L[1], Lz = g.L[2], Lt = g.L[3];
  const int ty = Ly / C3T_ROWS;
  const int y0 = (tile % ty) * C3T_ROWS;
  const int z = (tile / ty) % Lz, t = tile / (ty * Lz);
  auto rowcb = [&](int y, int zz, int tt) { return W * (y + Ly * (zz + Lz * tt)); };
  const int ym1 = (y0 + Ly - 1) % Ly, yp = (y0 + C3T_ROWS) % Ly;
  const int zm = (z + Lz - 1) % Lz, zp = (z + 1) % Lz, tm = (t + Lt - 1) % Lt, tp = (t + 1) % Lt;
  const int cb0 = rowcb(y0, z, t);
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthr = blockDim.x * blockDim.y;

  if (tid == 0) {
    for (int i = 0; i < 3; i++) c3t_bar_init(&bar[i]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  auto active = [&](int r) { return !A.active || A.active[r]; };
  auto next_active = [&](int r) {
    for (r++; r < A.nrhs; r++)
      if (active(r)) break;
    return r;
  };
  // the staged spinor boxes of right-hand side r into buffer b
  auto issue_spin = [&](int r, int b) {
    const int row = 12 * r;
    unsigned char* base = sm + b * lay.spin_stride;
    c3t_expect(&bar[b], (uint32_t)lay.spin_bytes);
    c3t_load(base + lay.spin_off[0], &M.in4[q], 2 * cb0, row, &bar[b]);
    c3t_load(base + lay.spin_off[1], &M.in1[q], 2 * rowcb(ym1, z, t), row, &bar[b]);
    c3t_load(base + lay.spin_off[2], &M.in1[q], 2 * rowcb(yp, z, t), row, &bar[b]);
    c3t_load(base + lay.spin_off[3], &M.in4[q], 2 * rowcb(y0, zm, t), row, &bar[b]);
    c3t_load(base + lay.spin_off[4], &M.in4[q], 2 * rowcb(y0, zp, t), row, &bar[b]);
    c3t_load(base + lay.spin_off[5], &M.in4[q], 2 * rowcb(y0, z, tm), row, &bar[b]);
    c3t_load(base + lay.spin_off[6], &M.in4[q], 2 * rowcb(y0, z, tp), row, &bar[b]);
  };

  int r_cur = next_active(-1);
  bool pend[3] = {false, false, false};  // copies in flight per barrier (thread 0's view)
  int phase[2] = {0, 0};                 // completed uses of each spinor buffer
  if (tid == 0) {
    c3t_expect(&bar[2], (uint32_t)lay.link_bytes);
    for (int mu = 0; mu < 4; mu++)
      c3t_load(sm + lay.link_off[mu], &M.l4, 2 * cb0, (par * 4 + mu) * 9, &bar[2]);
    c3t_load(sm + lay.link_off[4], &M.l4, 2 * cb0, (q * 4 + 0) * 9, &bar[2]);
    c3t_load(sm + lay.link_off[5], &M.l1, 2 * rowcb(ym1, z, t), (q * 4 + 1) * 9, &bar[2]);
    c3t_load(sm + lay.link_off[6], &M.l3, 2 * cb0, (q * 4 + 1) * 9, &bar[2]);
    c3t_load(sm + lay.link_off[7], &M.l4, 2 * rowcb(y0, zm, t), (q * 4 + 2) * 9, &bar[2]);
    c3t_load(sm + lay.link_off[8], &M.l4, 2 * rowcb(y0, z, tm), (q * 4 + 3) * 9, &bar[2]);
    pend[2] = true;
    if (r_cur < A.nrhs) {
      issue_spin(r_cur, 0);
      pend[0] = true;
    }
  }

  // this thread's site in the tile and its output coordinates
  const int s = threadIdx.x, a = threadIdx.y;
  const int rr = s / W, i = s % W;
  const int y = y0 + rr;
  const int off = (y + z + t + par) & 1;  // x = 2i + off
  const int ip = off ? (i + 1 == W ? 0 : i + 1) : i;  // the +x neighbour's index in the row
  const int im = off ? i : (i == 0 ? W - 1 : i - 1);  // the -x neighbour's
  const int cb = cb0 + s;
  const bool flip_f = g.bc_sign < 0 && t == Lt - 1, flip_b = g.bc_sign < 0 && t == 0;
  auto lk = [&](int k) { return reinterpret_cast<const double2*>(sm + lay.link_off[k]); };
  const int n4 = C3T_ROWS * W;

  bool links_ready = false;
  int use = 0;
  bool failed = false;
  for (int r = 0; r < A.nrhs; r++) {
    double* slot = A.norm_part ? A.norm_part + (size_t)r * A.nblk + blk : nullptr;
    if (!active(r)) {
      if (slot && tid == 0) *slot = 0.0;
      continue;
    }
    const int b = use & 1;
    const int r_next = next_active(r);
    if (tid == 0 && r_next < A.nrhs) {
      // the other buffer was last read in the previous step, which ended with a block barrier
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_spin(r_next, b ^ 1);
      pend[b ^ 1] = true;
    }
    bool ok = true;
    if (!links_ready) ok = c3t_wait(&bar[2], 0);
    ok = ok && c3t_wait(&bar[b], (uint32_t)(phase[b] & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    if (tid == 0) {
      if (!links_ready) pend[2] = false;
      pend[b] = false;
    }
    phase[b]++;
    links_ready = true;
    const unsigned char* sbase = sm + b * lay.spin_stride;
    auto sp = [&](int k) { return reinterpret_cast<const double2*>(sbase + lay.spin_off[k]); };
    Spin4<double> acc;
#pragma unroll
    for (int k = 0; k < 4; k++) acc.s[k] = {0.0, 0.0};
    // x
    hop_side_c3t<B, DAG, 0, true>(sp(0), n4, rr * W + ip, lk(0), n4, s, false, a, acc);
    hop_side_c3t<B, DAG, 0, false>(sp(0), n4, rr * W + im, lk(4), n4, rr * W + im, false, a, acc);
    // y
    if (rr + 1 < C3T_ROWS) hop_side_c3t<B, DAG, 1, true>(sp(0), n4, s + W, lk(1), n4, s, false, a, acc);
    else hop_side_c3t<B, DAG, 1, true>(sp(2), W, i, lk(1), n4, s, false, a, acc);
    if (rr > 0) hop_side_c3t<B, DAG, 1, false>(sp(0), n4, s - W, lk(6), (C3T_ROWS - 1) * W, s - W, false, a, acc);
    else hop_side_c3t<B, DAG, 1, false>(sp(1), W, i, lk(5), W, i, false, a, acc);
    // z
    hop_side_c3t<B, DAG, 2, true>(sp(4), n4, s, lk(2), n4, s, false, a, acc);
    hop_side_c3t<B, DAG, 2, false>(sp(3), n4, s, lk(7), n4, s, false, a, acc);
    // t
    hop_side_c3t<B, DAG, 3, true>(sp(6), n4, s, lk(3), n4, s, flip_f, a, acc);
    hop_side_c3t<B, DAG, 3, false>(sp(5), n4, s, lk(8), n4, s, flip_b, a, acc);
    const double nrm = c3_epilogue<SpinorF64, B, EPI>(A, Rz, r, par, cb, a, acc);
    if (slot) {
      // 12W threads: the last warp may be partial (W = 2, 4, 6, 12, ...); shuffle among the
      // lanes that exist and add only what comes from them
      const int lane = tid & 31, nl = min(32, nthr - (tid & ~31));
      const unsigned lanes = nl == 32 ? 0xffffffffu : ((1u << nl) - 1u);
      double w = nrm;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_down_sync(lanes, w, o);
        if (lane + o < nl) w += v;
      }
      if (lane == 0) red[tid >> 5] = w;
    }
    __syncthreads();  // every thread is done with buffer b (and red is complete)
    if (slot && tid == 0) {
      double tsum = 0.0;
      const int nw = (nthr + 31) / 32;
      for (int k = 0; k < nw; k++) tsum += red[k];
      *slot = tsum;
    }
    __syncthreads();  // red is free again
    use++;
  }
  if (tid == 0) {
    // the copies still in flight (after a failed wait, or the links of a block whose
    // right-hand sides are all inactive) land before the block's shared memory is released
    bool drained = true;
    for (int k = 0; k < 3; k++)
      if (pend[k]) drained = c3t_wait(&bar[k], k == 2 ? 0u : (uint32_t)(phase[k] & 1)) && drained;
    if (failed || !drained) atomicExch(err, 1);
  }
}

// tile geometry the kernel supports: an even Lx with W = Lx/2 <= 16, Ly a multiple of
// C3T_ROWS, and the layout within the shared memory an SM offers
inline bool c3t_supported(const Geom& g, int smem_max) {
  const int W = g.L[0] / 2;
  if (g.L[0] % 2 || W < 1 || W > 16 || g.L[1] % C3T_ROWS) return false;
  return C3tLayout(W).bytes + 128 <= smem_max;
}

inline int c3t_blocks(const Geom& g, int out_parity) {
  const int tiles = (g.L[1] / C3T_ROWS) * g.L[2] * g.L[3];
  return out_parity < 0 ? 2 * tiles : tiles;
}

}  // namespace qkx
