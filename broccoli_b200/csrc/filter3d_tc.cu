// filter3d_tc.cu -- 7x7x7 complex filtering on the tcgen05 tensor cores in
// BF16 split precision with FP32 accumulation (BRC_PREC_BF16X3).
//
// The contraction q_f(z,y,x) = sum_{dz,dy,dx} F_f[3-dz][3-dy][3-dx] V(z+dz,
// y+dy, x+dx) (NonseparableConvolution3D, broccoli_lib.cpp:4974-5027, true
// convolution with zero padding) is recast as 49 (or 56) GEMMs per tile,
// one per (input-plane offset, dy):
//
//   D[m][n] += A_{c,dy}[m][k] * B[k][n]
//     m = (s, f, xo)  128 rows: real filter f (re/im of each complex filter),
//                     output x offset xo in [0,10), stacked output plane s
//     k = x_in        16 input samples along x (the window of the 10 outputs
//                     plus the 6-sample halo): A is a banded Toeplitz matrix
//                     with the 7 taps of row (dz, dy) of filter f
//     n = (j, y)      output rows of the tile: plane group j, row y
//
// B is never materialised per GEMM: the input tile sits in shared memory as
// K-major 8x16-byte core matrices (one 16-byte row per (plane, y) and half
// window of x), so the dy / dz shift of a GEMM is a shift of its smem
// descriptor's start address by whole rows.  With 3 complex filters (6 real
// outputs = 60 rows) two output planes share M (s in {0,1}): the GEMM for
// input-plane offset c feeds plane s with the taps of dz = c - s.  Input
// planes are stored by parity then so that the rows of plane groups j are
// evenly spaced for every c.
//
// Split precision: x = x_hi + x_lo with both parts BF16 (x_lo the BF16
// rounding of x - x_hi), for the data and the taps; each GEMM is issued as
// A_hi B_hi + A_hi B_lo + A_lo B_hi into the same FP32 TMEM accumulator
// (relative error of a product ~2^-16; the dropped A_lo B_lo ~2^-18).
//
// Per CTA (128 threads, one tile = 10 x positions x Ty rows x SP*J planes of
// one volume): all threads stage the input tile (FP32 -> BF16 hi/lo); then
// thread 32 streams the packed taps of each GEMM (8 KB, hi + lo) through a
// 6-slot shared-memory ring with cp.async.bulk + mbarriers while thread 0
// issues the tcgen05.mma's, each stage's tcgen05.commit freeing its slot;
// at the end all threads read the accumulator back with tcgen05.ld.  Two
// CTAs per SM overlap one tile's staging/epilogue with the other's GEMMs.
// Every wait is bounded (about 2 s); a CTA that gives up sets *err, still
// waits (bounded) for its GEMMs and copies, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "common.cuh"
#include "filter3d_tc.h"

namespace brc {
namespace tc {

constexpr int kThreads = 128;
constexpr int kRing = 6;
constexpr int kStageHalves = kM * kK;              // BF16 elements of one A (hi or lo)
constexpr int kStageBytes = 2 * kStageHalves * 2;  // hi + lo
constexpr uint32_t kTmemCols = 256;
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Shared-memory matrix descriptor, K-major, no swizzle: start address, LBO
// (byte distance between the two 8-element K halves), SBO (between groups
// of 8 rows), descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity; false after limit_ns
// (default ~2 s).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          unsigned long long limit_ns = kWaitNs) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Plain (non-multicast) bulk copy global -> own shared memory.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo_elem, __nv_bfloat16 hi_elem) {
  return (uint32_t)__bfloat16_as_ushort(lo_elem) | ((uint32_t)__bfloat16_as_ushort(hi_elem) << 16);
}

__global__ void __launch_bounds__(kThreads, 2)
filter3d_tc_kernel(const float* __restrict__ vol, int W, int H, int D, long long vstride,
                   const uint16_t* __restrict__ taps, float* __restrict__ out, int nfilt, Geometry g,
                   int n_xchunks, const int* __restrict__ conv_iter, int it, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int b = blockIdx.z;
  if (instance_done(conv_iter, b, it)) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int xc = blockIdx.x % n_xchunks, yt = blockIdx.x / n_xchunks;
  const int x0 = xc * kXo, y0 = yt * g.Ty, z0 = blockIdx.y * g.SP * g.J;
  const long long V = (long long)W * H * D;

  uint8_t* ring = smem;
  uint8_t* dhi = smem + kRing * kStageBytes;
  const uint32_t hl_bytes = 32u * (uint32_t)g.NR;  // two K halves of NR 16-byte rows
  uint8_t* dlo = dhi + hl_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(dlo + hl_bytes);
  uint64_t* empty = full + kRing;
  uint64_t* done = empty + kRing;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* flags = reinterpret_cast<int*>(tmem_slot + 1);  // [0] GEMM stages issued, [1] tap stages loaded

  if (tid == 0) {
    for (int s = 0; s < kRing; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();

  const int nst = g.nstage;
  if (tid == 0)
    for (int s = 0; s < kRing && s < nst; s++) {
      mbar_expect_tx(&full[s], kStageBytes);
      bulk_load(ring + s * kStageBytes, taps + (size_t)s * (kStageBytes / 2), kStageBytes, &full[s]);
    }

  // Stage the input tile: row (parity p, plane slot qq, y row yl) holds the
  // 16 samples x0-3 .. x0+12 of input plane z0-3 + SP*qq + p, row y0-3+yl,
  // as two 16-byte K halves (hi and lo arrays).  Rows past the tile are 0.
  const float* src = vol + (long long)b * vstride;
  const int NQ = g.SP * g.J + 6;
  // consecutive threads take consecutive rows of one K half: each warp's
  // 16-byte stores cover 512 contiguous bytes (no bank conflicts)
  // rows are 16-byte aligned when W is a multiple of 4 (and the volume is):
  // a window inside the row then takes three aligned float4 loads
  const bool vec_rows = (W & 3) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0;
#pragma unroll 2
  for (int item = tid; item < 2 * g.NR; item += kThreads) {
    const int kh = item >= g.NR ? 1 : 0, row = item - kh * g.NR;
    const int par = row / g.RP, rr = row - par * g.RP;
    const int qq = rr / g.Hp, yl = rr - qq * g.Hp;
    const int q = qq * g.SP + par;
    const int zg = z0 - 3 + q, yg = y0 - 3 + yl;
    const bool rowok = q < NQ && zg >= 0 && zg < D && yg >= 0 && yg < H;
    const int xs = x0 - 3 + 8 * kh;
    float v[8];
    if (rowok && vec_rows && xs >= 0 && (xs & ~3) + 12 <= W) {
      const int a = xs & 3;
      const float4* p4 = reinterpret_cast<const float4*>(src + ((long long)zg * H + yg) * W + (xs - a));
      const float4 f0 = __ldg(p4), f1 = __ldg(p4 + 1), f2 = __ldg(p4 + 2);
      const float w[12] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w};
#pragma unroll
      for (int e = 0; e < 8; e++) v[e] = a == 0 ? w[e] : (a == 1 ? w[e + 1] : (a == 2 ? w[e + 2] : w[e + 3]));
    } else {
      const float* rp = src + ((long long)zg * H + yg) * W;
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int xg = xs + e;
        v[e] = (rowok && xg >= 0 && xg < W) ? __ldg(rp + xg) : 0.f;
      }
    }
    uint32_t ph[4], pl[4];
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      const __nv_bfloat16 h0 = __float2bfloat16_rn(v[e]), h1 = __float2bfloat16_rn(v[e + 1]);
      const __nv_bfloat16 l0 = __float2bfloat16_rn(v[e] - __bfloat162float(h0));
      const __nv_bfloat16 l1 = __float2bfloat16_rn(v[e + 1] - __bfloat162float(h1));
      ph[e / 2] = pack_bf16(h0, h1);
      pl[e / 2] = pack_bf16(l0, l1);
    }
    const uint32_t off = (uint32_t)kh * (uint32_t)g.NR * 16u + (uint32_t)row * 16u;
    *reinterpret_cast<uint4*>(dhi + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
    *reinterpret_cast<uint4*>(dlo + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // Roles: thread 0 issues the GEMMs, thread 32 refills the tap ring.
  // Stage s = (c+3)*7 + (dy+3) uses ring slot s % kRing.
  if (tid == 0) {
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(g.N >> 3) << 17) |
                           ((uint32_t)(kM >> 4) << 24);
    const uint32_t ring_a = smem_u32(ring), dhi_a = smem_u32(dhi), dlo_a = smem_u32(dlo);
    const uint32_t lbo_b = (uint32_t)g.NR * 16u;
    int s = 0;
    for (; s < nst; s++) {
      const int slot = s % kRing;
      if (!mbar_wait(&full[slot], (uint32_t)(s / kRing) & 1u)) break;
      const int cq = s / 7, dyq = s % 7;  // c + 3, dy + 3
      const int par = cq % g.SP, qoff = cq / g.SP;
      const uint32_t brow = (uint32_t)(par * g.RP + qoff * g.Hp + dyq);
      const uint32_t a_hi = ring_a + (uint32_t)slot * kStageBytes, a_lo = a_hi + kStageBytes / 2;
      const uint64_t dah = sdesc(a_hi, kM * 16, 128), dal = sdesc(a_lo, kM * 16, 128);
      const uint64_t dbh = sdesc(dhi_a + brow * 16u, lbo_b, 128), dbl = sdesc(dlo_a + brow * 16u, lbo_b, 128);
      mma_bf16(tmem, dah, dbh, idesc, s > 0 ? 1u : 0u);
      mma_bf16(tmem, dah, dbl, idesc, 1u);
      mma_bf16(tmem, dal, dbh, idesc, 1u);
      mma_commit(&empty[slot]);  // the slot is free once these GEMMs retire
    }
    flags[0] = s;  // stages issued
    mma_commit(done);
  } else if (tid == 32) {
    int s = kRing;
    for (; s < nst; s++) {
      const int slot = s % kRing;
      if (!mbar_wait(&empty[slot], (uint32_t)(s / kRing - 1) & 1u)) break;
      mbar_expect_tx(&full[slot], kStageBytes);
      bulk_load(ring + slot * kStageBytes, taps + (size_t)s * (kStageBytes / 2), kStageBytes, &full[slot]);
    }
    flags[1] = s < nst ? s : nst;  // stages loaded
  }
  __syncthreads();
  const int issued = flags[0], loaded = flags[1];
  int ok = issued == nst;
  // a wait gave up: bounded drain of the tap copies no GEMM consumed
  if (tid == 32)
    for (int t = issued; t < loaded; t++) mbar_wait(&full[t % kRing], (uint32_t)(t / kRing) & 1u);
  const int dok = mbar_wait(done, 0) ? 1 : 0;
  tc_fence_after();

  // Epilogue: TMEM lane r = M row (s, f, xo); columns n = (j, y).
  const int r = warp * 32 + lane;
  int sp, f, xo;
  bool rvalid;
  if (g.SP == 2) {
    sp = r >> 6;
    const int rr = r & 63;
    f = rr / kXo;
    xo = rr - f * kXo;
    rvalid = rr < 2 * nfilt * kXo;
  } else {
    sp = 0;
    f = r / kXo;
    xo = r - f * kXo;
    rvalid = r < 2 * nfilt * kXo;
  }
  rvalid = rvalid && ok && dok;
  // The accumulator is transposed through the shared memory the GEMMs no
  // longer need (tap ring + input tile): element (column n, plane s, filter
  // k, x offset xo, re/im) at E[((n - cbase) * SP + s) * 20 nfilt + 20 k +
  // 2 xo + ri], so each output row (z, y) of a filter is 80 contiguous
  // bytes (10 complex samples), written with 16-byte stores.
  float* E = reinterpret_cast<float*>(smem);
  const int rowf = 20 * nfilt;  // floats per (column, plane) row
  const uint32_t avail = (uint32_t)(kRing * kStageBytes) + 2u * hl_bytes;
  int C = (int)(avail / (uint32_t)(4 * rowf * g.SP)) / 16 * 16;
  if (C > g.N) C = g.N;
  const int ke = (f >> 1) * 20 + xo * 2 + (f & 1);
  const bool vec16 = ((W & 1) == 0) && ((V & 1) == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
  for (int cbase = 0; cbase < g.N; cbase += C) {
    const int cend = cbase + C < g.N ? cbase + C : g.N;
    for (int c0 = cbase; c0 < cend; c0 += 16) {
      uint32_t v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (rvalid) {
#pragma unroll
        for (int e = 0; e < 16; e++) E[((c0 + e - cbase) * g.SP + sp) * rowf + ke] = __uint_as_float(v[e]);
      }
    }
    __syncthreads();
    const int segs = (cend - cbase) * g.SP * nfilt;
    for (int item = tid; item < segs * 5; item += kThreads) {
      const int seg = item / 5, part = item - seg * 5;
      const int nl = seg / (g.SP * nfilt), rem = seg - nl * (g.SP * nfilt);
      const int s2 = rem / nfilt, k = rem - s2 * nfilt;
      const int n = cbase + nl;
      const int j = n / g.Hp, yl = n - j * g.Hp;
      const int z = z0 + j * g.SP + s2, y = y0 + yl, xs = x0 + 2 * part;
      if (j >= g.J || yl >= g.Ty || y >= H || z >= D || xs >= W) continue;
      const float4 q = *reinterpret_cast<const float4*>(E + (nl * g.SP + s2) * rowf + k * 20 + part * 4);
      float* dst = out + (((long long)b * nfilt + k) * V + ((long long)z * H + y) * W + xs) * 2;
      if (xs + 1 < W && vec16) {
        *reinterpret_cast<float4*>(dst) = q;
      } else {
        *reinterpret_cast<float2*>(dst) = make_float2(q.x, q.y);
        if (xs + 1 < W) *reinterpret_cast<float2*>(dst + 2) = make_float2(q.z, q.w);
      }
    }
    __syncthreads();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  if (tid == 0 && (!ok || !dok)) atomicExch(err, 1);
}

// ---------------------------------------------------------------------------
// Persistent form: one CTA per SM walks the tiles of the launch with its
// warps specialised.  The input comes pre-converted (pack_windows_kernel)
// so that a tile's B operand is eight TMA box loads, and two TMEM
// accumulators let the epilogue of one tile run under the GEMMs of the next.
//
//   warp 0, lane 0   TMA loads of the packed input tile (two buffers)
//   warp 1, lane 0   tcgen05.mma issue (the 3 split products of each stage)
//   warp 2, lane 0   tap stages through the ring (cp.async.bulk)
//   warps 4-7        epilogue: tcgen05.ld of TMEM lanes 32 (warp - 4) ..,
//                    transpose through shared memory, 16-byte stores
//
// Packed layout (uint16 BF16): element e of row (b, part, xc, z, y) at
// ((((b * 2 + part) * nxc + xc) * Dp + z) * H + y) * 16 + e is the
// sample x = 10 xc - 3 + e of plane z, row y (part 0 the BF16 rounding of
// the sample, part 1 the BF16 rounding of the remainder; zero outside the
// volume, Dp = D rounded up to SP).  Its tensor map has five dimensions
// (e: 16, y: H, plane parity: SP, plane pair: Dp / SP, (b, part, xc)), so
// one box {8, Hp, 1, NQ / SP, 1} brings the 16-byte K-half rows of one plane
// parity of a tile in the order (plane slot, row) the GEMMs read them.
// ---------------------------------------------------------------------------

struct PArgs {
  int W, H, D, Dp, nxc, nyt, nzt, batch, nfilt, ntiles;
  int nqp;                 // planes per parity in a tile (NQ / SP)
  uint32_t in_off;         // shared offset of the input buffers
  uint32_t e_off;          // shared offset of the epilogue transpose buffer
  uint32_t bar_off;        // shared offset of the barriers
  int ecols;               // accumulator columns per epilogue chunk
};

constexpr int kPThreads = 256;
constexpr int kPRing = 8;
constexpr uint32_t kPTmemCols = 512;  // two accumulators of up to 256 columns
// barrier block: full_in, empty_in, acc_full, acc_empty (2 each), the ring's
// full / empty (kPRing each), done; then the TMEM address and 6 flags
constexpr int kPBarBytes = ((8 + 2 * kPRing + 1) * 8 + 4 + 6 * 4 + 15) / 16 * 16;

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Tile t -> (b, zt, yt, xc), xc fastest.
__device__ __forceinline__ void decode_tile(const PArgs& a, int t, int& b, int& zt, int& yt, int& xc) {
  xc = t % a.nxc;
  int r = t / a.nxc;
  yt = r % a.nyt;
  r /= a.nyt;
  zt = r % a.nzt;
  b = r / a.nzt;
}

__global__ void __launch_bounds__(kPThreads, 1)
filter3d_tcp_kernel(const __grid_constant__ CUtensorMap tmap, const uint16_t* __restrict__ taps,
                    float* __restrict__ out, const PArgs a, const Geometry g, const int* __restrict__ conv_iter,
                    int it, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t* ring = smem;
  uint8_t* inb = smem + a.in_off;
  float* E = reinterpret_cast<float*>(smem + a.e_off);
  uint64_t* full_in = reinterpret_cast<uint64_t*>(smem + a.bar_off);
  uint64_t* empty_in = full_in + 2;
  uint64_t* acc_full = empty_in + 2;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* tfull = acc_empty + 2;
  uint64_t* tempty = tfull + kPRing;
  uint64_t* done = tempty + kPRing;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  // [0] tiles produced, [1] tiles consumed, [2] tap stages loaded, [3] consumed,
  // [4] a wait gave up, [5] epilogue: accumulator ready
  int* flags = reinterpret_cast<int*>(tmem_slot + 1);

  const uint32_t rowbytes = 16u * (uint32_t)g.NR;  // one K half of one part of one buffer
  const int nst = g.nstage;
  const long long V = (long long)a.W * a.H * a.D;

  if (tid == 0) {
    for (int i = 0; i < 2; i++) {
      mbar_init(&full_in[i], 1);
      mbar_init(&empty_in[i], 1);
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 128);
    }
    for (int s = 0; s < kPRing; s++) {
      mbar_init(&tfull[s], 1);
      mbar_init(&tempty[s], 1);
    }
    mbar_init(done, 1);
    for (int i = 0; i < 6; i++) flags[i] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kPTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer: packed input tiles by TMA
    const uint32_t tx = 64u * (uint32_t)g.SP * (uint32_t)g.Hp * (uint32_t)a.nqp;
    int i = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, t, b, zt, yt, xc);
      if (instance_done(conv_iter, b, it)) continue;
      const int buf = i & 1;
      if (i >= 2 && !mbar_wait(&empty_in[buf], (uint32_t)((i >> 1) - 1) & 1u)) {
        ok = false;
        break;
      }
      mbar_expect_tx(&full_in[buf], tx);
      const int z0 = zt * g.SP * g.J, y0 = yt * g.Ty;
      for (int part = 0; part < 2; part++)
        for (int kh = 0; kh < 2; kh++)
          for (int p = 0; p < g.SP; p++) {
            uint8_t* dst = inb + (uint32_t)((buf * 2 + part) * 2 + kh) * rowbytes + (uint32_t)(p * g.RP) * 16u;
            const int gpar = g.SP == 2 ? ((p + 1) & 1) : 0;
            const int zp0 = g.SP == 2 ? (z0 / 2 - 2 + p) : (z0 - 3);
            tma_load_5d(dst, &tmap, 8 * kh, y0 - 3, gpar, zp0, (b * 2 + part) * a.nxc + xc, &full_in[buf]);
          }
      i++;
    }
    flags[0] = i;
    if (!ok) flags[4] = 1;
  } else if (warp == 1 && lane == 0) {
    // ---- GEMM issue.  The descriptors are built once; a stage only adds
    // offsets to their start-address fields (one 16-byte row = 1), so that
    // the issuing thread spends its time in tcgen05.mma, not in address
    // arithmetic (which delays every GEMM it precedes).
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(g.N >> 3) << 17) |
                           ((uint32_t)(kM >> 4) << 24);
    const uint64_t da0 = sdesc(smem_u32(ring), kM * 16, 128);  // slot 0, hi taps
    const uint64_t db0 = sdesc(smem_u32(inb), rowbytes, 128);  // buffer 0, hi part, row 0
    const uint64_t dslot = kStageBytes >> 4, dalo = kStageBytes >> 5;
    const uint64_t dbuf = (4u * rowbytes) >> 4, dblo = (2u * rowbytes) >> 4;
    const int ncq = nst / 7;
    int i = 0, slot = 0;
    uint32_t ph = 0, G = 0;
    uint64_t ah = da0;
    bool ok = true;
    for (int t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, t, b, zt, yt, xc);
      if (instance_done(conv_iter, b, it)) continue;
      const int buf = i & 1, acc = i & 1;
      if (!mbar_wait(&full_in[buf], (uint32_t)(i >> 1) & 1u) ||
          (i >= 2 && !mbar_wait(&acc_empty[acc], (uint32_t)((i >> 1) - 1) & 1u))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint64_t bh0 = db0 + (uint64_t)buf * dbuf;
      const uint32_t dcol = tmem + (uint32_t)(acc * 256);
      uint32_t accf = 0;
      for (int cq = 0; cq < ncq && ok; cq++) {
        // rows of input-plane offset c = cq - 3: parity array cq % SP, plane slot cq / SP
        const uint64_t bh = bh0 + (uint64_t)((cq % g.SP) * g.RP + (cq / g.SP) * g.Hp), bl = bh + dblo;
#pragma unroll
        for (int dyq = 0; dyq < 7; dyq++) {
          if (!mbar_wait(&tfull[slot], ph)) {
            ok = false;
            break;
          }
          mma_bf16(dcol, ah, bh + dyq, idesc, accf);
          mma_bf16(dcol, ah, bl + dyq, idesc, 1u);
          mma_bf16(dcol, ah + dalo, bh + dyq, idesc, 1u);
          mma_commit(&tempty[slot]);
          accf = 1u;
          G++;
          ah += dslot;
          if (++slot == kPRing) {
            slot = 0;
            ph ^= 1u;
            ah = da0;
          }
        }
      }
      if (!ok) break;
      mma_commit(&empty_in[buf]);
      mma_commit(&acc_full[acc]);
      i++;
    }
    flags[1] = i;
    flags[3] = (int)G;
    if (!ok) flags[4] = 1;
    mma_commit(done);
    if (!mbar_wait(done, 0)) flags[4] = 1;
  } else if (warp == 2 && lane == 0) {
    // ---- tap stages
    uint32_t G = 0, ph = 0;
    int slot = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, t, b, zt, yt, xc);
      if (instance_done(conv_iter, b, it)) continue;
      const uint16_t* src = taps;
      for (int s = 0; s < nst; s++, G++) {
        // the slot's previous stage (G - kPRing) must have been consumed
        if (G >= (uint32_t)kPRing && !mbar_wait(&tempty[slot], ph ^ 1u)) {
          ok = false;
          break;
        }
        mbar_expect_tx(&tfull[slot], kStageBytes);
        bulk_load(ring + slot * kStageBytes, src, kStageBytes, &tfull[slot]);
        src += kStageBytes / 2;
        if (++slot == kPRing) {
          slot = 0;
          ph ^= 1u;
        }
      }
    }
    flags[2] = (int)G;
    if (!ok) flags[4] = 1;
  } else if (warp >= 4) {
    // ---- epilogue
    const int q = warp - 4;
    const int r = q * 32 + lane;
    int sp, f, xo;
    bool rvalid;
    if (g.SP == 2) {
      sp = r >> 6;
      const int rr = r & 63;
      f = rr / kXo;
      xo = rr - f * kXo;
      rvalid = rr < 2 * a.nfilt * kXo;
    } else {
      sp = 0;
      f = r / kXo;
      xo = r - f * kXo;
      rvalid = r < 2 * a.nfilt * kXo;
    }
    const int rowf = 20 * a.nfilt;
    const int ke = (f >> 1) * 20 + xo * 2 + (f & 1);
    const int et = tid - 128;
    // stores: SP * nfilt * 5 = 30 16-byte pieces per accumulator column
    // (plane s2, filter k, x pair); threads et < 120 take piece et % 30 of
    // every fourth column, starting at column et / 30
    const int piece = et % 30, cgrp = et / 30;
    const int part = piece % 5, sk = piece / 5;
    const int s2 = sk / a.nfilt, k = sk - s2 * a.nfilt;
    const bool vec16 = ((a.W & 1) == 0) && ((V & 1) == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    int i = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, t, b, zt, yt, xc);
      if (instance_done(conv_iter, b, it)) continue;
      const int acc = i & 1;
      // one thread waits and tells the other 127, so that all of them leave
      // together if the wait gives up (they meet at named barriers below)
      if (et == 0) flags[5] = mbar_wait(&acc_full[acc], (uint32_t)(i >> 1) & 1u) ? 1 : 0;
      epi_sync();
      const bool ready = *reinterpret_cast<volatile int*>(&flags[5]) != 0;
      epi_sync();
      if (!ready) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int x0 = xc * kXo, y0 = yt * g.Ty, z0 = zt * g.SP * g.J;
      const uint32_t lanecol = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * 256);
      for (int cbase = 0; cbase < g.N; cbase += a.ecols) {
        const int cend = cbase + a.ecols < g.N ? cbase + a.ecols : g.N;
        for (int c0 = cbase; c0 < cend; c0 += 16) {
          uint32_t v[16];
          tmem_ld16(lanecol + (uint32_t)c0, v);
          if (rvalid) {
#pragma unroll
            for (int e = 0; e < 16; e++) E[((c0 + e - cbase) * g.SP + sp) * rowf + ke] = __uint_as_float(v[e]);
          }
        }
        if (cend >= g.N) {
          // this accumulator is read out: the GEMMs of tile i + 2 may start
          tc_fence_before();
          mbar_arrive(&acc_empty[acc]);
        }
        epi_sync();
        if (et < 120) {
          int nl = cgrp;
          int j = (cbase + nl) / g.Hp, yl = cbase + nl - j * g.Hp;
          const int xs = x0 + 2 * part;
          for (; nl < cend - cbase; nl += 4) {
            const int z = z0 + j * g.SP + s2, y = y0 + yl;
            if (j < g.J && yl < g.Ty && y < a.H && z < a.D && xs < a.W) {
              const float4 qv = *reinterpret_cast<const float4*>(E + (nl * g.SP + s2) * rowf + k * 20 + part * 4);
              float* dst = out + (((long long)b * a.nfilt + k) * V + ((long long)z * a.H + y) * a.W + xs) * 2;
              if (xs + 1 < a.W && vec16) {
                *reinterpret_cast<float4*>(dst) = qv;
              } else {
                *reinterpret_cast<float2*>(dst) = make_float2(qv.x, qv.y);
                if (xs + 1 < a.W) *reinterpret_cast<float2*>(dst + 2) = make_float2(qv.z, qv.w);
              }
            }
            yl += 4;  // Hp >= 7 > 4: at most one wrap
            if (yl >= g.Hp) {
              yl -= g.Hp;
              j++;
            }
          }
        }
        epi_sync();
      }
      i++;
    }
    if (!ok) flags[4] = 1;
  }

  __syncthreads();
  // a wait gave up somewhere: bounded drain of the copies nothing consumed
  if (tid == 0)
    for (int j = flags[1]; j < flags[0]; j++) mbar_wait(&full_in[j & 1], (uint32_t)(j >> 1) & 1u);
  if (tid == 64)
    for (int s = flags[3]; s < flags[2]; s++) mbar_wait(&tfull[s % kPRing], (uint32_t)(s / kPRing) & 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPTmemCols) : "memory");
  if (tid == 0 && flags[4]) atomicExch(err, 1);
}

// One thread per packed row (b, xc, z, y), y fastest: the 16 samples of the
// window, split into BF16 hi and lo.
__global__ void pack_windows_kernel(const float* __restrict__ vol, long long vstride, int W, int H, int D, int Dp,
                                    int nxc, uint4* __restrict__ packed, const int* __restrict__ conv_iter,
                                    int it) {
  const int b = blockIdx.y;
  if (instance_done(conv_iter, b, it)) return;
  const long long rows = (long long)nxc * Dp * H;
  const float* src = vol + (long long)b * vstride;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(r % H);
    const long long t = r / H;
    const int z = (int)(t % Dp), xc = (int)(t / Dp);
    const int xs = xc * kXo - 3;
    const bool rowok = z < D;
    const float* rp = src + ((long long)(rowok ? z : 0) * H + y) * W;
    uint32_t ph[8], pl[8];
#pragma unroll
    for (int e = 0; e < 16; e += 2) {
      const int xa = xs + e, xb = xs + e + 1;
      const float va = (rowok && xa >= 0 && xa < W) ? __ldg(rp + xa) : 0.f;
      const float vb = (rowok && xb >= 0 && xb < W) ? __ldg(rp + xb) : 0.f;
      const __nv_bfloat16 ha = __float2bfloat16_rn(va), hb = __float2bfloat16_rn(vb);
      const __nv_bfloat16 la = __float2bfloat16_rn(va - __bfloat162float(ha));
      const __nv_bfloat16 lb = __float2bfloat16_rn(vb - __bfloat162float(hb));
      ph[e / 2] = pack_bf16(ha, hb);
      pl[e / 2] = pack_bf16(la, lb);
    }
    const long long hrow = (((long long)(b * 2) * nxc + xc) * Dp + z) * H + y;
    const long long lrow = hrow + (long long)nxc * Dp * H;
    packed[2 * hrow] = make_uint4(ph[0], ph[1], ph[2], ph[3]);
    packed[2 * hrow + 1] = make_uint4(ph[4], ph[5], ph[6], ph[7]);
    packed[2 * lrow] = make_uint4(pl[0], pl[1], pl[2], pl[3]);
    packed[2 * lrow + 1] = make_uint4(pl[4], pl[5], pl[6], pl[7]);
  }
}

// Self-test of the bounded wait and the error flag: thread 0 waits on an
// mbarrier that nothing arrives on, gives up after limit_ns and sets *err,
// as a CTA of filter3d_tc_kernel does when a wait runs out.
__global__ void bounded_wait_probe_kernel(unsigned long long limit_ns, int* __restrict__ err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, limit_ns)) atomicExch(err, 1);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

static uint16_t bf16_rn(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
static float bf16_to_f(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

int stacked_planes(int nfilt) { return nfilt == 3 ? 2 : 1; }
int num_stages(int nfilt) { return (7 + stacked_planes(nfilt) - 1) * 7; }
size_t packed_tap_bytes(int nfilt) { return (size_t)num_stages(nfilt) * kStageBytes; }

void pack_taps(const float* h_filters, int nfilt, uint16_t* dst) {
  const int SP = stacked_planes(nfilt);
  const int nst = num_stages(nfilt);
  memset(dst, 0, (size_t)nst * kStageBytes);
  for (int st = 0; st < nst; st++) {
    const int c = st / 7 - 3, dy = st % 7 - 3;
    uint16_t* hi = dst + (size_t)st * 2 * kStageHalves;
    uint16_t* lo = hi + kStageHalves;
    for (int r = 0; r < kM; r++) {
      int s, f, xo;
      if (SP == 2) {
        s = r >> 6;
        const int rr = r & 63;
        if (rr >= 2 * nfilt * kXo) continue;
        f = rr / kXo;
        xo = rr % kXo;
      } else {
        s = 0;
        if (r >= 2 * nfilt * kXo) continue;
        f = r / kXo;
        xo = r % kXo;
      }
      const int dz = c - s;
      if (dz < -3 || dz > 3) continue;
      const float* F = h_filters + (size_t)(f >> 1) * kFilterFloats + (f & 1) * kTaps;
      for (int kx = xo; kx <= xo + 6; kx++) {
        const int dx = kx - 3 - xo;
        const float w = F[(3 - dz) * 49 + (3 - dy) * 7 + (3 - dx)];
        const uint16_t wh = bf16_rn(w);
        const uint16_t wl = bf16_rn(w - bf16_to_f(wh));
        const size_t e = (size_t)(kx / 8) * (kM * 8) + (size_t)r * 8 + (kx % 8);
        hi[e] = wh;
        lo[e] = wl;
      }
    }
  }
}

Geometry make_geometry(int nfilt, int H, int D, int Ty) {
  Geometry g;
  g.SP = stacked_planes(nfilt);
  g.Ty = Ty < H ? Ty : H;
  g.Hp = g.Ty + 6;
  g.J = kMaxN / g.Hp;
  if (g.J < 1) g.J = 1;
  // no more plane groups than the volume needs
  const int jmax = (D + g.SP - 1) / g.SP;
  if (g.J > jmax) g.J = jmax;
  g.N = ((g.J * g.Hp + 15) / 16) * 16;
  const int qmax = (5 + g.SP) / g.SP;  // largest plane-slot offset of a GEMM: (c+3)/SP, c <= 2+SP
  g.RP = ((qmax * g.Hp + 6 + g.N) + 7) / 8 * 8;
  g.NR = g.SP * g.RP;
  g.nstage = num_stages(nfilt);
  g.smem = kRing * kStageBytes + 2 * 32 * g.NR + (2 * kRing + 1) * 8 + 32;
  return g;
}

bool geometry_ok(const Geometry& g) {
  return g.Hp <= kMaxN && g.N >= 16 && g.N <= kMaxN && g.smem <= 227 * 1024;
}

// Cost model of a tile shape: GEMM columns issued over the volume (tiles x
// (N + 32), the 32 standing for a tile's staging and epilogue), x1.3 when
// the tile leaves no room for a second CTA on the SM.
static long long tile_cost(const Geometry& g, int H, int D, bool persistent) {
  const long long ny = (H + g.Ty - 1) / g.Ty;
  const long long nz = (D + g.SP * g.J - 1) / (g.SP * g.J);
  if (persistent) return ny * nz * (g.N + 16);
  long long cost = ny * nz * (g.N + 32);
  if (g.smem > 113 * 1024) cost = cost * 13 / 10;
  return cost;
}

int persistent_smem(const Geometry& g);
bool persistent_ok(const Geometry& g);

int candidate_tys(int nfilt, int H, int D, int* tys, int max_n, bool persistent) {
  // the cheapest tile height for each plane-group count J (ties to the
  // taller tile), then the max_n cheapest of those
  long long best_cost[kMaxN + 1];
  int best_ty[kMaxN + 1];
  for (int j = 0; j <= kMaxN; j++) best_ty[j] = -1;
  const int lo = H < 10 ? H : 10;
  const int hi = H < kMaxN - 6 ? H : kMaxN - 6;
  for (int ty = hi; ty >= lo; ty--) {
    const Geometry g = make_geometry(nfilt, H, D, ty);
    if (persistent ? !persistent_ok(g) : !geometry_ok(g)) continue;
    const long long c = tile_cost(g, H, D, persistent);
    if (best_ty[g.J] < 0 || c < best_cost[g.J]) {
      best_ty[g.J] = g.Ty;
      best_cost[g.J] = c;
    }
  }
  int n = 0;
  for (; n < max_n; n++) {
    int pick = -1;
    for (int j = 1; j <= kMaxN; j++)
      if (best_ty[j] >= 0 && (pick < 0 || best_cost[j] < best_cost[pick])) pick = j;
    if (pick < 0) break;
    tys[n] = best_ty[pick];
    best_ty[pick] = -1;
  }
  return n;
}

int pick_ty(int nfilt, int H, int D, bool persistent) {
  int ty = -1;
  return candidate_tys(nfilt, H, D, &ty, 1, persistent) == 1 ? ty : -1;
}

// ---- persistent form -------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static int g_num_sms = 0;

static int dpad(int D, int SP) { return (D + SP - 1) / SP * SP; }

size_t packed_bytes(int W, int H, int D, int batch, int nfilt) {
  const int SP = stacked_planes(nfilt);
  const long long nxc = (W + kXo - 1) / kXo;
  return (size_t)batch * 2 * (size_t)nxc * (size_t)dpad(D, SP) * (size_t)H * 32u;
}

static int epi_cols() { return 64; }

int persistent_smem(const Geometry& g) {
  const int ebytes = epi_cols() * 6 * 20 * 4;  // SP * nfilt = 6 for both banks
  const int need = kPRing * kStageBytes + 128 * g.NR + ebytes + kPBarBytes;
  return need > 116 * 1024 ? need : 116 * 1024;  // one CTA (and 512 TMEM columns) per SM
}

bool persistent_ok(const Geometry& g) {
  return g.Hp <= kMaxN && g.N >= 16 && g.N <= kMaxN && persistent_smem(g) <= 227 * 1024;
}

cudaError_t pack(const float* vol, int W, int H, int D, int batch, long long stride, int nfilt, uint16_t* packed,
                 const int* conv_iter, int it, cudaStream_t st) {
  if (batch <= 0 || batch > 65535 || (nfilt != 3 && nfilt != 6)) return cudaErrorInvalidValue;
  const int SP = stacked_planes(nfilt);
  const int nxc = (W + kXo - 1) / kXo, Dp = dpad(D, SP);
  const long long rows = (long long)nxc * Dp * H;
  long long nb = (rows + 255) / 256;
  const long long cap = 4LL * (g_num_sms > 0 ? g_num_sms : 148);
  if (nb > cap) nb = cap;
  dim3 grid((unsigned)nb, (unsigned)batch);
  pack_windows_kernel<<<grid, 256, 0, st>>>(vol, stride, W, H, D, Dp, nxc, reinterpret_cast<uint4*>(packed),
                                            conv_iter, it);
  return cudaGetLastError();
}

cudaError_t launch_packed(const uint16_t* packed, int W, int H, int D, int batch, const uint16_t* d_taps, int nfilt,
                          float* out, const int* conv_iter, int it, int* d_err, const Geometry& g, cudaStream_t st) {
  if (!g_encode || g_num_sms <= 0) return cudaErrorInitializationError;
  if (!persistent_ok(g) || (nfilt != 3 && nfilt != 6) || g.SP != stacked_planes(nfilt)) return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(packed) & 15) != 0 || batch <= 0) return cudaErrorInvalidValue;
  PArgs a;
  a.W = W;
  a.H = H;
  a.D = D;
  a.Dp = dpad(D, g.SP);
  a.nxc = (W + kXo - 1) / kXo;
  a.nyt = (H + g.Ty - 1) / g.Ty;
  a.nzt = (D + g.SP * g.J - 1) / (g.SP * g.J);
  a.batch = batch;
  a.nfilt = nfilt;
  const long long ntiles = (long long)a.nxc * a.nyt * a.nzt * batch;
  if (ntiles > 0x7fffffffLL || (long long)batch * 2 * a.nxc > 0x7fffffffLL) return cudaErrorInvalidValue;
  a.ntiles = (int)ntiles;
  a.nqp = (g.SP * g.J + 6) / g.SP;
  a.ecols = epi_cols();
  a.in_off = (uint32_t)(kPRing * kStageBytes);
  a.e_off = a.in_off + 128u * (uint32_t)g.NR;
  a.bar_off = a.e_off + (uint32_t)(a.ecols * 6 * 20 * 4);
  const int smem = persistent_smem(g);

  CUtensorMap map;
  const cuuint64_t dims[5] = {16, (cuuint64_t)H, (cuuint64_t)g.SP, (cuuint64_t)(a.Dp / g.SP),
                              (cuuint64_t)batch * 2 * (cuuint64_t)a.nxc};
  const cuuint64_t strides[4] = {32, 32 * (cuuint64_t)H, 32 * (cuuint64_t)H * g.SP, 32 * (cuuint64_t)H * a.Dp};
  const cuuint32_t box[5] = {8, (cuuint32_t)g.Hp, 1, (cuuint32_t)a.nqp, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult cr = g_encode(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<uint16_t*>(packed), dims,
                               strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const int grid = a.ntiles < g_num_sms ? a.ntiles : g_num_sms;
  filter3d_tcp_kernel<<<grid, kPThreads, smem, st>>>(map, d_taps, out, a, g, conv_iter, it, d_err);
  return cudaGetLastError();
}

cudaError_t bounded_wait_probe(int wait_ms, int* d_err, cudaStream_t st) {
  if (wait_ms < 1 || wait_ms > 1000) return cudaErrorInvalidValue;
  bounded_wait_probe_kernel<<<1, 32, 0, st>>>((unsigned long long)wait_ms * 1000000ull, d_err);
  return cudaGetLastError();
}

cudaError_t init() {
  cudaError_t e = cudaFuncSetAttribute(filter3d_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(filter3d_tcp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e != cudaSuccess) return e;
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if (!g_encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return e != cudaSuccess ? e : cudaErrorNotSupported;
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return cudaSuccess;
}

cudaError_t launch(const float* vol, int W, int H, int D, int batch, long long stride, const uint16_t* d_taps,
                   int nfilt, float* out, const int* conv_iter, int it, int* d_err, const Geometry& g,
                   cudaStream_t st) {
  if (!geometry_ok(g) || (nfilt != 3 && nfilt != 6) || g.SP != stacked_planes(nfilt)) return cudaErrorInvalidValue;
  const int nxc = (W + kXo - 1) / kXo;
  const int nyt = (H + g.Ty - 1) / g.Ty;
  const int nzt = (D + g.SP * g.J - 1) / (g.SP * g.J);
  if ((long long)nxc * nyt > 0x7fffffffLL || nzt > 65535 || batch > 65535) return cudaErrorInvalidValue;
  // at least 77 KB per CTA: at most two CTAs (2 x 256 TMEM columns) per SM
  const int smem = g.smem > 77 * 1024 ? g.smem : 77 * 1024;
  dim3 grid((unsigned)(nxc * nyt), (unsigned)nzt, (unsigned)batch);
  filter3d_tc_kernel<<<grid, kThreads, smem, st>>>(vol, W, H, D, stride, d_taps, out, nfilt, g, nxc, conv_iter,
                                                   it, d_err);
  return cudaGetLastError();
}

}  // namespace tc
}  // namespace brc
