// filter3d_tc.cu -- 7x7x7 complex filtering on the tcgen05 tensor cores in
// BF16 split precision (BRC_PREC_BF16X3) or TF32 (BRC_PREC_TF32), with FP32
// accumulation.
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
// TF32: data and taps rounded to TF32 (10-bit mantissa, round to nearest,
// ties away), one product per tap (relative error ~2^-10), as ONE
// structured-sparse MMA of K = 16 per GEMM (tcgen05.mma.sp, kind::tf32,
// 1:2 sparsity): the banded A holds 7 taps in 16 K columns, and pairing
// sample P with sample P + 8 (P < 8) puts at most one tap in each pair, so
// A is stored as one value per pair (half the tap bytes) and a fixed
// metadata column in TMEM says which of the pair it is.  B's 16 samples of
// a row sit in four 16-byte quarters in that pair order (quarter q:
// samples 2q, 2q + 8, 2q + 1, 2q + 9), the bytes and descriptor strides of
// the BF16 form's hi and lo parts of two 8-sample halves.
//
// One persistent CTA per SM walks the tiles of the launch (10 x positions x
// Ty rows x SP*J planes of one volume each) with its warps specialised:
//
//   warps 12-19    stage a tile's input (FP32 -> BF16 hi/lo or TF32 rows)
//                  into one of two shared-memory buffers while the GEMMs
//                  read the other
//   warp 1, lane 0 issues the tcgen05.mma's: three split products (BF16X3)
//                  or one sparse MMA (TF32) per stage, descriptors built
//                  once and advanced by adds (every cycle of address
//                  arithmetic in this thread delays the GEMMs)
//   warp 2, lane 0 streams the packed taps, two stages (BF16X3: 16 KB, hi
//                  + lo of each; TF32: 8 KB) per slot, through a 3-slot
//                  ring with cp.async.bulk + mbarriers (one wait and one
//                  commit per two GEMMs)
//   warps 4-11     epilogue: tcgen05.ld of the accumulator (TMEM lanes
//                  32 (warp % 4) .., the two warps of a lane quarter on
//                  alternate 16-column groups); TF32 stores each lane's
//                  values straight to global memory (a warp's store: 80
//                  contiguous bytes per filter), BF16X3 transposes them
//                  through shared memory into 16-byte stores (its GEMMs
//                  bound the launch, and the direct stores slowed them)
//
// Two TMEM accumulators (2 x 256 of the SM's 512 columns) let the epilogue
// of tile i run under the GEMMs of tile i + 1.  Every wait is bounded
// (about 2 s); a CTA that gives up sets *err, waits (bounded) for its MMAs
// and copies in flight, frees its TMEM and returns.  The responses of a
// launch that timed out are undefined.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "common.cuh"
#include "filter3d_tc.h"

namespace brc {
namespace tc {

// Group sizes measured on 199 volumes of 64x64x33 (dense TF32 / BF16X3 ms):
// 4 + 4 warps 0.58 / 0.72, 8 + 4 0.57 / 0.74, 4 + 8 0.66 / 0.72, 8 + 8
// 0.534 / 0.696, 12 + 8 and 8 + 12 0.54-0.55 / 0.70.
constexpr int kEpiWarps = 8;         // epilogue warps (a multiple of 4: kEpiWarps / 4 per TMEM lane quarter)
constexpr int kStageWarps = 8;       // staging warps
constexpr int kStageWarp = 4 + kEpiWarps;                    // first staging warp
constexpr int kThreads = 32 * (4 + kEpiWarps + kStageWarps);  // roles above
constexpr int kEpiThreads = 32 * kEpiWarps, kStageThreads = 32 * kStageWarps;
constexpr int kEpiGroups = kEpiThreads / 30;  // accumulator columns stored at once (30 pieces each)
constexpr int kRing = 3;             // tap slots in flight (two stages each; 2, 4, 5, 6 measured slower)
constexpr int kEpiCols = 64;         // accumulator columns per epilogue chunk
constexpr uint32_t kTmemCols = 512;  // two accumulators of up to 256 columns
constexpr int kStageHalves = kM * kK;              // BF16 elements of one A (hi or lo)
constexpr int kStageBytes = 2 * kStageHalves * 2;  // hi + lo
constexpr int kSlotBytes = 2 * kStageBytes;        // a ring slot: two stages
constexpr int kSlotsPerTile = 28;                  // 7 dy x 4 pairs of input-plane offsets
// TF32: structured-sparse A, kM rows x 8 stored values (16 K samples)
constexpr int kStageBytesSp = kM * 8 * 4;
constexpr int kSlotBytesSp = 2 * kStageBytesSp;
constexpr uint32_t kMetaCol = 508;  // TMEM column of the sparsity metadata (N <= 240: free)
constexpr int kEpiBytes = kEpiCols * 6 * 20 * 4;   // SP * nfilt = 6 for both banks
// barrier block: full_in, empty_in, acc_full, acc_empty (2 each), the ring's
// full / empty (kRing each), done; then the TMEM address and 7 flags
constexpr int kBarBytes = ((8 + 2 * kRing + 1) * 8 + 4 + 7 * 4 + 15) / 16 * 16;
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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Named barriers of the 128-thread groups (0 is __syncthreads).
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory"); }
__device__ __forceinline__ void stage_sync() { asm volatile("bar.sync 2, %0;" ::"n"(kStageThreads) : "memory"); }

struct TileArgs {
  long long vstride;       // floats between volumes
  int W, H, D, nxc, nyt, nzt, nfilt, batch;
  int tiles_per;           // tiles of one volume
  int nqp;                 // input plane slots per parity array: (SP J + 6) / SP
  uint32_t in_off;         // shared offsets: input buffers, epilogue buffer, barriers
  uint32_t e_off;
  uint32_t bar_off;
};

// Tile t of the launch -> (instance b, zt, yt, xc), xc fastest; the
// instances are those of the active set, in its order.
__device__ __forceinline__ void decode_tile(const TileArgs& a, const ActiveSet& act, int t, int& b, int& zt,
                                            int& yt, int& xc) {
  const int li = t / a.tiles_per;
  int r = t - li * a.tiles_per;
  xc = r % a.nxc;
  r /= a.nxc;
  yt = r % a.nyt;
  zt = r / a.nyt;
  b = active_instance(act, li);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// One structured-sparse TF32 MMA (K = 16 samples, 8 stored per A row), its
// metadata in TMEM column tmem_e.
__device__ __forceinline__ void mma_tf32_sp(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t tmem_e,
                                            uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.sp.cta_group::1.kind::tf32 [%0], %1, %2, [%5], %3, {%6, %7, %8, %9}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(tmem_e), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Sparsity metadata of TMEM lane L for the banded A (the same for every
// stage): lane L = m0 + 8 k1 + 16 m2 holds rows m0 + 8 m1 + 16 m2 (m1 = 0,
// 1) in bits 16 m1 .., K half k1; a nibble per sample pair j of that half
// (pair P = 4 k1 + j: samples P and P + 8), 0b0100 keeping the first and
// 0b1110 the second; row r's taps are samples xo .. xo + 6.
__host__ __device__ __forceinline__ uint32_t sparse_metadata_word(int L, int SP, int nfilt) {
  const int m0 = L & 7, k1 = (L >> 3) & 1, m2 = L >> 4;
  uint32_t word = 0;
  for (int m1 = 0; m1 < 2; m1++) {
    const int r = m0 + 8 * m1 + 16 * m2;
    const int rr = SP == 2 ? (r & 63) : r;
    const bool valid = rr < 2 * nfilt * kXo;
    const int xo = rr % kXo;
    for (int j = 0; j < 4; j++) {
      const int P = 4 * k1 + j;
      const bool second = valid && !(P >= xo && P <= xo + 6) && (P + 8 >= xo && P + 8 <= xo + 6);
      word |= (second ? 0xEu : 0x4u) << (16 * m1 + 4 * j);
    }
  }
  return word;
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

template <bool TF32>
__global__ void __launch_bounds__(kThreads, 1)
filter3d_tc_kernel(const float* __restrict__ vol, const uint16_t* __restrict__ taps, float* __restrict__ out,
                   const TileArgs a, const Geometry g, const ActiveSet act, int* __restrict__ err) {
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
  uint64_t* tempty = tfull + kRing;
  uint64_t* done = tempty + kRing;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  // [1] tiles the GEMMs finished, [2] tap stages loaded, [3] tap stages
  // consumed, [4] a wait gave up, [5] / [6] epilogue / staging broadcasts
  int* flags = reinterpret_cast<int*>(tmem_slot + 1);

  // one K half of one part (hi or lo) of one input buffer: NR 16-byte rows
  const uint32_t rowbytes = 16u * (uint32_t)g.NR;
  const long long V = (long long)a.W * a.H * a.D;
  // every role walks the same tiles: those of the active instances
  const int ntiles = active_count(act, a.batch) * a.tiles_per;

  if (tid == 0) {
    for (int i = 0; i < 2; i++) {
      mbar_init(&full_in[i], kStageThreads);
      mbar_init(&empty_in[i], 1);
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], kEpiThreads);
    }
    for (int s = 0; s < kRing; s++) {
      mbar_init(&tfull[s], 1);
      mbar_init(&tempty[s], 1);
    }
    mbar_init(done, 1);
    for (int i = 0; i < 7; i++) flags[i] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  if (TF32) {
    // the sparsity metadata, one column for every MMA of the launch
    if (warp >= 4 && warp < 8) {
      const int q = warp - 4;
      const uint32_t word = sparse_metadata_word(32 * q + lane, g.SP, a.nfilt);
      asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(tmem + ((uint32_t)(32 * q) << 16) +
                                                                             kMetaCol),
                   "r"(word)
                   : "memory");
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }

  if (warp >= kStageWarp) {
    // ---- staging: row (parity p, plane slot qq, y row yl) of K half kh
    // holds the 8 samples x0-3+8kh .. x0+4+8kh of input plane z0-3+SP*qq+p,
    // row y0-3+yl (zero outside the volume), as BF16 hi and lo.
    const int st = tid - kStageWarp * 32;
    const int prow = a.nqp * g.Hp;   // staged rows per parity array
    const int nrows = g.SP * prow;   // staged rows per K half
    int i = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, act, t, b, zt, yt, xc);
      const int buf = i & 1;
      // one thread waits for the buffer and tells the others
      if (st == 0) flags[6] = (i < 2 || mbar_wait(&empty_in[buf], (uint32_t)((i >> 1) - 1) & 1u)) ? 1 : 0;
      stage_sync();
      const bool go = *reinterpret_cast<volatile int*>(&flags[6]) != 0;
      stage_sync();
      if (!go) {
        ok = false;
        break;
      }
      const int x0 = xc * kXo, y0 = yt * g.Ty, z0 = zt * g.SP * g.J;
      const float* src = vol + (long long)b * a.vstride;
      // rows are 16-byte aligned when W is a multiple of 4 (and the volume
      // is): a window inside the row then takes three aligned float4 loads
      const bool vec_rows = (a.W & 3) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0;
      uint8_t* hi = inb + (uint32_t)(buf * 4) * rowbytes;
      uint8_t* lo = hi + 2u * rowbytes;
      if (TF32) {
        // whole rows of 16 samples x0 - 3 .. x0 + 12, in the K order of the
        // sparse MMA: quarter q holds samples 2q, 2q + 8, 2q + 1, 2q + 9
        for (int row = st; row < nrows; row += kStageThreads) {
          const int par = row / prow, rr = row - par * prow;
          const int qq = rr / g.Hp, yl = rr - qq * g.Hp;
          const int zg = z0 - 3 + qq * g.SP + par, yg = y0 - 3 + yl;
          const bool rowok = zg >= 0 && zg < a.D && yg >= 0 && yg < a.H;
          const int xs = x0 - 3;
          float v[16];
          if (rowok && vec_rows && xs >= 0 && (xs & ~3) + 20 <= a.W) {
            const int al = xs & 3;
            const float4* p4 = reinterpret_cast<const float4*>(src + ((long long)zg * a.H + yg) * a.W + (xs - al));
            const float4 f0 = __ldg(p4), f1 = __ldg(p4 + 1), f2 = __ldg(p4 + 2), f3 = __ldg(p4 + 3),
                         f4 = __ldg(p4 + 4);
            const float w[20] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f2.x, f2.y,
                                 f2.z, f2.w, f3.x, f3.y, f3.z, f3.w, f4.x, f4.y, f4.z, f4.w};
#pragma unroll
            for (int e = 0; e < 16; e++)
              v[e] = al == 0 ? w[e] : (al == 1 ? w[e + 1] : (al == 2 ? w[e + 2] : w[e + 3]));
          } else {
            const float* rp = src + ((long long)(rowok ? zg : 0) * a.H + (rowok ? yg : 0)) * a.W;
#pragma unroll
            for (int e = 0; e < 16; e++) {
              const int xg = xs + e;
              v[e] = (rowok && xg >= 0 && xg < a.W) ? __ldg(rp + xg) : 0.f;
            }
          }
          const uint32_t rowoff = (uint32_t)(par * g.RP + qq * g.Hp + yl) * 16u;
#pragma unroll
          for (int q = 0; q < 4; q++)
            *reinterpret_cast<uint4*>(hi + (uint32_t)q * rowbytes + rowoff) =
                make_uint4(tf32_rna(v[2 * q]), tf32_rna(v[2 * q + 8]), tf32_rna(v[2 * q + 1]), tf32_rna(v[2 * q + 9]));
        }
      }
      for (int item = st; !TF32 && item < 2 * nrows; item += kStageThreads) {
        const int kh = item >= nrows ? 1 : 0, row = item - kh * nrows;
        const int par = row / prow, rr = row - par * prow;
        const int qq = rr / g.Hp, yl = rr - qq * g.Hp;
        const int zg = z0 - 3 + qq * g.SP + par, yg = y0 - 3 + yl;
        const bool rowok = zg >= 0 && zg < a.D && yg >= 0 && yg < a.H;
        const int xs = x0 - 3 + 8 * kh;
        float v[8];
        if (rowok && vec_rows && xs >= 0 && (xs & ~3) + 12 <= a.W) {
          const int al = xs & 3;
          const float4* p4 = reinterpret_cast<const float4*>(src + ((long long)zg * a.H + yg) * a.W + (xs - al));
          const float4 f0 = __ldg(p4), f1 = __ldg(p4 + 1), f2 = __ldg(p4 + 2);
          const float w[12] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w};
#pragma unroll
          for (int e = 0; e < 8; e++) v[e] = al == 0 ? w[e] : (al == 1 ? w[e + 1] : (al == 2 ? w[e + 2] : w[e + 3]));
        } else {
          const float* rp = src + ((long long)(rowok ? zg : 0) * a.H + (rowok ? yg : 0)) * a.W;
#pragma unroll
          for (int e = 0; e < 8; e++) {
            const int xg = xs + e;
            v[e] = (rowok && xg >= 0 && xg < a.W) ? __ldg(rp + xg) : 0.f;
          }
        }
        const uint32_t rowoff = (uint32_t)(par * g.RP + qq * g.Hp + yl) * 16u;
        {
          uint32_t ph4[4], pl4[4];
#pragma unroll
          for (int e = 0; e < 8; e += 2) {
            const __nv_bfloat16 h0 = __float2bfloat16_rn(v[e]), h1 = __float2bfloat16_rn(v[e + 1]);
            const __nv_bfloat16 l0 = __float2bfloat16_rn(v[e] - __bfloat162float(h0));
            const __nv_bfloat16 l1 = __float2bfloat16_rn(v[e + 1] - __bfloat162float(h1));
            ph4[e / 2] = pack_bf16(h0, h1);
            pl4[e / 2] = pack_bf16(l0, l1);
          }
          const uint32_t off = (uint32_t)kh * rowbytes + rowoff;
          *reinterpret_cast<uint4*>(hi + off) = make_uint4(ph4[0], ph4[1], ph4[2], ph4[3]);
          *reinterpret_cast<uint4*>(lo + off) = make_uint4(pl4[0], pl4[1], pl4[2], pl4[3]);
        }
      }
      // the GEMMs read the buffer through the async proxy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full_in[buf]);
      i++;
    }
    if (!ok) flags[4] = 1;
  } else if (warp == 1 && lane == 0) {
    // ---- GEMM issue.  The descriptors are built once; a stage only adds
    // offsets to their start-address fields (one 16-byte row = 1), so that
    // the issuing thread spends its time in tcgen05.mma, not in address
    // arithmetic (which delays every GEMM it precedes).
    // D F32; A, B BF16 (1) or TF32 (2); K-major; N, M
    // (TF32: structured-sparse MMAs, sparse flag bit 2, metadata in TMEM
    // column kMetaCol)
    const uint32_t ab = TF32 ? 2u : 1u;
    const uint32_t idesc = (TF32 ? (1u << 2) : 0u) | (1u << 4) | (ab << 7) | (ab << 10) |
                           ((uint32_t)(g.N >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
    const uint32_t tmem_e = tmem + kMetaCol;
    const uint64_t da0 = sdesc(smem_u32(ring), kM * 16, 128);  // slot 0, hi taps
    const uint64_t db0 = sdesc(smem_u32(inb), rowbytes, 128);  // buffer 0, hi part, row 0
    const uint64_t dslot = (TF32 ? kSlotBytesSp : kSlotBytes) >> 4;
    const uint64_t dstage = (TF32 ? kStageBytesSp : kStageBytes) >> 4, dalo = kStageBytes >> 5;
    const uint64_t dbuf = (4u * rowbytes) >> 4, dblo = (2u * rowbytes) >> 4;
    // slot m of dy row dyq holds the taps of input-plane offsets cq = 2m and
    // 2m + 1 (c = cq - 3); their B rows start at parity array cq % SP, plane
    // slot cq / SP, row dyq.  The last slot's second stage (cq = 7) exists
    // only with two stacked planes.
    uint64_t offa[4], offb[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
      offa[m] = (uint64_t)(((2 * m) % g.SP) * g.RP + ((2 * m) / g.SP) * g.Hp);
      offb[m] = (uint64_t)(((2 * m + 1) % g.SP) * g.RP + ((2 * m + 1) / g.SP) * g.Hp);
    }
    const bool last_pair = g.SP == 2;
    int i = 0, slot = 0;
    uint32_t ph = 0, G = 0;
    uint64_t ah = da0;
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, act, t, b, zt, yt, xc);
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
      for (int dyq = 0; dyq < 7 && ok; dyq++) {
#pragma unroll
        for (int m = 0; m < 4; m++) {
          if (!mbar_wait(&tfull[slot], ph)) {
            ok = false;
            break;
          }
          const uint64_t b1 = bh0 + offa[m] + (uint64_t)dyq;
          if (TF32) {
            mma_tf32_sp(dcol, ah, b1, tmem_e, idesc, accf);
          } else {
            mma_bf16(dcol, ah, b1, idesc, accf);
            mma_bf16(dcol, ah, b1 + dblo, idesc, 1u);
            mma_bf16(dcol, ah + dalo, b1, idesc, 1u);
          }
          accf = 1u;
          if (m < 3 || last_pair) {
            const uint64_t b2 = bh0 + offb[m] + (uint64_t)dyq, a2 = ah + dstage;
            if (TF32) {
              mma_tf32_sp(dcol, a2, b2, tmem_e, idesc, 1u);
            } else {
              mma_bf16(dcol, a2, b2, idesc, 1u);
              mma_bf16(dcol, a2, b2 + dblo, idesc, 1u);
              mma_bf16(dcol, a2 + dalo, b2, idesc, 1u);
            }
          }
          mma_commit(&tempty[slot]);
          G++;
          ah += dslot;
          if (++slot == kRing) {
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
    // on every exit, the give-up path included: one commit that tracks all
    // MMAs this thread issued, waited on (bounded) before the TMEM and the
    // shared-memory stages are released below
    mma_commit(done);
    if (!mbar_wait(done, 0)) flags[4] = 1;
  } else if (warp == 2 && lane == 0) {
    // ---- tap stages
    uint32_t G = 0, ph = 0;
    int slot = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, act, t, b, zt, yt, xc);
      const uint16_t* src = taps;
      for (int s = 0; s < kSlotsPerTile; s++, G++) {
        // the slot's previous pair (G - kRing) must have been consumed
        if (G >= (uint32_t)kRing && !mbar_wait(&tempty[slot], ph ^ 1u)) {
          ok = false;
          break;
        }
        constexpr int kSl = TF32 ? kSlotBytesSp : kSlotBytes;
        mbar_expect_tx(&tfull[slot], kSl);
        bulk_load(ring + slot * kSl, src, kSl, &tfull[slot]);
        src += kSl / 2;
        if (++slot == kRing) {
          slot = 0;
          ph ^= 1u;
        }
      }
    }
    flags[2] = (int)G;
    if (!ok) flags[4] = 1;
  } else if (warp >= 4 && warp < 4 + kEpiWarps) {
    // ---- epilogue: warp w reads TMEM lane quarter w % 4; with 8 warps the
    // two of a quarter take alternate 16-column groups
    const int q = (warp - 4) & 3, half = (warp - 4) >> 2;
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
    // (plane s2, filter k, x pair); threads et < 30 kEpiGroups take piece
    // et % 30 of every kEpiGroups-th column, starting at column et / 30
    const int piece = et % 30, cgrp = et / 30;
    const int part = piece % 5, sk = piece / 5;
    const int s2 = sk / a.nfilt, k = sk - s2 * a.nfilt;
    const bool vec16 = ((a.W & 1) == 0) && ((V & 1) == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    int i = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int b, zt, yt, xc;
      decode_tile(a, act, t, b, zt, yt, xc);
      const int acc = i & 1;
      // one thread waits and tells the others, so that all of them leave
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
      if (TF32) {
        // each thread stores its row's outputs (filter f >> 1, re/im f & 1,
        // x0 + xo) column by column straight from the accumulator: a warp's
        // store covers 20 consecutive lanes = 80 contiguous bytes per filter
        const int xg = x0 + xo;
        const bool lane_ok = rvalid && xg < a.W;
        const int ylim = g.Ty < a.H - y0 ? g.Ty : a.H - y0;
        const int zrem = a.D - z0 - sp;
        const int jl0 = zrem > 0 ? (zrem + g.SP - 1) / g.SP : 0;
        const int jl = jl0 < g.J ? jl0 : g.J;
        float* obase = out + (((long long)b * a.nfilt + (rvalid ? (f >> 1) : 0)) * V + xg) * 2 + (f & 1);
        const long long ystep = 2ll * a.W, zwrap = 2ll * a.W * ((long long)g.SP * a.H - g.Hp);
        constexpr int kStep = 16 * (kEpiWarps / 4);
        bool arrived = false;
        for (int c0 = 16 * half; c0 < g.N; c0 += kStep) {
          uint32_t v[16];
          tmem_ld16(lanecol + (uint32_t)c0, v);
          if (c0 + kStep >= g.N) {
            // this thread's last read of the accumulator: the GEMMs of tile
            // i + 2 may start once every epilogue thread is here
            tc_fence_before();
            mbar_arrive(&acc_empty[acc]);
            arrived = true;
          }
          int j = c0 / g.Hp, yl = c0 - j * g.Hp;
          float* p = obase + ((long long)(z0 + j * g.SP + sp) * a.H + y0 + yl) * ystep;
#pragma unroll
          for (int e = 0; e < 16; e++) {
            if (lane_ok && j < jl && yl < ylim) *p = __uint_as_float(v[e]);
            p += ystep;
            if (++yl == g.Hp) {
              yl = 0;
              j++;
              p += zwrap;
            }
          }
        }
        if (!arrived) {
          tc_fence_before();
          mbar_arrive(&acc_empty[acc]);
        }
      } else {
        // BF16X3 (tensor-bound: the direct stores above slow its GEMMs):
        // chunks of kEpiCols columns transposed through shared memory
        // into 16-byte stores of ten complex samples
        for (int cbase = 0; cbase < g.N; cbase += kEpiCols) {
          const int cend = cbase + kEpiCols < g.N ? cbase + kEpiCols : g.N;
          for (int c0 = cbase + 16 * half; c0 < cend; c0 += 16 * (kEpiWarps / 4)) {
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
          if (et < 30 * kEpiGroups) {
            int nl = cgrp;
            int j = (cbase + nl) / g.Hp, yl = cbase + nl - j * g.Hp;
            const int xs = x0 + 2 * part;
            for (; nl < cend - cbase; nl += kEpiGroups) {
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
              yl += kEpiGroups;  // Hp >= 7 and kEpiGroups <= 12: at most two wraps
              if (yl >= g.Hp) {
                yl -= g.Hp;
                j++;
                if (yl >= g.Hp) {
                  yl -= g.Hp;
                  j++;
                }
              }
            }
          }
          epi_sync();
        }
      }
      i++;
    }
    if (!ok) flags[4] = 1;
  }

  __syncthreads();
  // a wait gave up somewhere: bounded drain of the tap copies no GEMM consumed
  if (tid == 64)
    for (int s = flags[3]; s < flags[2]; s++) mbar_wait(&tfull[s % kRing], (uint32_t)(s / kRing) & 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  if (tid == 0 && flags[4]) atomicExch(err, 1);
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

uint32_t metadata_word(int lane, int SP, int nfilt) { return sparse_metadata_word(lane, SP, nfilt); }

int stacked_planes(int nfilt) { return nfilt == 3 ? 2 : 1; }
int num_stages(int nfilt) { return (7 + stacked_planes(nfilt) - 1) * 7; }
size_t packed_tap_bytes(int nfilt, bool tf32) {
  (void)nfilt;
  return (size_t)kSlotsPerTile * (tf32 ? kSlotBytesSp : kSlotBytes);
}

static uint32_t tf32_rna_host(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return u & 0xffffe000u;  // inf / nan
  return (u + 0x1000u) & 0xffffe000u;  // nearest, ties away from zero
}

// Stage (input-plane offset c = cq - 3, dy = dyq - 3) goes to ring slot
// dyq * 4 + cq / 2, half cq % 2.  BF16X3: each half is hi (kM x 16 BF16)
// then lo, as two K-major 8-row x 16-byte core-matrix blocks.  TF32: each
// half is the structured-sparse A of the stage: the 16 K samples of a row
// pair up as (P, P + 8), P < 8, and a row's 7 taps (samples xo .. xo + 6)
// never hold both of a pair, so each row keeps one value per pair -- stored
// position P, two K-major blocks of kM x 4 TF32 -- and the MMA's metadata
// says which of the pair it is (sparse_metadata_word).  Halves without a
// stage (cq = 7 with one stacked plane) stay zero.
void pack_taps(const float* h_filters, int nfilt, uint16_t* dst, bool tf32) {
  const int SP = stacked_planes(nfilt);
  const int ncq = 6 + SP;
  memset(dst, 0, packed_tap_bytes(nfilt, tf32));
  for (int cq = 0; cq < ncq; cq++)
    for (int dyq = 0; dyq < 7; dyq++) {
      const int c = cq - 3, dy = dyq - 3;
      const size_t stage = (size_t)(dyq * 4 + cq / 2) * 2 + (cq & 1);
      uint16_t* hi = dst + stage * (tf32 ? kStageBytesSp / 2 : 2 * kStageHalves);
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
          if (tf32) {
            const uint32_t t = tf32_rna_host(w);
            const int P = kx & 7;  // pair (P, P + 8): stored position P
            const size_t e = (size_t)(P / 4) * (kM * 4) + (size_t)r * 4 + (P % 4);
            memcpy(hi + 2 * e, &t, 4);
          } else {
            const uint16_t wh = bf16_rn(w);
            const uint16_t wl = bf16_rn(w - bf16_to_f(wh));
            const size_t e = (size_t)(kx / 8) * (kM * 8) + (size_t)r * 8 + (kx % 8);
            hi[e] = wh;
            lo[e] = wl;
          }
        }
      }
    }
}

static int g_num_sms = 0;

// Dynamic shared memory of a geometry: tap ring, two input buffers (hi and
// lo, two K halves each), epilogue transpose buffer, barriers; at least
// 116 KB, so that one CTA (and its 512 TMEM columns) is alone on its SM.
static int smem_bytes(int NR) {
  const int need = kRing * kSlotBytes + 128 * NR + kEpiBytes + kBarBytes;
  return need > 116 * 1024 ? need : 116 * 1024;
}

Geometry make_geometry(int nfilt, int H, int D, int Ty, bool tf32) {
  Geometry g;
  g.maxN = tf32 ? kMaxNSparse : kMaxN;
  g.SP = stacked_planes(nfilt);
  g.Ty = Ty < H ? Ty : H;
  g.Hp = g.Ty + 6;
  g.J = g.maxN / g.Hp;
  if (g.J < 1) g.J = 1;
  // no more plane groups than the volume needs
  const int jmax = (D + g.SP - 1) / g.SP;
  if (g.J > jmax) g.J = jmax;
  g.N = ((g.J * g.Hp + 15) / 16) * 16;
  // rows a GEMM may read: start row up to (qmax Hp + 6), then N rows
  const int qmax = (5 + g.SP) / g.SP;  // largest plane-slot offset of a GEMM: (c+3)/SP, c <= 2+SP
  g.RP = ((qmax * g.Hp + 6 + g.N) + 7) / 8 * 8;
  g.NR = g.SP * g.RP;
  g.nstage = num_stages(nfilt);
  g.smem = smem_bytes(g.NR);
  return g;
}

bool geometry_ok(const Geometry& g) {
  return g.Hp <= g.maxN && g.N >= 16 && g.N <= g.maxN && g.smem <= 227 * 1024;
}

// Cost model of a tile shape: GEMM columns issued over the volume (tiles x
// N; a GEMM's time is proportional to N), plus 16 columns' worth per tile for
// its waits and commits.
static long long tile_cost(const Geometry& g, int H, int D) {
  const long long ny = (H + g.Ty - 1) / g.Ty;
  const long long nz = (D + g.SP * g.J - 1) / (g.SP * g.J);
  return ny * nz * (g.N + 16);
}

int candidate_tys(int nfilt, int H, int D, int* tys, int max_n, bool tf32) {
  // the cheapest tile height for each plane-group count J (ties to the
  // taller tile), then the max_n cheapest of those
  long long best_cost[kMaxN + 1];
  int best_ty[kMaxN + 1];
  for (int j = 0; j <= kMaxN; j++) best_ty[j] = -1;
  const int lo = H < 10 ? H : 10;
  const int maxN = tf32 ? kMaxNSparse : kMaxN;
  const int hi = H < maxN - 6 ? H : maxN - 6;
  for (int ty = hi; ty >= lo; ty--) {
    const Geometry g = make_geometry(nfilt, H, D, ty, tf32);
    if (!geometry_ok(g)) continue;
    const long long c = tile_cost(g, H, D);
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

int pick_ty(int nfilt, int H, int D, bool tf32) {
  int ty = -1;
  return candidate_tys(nfilt, H, D, &ty, 1, tf32) == 1 ? ty : -1;
}

cudaError_t bounded_wait_probe(int wait_ms, int* d_err, cudaStream_t st) {
  if (wait_ms < 1 || wait_ms > 1000) return cudaErrorInvalidValue;
  bounded_wait_probe_kernel<<<1, 32, 0, st>>>((unsigned long long)wait_ms * 1000000ull, d_err);
  return cudaGetLastError();
}

cudaError_t init() {
  cudaError_t e = cudaFuncSetAttribute(filter3d_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       227 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(filter3d_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e != cudaSuccess) return e;
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  return cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
}

cudaError_t launch(const float* vol, int W, int H, int D, int batch, long long stride, const uint16_t* d_taps,
                   int nfilt, float* out, ActiveSet act, int* d_err, const Geometry& g, cudaStream_t st, bool tf32) {
  if (g_num_sms <= 0) return cudaErrorInitializationError;
  if (!geometry_ok(g) || (nfilt != 3 && nfilt != 6) || g.SP != stacked_planes(nfilt) || batch <= 0 ||
      (tf32 && g.N > kMaxNSparse))
    return cudaErrorInvalidValue;
  TileArgs a;
  a.vstride = stride;
  a.W = W;
  a.H = H;
  a.D = D;
  a.nxc = (W + kXo - 1) / kXo;
  a.nyt = (H + g.Ty - 1) / g.Ty;
  a.nzt = (D + g.SP * g.J - 1) / (g.SP * g.J);
  a.nfilt = nfilt;
  a.batch = batch;
  const long long ntiles = (long long)a.nxc * a.nyt * a.nzt * batch;
  if (ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
  a.tiles_per = a.nxc * a.nyt * a.nzt;
  a.nqp = (g.SP * g.J + 6) / g.SP;
  a.in_off = (uint32_t)(kRing * kSlotBytes);
  a.e_off = a.in_off + 128u * (uint32_t)g.NR;
  a.bar_off = a.e_off + (uint32_t)kEpiBytes;
  const int grid = ntiles < g_num_sms ? (int)ntiles : g_num_sms;
  if (tf32)
    filter3d_tc_kernel<true><<<grid, kThreads, g.smem, st>>>(vol, d_taps, out, a, g, act, d_err);
  else
    filter3d_tc_kernel<false><<<grid, kThreads, g.smem, st>>>(vol, d_taps, out, a, g, act, d_err);
  return cudaGetLastError();
}

}  // namespace tc
}  // namespace brc
