// filter3d.cu -- 7x7x7 complex quadrature filtering, FP32 on the CUDA cores.
//
// One CTA computes a 32 (x) x 8 (y) x TZ (z) block of outputs for all NF
// complex filters of one volume of the batch.  The input block with its
// +-3 halo is staged in shared memory once (zero padding outside the
// volume, rows padded to 44 floats so that the 16-byte row loads of a
// quarter-warp hit distinct banks); the tap-major filter bank is staged in
// shared memory from the kernel parameters.  Each thread owns a run of R
// consecutive x outputs and keeps 2*NF*R accumulators in registers: per
// (dz,dy) it loads one row segment of R+6 samples with 16-byte loads, then
// for each of the 7 dx taps it loads the 2*NF coefficients (a broadcast)
// and issues 2*NF*R FMAs.  FMAs per shared-memory load is ~40, so the
// kernel is bound by the FP32 pipe.
//
// Algorithm (what is computed, not how): NonseparableConvolution3D,
// broccoli_lib.cpp:4974-5027, with the 2D passes of
// kernelConvolution.cpp:2802-3693.
#include <type_traits>

#include "common.cuh"

namespace brc {

constexpr int kTX = 32;   // outputs per CTA along x
constexpr int kTY = 8;    // outputs per CTA along y
constexpr int kRowPad = 44;  // shared row length (38 used)

template <int NF, int R, int TZ>
struct Filter3dCfg {
  static constexpr int kThreadsX = kTX / R;
  static constexpr int kThreads = kThreadsX * kTY * TZ;
  static constexpr int kCP = (2 * NF + 3) / 4 * 4;  // coefficient stride per tap
  static constexpr int kSlices = TZ + 6;
  static constexpr int kRows = kTY + 6;
  static constexpr int kVolFloats = kSlices * kRows * kRowPad;
  static constexpr int kCoefFloats = kTaps * kCP;
  static constexpr size_t kSmemBytes = sizeof(float) * (kVolFloats + kCoefFloats);
};

template <int NF, int R, int TZ>
__global__ void __launch_bounds__(Filter3dCfg<NF, R, TZ>::kThreads)
filter3d_fp32_kernel(const float* __restrict__ vol, int W, int H, int D, long long vol_stride,
                     const __grid_constant__ FilterBank<NF> bank, float* __restrict__ out,
                     const ActiveSet act) {
  using Cfg = Filter3dCfg<NF, R, TZ>;
  extern __shared__ __align__(16) float smem[];
  float* s_vol = smem;
  float* s_coef = smem + Cfg::kVolFloats;

  if ((int)blockIdx.z >= active_count(act, (int)gridDim.z)) return;
  const int b = active_instance(act, blockIdx.z);
  const int z_tiles = (D + TZ - 1) / TZ;
  const int tile_x0 = blockIdx.x * kTX;
  const int tile_y0 = (blockIdx.y / z_tiles) * kTY;
  const int tile_z0 = (blockIdx.y % z_tiles) * TZ;
  const float* src = vol + (long long)b * vol_stride;
  const long long V = (long long)W * H * D;

  // Stage the coefficients: tap-major, 2*NF values per tap, padded to kCP.
  for (int i = threadIdx.x; i < kTaps * Cfg::kCP; i += Cfg::kThreads) {
    const int t = i / Cfg::kCP, c = i % Cfg::kCP;
    s_coef[i] = c < 2 * NF ? bank.coef[t * 2 * NF + c] : 0.f;
  }
  // Stage the input block: x from tile_x0-4 (16-byte aligned in shared
  // memory), y from tile_y0-3, z from tile_z0-3; zero outside the volume.
  for (int i = threadIdx.x; i < Cfg::kVolFloats; i += Cfg::kThreads) {
    const int xs = i % kRowPad;
    const int ys = (i / kRowPad) % Cfg::kRows;
    const int zs = i / (kRowPad * Cfg::kRows);
    const int x = tile_x0 - 4 + xs, y = tile_y0 - 3 + ys, z = tile_z0 - 3 + zs;
    float v = 0.f;
    if (x >= 0 && x < W && y >= 0 && y < H && z >= 0 && z < D)
      v = __ldg(src + x + (long long)y * W + (long long)z * W * H);
    s_vol[i] = v;
  }
  __syncthreads();

  const int tx = threadIdx.x % Cfg::kThreadsX;
  const int ty = (threadIdx.x / Cfg::kThreadsX) % kTY;
  const int tz = threadIdx.x / (Cfg::kThreadsX * kTY);

  float acc[2 * NF][R];
#pragma unroll
  for (int f = 0; f < 2 * NF; f++)
#pragma unroll
    for (int r = 0; r < R; r++) acc[f][r] = 0.f;

  constexpr int kSeg = (R + 8) / 4;  // float4 loads per row segment
  // Runtime loops over the 49 (dz, dy) rows keep the loop body (7 dx taps x
  // 2*NF*R FMAs) small enough for the instruction cache.
#pragma unroll 1
  for (int dz = 0; dz < 7; dz++) {
#pragma unroll 1
    for (int dy = 0; dy < 7; dy++) {
      const float4* row = reinterpret_cast<const float4*>(
          s_vol + ((tz + dz) * Cfg::kRows + (ty + dy)) * kRowPad + R * tx);
      float d[4 * kSeg];
#pragma unroll
      for (int s = 0; s < kSeg; s++) {
        const float4 q = row[s];
        d[4 * s] = q.x;
        d[4 * s + 1] = q.y;
        d[4 * s + 2] = q.z;
        d[4 * s + 3] = q.w;
      }
      const float* ct = s_coef + (dz * 49 + dy * 7) * Cfg::kCP;
#pragma unroll
      for (int dx = 0; dx < 7; dx++) {
        float c[Cfg::kCP];
#pragma unroll
        for (int s = 0; s < Cfg::kCP / 4; s++) {
          const float4 q = reinterpret_cast<const float4*>(ct + dx * Cfg::kCP)[s];
          c[4 * s] = q.x;
          c[4 * s + 1] = q.y;
          c[4 * s + 2] = q.z;
          c[4 * s + 3] = q.w;
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
          const float px = d[1 + r + dx];
#pragma unroll
          for (int f = 0; f < 2 * NF; f++) acc[f][r] = fmaf(px, c[f], acc[f][r]);
        }
      }
    }
  }

  const int x0 = tile_x0 + R * tx;
  const int y = tile_y0 + ty;
  const int z = tile_z0 + tz;
  if (y >= H || z >= D || x0 >= W) return;
  const long long idx0 = x0 + (long long)y * W + (long long)z * W * H;
  float* o = out + (long long)b * NF * 2 * V;
  const bool full = x0 + R <= W;
#pragma unroll
  for (int k = 0; k < NF; k++) {
    float* ok = o + (long long)k * 2 * V + 2 * idx0;
    if (full && (reinterpret_cast<uintptr_t>(ok) & 15) == 0) {
#pragma unroll
      for (int r = 0; r < R; r += 2)
        reinterpret_cast<float4*>(ok)[r / 2] =
            make_float4(acc[2 * k][r], acc[2 * k + 1][r], acc[2 * k][r + 1], acc[2 * k + 1][r + 1]);
    } else {
#pragma unroll
      for (int r = 0; r < R; r++)
        if (x0 + r < W) {
          ok[2 * r] = acc[2 * k][r];
          ok[2 * r + 1] = acc[2 * k + 1][r];
        }
    }
  }
}

// ---------------------------------------------------------------------------
// Even/odd variant.  Quadrature filters have an even real part and an odd
// imaginary part (W(-d) = conj W(d) for the tap weights W(d) of offset d),
// so the responses need only half the taps:
//   q_re(x) = W_re(0) V(x) + sum_{d in half} W_re(d) (V(x+d) + V(x-d))
//   q_im(x) =                sum_{d in half} W_im(d) (V(x+d) - V(x-d))
// The host checks the symmetry of the bank (to 1e-6 of its largest tap; the
// shipped and the lognormal filters are symmetric to 1e-7) and passes the
// symmetrised weights; other banks take the general kernel.  Rows pair up
// as (dy, dz) with (-dy, -dz): 24 row pairs plus the centre row, whose dx
// taps pair within the row.  Per pair and output: one add, one subtract and
// 2*NF FMAs instead of 4*NF FMAs.
// ---------------------------------------------------------------------------

// Symmetrised bank: pair p in [0, 24) (rows (dy,dz) of the positive half,
// offsets in -3..3), dx in -3..3, 2*NF weights (re0, im0, re1, ...); then
// the centre row, dx in 0..3 (dx = 0 uses re only).
template <int NF>
struct SymBank {
  float coef[(24 * 7 + 4) * 2 * NF];
};

template <int NF, int R, int TZ>
__global__ void __launch_bounds__(Filter3dCfg<NF, R, TZ>::kThreads)
filter3d_sym_kernel(const float* __restrict__ vol, int W, int H, int D, long long vol_stride,
                    const __grid_constant__ SymBank<NF> bank, float* __restrict__ out,
                    const ActiveSet act) {
  using Cfg = Filter3dCfg<NF, R, TZ>;
  constexpr int kTapsSym = 24 * 7 + 4;
  extern __shared__ __align__(16) float smem[];
  float* s_vol = smem;
  float* s_coef = smem + Cfg::kVolFloats;  // kTapsSym x kCP

  if ((int)blockIdx.z >= active_count(act, (int)gridDim.z)) return;
  const int b = active_instance(act, blockIdx.z);
  const int z_tiles = (D + TZ - 1) / TZ;
  const int tile_x0 = blockIdx.x * kTX;
  const int tile_y0 = (blockIdx.y / z_tiles) * kTY;
  const int tile_z0 = (blockIdx.y % z_tiles) * TZ;
  const float* src = vol + (long long)b * vol_stride;
  const long long V = (long long)W * H * D;

  for (int i = threadIdx.x; i < kTapsSym * Cfg::kCP; i += Cfg::kThreads) {
    const int t = i / Cfg::kCP, c = i % Cfg::kCP;
    s_coef[i] = c < 2 * NF ? bank.coef[t * 2 * NF + c] : 0.f;
  }
  for (int i = threadIdx.x; i < Cfg::kVolFloats; i += Cfg::kThreads) {
    const int xs = i % kRowPad;
    const int ys = (i / kRowPad) % Cfg::kRows;
    const int zs = i / (kRowPad * Cfg::kRows);
    const int x = tile_x0 - 4 + xs, y = tile_y0 - 3 + ys, z = tile_z0 - 3 + zs;
    float v = 0.f;
    if (x >= 0 && x < W && y >= 0 && y < H && z >= 0 && z < D)
      v = __ldg(src + x + (long long)y * W + (long long)z * W * H);
    s_vol[i] = v;
  }
  __syncthreads();

  const int tx = threadIdx.x % Cfg::kThreadsX;
  const int ty = (threadIdx.x / Cfg::kThreadsX) % kTY;
  const int tz = threadIdx.x / (Cfg::kThreadsX * kTY);

  float acc[2 * NF][R];
#pragma unroll
  for (int f = 0; f < 2 * NF; f++)
#pragma unroll
    for (int r = 0; r < R; r++) acc[f][r] = 0.f;

  constexpr int kSeg = (R + 8) / 4;
  auto load_row = [&](int dy, int dz, float* d) {
    const float4* row = reinterpret_cast<const float4*>(
        s_vol + ((tz + 3 + dz) * Cfg::kRows + (ty + 3 + dy)) * kRowPad + R * tx);
#pragma unroll
    for (int s = 0; s < kSeg; s++) {
      const float4 q = row[s];
      d[4 * s] = q.x;
      d[4 * s + 1] = q.y;
      d[4 * s + 2] = q.z;
      d[4 * s + 3] = q.w;
    }
  };
  // sample at offset dx (-3..3) of output r sits at d[4 + r + dx]
#pragma unroll 1
  for (int p = 0; p < 24; p++) {
    // positive half of the (dy, dz) rows: dz = 1..3 (all dy), then dz = 0, dy = 1..3
    const int dz = p < 21 ? 1 + p / 7 : 0;
    const int dy = p < 21 ? p % 7 - 3 : p - 20;
    float da[4 * kSeg], db[4 * kSeg];
    load_row(dy, dz, da);
    load_row(-dy, -dz, db);
    const float* ct = s_coef + p * 7 * Cfg::kCP;
#pragma unroll
    for (int j = 0; j < 7; j++) {
      const int dx = j - 3;
      float c[Cfg::kCP];
#pragma unroll
      for (int s = 0; s < Cfg::kCP / 4; s++) {
        const float4 q = reinterpret_cast<const float4*>(ct + j * Cfg::kCP)[s];
        c[4 * s] = q.x;
        c[4 * s + 1] = q.y;
        c[4 * s + 2] = q.z;
        c[4 * s + 3] = q.w;
      }
#pragma unroll
      for (int r = 0; r < R; r++) {
        const float a = da[4 + r + dx], bb = db[4 + r - dx];
        const float sp = a + bb, sm = a - bb;
#pragma unroll
        for (int k = 0; k < NF; k++) {
          acc[2 * k][r] = fmaf(sp, c[2 * k], acc[2 * k][r]);
          acc[2 * k + 1][r] = fmaf(sm, c[2 * k + 1], acc[2 * k + 1][r]);
        }
      }
    }
  }
  {  // centre row: dx pairs within the row, and the centre tap (real only)
    float d0[4 * kSeg];
    load_row(0, 0, d0);
    const float* ct = s_coef + 24 * 7 * Cfg::kCP;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      float c[Cfg::kCP];
#pragma unroll
      for (int s = 0; s < Cfg::kCP / 4; s++) {
        const float4 q = reinterpret_cast<const float4*>(ct + j * Cfg::kCP)[s];
        c[4 * s] = q.x;
        c[4 * s + 1] = q.y;
        c[4 * s + 2] = q.z;
        c[4 * s + 3] = q.w;
      }
#pragma unroll
      for (int r = 0; r < R; r++) {
        if (j == 0) {
#pragma unroll
          for (int k = 0; k < NF; k++) acc[2 * k][r] = fmaf(d0[4 + r], c[2 * k], acc[2 * k][r]);
        } else {
          const float a = d0[4 + r + j], bb = d0[4 + r - j];
          const float sp = a + bb, sm = a - bb;
#pragma unroll
          for (int k = 0; k < NF; k++) {
            acc[2 * k][r] = fmaf(sp, c[2 * k], acc[2 * k][r]);
            acc[2 * k + 1][r] = fmaf(sm, c[2 * k + 1], acc[2 * k + 1][r]);
          }
        }
      }
    }
  }

  const int x0 = tile_x0 + R * tx;
  const int y = tile_y0 + ty;
  const int z = tile_z0 + tz;
  if (y >= H || z >= D || x0 >= W) return;
  const long long idx0 = x0 + (long long)y * W + (long long)z * W * H;
  float* o = out + (long long)b * NF * 2 * V;
  const bool full = x0 + R <= W;
#pragma unroll
  for (int k = 0; k < NF; k++) {
    float* ok = o + (long long)k * 2 * V + 2 * idx0;
    if (full && (reinterpret_cast<uintptr_t>(ok) & 15) == 0) {
#pragma unroll
      for (int r = 0; r < R; r += 2)
        reinterpret_cast<float4*>(ok)[r / 2] =
            make_float4(acc[2 * k][r], acc[2 * k + 1][r], acc[2 * k][r + 1], acc[2 * k + 1][r + 1]);
    } else {
#pragma unroll
      for (int r = 0; r < R; r++)
        if (x0 + r < W) {
          ok[2 * r] = acc[2 * k][r];
          ok[2 * r + 1] = acc[2 * k + 1][r];
        }
    }
  }
}

// Tap weight of filter k, component c (0 re, 1 im) at offset (dx,dy,dz):
// the reference convolves, so the weight of offset d is F[3-d]
// (kernelConvolution.cpp:2840-2858).
static inline float tap_weight(const float* h_filters, int k, int c, int dx, int dy, int dz) {
  return h_filters[k * kFilterFloats + c * kTaps + (3 - dx) + 7 * (3 - dy) + 49 * (3 - dz)];
}

// True (and the symmetrised bank) when every filter of the bank has an even
// real and odd imaginary part to 1e-6 of its largest tap.
template <int NF>
static bool pack_sym_bank(const float* h_filters, SymBank<NF>& bank) {
  for (int k = 0; k < NF; k++) {
    float mx = 0.f;
    for (int i = 0; i < kFilterFloats; i++) mx = fmaxf(mx, fabsf(h_filters[k * kFilterFloats + i]));
    const float tol = 1e-6f * mx;
    for (int dz = -3; dz <= 3; dz++)
      for (int dy = -3; dy <= 3; dy++)
        for (int dx = -3; dx <= 3; dx++) {
          const float re = tap_weight(h_filters, k, 0, dx, dy, dz);
          const float rm = tap_weight(h_filters, k, 0, -dx, -dy, -dz);
          const float im = tap_weight(h_filters, k, 1, dx, dy, dz);
          const float imm = tap_weight(h_filters, k, 1, -dx, -dy, -dz);
          if (fabsf(re - rm) > tol || fabsf(im + imm) > tol) return false;
        }
  }
  auto put = [&](int slot, int dx, int dy, int dz) {
    for (int k = 0; k < NF; k++) {
      const float re = 0.5f * (tap_weight(h_filters, k, 0, dx, dy, dz) + tap_weight(h_filters, k, 0, -dx, -dy, -dz));
      const float im = 0.5f * (tap_weight(h_filters, k, 1, dx, dy, dz) - tap_weight(h_filters, k, 1, -dx, -dy, -dz));
      bank.coef[slot * 2 * NF + 2 * k] = re;
      bank.coef[slot * 2 * NF + 2 * k + 1] = im;
    }
  };
  for (int p = 0; p < 24; p++) {
    const int dz = p < 21 ? 1 + p / 7 : 0;
    const int dy = p < 21 ? p % 7 - 3 : p - 20;
    for (int j = 0; j < 7; j++) put(p * 7 + j, j - 3, dy, dz);
  }
  for (int j = 0; j < 4; j++) put(24 * 7 + j, j, 0, 0);
  for (int k = 0; k < NF; k++) bank.coef[24 * 7 * 2 * NF + 2 * k + 1] = 0.f;  // centre: real only
  return true;
}

template <int NF>
static void pack_bank(const float* h_filters, FilterBank<NF>& bank) {
  for (int t = 0; t < kTaps; t++) {
    const int dx = t % 7, dy = (t / 7) % 7, dz = t / 49;
    const int src = (6 - dx) + 7 * (6 - dy) + 49 * (6 - dz);
    for (int k = 0; k < NF; k++) {
      bank.coef[t * 2 * NF + 2 * k] = h_filters[k * kFilterFloats + src];
      bank.coef[t * 2 * NF + 2 * k + 1] = h_filters[k * kFilterFloats + kTaps + src];
    }
  }
}

template <int NF, int R, int TZ>
static cudaError_t launch_fp32(const float* vol, int W, int H, int D, int batch, long long stride,
                               const FilterBank<NF>& bank, float* out, ActiveSet act,
                               cudaStream_t st) {
  using Cfg = Filter3dCfg<NF, R, TZ>;
  const int z_tiles = (D + TZ - 1) / TZ;
  dim3 grid((W + kTX - 1) / kTX, ((H + kTY - 1) / kTY) * z_tiles, batch);
  filter3d_fp32_kernel<NF, R, TZ><<<grid, Cfg::kThreads, Cfg::kSmemBytes, st>>>(
      vol, W, H, D, stride, bank, out, act);
  return cudaGetLastError();
}

template <int NF, int R, int TZ>
static cudaError_t launch_sym(const float* vol, int W, int H, int D, int batch, long long stride,
                              const SymBank<NF>& bank, float* out, ActiveSet act,
                              cudaStream_t st) {
  using Cfg = Filter3dCfg<NF, R, TZ>;
  const int z_tiles = (D + TZ - 1) / TZ;
  dim3 grid((W + kTX - 1) / kTX, ((H + kTY - 1) / kTY) * z_tiles, batch);
  filter3d_sym_kernel<NF, R, TZ><<<grid, Cfg::kThreads, Cfg::kSmemBytes, st>>>(
      vol, W, H, D, stride, bank, out, act);
  return cudaGetLastError();
}

template <int NF, int R, int TZ>
static cudaError_t set_smem_attr() {
  cudaError_t e = cudaFuncSetAttribute(filter3d_fp32_kernel<NF, R, TZ>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)Filter3dCfg<NF, R, TZ>::kSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(filter3d_sym_kernel<NF, R, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Filter3dCfg<NF, R, TZ>::kSmemBytes);
}

// z depths of the output block the kernels are instantiated for; the
// context's tuner times them per volume shape (pick_tz is the untimed
// choice).
constexpr int kTzCandidates[] = {2, 3, 4, 6, 8};

// Raises the dynamic shared-memory limit of every instantiation; called
// once per device when a context is created.
cudaError_t filter3d_init() {
  cudaError_t e;
#define BRC_TZ_ATTR(TZ)                                                \
  if ((e = set_smem_attr<3, 8, TZ>()) != cudaSuccess) return e;        \
  if ((e = set_smem_attr<6, 4, TZ>()) != cudaSuccess) return e;
  BRC_TZ_ATTR(2)
  BRC_TZ_ATTR(3)
  BRC_TZ_ATTR(4)
  BRC_TZ_ATTR(6)
  BRC_TZ_ATTR(8)
#undef BRC_TZ_ATTR
  return cudaSuccess;
}

// Chooses the z depth of the tile without timing: 3 when it divides D
// exactly and 4 does not (e.g. D = 33), else 4.
static int pick_tz(int D) { return (D % 4 != 0 && D % 3 == 0) ? 3 : 4; }

int filter3d_tz_candidates(int* tz, int max_n) {
  const int n = (int)(sizeof(kTzCandidates) / sizeof(kTzCandidates[0]));
  for (int i = 0; i < n && i < max_n; i++) tz[i] = kTzCandidates[i];
  return n < max_n ? n : max_n;
}

int filter3d_default_tz(int D) { return pick_tz(D); }

bool filter3d_bank_symmetric(const float* h_filters, int nfilt) {
  if (nfilt == 3) {
    SymBank<3> sb;
    return pack_sym_bank<3>(h_filters, sb);
  }
  if (nfilt == 6) {
    SymBank<6> sb;
    return pack_sym_bank<6>(h_filters, sb);
  }
  return false;
}

template <typename Launch>
static cudaError_t dispatch_tz(int tz, Launch launch) {
  switch (tz) {
    case 2: return launch(std::integral_constant<int, 2>());
    case 3: return launch(std::integral_constant<int, 3>());
    case 4: return launch(std::integral_constant<int, 4>());
    case 6: return launch(std::integral_constant<int, 6>());
    case 8: return launch(std::integral_constant<int, 8>());
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t filter3d_fp32(const float* vol, int W, int H, int D, int batch, long long stride,
                          const float* h_filters, int nfilt, float* out, ActiveSet act, cudaStream_t st,
                          bool allow_symmetric, int tz) {
  if (tz <= 0) tz = pick_tz(D);
  if (allow_symmetric && nfilt == 3) {
    SymBank<3> sb;
    if (pack_sym_bank<3>(h_filters, sb))
      return dispatch_tz(tz, [&](auto T) {
        return launch_sym<3, 8, decltype(T)::value>(vol, W, H, D, batch, stride, sb, out, act, st);
      });
  }
  if (allow_symmetric && nfilt == 6) {
    SymBank<6> sb;
    if (pack_sym_bank<6>(h_filters, sb))
      return dispatch_tz(tz, [&](auto T) {
        return launch_sym<6, 4, decltype(T)::value>(vol, W, H, D, batch, stride, sb, out, act, st);
      });
  }
  if (nfilt == 3) {
    FilterBank<3> bank;
    pack_bank<3>(h_filters, bank);
    return dispatch_tz(tz, [&](auto T) {
      return launch_fp32<3, 8, decltype(T)::value>(vol, W, H, D, batch, stride, bank, out, act, st);
    });
  }
  if (nfilt == 6) {
    FilterBank<6> bank;
    pack_bank<6>(h_filters, bank);
    return dispatch_tz(tz, [&](auto T) {
      return launch_fp32<6, 4, decltype(T)::value>(vol, W, H, D, batch, stride, bank, out, act, st);
    });
  }
  return cudaErrorInvalidValue;
}

}  // namespace brc
