// registration.cu -- the per-iteration kernels of batched linear registration
// and the volume helpers around it (warps, separable smoothing, rescale).
//
// Per affine iteration and instance:
//   normal_eq_partial_kernel  phase difference, certainty and phase gradient
//                             of the three filter pairs, reduced to the 42
//                             distinct sums of the 12x12 system (FP64).
//   solve_update_kernel       reduces the partial sums in a fixed order,
//                             solves the three decoupled 4x4 systems in FP64,
//                             applies the TRANSLATION / RIGID / AFFINE update
//                             and the convergence test.
//   warp_affine_kernel        exact-weight trilinear resampling of the
//                             original volume with the total parameters.
#include <math.h>

#include <type_traits>

#include "common.cuh"
#include "internal.h"

namespace brc {

// ---------------------------------------------------------------------------
// Normal equations
// ---------------------------------------------------------------------------

constexpr int kNEThreads = 256;
// Largest volume the 32-bit voxel indexing of the resampling kernels takes.
constexpr long long kMaxVoxels = 0x7fffff00LL;

// Phase difference and certainty of one response pair
// (CalculatePhaseDifferencesAndCertainties, kernelRegistration.cpp:173-211):
// dphi = arg(q1 q2*), c = |q1 q2| cos^2(dphi/2).  With cos^2(t/2) =
// (1 + cos t)/2 and cos dphi = Re(q1 q2*)/|q1 q2*|, c = (|q1 q2*| + Re(q1 q2*))/2:
// the same value without the cosine (|q1 q2| = |q1 q2*|).
__device__ __forceinline__ void phase_diff_cert(float2 a, float2 c, float& pd, float& cert) {
  // products rounded separately (no FMA contraction), as in the reference's
  // arithmetic: identical responses then give exactly zero phase difference
  const float re = __fadd_rn(__fmul_rn(a.x, c.x), __fmul_rn(a.y, c.y));
  const float im = __fsub_rn(__fmul_rn(a.y, c.x), __fmul_rn(a.x, c.y));
  pd = phase_atan2(im, re);
  cert = 0.5f * (sqrt_approx(re * re + im * im) + re);
}

// Phase gradient from the neighbours along one axis
// (CalculatePhaseGradientsX/Y/Z, kernelRegistration.cpp:213-382).
__device__ __forceinline__ float phase_grad(float2 a_p, float2 a_c, float2 a_m, float2 c_p,
                                            float2 c_c, float2 c_m) {
  float tr = 0.f, ti = 0.f;
  tr += a_p.x * a_c.x + a_p.y * a_c.y;
  ti += a_p.y * a_c.x - a_p.x * a_c.y;
  tr += a_c.x * a_m.x + a_c.y * a_m.y;
  ti += a_c.y * a_m.x - a_c.x * a_m.y;
  tr += c_p.x * c_c.x + c_p.y * c_c.y;
  ti += c_p.y * c_c.x - c_p.x * c_c.y;
  tr += c_c.x * c_m.x + c_c.y * c_m.y;
  ti += c_c.y * c_m.x - c_c.x * c_m.y;
  return phase_atan2(ti, tr);
}

// Sum e (0..13) of one axis as (row moment) x y^py x z^pz: moments
// [sum w, sum w x, sum w x^2, sum v, sum v x] of the row, y and z relative
// to the volume centre.
__constant__ signed char c_sum_moment[14] = {0, 1, 0, 0, 2, 1, 1, 0, 0, 0, 3, 4, 3, 3};
__constant__ signed char c_sum_ypow[14] = {0, 0, 1, 0, 0, 1, 0, 2, 1, 0, 0, 0, 1, 0};
__constant__ signed char c_sum_zpow[14] = {0, 0, 0, 1, 0, 0, 1, 0, 1, 2, 0, 0, 0, 1};

__device__ __forceinline__ double pick_moment(const float (&m)[3][5], int sel) {
  float r = 0.f;
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int q = 0; q < 5; q++) r = (sel == 5 * k + q) ? m[k][q] : r;
  return (double)r;
}
__device__ __forceinline__ double ypow(double y, int e) {
  const int p = c_sum_ypow[e];
  return p == 0 ? 1.0 : (p == 1 ? y : y * y);
}
__device__ __forceinline__ double zpow(double z, int e) {
  const int p = c_sum_zpow[e];
  return p == 0 ? 1.0 : (p == 1 ? z : z * z);
}

// Sums over the interior (3 voxels from every face) of
//   c g^2 [1, x, y, z, xx, xy, xz, yy, yz, zz]  and  c g dphi [1, x, y, z]
// for each axis k (sum index 14k + e), coordinates relative to the volume
// centre: the 30 + 12 values that CalculateAMatrixAndHVector2DValuesX/Y/Z,
// CalculateAMatrix1DValues / HVector1DValues and CalculateAMatrix /
// HVector accumulate (kernelRegistration.cpp:387-800).  One CTA handles
// `zpb` interior slices of one instance and writes 42 FP64 partial sums.
//
// One warp walks one (y, z) row at a time, lanes along x (coalesced float2
// loads).  Within a row y and z are constant, so the 42 sums factor into 15
// row moments per lane, sum_x w [1, x, x^2] and sum_x v [1, x] for the three
// axes, reduced over the warp in FP32 and expanded into the 42 sums in FP64
// (lane j owns sums j and 32 + j).  The same order on every run: results
// are deterministic.
__global__ void __launch_bounds__(kNEThreads, 4)
normal_eq_partial_kernel(const float2* __restrict__ q1, long long q1_stride,
                         const float2* __restrict__ q2, int W, int H, int D, int zpb,
                         double* __restrict__ partials) {
  const int b = blockIdx.y;
  const long long V = (long long)W * H * D;
  const long long WH = (long long)W * H;
  const float2* Q1 = q1 + (long long)b * q1_stride;
  const float2* Q2 = q2 + (long long)b * 3 * V;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  const int nx = W - 6, ny = H - 6;
  const int z0 = 3 + blockIdx.x * zpb;
  const int z1 = min(D - 3, z0 + zpb);
  const int nrows = (nx > 0 && ny > 0 && z1 > z0) ? ny * (z1 - z0) : 0;
  const float cxf = 0.5f * (float)(W - 1);
  const double cy = 0.5 * (H - 1), cz = 0.5 * (D - 1);

  // lane j accumulates sums j and 32 + j (the latter for j < 10)
  double acc_lo = 0.0, acc_hi = 0.0;
  const int jlo = lane, jhi = 32 + lane;
  const int elo = jlo % 14, ehi = jhi % 14;
  const int slo = 5 * (jlo / 14) + c_sum_moment[elo];
  const int shi = jhi < kNSums ? 5 * (jhi / 14) + c_sum_moment[ehi] : 0;

  for (int r = warp; r < nrows; r += kNEThreads / 32) {
    const int y = 3 + r % ny;
    const int z = z0 + r / ny;
    const long long row = (long long)y * W + (long long)z * WH;
    // [k][0..4] = sum w, sum w x, sum w x^2, sum v, sum v x
    float m[3][5];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int q = 0; q < 5; q++) m[k][q] = 0.f;
    // all lanes run every chunk (shuffles need the full warp); lanes past
    // the interior load their clamped centre for their neighbours' use and
    // add nothing
    for (int xb = 3; xb < W - 3; xb += 32) {
      const int x = xb + lane;
      const bool act = x < W - 3;
      const long long i = row + (x < W ? x : W - 1);
      const float xf = (float)x - cxf;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const float2* A = Q1 + k * V;
        const float2* C = Q2 + k * V;
        const float2 a = __ldg(A + i), c = __ldg(C + i);
        float2 ap, am, cp, cm;
        if (k == 0) {
          // x neighbours from the adjacent lanes; the warp's end lanes load
          ap = make_float2(__shfl_down_sync(0xffffffffu, a.x, 1), __shfl_down_sync(0xffffffffu, a.y, 1));
          cp = make_float2(__shfl_down_sync(0xffffffffu, c.x, 1), __shfl_down_sync(0xffffffffu, c.y, 1));
          am = make_float2(__shfl_up_sync(0xffffffffu, a.x, 1), __shfl_up_sync(0xffffffffu, a.y, 1));
          cm = make_float2(__shfl_up_sync(0xffffffffu, c.x, 1), __shfl_up_sync(0xffffffffu, c.y, 1));
          if (lane == 31 && act) {
            ap = __ldg(A + i + 1);
            cp = __ldg(C + i + 1);
          }
          if (lane == 0) {
            am = __ldg(A + i - 1);
            cm = __ldg(C + i - 1);
          }
        } else {
          const long long st = k == 1 ? (long long)W : WH;
          ap = act ? __ldg(A + i + st) : a;
          am = act ? __ldg(A + i - st) : a;
          cp = act ? __ldg(C + i + st) : c;
          cm = act ? __ldg(C + i - st) : c;
        }
        float pd, cert;
        phase_diff_cert(a, c, pd, cert);
        const float g = phase_grad(ap, a, am, cp, c, cm);
        const float cg = act ? cert * g : 0.f;
        const float w = cg * g;
        const float v = cg * pd;
        m[k][0] += w;
        m[k][1] += w * xf;
        m[k][2] += w * xf * xf;
        m[k][3] += v;
        m[k][4] += v * xf;
      }
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int q = 0; q < 5; q++) {
        float t = m[k][q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        m[k][q] = t;
      }
    const double yf = (double)y - cy, zf = (double)z - cz;
    acc_lo += pick_moment(m, slo) * ypow(yf, elo) * zpow(zf, elo);
    if (jhi < kNSums) acc_hi += pick_moment(m, shi) * ypow(yf, ehi) * zpow(zf, ehi);
  }

  // Deterministic block reduction: warps in order.
  __shared__ double s_part[kNEThreads / 32][kNSums];
  s_part[warp][jlo] = acc_lo;
  if (jhi < kNSums) s_part[warp][jhi] = acc_hi;
  __syncthreads();
  if (threadIdx.x < kNSums) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kNEThreads / 32; w++) v += s_part[w][threadIdx.x];
    partials[((long long)b * gridDim.x + blockIdx.x) * kNSums + threadIdx.x] = v;
  }
}

// ---------------------------------------------------------------------------
// Normal equations, z-marching form: certainty smoothing fused in.
//
// One CTA of 10 warps x 32 lanes covers a patch of 30 x 8 interior voxels
// (x, y) with a one-voxel halo (lanes 0 and 31, warps 0 and 9) and walks a
// slab of interior planes z0..z1-1, reading each plane's responses once:
//   * certainties of a plane are smoothed along x by shuffles, along y
//     through shared memory and along z through a three-plane window kept
//     in shared memory (the separable 3x3x3 Gaussian in the order x, y, z);
//   * phase-gradient neighbours come from the adjacent lanes (x), from the
//     shared-memory copy of the axis-1 responses of the adjacent warps (y)
//     and from the previous / next plane held in registers (z);
//   * each lane accumulates, over the planes, the FP32 moments
//     sum w [1, z, z^2] and sum v [1, z] of its (x, y) column per axis and
//     expands them once into the 42 FP64 sums with its x and y.
// The next plane's responses are loaded while the current plane's sums are
// computed.  Without smoothing, the same sums as normal_eq_partial_kernel
// up to FP32 summation order.
// ---------------------------------------------------------------------------

constexpr int kMarchWarps = 10;              // 8 output rows + 2 halo rows
constexpr int kMarchCols = 30;               // output columns per warp
constexpr int kMarchZs = 32;                 // at most this many planes per slab (16: 1 % slower)

struct PlaneQ {
  float2 a[3], c[3];  // q1, q2 of the three filters at this lane's (x, y)
};

__device__ __forceinline__ void load_plane_q(const float2* __restrict__ Q1, const float2* __restrict__ Q2,
                                             long long V, long long i, bool in, PlaneQ& q) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    q.a[k] = in ? __ldg(Q1 + k * V + i) : make_float2(0.f, 0.f);
    q.c[k] = in ? __ldg(Q2 + k * V + i) : make_float2(0.f, 0.f);
  }
}

template <bool SMOOTH>
__global__ void __launch_bounds__(kMarchWarps * 32, 2)
normal_eq_march_kernel(const float2* __restrict__ q1, long long q1_stride, const float2* __restrict__ q2, int W,
                       int H, int D, int ntx, int nty, int zs, double* __restrict__ partials,
                       const ActiveSet act, float cw0, float cw1) {
  if ((int)blockIdx.y >= active_count(act, (int)gridDim.y)) return;
  const int b = active_instance(act, blockIdx.y);
  // Shared slots are numbered by step: the plane of step s (p = z0 - 1 + s)
  // uses slot s % 3, a constant in each of the three unrolled copies below.
  __shared__ float sxr[kMarchWarps][3][32];     // x-smoothed certainties of the newest plane
  // x/y-smoothed certainties of the last three planes; each thread reads
  // back only its own entries, so no barrier guards them
  __shared__ float cxr[SMOOTH ? 3 : 1][kMarchWarps][3][32];
  __shared__ float2 qy1[3][kMarchWarps][32];    // axis-1 responses (q1) of the last planes
  __shared__ float2 qy2[3][kMarchWarps][32];    // axis-1 responses (q2)
  __shared__ double s_part[kMarchWarps][kNSums];
  const long long V = (long long)W * H * D;
  const long long WH = (long long)W * H;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nzs = gridDim.x / (ntx * nty);
  const int zsl = blockIdx.x / (ntx * nty), rem = blockIdx.x - zsl * (ntx * nty);
  const int yt = rem / ntx, xt = rem - yt * ntx;
  const int x = 3 + xt * kMarchCols - 1 + lane;  // lanes 0 and 31: halo columns
  const int y = 3 + yt * 8 - 1 + warp;           // warps 0 and 9: halo rows
  const int z0 = 3 + zsl * zs;
  const int z1 = min(D - 3, z0 + zs);
  (void)nzs;
  const bool empty = W <= 6 || H <= 6 || z1 <= z0;  // no interior voxel: zero sums
  const float2* Q1 = q1 + (long long)b * q1_stride;
  const float2* Q2 = q2 + (long long)b * 3 * V;
  const bool in = x < W && y < H;                         // loads stay inside the volume
  const bool cin = x <= W - 3 && y <= H - 3;              // certainty defined (smoothing support)
  const bool out = lane >= 1 && lane <= kMarchCols && warp >= 1 && warp <= 8 && x <= W - 4 && y <= H - 4;
  const long long col = (long long)y * W + x;
  const float xf = (float)x - 0.5f * (float)(W - 1);
  const float w0 = cw0, w1 = cw1;

  // per-lane moments over the planes: [k][sum w, sum w z, sum w z^2, sum v, sum v z]
  float m[3][5];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int q = 0; q < 5; q++) m[k][q] = 0.f;

  // Three plane buffers whose roles rotate by step: at step s (plane p) the
  // current one holds plane p - 1 (the output plane), the newest plane p,
  // and the third, which held plane p - 2, receives plane p + 1.  The loop
  // is unrolled three times so that the rotation costs no register moves.
  PlaneQ pb0, pb1, pb2;
  float2 prev_a2 = make_float2(0.f, 0.f), prev_c2 = make_float2(0.f, 0.f);  // axis 2 at z - 1
#pragma unroll
  for (int k = 0; k < 3; k++) pb0.a[k] = pb0.c[k] = pb2.a[k] = pb2.c[k] = make_float2(0.f, 0.f);
  if (!empty) load_plane_q(Q1, Q2, V, (long long)(z0 - 1) * WH + col, in, pb1);

  auto step = [&](auto slot, int p, PlaneQ& cur, PlaneQ& nw, PlaneQ& nxt) {
    constexpr int j = decltype(slot)::value;  // slot of plane p
    constexpr int j1 = (j + 2) % 3;            // plane p - 1
    constexpr int j2 = (j + 1) % 3;            // plane p - 2
    // [A] certainties of plane p, x pass, axis-1 responses to shared memory
    if (SMOOTH) {
#pragma unroll
      for (int k = 0; k < 3; k++) {
        float pd, cv = 0.f;
        phase_diff_cert(nw.a[k], nw.c[k], pd, cv);
        cv = cin ? cv : 0.f;
        const float cl = __shfl_up_sync(0xffffffffu, cv, 1), cr = __shfl_down_sync(0xffffffffu, cv, 1);
        sxr[warp][k][lane] = w1 * cl + w0 * cv + w1 * cr;
      }
    }
    qy1[j][warp][lane] = nw.a[1];
    qy2[j][warp][lane] = nw.c[1];
    __syncthreads();
    // axis 2 of plane p - 2, then the next plane in flight during the rest
    // of this step
    prev_a2 = nxt.a[2];
    prev_c2 = nxt.c[2];
    if (p + 1 <= z1) load_plane_q(Q1, Q2, V, (long long)(p + 1) * WH + col, in, nxt);
    // [B] y pass: smoothed certainty of plane p in the register window
    if (SMOOTH && warp >= 1 && warp <= 8) {
#pragma unroll
      for (int k = 0; k < 3; k++)
        cxr[SMOOTH ? j : 0][warp][k][lane] =
            w1 * sxr[warp - 1][k][lane] + w0 * sxr[warp][k][lane] + w1 * sxr[warp + 1][k][lane];
    }
    // [C] sums of output plane z = p - 1
    if (p >= z0 + 1) {
      const int z = p - 1;
      const float zf = (float)z - 0.5f * (float)(D - 1);
      // x neighbours of axis 0 from the adjacent lanes (all lanes shuffle)
      const float2 a0p = make_float2(__shfl_down_sync(0xffffffffu, cur.a[0].x, 1),
                                     __shfl_down_sync(0xffffffffu, cur.a[0].y, 1));
      const float2 c0p = make_float2(__shfl_down_sync(0xffffffffu, cur.c[0].x, 1),
                                     __shfl_down_sync(0xffffffffu, cur.c[0].y, 1));
      const float2 a0m = make_float2(__shfl_up_sync(0xffffffffu, cur.a[0].x, 1),
                                     __shfl_up_sync(0xffffffffu, cur.a[0].y, 1));
      const float2 c0m = make_float2(__shfl_up_sync(0xffffffffu, cur.c[0].x, 1),
                                     __shfl_up_sync(0xffffffffu, cur.c[0].y, 1));
      if (out) {
        float2 ap[3], am[3], cp[3], cm[3];
        ap[0] = a0p; am[0] = a0m; cp[0] = c0p; cm[0] = c0m;
        ap[1] = qy1[j1][warp + 1][lane]; am[1] = qy1[j1][warp - 1][lane];
        cp[1] = qy2[j1][warp + 1][lane]; cm[1] = qy2[j1][warp - 1][lane];
        ap[2] = nw.a[2]; am[2] = prev_a2; cp[2] = nw.c[2]; cm[2] = prev_c2;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          float pd, cert;
          phase_diff_cert(cur.a[k], cur.c[k], pd, cert);
          if (SMOOTH)
            cert = w1 * cxr[SMOOTH ? j2 : 0][warp][k][lane] + w0 * cxr[SMOOTH ? j1 : 0][warp][k][lane] +
                   w1 * cxr[SMOOTH ? j : 0][warp][k][lane];  // planes z - 1, z, z + 1
          const float g = phase_grad(ap[k], cur.a[k], am[k], cp[k], cur.c[k], cm[k]);
          const float cg = cert * g;
          const float wv = cg * g;
          const float vv = cg * pd;
          m[k][0] += wv;
          m[k][1] += wv * zf;
          m[k][2] += wv * zf * zf;
          m[k][3] += vv;
          m[k][4] += vv * zf;
        }
      }
    }
    __syncthreads();  // sxr and the qy slot of plane p - 2 are rewritten next step
  };

  if (!empty) {
    for (int p = z0 - 1;; p += 3) {
      step(std::integral_constant<int, 0>(), p, pb0, pb1, pb2);
      if (p + 1 > z1) break;
      step(std::integral_constant<int, 1>(), p + 1, pb1, pb2, pb0);
      if (p + 2 > z1) break;
      step(std::integral_constant<int, 2>(), p + 2, pb2, pb0, pb1);
      if (p + 3 > z1) break;
    }
  }

  // expand the column moments into the 42 sums (FP64), warp sums, block sum
  const double xd = (double)xf, yd = (double)y - 0.5 * (double)(H - 1);
#pragma unroll
  for (int j = 0; j < kNSums; j++) {
    const int k = j / 14, e = j % 14;
    double v = 0.0;
    if (out) {
      const double s0 = m[k][0], sz = m[k][1], szz = m[k][2], v0 = m[k][3], vz = m[k][4];
      switch (e) {
        case 0: v = s0; break;
        case 1: v = xd * s0; break;
        case 2: v = yd * s0; break;
        case 3: v = sz; break;
        case 4: v = xd * xd * s0; break;
        case 5: v = xd * yd * s0; break;
        case 6: v = xd * sz; break;
        case 7: v = yd * yd * s0; break;
        case 8: v = yd * sz; break;
        case 9: v = szz; break;
        case 10: v = v0; break;
        case 11: v = xd * v0; break;
        case 12: v = yd * v0; break;
        default: v = vz; break;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s_part[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNSums) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kMarchWarps; w++) v += s_part[w][threadIdx.x];
    partials[((long long)b * gridDim.x + blockIdx.x) * kNSums + threadIdx.x] = v;
  }
}

// (row, column) of the 10 A entries of one axis, monomial order
// [1, x, y, z, xx, xy, xz, yy, yz, zz]; axis k owns parameters
// {k, 3+3k, 4+3k, 5+3k} (the GetParameterIndices table,
// kernelRegistration.cpp:43-171).
__constant__ int c_mono_a[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
__constant__ int c_mono_b[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};

__device__ __forceinline__ int axis_param(int k, int m) { return m == 0 ? k : 2 + 3 * k + m; }

// Threads [0, 42) of the CTA sum the nblk partial rows of instance b.
__device__ void reduce_partials(const double* __restrict__ partials, int nblk, int b, double* s) {
  if (threadIdx.x < kNSums) {
    double v = 0.0;
    for (int r = 0; r < nblk; r++) v += partials[((long long)b * nblk + r) * kNSums + threadIdx.x];
    s[threadIdx.x] = v;
  }
  __syncthreads();
}

// Full symmetric 12x12 A (column-major) and h of one instance.
__global__ void assemble_kernel(const double* __restrict__ partials, int nblk, double* __restrict__ A,
                                double* __restrict__ h) {
  __shared__ double s[kNSums];
  const int b = blockIdx.x;
  reduce_partials(partials, nblk, b, s);
  double* Ab = A + (long long)b * 144;
  for (int j = threadIdx.x; j < 144; j += blockDim.x) Ab[j] = 0.0;
  __syncthreads();
  if (threadIdx.x < 30) {
    const int k = threadIdx.x / 10, e = threadIdx.x % 10;
    const int i = axis_param(k, c_mono_a[e]), j = axis_param(k, c_mono_b[e]);
    Ab[i + 12 * j] = s[14 * k + e];
    Ab[j + 12 * i] = s[14 * k + e];
  } else if (threadIdx.x >= 32 && threadIdx.x < 44) {
    const int t = threadIdx.x - 32, k = t / 4, m = t % 4;
    h[(long long)b * 12 + axis_param(k, m)] = s[14 * k + 10 + m];
  }
}

// Solves the 4x4 block of axis k by Gaussian elimination with complete
// pivoting.  Pivots at or below `thresh` end the elimination and the
// remaining unknowns are 0, the rank rule of the reference's full-pivoting
// QR solve (SolveEquationSystem, broccoli_lib.cpp:17157-17186).
__device__ void solve4(double M[4][4], double r[4], double thresh, double x[4]) {
  int perm[4] = {0, 1, 2, 3};
  int rank = 0;
  for (int k = 0; k < 4; k++) {
    int pr = k, pc = k;
    double best = -1.0;
    for (int i = k; i < 4; i++)
      for (int j = k; j < 4; j++)
        if (fabs(M[i][j]) > best) {
          best = fabs(M[i][j]);
          pr = i;
          pc = j;
        }
    if (best <= thresh || best == 0.0) break;
    rank++;
    if (pr != k) {
      for (int j = 0; j < 4; j++) {
        const double t = M[k][j];
        M[k][j] = M[pr][j];
        M[pr][j] = t;
      }
      const double t = r[k];
      r[k] = r[pr];
      r[pr] = t;
    }
    if (pc != k) {
      for (int i = 0; i < 4; i++) {
        const double t = M[i][k];
        M[i][k] = M[i][pc];
        M[i][pc] = t;
      }
      const int t = perm[k];
      perm[k] = perm[pc];
      perm[pc] = t;
    }
    for (int i = k + 1; i < 4; i++) {
      const double m = M[i][k] / M[k][k];
      if (m == 0.0) continue;
      for (int j = k; j < 4; j++) M[i][j] -= m * M[k][j];
      r[i] -= m * r[k];
    }
  }
  double y[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = rank - 1; i >= 0; i--) {
    double s = r[i];
    for (int j = i + 1; j < rank; j++) s -= M[i][j] * y[j];
    y[i] = s / M[i][i];
  }
  for (int i = 0; i < 4; i++) x[perm[i]] = y[i];
}

// p = A^-1 h for the 12-parameter system given by the 42 sums, FP64,
// rounded to float (the reference casts its Eigen solution to float).
__device__ void solve12_from_sums(const double* s, float p[12]) {
  double maxabs = 0.0;
  for (int j = 0; j < kNSums; j++)
    if ((j % 14) < 10) maxabs = fmax(maxabs, fabs(s[j]));
  const double thresh = maxabs * 2.220446049250313e-16 * 12.0;
  for (int k = 0; k < 3; k++) {
    double M[4][4], r[4], x[4];
    for (int e = 0; e < 10; e++) {
      const int a = c_mono_a[e], bb = c_mono_b[e];
      M[a][bb] = s[14 * k + e];
      M[bb][a] = s[14 * k + e];
    }
    for (int m = 0; m < 4; m++) r[m] = s[14 * k + 10 + m];
    solve4(M, r, thresh, x);
    for (int m = 0; m < 4; m++) p[axis_param(k, m)] = (float)x[m];
  }
}

// Orthogonal polar factor U V^T of a 3x3 matrix (row-major) from one-sided
// Jacobi sweeps, FP64 (the reference takes U V^T of Eigen's JacobiSVD in
// RemoveTransformationScaling, broccoli_lib.cpp:6153-6194).
__device__ void polar3(const double* M, double* R) {
  double A[9], Vm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 9; i++) A[i] = M[i];
  for (int sweep = 0; sweep < 60; sweep++) {
    bool rotated = false;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        double al = 0, be = 0, ga = 0;
        for (int i = 0; i < 3; i++) {
          al += A[i * 3 + p] * A[i * 3 + p];
          be += A[i * 3 + q] * A[i * 3 + q];
          ga += A[i * 3 + p] * A[i * 3 + q];
        }
        if (fabs(ga) <= 1e-300 || fabs(ga) <= 2.220446049250313e-16 * sqrt(al * be)) continue;
        rotated = true;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
        for (int i = 0; i < 3; i++) {
          const double ap = A[i * 3 + p], aq = A[i * 3 + q];
          A[i * 3 + p] = c * ap - sn * aq;
          A[i * 3 + q] = sn * ap + c * aq;
          const double vp = Vm[i * 3 + p], vq = Vm[i * 3 + q];
          Vm[i * 3 + p] = c * vp - sn * vq;
          Vm[i * 3 + q] = sn * vp + c * vq;
        }
      }
    if (!rotated) break;
  }
  double U[9], sig[3];
  for (int j = 0; j < 3; j++) {
    sig[j] = sqrt(A[j] * A[j] + A[3 + j] * A[3 + j] + A[6 + j] * A[6 + j]);
    for (int i = 0; i < 3; i++) U[i * 3 + j] = sig[j] > 0 ? A[i * 3 + j] / sig[j] : 0.0;
  }
  for (int j = 0; j < 3; j++)
    if (!(sig[j] > 0)) {
      const int a = (j + 1) % 3, bb = (j + 2) % 3;
      U[0 * 3 + j] = U[1 * 3 + a] * U[2 * 3 + bb] - U[2 * 3 + a] * U[1 * 3 + bb];
      U[1 * 3 + j] = U[2 * 3 + a] * U[0 * 3 + bb] - U[0 * 3 + a] * U[2 * 3 + bb];
      U[2 * 3 + j] = U[0 * 3 + a] * U[1 * 3 + bb] - U[1 * 3 + a] * U[0 * 3 + bb];
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s += U[i * 3 + k] * Vm[j * 3 + k];
      R[i * 3 + j] = s;
    }
}

__device__ void remove_scaling(float* p) {
  double M[9], R[9];
  for (int i = 0; i < 9; i++) M[i] = (double)p[3 + i];
  M[0] += 1.0;
  M[4] += 1.0;
  M[8] += 1.0;
  polar3(M, R);
  R[0] -= 1.0;
  R[4] -= 1.0;
  R[8] -= 1.0;
  for (int i = 0; i < 9; i++) p[3 + i] = (float)R[i];
}

// Total = New * Old on 4x4 homogeneous matrices in FP64, the diagonal ones
// added in float first (AddAffineRegistrationParameters,
// broccoli_lib.cpp:7252-7340).
__device__ void compose(float* old12, const float* n12) {
  double O[16], N[16], T[16];
  const float* src[2] = {old12, n12};
  double* dst[2] = {O, N};
  for (int m = 0; m < 2; m++) {
    const float* p = src[m];
    double* Mt = dst[m];
    Mt[0] = (double)(p[3] + 1.0f); Mt[1] = (double)p[4]; Mt[2] = (double)p[5]; Mt[3] = (double)p[0];
    Mt[4] = (double)p[6]; Mt[5] = (double)(p[7] + 1.0f); Mt[6] = (double)p[8]; Mt[7] = (double)p[1];
    Mt[8] = (double)p[9]; Mt[9] = (double)p[10]; Mt[10] = (double)(p[11] + 1.0f); Mt[11] = (double)p[2];
    Mt[12] = 0; Mt[13] = 0; Mt[14] = 0; Mt[15] = 1;
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0;
      for (int k = 0; k < 4; k++) s += N[i * 4 + k] * O[k * 4 + j];
      T[i * 4 + j] = s;
    }
  old12[0] = (float)T[3];
  old12[1] = (float)T[7];
  old12[2] = (float)T[11];
  old12[3] = (float)(T[0] - 1.0); old12[4] = (float)T[1]; old12[5] = (float)T[2];
  old12[6] = (float)T[4]; old12[7] = (float)(T[5] - 1.0); old12[8] = (float)T[6];
  old12[9] = (float)T[8]; old12[10] = (float)T[9]; old12[11] = (float)(T[10] - 1.0);
}

// Euler angles in degrees (CalculateRotationAnglesFromRotationMatrix,
// broccoli_lib.cpp:6199-6244).
__device__ void rotation_angles(const float* p, float* rot) {
  const double PI_ = 3.14159265358979323846;
  double m[9];
  for (int i = 0; i < 9; i++) m[i] = (double)p[3 + i];
  m[0] += 1.0;
  m[4] += 1.0;
  m[8] += 1.0;
  const double a1 = -atan2(m[5], m[8]) * 180.0 / PI_;
  const double c2 = sqrt(m[0] * m[0] + m[1] * m[1]);
  const double a2 = -atan2(-m[2], c2) * 180.0 / PI_;
  const double s1 = sin(a1 * PI_ / 180.0), c1 = cos(a1 * PI_ / 180.0);
  const double a3 = -atan2(s1 * m[6] - c1 * m[3], c1 * m[4] - s1 * m[7]) * 180.0 / PI_;
  rot[0] = (float)a1;
  rot[1] = (float)a2;
  rot[2] = (float)a3;
}

// Largest displacement (voxels) of the update p over the 8 volume corners.
__device__ double update_magnitude(const float* p, int W, int H, int D) {
  const double hx = 0.5 * (W - 1), hy = 0.5 * (H - 1), hz = 0.5 * (D - 1);
  double best = 0.0;
  for (int c = 0; c < 8; c++) {
    const double x = (c & 1) ? hx : -hx, y = (c & 2) ? hy : -hy, z = (c & 4) ? hz : -hz;
    const double dx = p[0] + p[3] * x + p[4] * y + p[5] * z;
    const double dy = p[1] + p[6] * x + p[7] * y + p[8] * z;
    const double dz = p[2] + p[9] * x + p[10] * y + p[11] * z;
    best = fmax(best, sqrt(dx * dx + dy * dy + dz * dz));
  }
  return best;
}

// One iteration's solve and parameter update for every active instance
// (AlignTwoVolumesLinear, broccoli_lib.cpp:5380-5421), iteration it of
// act; instances whose update is not yet below tol go to list
// (it + 1) % 3, and list (it + 2) % 3 (the one iteration it - 1 used) is
// emptied for the next solve.
__global__ void solve_update_kernel(const double* __restrict__ partials, int nblk, int type,
                                    float tol, int W, int H, int D, float* __restrict__ params,
                                    float* __restrict__ rotations, int* __restrict__ conv_iter,
                                    int* __restrict__ iterations, int* __restrict__ status,
                                    const ActiveSet act, int* __restrict__ lists, int* __restrict__ counts) {
  __shared__ double s[kNSums];
  const int it = active_iteration(act);
  int* next_list = lists + ((it + 1) % 3) * act.stride;
  int* next_count = counts + (it + 1) % 3;
  if (blockIdx.x == 0 && threadIdx.x == 0) counts[(it + 2) % 3] = 0;
  if ((int)blockIdx.x >= active_count(act, (int)gridDim.x)) return;
  const int b = active_instance(act, blockIdx.x);
  reduce_partials(partials, nblk, b, s);
  if (threadIdx.x != 0) return;
  float p[12];
  solve12_from_sums(s, p);
  bool finite = true;
  for (int i = 0; i < 12; i++) finite = finite && isfinite(p[i]);
  if (!finite) {
    for (int i = 0; i < 12; i++) p[i] = 0.f;
    if (status) atomicOr(status, 1);
  }
  float* tot = params + (long long)b * 12;
  float t[12];
  for (int i = 0; i < 12; i++) t[i] = tot[i];
  if (type == 0) {
    t[0] += p[0];
    t[1] += p[1];
    t[2] += p[2];
    for (int i = 3; i < 12; i++) t[i] = 0.f;
    for (int i = 3; i < 12; i++) p[i] = 0.f;
  } else if (type == 1) {
    remove_scaling(p);
    compose(t, p);
  } else {
    compose(t, p);
  }
  for (int i = 0; i < 12; i++) tot[i] = t[i];
  if (iterations) iterations[b] = it + 1;
  if (rotations && type == 1) rotation_angles(t, rotations + (long long)b * 3);
  const bool converged = tol > 0.f && update_magnitude(p, W, H, D) < (double)tol;
  if (converged && conv_iter != nullptr) conv_iter[b] = it;
  if (!converged) next_list[atomicAdd(next_count, 1)] = b;
}

// End of an iteration of the loop: advances the device iteration counter,
// and, when the loop runs as a graph's conditional WHILE node, sets its
// condition: another iteration while iterations remain and the list the
// solve just filled is not empty (then *iters_run counts the iteration).
__global__ void iteration_control_kernel(int* __restrict__ iter, const int* __restrict__ counts, int max_it,
                                         cudaGraphConditionalHandle cond, int use_cond,
                                         unsigned long long* __restrict__ iters_run) {
  const int next = *iter + 1;
  *iter = next;
  if (use_cond) {
    atomicAdd(iters_run, 1ull);
    cudaGraphSetConditional(cond, (next < max_it && counts[next % 3] > 0) ? 1u : 0u);
  }
}

__global__ void active_init_kernel(int* __restrict__ list0, int* __restrict__ counts, int batch) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) list0[i] = i;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counts[0] = batch;
    counts[1] = 0;
    counts[2] = 0;
  }
}

// Plain solve of given A/h (brc_solve_affine_fp64): A column-major 12x12.
__global__ void solve_given_kernel(const double* __restrict__ A, const double* __restrict__ h,
                                   float* __restrict__ p) {
  const int b = blockIdx.x;
  if (threadIdx.x != 0) return;
  const double* Ab = A + (long long)b * 144;
  const double* hb = h + (long long)b * 12;
  // The 12x12 of this path is block diagonal; solve it as a general 12x12
  // with complete pivoting so that any symmetric system is handled.
  double M[144], r[12], x[12];
  int perm[12];
  for (int i = 0; i < 12; i++) {
    r[i] = hb[i];
    perm[i] = i;
    for (int j = 0; j < 12; j++) M[i * 12 + j] = Ab[i + 12 * j];
  }
  double maxpiv = 0.0;
  int rank = 0;
  for (int k = 0; k < 12; k++) {
    int pr = k, pc = k;
    double best = -1.0;
    for (int i = k; i < 12; i++)
      for (int j = k; j < 12; j++)
        if (fabs(M[i * 12 + j]) > best) {
          best = fabs(M[i * 12 + j]);
          pr = i;
          pc = j;
        }
    if (k == 0) maxpiv = best;
    if (best <= maxpiv * 2.220446049250313e-16 * 12.0 || best == 0.0) break;
    rank++;
    if (pr != k) {
      for (int j = 0; j < 12; j++) {
        const double t = M[k * 12 + j];
        M[k * 12 + j] = M[pr * 12 + j];
        M[pr * 12 + j] = t;
      }
      const double t = r[k];
      r[k] = r[pr];
      r[pr] = t;
    }
    if (pc != k) {
      for (int i = 0; i < 12; i++) {
        const double t = M[i * 12 + k];
        M[i * 12 + k] = M[i * 12 + pc];
        M[i * 12 + pc] = t;
      }
      const int t = perm[k];
      perm[k] = perm[pc];
      perm[pc] = t;
    }
    for (int i = k + 1; i < 12; i++) {
      const double m = M[i * 12 + k] / M[k * 12 + k];
      if (m == 0.0) continue;
      for (int j = k; j < 12; j++) M[i * 12 + j] -= m * M[k * 12 + j];
      r[i] -= m * r[k];
    }
  }
  double y[12];
  for (int i = 0; i < 12; i++) y[i] = 0.0;
  for (int i = rank - 1; i >= 0; i--) {
    double s = r[i];
    for (int j = i + 1; j < rank; j++) s -= M[i * 12 + j] * y[j];
    y[i] = s / M[i * 12 + i];
  }
  for (int i = 0; i < 12; i++) x[perm[i]] = y[i];
  for (int i = 0; i < 12; i++) p[(long long)b * 12 + i] = (float)x[i];
}

// ---------------------------------------------------------------------------
// Trilinear sampling
// ---------------------------------------------------------------------------

// out_b(x) = src_b(x + t + (A - I)(x - centre)), params_b of instance b
// (InterpolateVolumeLinearLinear, kernelRegistration.cpp:1066-1101).
// VEC: params is 16-byte aligned, and the 12 parameters of an instance are
// read as three 16-byte loads.
template <bool VEC>
__global__ void __launch_bounds__(256)
warp_affine_kernel(const float* __restrict__ src, long long src_stride, int W, int H, int D, int ntx, int batch,
                   const float* __restrict__ params, float* __restrict__ out, long long out_stride,
                   const ActiveSet act) {
  // block: 32 x 8 voxels of one plane; grid (x-y tiles, planes, a share of
  // the instances: blockIdx.z, + gridDim.z, ...)
  const int ty = blockIdx.x / ntx, tx = blockIdx.x - ty * ntx;
  const int x = tx * 32 + threadIdx.x, y = ty * 8 + threadIdx.y, z = blockIdx.y;
  if (x >= W || y >= H) return;
  const int n = active_count(act, batch);
  for (int li = blockIdx.z; li < n; li += gridDim.z) {
    const int b = active_instance(act, li);
    float p[12];
    if (VEC) {
      const float4* p4 = reinterpret_cast<const float4*>(params + (long long)b * 12);
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const float4 v = __ldg(p4 + q);
        p[4 * q] = v.x;
        p[4 * q + 1] = v.y;
        p[4 * q + 2] = v.z;
        p[4 * q + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < 12; q++) p[q] = __ldg(params + (long long)b * 12 + q);
    }
    out[(long long)b * out_stride + ((long long)z * H + y) * W + x] =
        affine_sample(src + (long long)b * src_stride, W, H, D, p, x, y, z);
  }
}

// Displacement-field warp (InterpolateVolumeLinearNonLinear,
// kernelRegistration.cpp:1111-1140).
__global__ void __launch_bounds__(256)
warp_field_kernel(const float* __restrict__ src, int W, int H, int D, const float* __restrict__ dx,
                  const float* __restrict__ dy, const float* __restrict__ dz, float* __restrict__ out,
                  long long src_stride, long long field_stride, long long out_stride) {
  const int V = W * H * D;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  // instance blockIdx.y
  const long long b = blockIdx.y;
  src += b * src_stride;
  dx += b * field_stride;
  dy += b * field_stride;
  dz += b * field_stride;
  out += b * out_stride;
  const int r = i / W;
  const int x = i - r * W, y = r % H, z = r / H;
  out[i] = sample_linear(src, W, H, D, (float)x + dx[i] + 0.5f, (float)y + dy[i] + 0.5f,
                         (float)z + dz[i] + 0.5f);
}

// Linear resample with spacing (N-1)/(N'-1) (RescaleVolumeLinear,
// kernelRegistration.cpp:1340-1366).
__global__ void __launch_bounds__(256)
rescale_linear_kernel(const float* __restrict__ src, int W, int H, int D, float* __restrict__ out,
                      int W2, int H2, int D2, float vx, float vy, float vz) {
  const int V2 = W2 * H2 * D2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V2) return;
  const int r = i / W2;
  const int x = i - r * W2, y = r % H2, z = r / H2;
  out[i] = sample_linear(src, W, H, D, x * vx + 0.5f, y * vy + 0.5f, z * vz + 0.5f);
}

// ---------------------------------------------------------------------------
// Separable 9-tap smoothing (three passes)
// ---------------------------------------------------------------------------

struct Taps9 {
  float f[9];
};

// The three separable 9-tap passes in one kernel: y over (vol * cert), then
// x, then z, divided by the smoothed certainty (SeparableConvolutionRows /
// Columns / Rods, kernelConvolution.cpp:52-91, :531-569, :1201-1240, zero
// padding).  Each output is the same sequence of terms as three separate
// passes (o = -4..4 in order, out-of-volume terms 0), and the volume is read
// from HBM once and written once.
//
// A block owns a 56 x 16 column tile and marches along z through a chunk of
// planes.  Per plane, the 64 x 24 input window (tile plus 4-voxel halo) is
// copied into shared memory with cp.async (zero-filled outside the volume)
// into a four-stage ring, three planes ahead of its use; with an even W the
// copies move 8-byte pairs (a pair never straddles the volume's edge), and a
// thread's copies lie in one window column, so its addresses advance by a
// constant.  Every thread then computes four y outputs of one window column
// (12 shared loads, 36 FMAs), and 224 of the 256 threads four consecutive x
// outputs of one tile row (three 16-byte shared loads, 36 FMAs), which enter
// a nine-plane register ring; the z pass (36 FMAs) writes the output plane
// to shared memory, from which all threads store it coalesced in the next
// phase.  The ring slot of a plane is its index modulo 9, dispatched by a
// switch over nine copies of the z pass so that every register index is a
// constant.  The y pass of plane k, the x and z passes of plane k - 1 and
// the stores of plane k - 2 run in the same phase (the y results and the
// output plane are double-buffered), so one barrier per plane separates
// every producer from its consumer.  With a certainty, its window is copied
// beside the volume's and the product is formed in the y pass.  `out` must
// not overlap the inputs.
constexpr int kSmTX = 56, kSmTY = 16;            // output tile
constexpr int kSmWX = kSmTX + 8, kSmWY = kSmTY + 8;  // input window 64 x 24
constexpr int kSmPitch = 68;                     // shared row pitch (floats, 16-byte rows)
constexpr int kSmThreads = 256;
constexpr int kSmXQ = kSmTX / 4;                 // 14 quads of x outputs per row
constexpr int kSmOwners = kSmXQ * kSmTY;         // 224 threads own outputs
constexpr int kSmStages = 4;                     // window ring (planes in flight + 1)
constexpr int kSmWin = kSmWY * kSmPitch;         // floats per window stage
constexpr int kSmYBuf = kSmTY * kSmPitch;        // floats per y-result buffer
constexpr int kSmOut = kSmTY * kSmTX;            // floats per output plane
static_assert(kSmWX == 64 && kSmTY == 16, "mappings assume 64 window columns and 16 tile rows");

inline size_t smooth_smem_bytes(bool cert) {
  return sizeof(float) * ((size_t)(cert ? 2 : 1) * kSmStages * kSmWin + 2 * kSmYBuf + 2 * kSmOut);
}

template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const float* src, uint32_t n) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(BYTES), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// VEC: floats per copy (2 needs an even W and 8-byte aligned volumes); DIV:
// divide by the smoothed certainty scert; ACC: add into `out`.
template <bool CERT, int VEC, bool DIV, bool ACC>
__global__ void __launch_bounds__(kSmThreads, 3)
smooth3d_kernel(const float* __restrict__ in, long long in_stride, const float* __restrict__ cert,
                const float* __restrict__ scert, int W, int H, int D, int zc, Taps9 tx, Taps9 ty, Taps9 tz,
                float* __restrict__ out, long long out_stride) {
  extern __shared__ __align__(16) float smem[];
  float* s_in = smem;                                       // kSmStages windows (+ certainty windows)
  float* s_y = smem + (CERT ? 2 : 1) * kSmStages * kSmWin;  // 2 y-result buffers
  float* s_o = s_y + 2 * kSmYBuf;                           // 2 output planes
  const int tid = threadIdx.x;
  const int ntx = (W + kSmTX - 1) / kSmTX;
  const int x0 = (int)(blockIdx.x % ntx) * kSmTX, y0 = (int)(blockIdx.x / ntx) * kSmTY;
  const int z0 = blockIdx.y * zc, z1 = min(D, z0 + zc);
  const int np = z1 - z0 + 8;  // planes z0 - 4 .. z1 + 3
  const long long WH = (long long)W * H;
  const float* src = in + (long long)blockIdx.z * in_stride;

  // copies: window column wc (VEC wide), rows wr0 + RS m for m < NC
  constexpr int CPR = kSmWX / VEC;            // copies per window row
  constexpr int RS = kSmThreads / CPR;        // row step between a thread's copies
  constexpr int NC = kSmWY / RS;              // copies per thread
  static_assert(NC * RS == kSmWY, "window rows / thread mismatch");
  const int wc = (tid % CPR) * VEC, wr0 = tid / CPR;
  const int gx = x0 - 4 + wc;
  const bool xin = gx >= 0 && gx < W;  // with VEC 2 and W even, gx + 1 < W too
  unsigned rowmask = 0;
#pragma unroll
  for (int m = 0; m < NC; m++) {
    const int gy = y0 - 4 + wr0 + RS * m;
    if (xin && gy >= 0 && gy < H) rowmask |= 1u << m;
  }
  // in-plane offset of copy 0 (outside the volume when its row is; only
  // copies of rows inside the volume use it)
  const long long off0 = (long long)(y0 - 4 + wr0) * W + gx;
  const long long rstep = (long long)RS * W;
  const uint32_t sdst0 = static_cast<uint32_t>(__cvta_generic_to_shared(s_in)) + 4u * (wr0 * kSmPitch + wc);
  auto issue = [&](int k) {
    const int p = z0 - 4 + k;
    const bool pin = p >= 0 && p < D;
    const unsigned mask = pin ? rowmask : 0u;
    const long long poff = (long long)(pin ? p : 0) * WH;
    const uint32_t d = sdst0 + 4u * (uint32_t)(((unsigned)k % kSmStages) * kSmWin);
#pragma unroll
    for (int m = 0; m < NC; m++) {
      const bool v = (mask >> m) & 1u;
      // copies outside the volume read nothing (size 0) from the volume's start
      const long long o = v ? poff + off0 + m * rstep : 0;
      cp_async<4 * VEC>(d + 4u * (uint32_t)(RS * m * kSmPitch), src + o, v ? 4u * VEC : 0u);
      if (CERT) cp_async<4 * VEC>(d + 4u * (uint32_t)(kSmStages * kSmWin + RS * m * kSmPitch), cert + o,
                                   v ? 4u * VEC : 0u);
    }
    cp_async_commit();
  };
  // y pass: window column yc, tile rows 4 yg .. 4 yg + 3
  const int yc = tid & 63, yg = tid >> 6;
  auto ypass = [&](int k) {
    const float* w = s_in + ((unsigned)k % kSmStages) * kSmWin + (4 * yg) * kSmPitch + yc;
    float* yb = s_y + (k & 1) * kSmYBuf + (4 * yg) * kSmPitch + yc;
    float a[12];
#pragma unroll
    for (int i = 0; i < 12; i++) {
      a[i] = w[i * kSmPitch];
      if (CERT) a[i] *= w[kSmStages * kSmWin + i * kSmPitch];
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      float sum = 0.f;
#pragma unroll
      for (int o = -4; o <= 4; o++) sum += a[i + 4 + o] * ty.f[4 - o];
      yb[i * kSmPitch] = sum;
    }
  };
  // x and z passes: tile row xr, outputs x0 + 4 xq .. + 3
  const bool owner = tid < kSmOwners;
  const int xr = tid / kSmXQ, xq = tid - (tid / kSmXQ) * kSmXQ;
  float ring[9][4];
#pragma unroll
  for (int u = 0; u < 9; u++)
#pragma unroll
    for (int i = 0; i < 4; i++) ring[u][i] = 0.f;
  // stores: tile row sr = tid / 16, columns sc + 16 i (i < 4, < 56)
  const int sr = tid >> 4, sc = tid & 15;
  unsigned colmask = 0;
#pragma unroll
  for (int i = 0; i < 4; i++)
    if (sc + 16 * i < kSmTX && x0 + sc + 16 * i < W) colmask |= 1u << i;
  if (y0 + sr >= H) colmask = 0;
  float* dst_row = out + (long long)blockIdx.z * out_stride + (long long)(y0 + sr) * W + x0 + sc;
  const float* scert_row = DIV ? scert + (long long)(y0 + sr) * W + x0 + sc : nullptr;
  auto store = [&](int j) {
    const long long zoff = (long long)(z0 + j - 8) * WH;
    const float* so = s_o + (j & 1) * kSmOut + sr * kSmTX + sc;
    float* o = dst_row + zoff;
#pragma unroll
    for (int i = 0; i < 4; i++)
      if ((colmask >> i) & 1u) {
        float q = so[16 * i];
        if (DIV) q = q / __ldg(scert_row + zoff + 16 * i);
        o[16 * i] = ACC ? o[16 * i] + q : q;
      }
  };

  // planes 0 .. kSmStages - 2 in flight; plane 0 complete and visible
#pragma unroll
  for (int k = 0; k < kSmStages - 1; k++) {
    if (k < np) issue(k);
    else cp_async_commit();
  }
  cp_async_wait<kSmStages - 2>();
  __syncthreads();
  // phase k: copies of plane k + 3 issued, y pass of plane k, x and z passes
  // of plane k - 1 (ring slot (k - 1) % 9), stores of plane k - 2; then plane
  // k + 1 complete and visible
  int slot = 0;
  for (int k = 0; k <= np + 1; k++) {
    if (k + kSmStages - 1 < np) issue(k + kSmStages - 1);
    else cp_async_commit();
    if (k < np) ypass(k);
    if (k >= 1 && k <= np) {
      if (owner) {
        const int j = k - 1;
        const float4* r4 = reinterpret_cast<const float4*>(s_y + (j & 1) * kSmYBuf + xr * kSmPitch + 4 * xq);
        const float4 f0 = r4[0], f1 = r4[1], f2 = r4[2];
        const float a[12] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w};
        float v[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          float sum = 0.f;
#pragma unroll
          for (int o = -4; o <= 4; o++) sum += a[i + 4 + o] * tx.f[4 - o];
          v[i] = sum;
        }
        float4* od = reinterpret_cast<float4*>(s_o + (j & 1) * kSmOut + xr * kSmTX + 4 * xq);
        // slot S holds plane j; the output plane z0 + j - 8 sums planes
        // j - 8 .. j, held in slots S + 1 .. S + 9 (mod 9), oldest first
#define BRC_SMOOTH_Z(S)                                                              \
  case S: {                                                                          \
    _Pragma("unroll") for (int i = 0; i < 4; i++) ring[S][i] = v[i];                 \
    if (j >= 8) {                                                                    \
      float zs[4];                                                                   \
      _Pragma("unroll") for (int i = 0; i < 4; i++) {                                \
        float sum = 0.f;                                                             \
        _Pragma("unroll") for (int jj = 0; jj < 9; jj++) sum += ring[(S + 1 + jj) % 9][i] * tz.f[8 - jj]; \
        zs[i] = sum;                                                                 \
      }                                                                              \
      *od = make_float4(zs[0], zs[1], zs[2], zs[3]);                                 \
    }                                                                                \
  } break;
        switch (slot) {
          BRC_SMOOTH_Z(0)
          BRC_SMOOTH_Z(1)
          BRC_SMOOTH_Z(2)
          BRC_SMOOTH_Z(3)
          BRC_SMOOTH_Z(4)
          BRC_SMOOTH_Z(5)
          BRC_SMOOTH_Z(6)
          BRC_SMOOTH_Z(7)
          BRC_SMOOTH_Z(8)
        }
#undef BRC_SMOOTH_Z
      }
      slot = slot == 8 ? 0 : slot + 1;
    }
    if (k >= 10) store(k - 2);
    cp_async_wait<kSmStages - 2>();
    __syncthreads();
  }
  cp_async_wait<0>();
}

// Planes per z chunk of smooth3d_kernel: enough chunks that the grid fills
// the 148 SMs about six blocks deep, at least 16 planes per chunk.
static int smooth_chunk(int D, long long tiles_x_batch) {
  const long long want = 148LL * 6;
  long long chunks = (want + tiles_x_batch - 1) / tiles_x_batch;
  const long long maxc = (D + 15) / 16;
  if (chunks > maxc) chunks = maxc;
  if (chunks < 1) chunks = 1;
  return (int)((D + chunks - 1) / chunks);
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

cudaError_t normal_eq_partials(const float* q1, long long q1_stride_floats, const float* q2, int W,
                               int H, int D, int batch, double* partials, int nblk, int zpb, cudaStream_t st) {
  dim3 grid(nblk, batch);
  normal_eq_partial_kernel<<<grid, kNEThreads, 0, st>>>(
      reinterpret_cast<const float2*>(q1), q1_stride_floats / 2, reinterpret_cast<const float2*>(q2),
      W, H, D, zpb, partials);
  return cudaGetLastError();
}

int normal_eq_march_blocks(int W, int H, int D, int* ntx, int* nty, int* zs) {
  const int nx = W - 6, ny = H - 6, nz = D - 6;
  *ntx = nx > 0 ? (nx + kMarchCols - 1) / kMarchCols : 1;
  *nty = ny > 0 ? (ny + 7) / 8 : 1;
  const int nzs = nz > 0 ? (nz + kMarchZs - 1) / kMarchZs : 1;
  *zs = nz > 0 ? (nz + nzs - 1) / nzs : 0;
  return *ntx * *nty * nzs;
}

cudaError_t normal_eq_march(const float* q1, long long q1_stride_floats, const float* q2, int W, int H, int D,
                            int batch, double* partials, int nblk, ActiveSet act, cudaStream_t st,
                            float cert_sigma) {
  int ntx, nty, zs;
  if (normal_eq_march_blocks(W, H, D, &ntx, &nty, &zs) != nblk) return cudaErrorInvalidValue;
  dim3 grid((unsigned)nblk, (unsigned)batch);
  const float2* a = reinterpret_cast<const float2*>(q1);
  const float2* c = reinterpret_cast<const float2*>(q2);
  if (cert_sigma > 0.f) {
    // 3-tap Gaussian, weights normalised to sum 1
    const float e = (float)exp(-1.0 / (2.0 * (double)cert_sigma * (double)cert_sigma));
    const float w0 = 1.0f / (1.0f + 2.0f * e), w1 = e * w0;
    normal_eq_march_kernel<true><<<grid, kMarchWarps * 32, 0, st>>>(a, q1_stride_floats / 2, c, W, H, D, ntx, nty,
                                                                     zs, partials, act, w0, w1);
  } else {
    normal_eq_march_kernel<false><<<grid, kMarchWarps * 32, 0, st>>>(a, q1_stride_floats / 2, c, W, H, D, ntx,
                                                                      nty, zs, partials, act, 1.f, 0.f);
  }
  return cudaGetLastError();
}

cudaError_t assemble_normal_eq(const double* partials, int nblk, int batch, double* A, double* h,
                               cudaStream_t st) {
  assemble_kernel<<<batch, 64, 0, st>>>(partials, nblk, A, h);
  return cudaGetLastError();
}

cudaError_t solve_update(const double* partials, int nblk, int batch, int type, float tol, int W,
                         int H, int D, float* params, float* rotations, int* conv_iter,
                         int* iterations, int* status, ActiveSet act, int* lists, int* counts, cudaStream_t st) {
  if (!act.list) return cudaErrorInvalidValue;
  solve_update_kernel<<<batch, 64, 0, st>>>(partials, nblk, type, tol, W, H, D, params, rotations,
                                            conv_iter, iterations, status, act, lists, counts);
  return cudaGetLastError();
}

cudaError_t iteration_control(int* iter, const int* counts, int max_it, cudaGraphConditionalHandle cond,
                              bool use_cond, unsigned long long* iters_run, cudaStream_t st) {
  iteration_control_kernel<<<1, 1, 0, st>>>(iter, counts, max_it, cond, use_cond ? 1 : 0, iters_run);
  return cudaGetLastError();
}

cudaError_t active_init(int* list0, int* counts, int batch, cudaStream_t st) {
  active_init_kernel<<<(batch + 255) / 256, 256, 0, st>>>(list0, counts, batch);
  return cudaGetLastError();
}

cudaError_t solve_given(const double* A, const double* h, int batch, float* p, cudaStream_t st) {
  solve_given_kernel<<<batch, 32, 0, st>>>(A, h, p);
  return cudaGetLastError();
}

cudaError_t warp_affine(const float* src, long long src_stride, int W, int H, int D, int batch,
                        const float* params, float* out, long long out_stride, ActiveSet act,
                        cudaStream_t st) {
  const long long V = (long long)W * H * D;
  if (V > kMaxVoxels) return cudaErrorInvalidValue;
  if (D > 65535 || batch > 65535 || batch <= 0) return cudaErrorInvalidValue;
  const int ntx = (W + 31) / 32, nty = (H + 7) / 8;
  // at most 16 instance shares: a launch whose instances have mostly
  // converged does not pay for blocks with nothing to do
  dim3 grid((unsigned)(ntx * nty), (unsigned)D, (unsigned)(batch < 16 ? batch : 16));
  if ((reinterpret_cast<uintptr_t>(params) & 15) == 0)
    warp_affine_kernel<true><<<grid, dim3(32, 8), 0, st>>>(src, src_stride, W, H, D, ntx, batch, params, out,
                                                         out_stride, act);
  else
    warp_affine_kernel<false><<<grid, dim3(32, 8), 0, st>>>(src, src_stride, W, H, D, ntx, batch, params, out,
                                                          out_stride, act);
  return cudaGetLastError();
}

cudaError_t warp_field(const float* src, int W, int H, int D, const float* dx, const float* dy,
                       const float* dz, float* out, cudaStream_t st, int batch, long long src_stride,
                       long long field_stride, long long out_stride) {
  const long long V = (long long)W * H * D;
  if (V > kMaxVoxels || batch <= 0 || batch > 65535) return cudaErrorInvalidValue;
  warp_field_kernel<<<dim3((unsigned)((V + 255) / 256), (unsigned)batch), 256, 0, st>>>(
      src, W, H, D, dx, dy, dz, out, src_stride, field_stride, out_stride);
  return cudaGetLastError();
}

cudaError_t rescale_linear(const float* src, int W, int H, int D, float* out, int W2, int H2, int D2,
                           cudaStream_t st) {
  const long long V2 = (long long)W2 * H2 * D2;
  if (V2 > kMaxVoxels || (long long)W * H * D > kMaxVoxels) return cudaErrorInvalidValue;
  const float vx = (float)(W - 1) / (float)(W2 - 1);
  const float vy = (float)(H - 1) / (float)(H2 - 1);
  const float vz = (float)(D - 1) / (float)(D2 - 1);
  rescale_linear_kernel<<<(unsigned)((V2 + 255) / 256), 256, 0, st>>>(src, W, H, D, out, W2, H2, D2,
                                                                     vx, vy, vz);
  return cudaGetLastError();
}

// vols[b][i] *= mask[i] for every volume b (MultiplyVolumes,
// kernelMisc.cpp, as PerformSmoothingNormalized ends, broccoli_lib.cpp:11359-11450).
__global__ void __launch_bounds__(256)
multiply_mask_kernel(float* __restrict__ vols, const float* __restrict__ mask, long long V) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  vols[(long long)blockIdx.y * V + i] *= __ldg(mask + i);
}

__global__ void phase_atan2_kernel(const float* __restrict__ y, const float* __restrict__ x,
                                   float* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = phase_atan2(y[i], x[i]);
}

// The reference's linear phase quantities of one filter pair, volume by
// volume (CalculatePhaseDifferencesAndCertainties, CalculatePhaseGradients
// X/Y/Z, kernelRegistration.cpp:173-382), with the library's own atan2f,
// cosf and sqrtf and no contraction into FMAs (the reference's order of
// operations).  Used for the debug outputs, not in the registration loop.
__global__ void __launch_bounds__(256)
phase_volumes_kernel(const float2* __restrict__ q1, const float2* __restrict__ q2, int W, int H, int D, int axis,
                     float* __restrict__ pd, float* __restrict__ cert, float* __restrict__ grad) {
  const long long V = (long long)W * H * D;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  if (pd || cert) {
    const float2 a = q1[i], c = q2[i];
    const float re = __fadd_rn(__fmul_rn(a.x, c.x), __fmul_rn(a.y, c.y));
    const float im = __fsub_rn(__fmul_rn(a.y, c.x), __fmul_rn(a.x, c.y));
    const float d = atan2f(im, re);
    if (pd) pd[i] = d;
    if (cert) {
      const float pr = __fsub_rn(__fmul_rn(a.x, c.x), __fmul_rn(a.y, c.y));
      const float pi = __fadd_rn(__fmul_rn(a.y, c.x), __fmul_rn(a.x, c.y));
      const float cc = cosf(__fmul_rn(d, 0.5f));
      cert[i] = __fmul_rn(__fmul_rn(sqrtf(__fadd_rn(__fmul_rn(pr, pr), __fmul_rn(pi, pi))), cc), cc);
    }
  }
  if (grad) {
    const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
    const int c = axis == 0 ? x : (axis == 1 ? y : z);
    const int n = axis == 0 ? W : (axis == 1 ? H : D);
    const long long step = axis == 0 ? 1 : (axis == 1 ? (long long)W : (long long)W * H);
    if (c - 1 < 0 || c + 1 >= n) {
      grad[i] = 0.f;
      return;
    }
    float tr = 0.f, ti = 0.f;
    const float2* qs[2] = {q1, q2};
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const float2 p = qs[k][i + step], o = qs[k][i], m = qs[k][i - step];
      tr = __fadd_rn(tr, __fadd_rn(__fmul_rn(p.x, o.x), __fmul_rn(p.y, o.y)));
      ti = __fadd_rn(ti, __fsub_rn(__fmul_rn(p.y, o.x), __fmul_rn(p.x, o.y)));
      tr = __fadd_rn(tr, __fadd_rn(__fmul_rn(o.x, m.x), __fmul_rn(o.y, m.y)));
      ti = __fadd_rn(ti, __fsub_rn(__fmul_rn(o.y, m.x), __fmul_rn(o.x, m.y)));
    }
    grad[i] = atan2f(ti, tr);
  }
}

cudaError_t phase_volumes(const float* q1, const float* q2, int W, int H, int D, int axis, float* pd, float* cert,
                          float* grad, cudaStream_t st) {
  const long long V = (long long)W * H * D;
  if (V <= 0 || V > kMaxVoxels || axis < 0 || axis > 2) return cudaErrorInvalidValue;
  phase_volumes_kernel<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(reinterpret_cast<const float2*>(q1),
                                                                   reinterpret_cast<const float2*>(q2), W, H, D,
                                                                   axis, pd, cert, grad);
  return cudaGetLastError();
}

cudaError_t phase_atan2_eval(const float* y, const float* x, float* out, long long n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const long long nb = (n + 255) / 256;
  phase_atan2_kernel<<<(unsigned)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, st>>>(y, x, out, n);
  return cudaGetLastError();
}

cudaError_t multiply_mask(float* vols, const float* mask, long long V, int batch, cudaStream_t st) {
  dim3 grid((unsigned)((V + 255) / 256), batch);
  multiply_mask_kernel<<<grid, 256, 0, st>>>(vols, mask, V);
  return cudaGetLastError();
}

// smooth3d_kernel instantiations indexed by (cert << 3) | (pairs << 2) |
// (divide << 1) | accumulate.
static const void* smooth_kernel_of(int v) {
#define BRC_SK(C, P, Q, A) reinterpret_cast<const void*>(smooth3d_kernel<C, (P) ? 2 : 1, Q, A>)
  static const void* const table[16] = {
      BRC_SK(false, false, false, false), BRC_SK(false, false, false, true), BRC_SK(false, false, true, false),
      BRC_SK(false, false, true, true),   BRC_SK(false, true, false, false), BRC_SK(false, true, false, true),
      BRC_SK(false, true, true, false),   BRC_SK(false, true, true, true),   BRC_SK(true, false, false, false),
      BRC_SK(true, false, false, true),   BRC_SK(true, false, true, false),  BRC_SK(true, false, true, true),
      BRC_SK(true, true, false, false),   BRC_SK(true, true, false, true),   BRC_SK(true, true, true, false),
      BRC_SK(true, true, true, true)};
#undef BRC_SK
  return table[v];
}

int smooth3d_default_chunk(int W, int H, int D, int batch) {
  const long long ntiles = (long long)((W + kSmTX - 1) / kSmTX) * ((H + kSmTY - 1) / kSmTY);
  return smooth_chunk(D, ntiles * batch);
}

int smooth3d_chunk_candidates(int D, int* zc, int max_n) {
  // D split into 1, 2, 3, 4, 6 or 8 chunks of at least 8 planes
  static const int parts[] = {1, 2, 3, 4, 6, 8};
  int n = 0;
  for (int c : parts) {
    const int z = (D + c - 1) / c;
    if (n >= max_n || (c > 1 && z < 8)) break;
    if (n == 0 || zc[n - 1] != z) zc[n++] = z;
  }
  return n;
}

cudaError_t smooth3d(const float* vol, int W, int H, int D, int batch, const float* fx,
                     const float* fy, const float* fz, const float* cert, const float* scert,
                     float* tmp1, float* tmp2, float* out, cudaStream_t st, int accumulate, int zchunk) {
  const long long V = (long long)W * H * D;
  Taps9 tx, ty, tz;
  for (int i = 0; i < 9; i++) {
    tx.f[i] = fx[i];
    ty.f[i] = fy[i];
    tz.f[i] = fz[i];
  }
  (void)tmp2;  // the fused kernel needs no second temporary
  // an output overlapping an input is computed into tmp1, then moved
  const size_t bytes = sizeof(float) * (size_t)V * batch;
  auto overlaps = [&](const float* a, size_t na) {
    const char *o0 = reinterpret_cast<const char*>(out), *a0 = reinterpret_cast<const char*>(a);
    return a != nullptr && o0 < a0 + na && a0 < o0 + bytes;
  };
  const bool alias = overlaps(vol, bytes) || overlaps(cert, sizeof(float) * (size_t)V) ||
                     overlaps(scert, sizeof(float) * (size_t)V);
  float* dst = alias ? tmp1 : out;
  const long long ntiles = (long long)((W + kSmTX - 1) / kSmTX) * ((H + kSmTY - 1) / kSmTY);
  if (ntiles > 0x7fffffffLL || batch > 65535 || V > kMaxVoxels) return cudaErrorInvalidValue;
  const int zc = zchunk > 0 ? (zchunk < D ? zchunk : D) : smooth_chunk(D, ntiles * batch);
  const dim3 grid((unsigned)ntiles, (unsigned)((D + zc - 1) / zc), (unsigned)batch);
  // the dynamic shared memory above 48 KB is a per-device function attribute
  static bool attr_set[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  // 8-byte copies need an even W (pairs never straddle the edge) and 8-byte
  // aligned volumes
  const bool pairs = (W & 1) == 0 && ((reinterpret_cast<uintptr_t>(vol) | reinterpret_cast<uintptr_t>(cert)) & 7) == 0;
  const bool acc = !alias && accumulate != 0;
  const int variant = (cert ? 8 : 0) | (pairs ? 4 : 0) | (scert ? 2 : 0) | (acc ? 1 : 0);
  if (!attr_set[dev]) {
    for (int v = 0; v < 16; v++) {
      const cudaError_t e0 = cudaFuncSetAttribute(smooth_kernel_of(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smooth_smem_bytes((v & 8) != 0));
      if (e0 != cudaSuccess) return e0;
    }
    attr_set[dev] = true;
  }
  void* args[] = {(void*)&vol, (void*)&V, (void*)&cert, (void*)&scert, (void*)&W, (void*)&H, (void*)&D, (void*)&zc,
                  (void*)&tx, (void*)&ty, (void*)&tz, (void*)&dst, (void*)&V};
  {
    const cudaError_t e0 = cudaLaunchKernel(smooth_kernel_of(variant), grid, dim3(kSmThreads), args,
                                            smooth_smem_bytes(cert != nullptr), st);
    if (e0 != cudaSuccess) return e0;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !alias) return e;
  if (accumulate) return add_volumes(out, out, tmp1, V * batch, st);
  return cudaMemcpyAsync(out, tmp1, bytes, cudaMemcpyDeviceToDevice, st);
}

}  // namespace brc
