// common.cuh -- shared definitions of the B200 registration/filtering kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace brc {

constexpr int kTaps = 343;          // 7 x 7 x 7
constexpr int kFilterFloats = 686;  // re[343] + im[343]
constexpr int kNParam = 12;
constexpr int kNSums = 42;          // 3 axes x (10 A sums + 4 h sums)
constexpr int kMaxFilters = 6;

// Filter bank passed to kernels by value (kernel parameter space).  Stored
// tap-major with the taps already reversed, so that coef[t][2k+c] is the
// weight that the sample at offset (dx,dy,dz) = (t%7-3, t/7%7-3, t/49-3)
// contributes to filter k's component c (0 re, 1 im): the reference's
// convolution uses F[(3-dx) + 7(3-dy) + 49(3-dz)] for that sample
// (kernelConvolution.cpp:2840-2858, broccoli_lib.cpp:5016-5017).
template <int NF>
struct FilterBank {
  float coef[kTaps * 2 * NF];
};

// The instances a kernel of the batched registration loop works on.  The
// loop keeps three lists of `stride` entries and their lengths; iteration
// it works on list it % 3, written by the solve of the previous iteration
// (instances whose update has not yet fallen below the tolerance).  The
// iteration is `it`, or *iter when iter is set (a device counter, so that
// one captured iteration serves every iteration of a graph's loop).  With
// list null: every instance 0 .. batch-1.
struct ActiveSet {
  const int* list;
  const int* count;
  const int* iter;
  int it;
  int stride;
};

inline ActiveSet all_instances() { return ActiveSet{nullptr, nullptr, nullptr, 0, 0}; }

__device__ __forceinline__ int active_iteration(const ActiveSet& a) { return a.iter ? *a.iter : a.it; }
__device__ __forceinline__ int active_count(const ActiveSet& a, int batch) {
  return a.list ? a.count[active_iteration(a) % 3] : batch;
}
__device__ __forceinline__ int active_instance(const ActiveSet& a, int i) {
  return a.list ? a.list[(active_iteration(a) % 3) * a.stride + i] : i;
}

// Four-quadrant arctangent of the phase kernels.  t = min(|x|,|y|) /
// max(|x|,|y|) with the hardware reciprocal (rcp.approx, about 1 ulp), atan(t)
// = t P(t^2) with P of degree 8 (a relative-error minimax fit made by
// broccoli_b200/fit_atan.py with Lawson's iteration, float32 relative error
// 1.4e-7 on [0, 1]), then pi/2 - r when |y| > |x|, pi - r when x < 0, and the sign
// of y.  Largest error about 2.5e-7 rad.  (0, 0) gives 0, and so does (+-0,
// -0), where atan2 gives +-pi; a larger magnitude below 2^-126 or from 2^126
// on gives a finite angle of lower accuracy.
__device__ __forceinline__ float phase_atan2(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  float rmx;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rmx) : "f"(fmaxf(mx, 1e-30f)));
  const float t = mn * rmx;
  const float s = t * t;
  float p = 2.849935787e-03f;
  p = fmaf(p, s, -1.606882550e-02f);
  p = fmaf(p, s, 4.269186407e-02f);
  p = fmaf(p, s, -7.504326850e-02f);
  p = fmaf(p, s, 1.064095125e-01f);
  p = fmaf(p, s, -1.420364976e-01f);
  p = fmaf(p, s, 1.999261975e-01f);
  p = fmaf(p, s, -3.333307207e-01f);
  p = fmaf(p, s, 1.0f);
  float r = p * t;
  r = ay > ax ? 1.57079632679489662f - r : r;
  r = x < 0.f ? 3.14159265358979324f - r : r;
  return copysignf(r, y);
}

// Square root by the hardware approximation (sqrt.approx, relative error
// about 2^-23); denormal inputs count as 0.
__device__ __forceinline__ float sqrt_approx(float v) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

// OpenCL 1.2 section 8.2 linear filtering with unnormalised coordinates and
// clamp-to-edge addressing, exact float weights (the sampler of
// kernelRegistration.cpp:1064).  u, v, w include the +0.5 texel offset.
__device__ __forceinline__ float sample_linear(const float* __restrict__ T, int W, int H, int D,
                                              float u, float v, float w) {
  // volumes hold fewer than 2^31 voxels (checked by the launchers)
  const float uu = u - 0.5f, vv = v - 0.5f, ww = w - 0.5f;
  const float fu = floorf(uu), fv = floorf(vv), fw = floorf(ww);
  const float a = uu - fu, bb = vv - fv, c = ww - fw;
  const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
  const int WH = W * H;
  float t000, t100, t010, t110, t001, t101, t011, t111;
  if ((unsigned)i0 < (unsigned)(W - 1) && (unsigned)j0 < (unsigned)(H - 1) && (unsigned)k0 < (unsigned)(D - 1)) {
    // all eight neighbours inside the volume (the clamps below leave them
    // as they are): one base address and constant offsets
    const float* p0 = T + (i0 + j0 * W + k0 * WH);
    const float* p1 = p0 + WH;
    t000 = __ldg(p0);
    t100 = __ldg(p0 + 1);
    t010 = __ldg(p0 + W);
    t110 = __ldg(p0 + W + 1);
    t001 = __ldg(p1);
    t101 = __ldg(p1 + 1);
    t011 = __ldg(p1 + W);
    t111 = __ldg(p1 + W + 1);
  } else {
    const int xi0 = min(max(i0, 0), W - 1), xi1 = min(max(i0 + 1, 0), W - 1);
    const int yj0 = min(max(j0, 0), H - 1), yj1 = min(max(j0 + 1, 0), H - 1);
    const int zk0 = min(max(k0, 0), D - 1), zk1 = min(max(k0 + 1, 0), D - 1);
    const int r00 = yj0 * W + zk0 * WH;
    const int r10 = yj1 * W + zk0 * WH;
    const int r01 = yj0 * W + zk1 * WH;
    const int r11 = yj1 * W + zk1 * WH;
    t000 = __ldg(T + xi0 + r00);
    t100 = __ldg(T + xi1 + r00);
    t010 = __ldg(T + xi0 + r10);
    t110 = __ldg(T + xi1 + r10);
    t001 = __ldg(T + xi0 + r01);
    t101 = __ldg(T + xi1 + r01);
    t011 = __ldg(T + xi0 + r11);
    t111 = __ldg(T + xi1 + r11);
  }
  // trilinear weights applied as seven linear interpolations
  const float c00 = fmaf(a, t100 - t000, t000), c10 = fmaf(a, t110 - t010, t010);
  const float c01 = fmaf(a, t101 - t001, t001), c11 = fmaf(a, t111 - t011, t011);
  const float c0 = fmaf(bb, c10 - c00, c00), c1 = fmaf(bb, c11 - c01, c01);
  return fmaf(c, c1 - c0, c0);
}

// The affine warp's sample of voxel (x, y, z): src at x + t + (A - I)(x -
// centre) with p = {t, A - I} (InterpolateVolumeLinearLinear,
// kernelRegistration.cpp:1066-1101).
__device__ __forceinline__ float affine_sample(const float* __restrict__ src, int W, int H, int D,
                                               const float* __restrict__ p, int x, int y, int z) {
  const float xf = (float)x - ((float)W - 1.0f) * 0.5f;
  const float yf = (float)y - ((float)H - 1.0f) * 0.5f;
  const float zf = (float)z - ((float)D - 1.0f) * 0.5f;
  const float u = (float)x + p[0] + p[3] * xf + p[4] * yf + p[5] * zf + 0.5f;
  const float v = (float)y + p[1] + p[6] * xf + p[7] * yf + p[8] * zf + 0.5f;
  const float w = (float)z + p[2] + p[9] * xf + p[10] * yf + p[11] * zf + 0.5f;
  return sample_linear(src, W, H, D, u, v, w);
}

}  // namespace brc
