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

// The instances a kernel of the batched registration loop works on: the
// first *count entries of list, written by the solve of the previous
// iteration (instances whose update has not yet fallen below the
// tolerance), or every instance 0 .. batch-1 when list is null.
struct ActiveSet {
  const int* list;
  const int* count;
};

inline ActiveSet all_instances() { return ActiveSet{nullptr, nullptr}; }

__device__ __forceinline__ int active_count(const ActiveSet& a, int batch) { return a.list ? *a.count : batch; }
__device__ __forceinline__ int active_instance(const ActiveSet& a, int i) { return a.list ? a.list[i] : i; }

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

}  // namespace brc
