// clshim.hpp -- just enough of OpenCL C, in C++, to compile the reference's
// kernel sources (code/Kernels/kernelConvolution.cpp and
// kernelRegistration.cpp of BROCCOLI) for the CPU.  TEST INFRASTRUCTURE ONLY:
// it exists so that oracle/_ref can run the reference's own kernel code as a
// cross-check of the C restatement in orc_impl.h.
//
// Work-items run one after another (no barriers); only kernels without
// __local memory or barriers are ever called.  The NDRange position of the
// current work-item lives in thread-local state set by the driver.
#pragma once
#include <cmath>
#include <cstdlib>

using std::atan2;
using std::cos;
using std::fabs;
using std::floor;
using std::round;
using std::sqrt;

#define __kernel
#define __global
#define __private
#define __constant const
#define __local
#define read_only
#define barrier(x) ((void)0)
#define CLK_LOCAL_MEM_FENCE 0
#define CLK_GLOBAL_MEM_FENCE 0

struct NDRangeState {
  int gid[3], lid[3], grp[3], lsz[3];
};
static thread_local NDRangeState g_ndr;
static inline int get_global_id(int d) { return g_ndr.gid[d]; }
static inline int get_local_id(int d) { return g_ndr.lid[d]; }
static inline int get_group_id(int d) { return g_ndr.grp[d]; }
static inline int get_local_size(int d) { return g_ndr.lsz[d]; }

struct float2 {
  float x, y;
  float2& operator+=(const float2& o) {
    x += o.x;
    y += o.y;
    return *this;
  }
};
static inline float2 make_float2(float a, float b) { return float2{a, b}; }

struct float3 {
  float x, y, z;
};
static inline float3 operator-(float3 a, float b) { return float3{a.x - b, a.y - b, a.z - b}; }
static inline float3 operator+(float3 a, float b) { return float3{a.x + b, a.y + b, a.z + b}; }
static inline float3 operator-(float3 a, float3 b) { return float3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline float3 floor(float3 a) { return float3{std::floor(a.x), std::floor(a.y), std::floor(a.z)}; }

struct float4 {
  float x, y, z, w;
};
static inline float4 make_float4(float a, float b, float c, float d) { return float4{a, b, c, d}; }

struct int3 {
  int x, y, z;
};

// Images: a dense float volume.  Samplers are the CLK_* flag words.
typedef int sampler_t;
#define CLK_NORMALIZED_COORDS_FALSE 0
#define CLK_ADDRESS_CLAMP_TO_EDGE 2
#define CLK_FILTER_NEAREST 0
#define CLK_FILTER_LINEAR 16

struct image3d_t {
  const float* data;
  int W, H, D;
};

static inline float img_texel(const image3d_t& im, int i, int j, int k) {
  i = i < 0 ? 0 : (i > im.W - 1 ? im.W - 1 : i);
  j = j < 0 ? 0 : (j > im.H - 1 ? im.H - 1 : j);
  k = k < 0 ? 0 : (k > im.D - 1 ? im.D - 1 : k);
  return im.data[i + (long)j * im.W + (long)k * im.W * im.H];
}

// OpenCL 1.2 section 8.2 filtering with unnormalised coordinates and
// CLK_ADDRESS_CLAMP_TO_EDGE, exact (not fixed-point) weights.
static inline float4 read_imagef(const image3d_t& im, sampler_t s, float4 c) {
  if (s & CLK_FILTER_LINEAR) {
    const float u = c.x - 0.5f, v = c.y - 0.5f, w = c.z - 0.5f;
    const float fu = std::floor(u), fv = std::floor(v), fw = std::floor(w);
    const float a = u - fu, b = v - fv, cc = w - fw;
    const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
    const int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
    const float r = (1 - a) * (1 - b) * (1 - cc) * img_texel(im, i0, j0, k0) +
                    a * (1 - b) * (1 - cc) * img_texel(im, i1, j0, k0) +
                    (1 - a) * b * (1 - cc) * img_texel(im, i0, j1, k0) +
                    a * b * (1 - cc) * img_texel(im, i1, j1, k0) +
                    (1 - a) * (1 - b) * cc * img_texel(im, i0, j0, k1) +
                    a * (1 - b) * cc * img_texel(im, i1, j0, k1) +
                    (1 - a) * b * cc * img_texel(im, i0, j1, k1) +
                    a * b * cc * img_texel(im, i1, j1, k1);
    return float4{r, 0.f, 0.f, 1.f};
  }
  const int i = (int)std::floor(c.x), j = (int)std::floor(c.y), k = (int)std::floor(c.z);
  return float4{img_texel(im, i, j, k), 0.f, 0.f, 1.f};
}
