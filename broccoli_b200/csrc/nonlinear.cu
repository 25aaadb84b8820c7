// nonlinear.cu -- per-voxel kernels of the nonlinear (displacement field)
// registration step, and the small helpers of the multi-scale drivers.
//
// One nonlinear iteration on the device (AlignTwoVolumesNonLinear,
// broccoli_lib.cpp:5748-6058), every arrow one launch:
//   filter3d<6> (+ fused structure tensor T = sum_k |q2_k| M_k)
//   -> smooth T (6 volumes, one batched launch per pass)
//   -> tensor_norm_max: |T| into a11 (the reference leaves it there) and the
//      global max into a device scalar (no host round trip)
//   -> nonlinear_ah: T scaled by 1/max, a += c TT, h += c dphi TT n for the
//      six filter pairs in registers (one pass instead of six)
//   -> smooth a, h (9 volumes)
//   -> displacement_update (3x3 per voxel, FP32 cofactors as the reference or
//      FP64 elimination)
//   -> smooth update, accumulated into the field by the last pass
//   -> warp_field
#include <math.h>

#include "common.cuh"

namespace brc {

struct NonlinearConsts {
  float m[6][6];    // projection tensor of filter k: m11 m12 m13 m22 m23 m33
  float dir[3][6];  // filter directions: x[6], y[6], z[6]
};

// |T| (Frobenius, symmetric) into a11 and the volume maximum into *maxbits
// (float bits of a non-negative value, so unsigned ordering is float
// ordering).  CalculateTensorNorms (kernelRegistration.cpp:847-875) and
// CalculateMax (broccoli_lib.cpp:10889-10928).
__global__ void __launch_bounds__(256)
tensor_norm_max_kernel(const float* __restrict__ t6, long long V, float* __restrict__ a11,
                       unsigned int* __restrict__ maxbits, long long t_stride, long long a_stride) {
  // instance blockIdx.y: its tensor, norm volume and maximum
  t6 += (long long)blockIdx.y * t_stride;
  a11 += (long long)blockIdx.y * a_stride;
  maxbits += blockIdx.y;
  float mx = 0.f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
       i += (long long)gridDim.x * blockDim.x) {
    const float a = t6[i], b = t6[V + i], c = t6[2 * V + i], d = t6[3 * V + i], e = t6[4 * V + i],
                f = t6[5 * V + i];
    const float n = sqrtf(a * a + 2.0f * b * b + 2.0f * c * c + d * d + 2.0f * e * e + f * f);
    a11[i] = n;
    mx = fmaxf(mx, n);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ float s[8];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmaxf(mx, s[w]);
    atomicMax(maxbits, __float_as_uint(mx));
  }
}

// a (6) and h (3) from the six filter pairs, T scaled by 1/max first; a11
// starts from the tensor norm already stored there.
// CalculateAMatricesAndHVectors, kernelRegistration.cpp:880-943.
__global__ void __launch_bounds__(256)
nonlinear_ah_kernel(const float2* __restrict__ q1, const float2* __restrict__ q2,
                    float* __restrict__ t6, long long V, const unsigned int* __restrict__ maxbits,
                    NonlinearConsts cst, float* __restrict__ a6, float* __restrict__ h3, long long ah_stride) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  // instance blockIdx.y (q1, the reference's responses, is shared): q2 6
  // complex volumes, t6 6 volumes, a6 / h3 ah_stride floats apart
  const int b = blockIdx.y;
  q2 += (long long)b * 6 * V;
  t6 += (long long)b * 6 * V;
  maxbits += b;
  a6 += (long long)b * ah_stride;
  h3 += (long long)b * ah_stride;
  const float mx = fmaxf(__uint_as_float(*maxbits), 1.17549435e-38f);
  const float f = 1.0f / mx;
  const float t11 = t6[i] * f, t12 = t6[V + i] * f, t13 = t6[2 * V + i] * f;
  const float t22 = t6[3 * V + i] * f, t23 = t6[4 * V + i] * f, t33 = t6[5 * V + i] * f;
  const float tt11 = t11 * t11 + t12 * t12 + t13 * t13;
  const float tt12 = t11 * t12 + t12 * t22 + t13 * t23;
  const float tt13 = t11 * t13 + t12 * t23 + t13 * t33;
  const float tt22 = t12 * t12 + t22 * t22 + t23 * t23;
  const float tt23 = t12 * t13 + t22 * t23 + t23 * t33;
  const float tt33 = t13 * t13 + t23 * t23 + t33 * t33;
  float a11 = a6[i], a12 = 0.f, a13 = 0.f, a22 = 0.f, a23 = 0.f, a33 = 0.f;
  float h1 = 0.f, h2 = 0.f, h3v = 0.f;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const float2 a = __ldg(q1 + k * V + i), c = __ldg(q2 + k * V + i);
    const float qr = __fadd_rn(__fmul_rn(a.x, c.x), __fmul_rn(a.y, c.y));
    const float qi = __fadd_rn(-__fmul_rn(a.x, c.y), __fmul_rn(a.y, c.x));
    const float pd = phase_atan2(qi, qr);
    // sqrt|q1 q2*| cos^2(pd/2) with cos^2(pd/2) = (1 + qr/|q1 q2*|)/2
    const float aqq = sqrt_approx(qr * qr + qi * qi);
    const float cert = aqq > 0.f ? 0.5f * (aqq + qr) * rsqrtf(aqq) : 0.f;
    a11 += cert * tt11;
    a12 += cert * tt12;
    a13 += cert * tt13;
    a22 += cert * tt22;
    a23 += cert * tt23;
    a33 += cert * tt33;
    const float cp = cert * pd;
    const float nx = cst.dir[0][k], ny = cst.dir[1][k], nz = cst.dir[2][k];
    h1 += cp * (nx * tt11 + ny * tt12 + nz * tt13);
    h2 += cp * (nx * tt12 + ny * tt22 + nz * tt23);
    h3v += cp * (nx * tt13 + ny * tt23 + nz * tt33);
  }
  a6[i] = a11;
  a6[V + i] = a12;
  a6[2 * V + i] = a13;
  a6[3 * V + i] = a22;
  a6[4 * V + i] = a23;
  a6[5 * V + i] = a33;
  h3[i] = h1;
  h3[V + i] = h2;
  h3[2 * V + i] = h3v;
  // the scaled tensor is what the reference keeps (MultiplyVolume in place)
  t6[i] = t11;
  t6[V + i] = t12;
  t6[2 * V + i] = t13;
  t6[3 * V + i] = t22;
  t6[4 * V + i] = t23;
  t6[5 * V + i] = t33;
}

// d = A^-1 h per voxel.  fp64 = 0: cofactors in FP32 with det + 1e-16f
// (CalculateDisplacementUpdate, kernelRegistration.cpp:948-988); fp64 = 1:
// the same regularised cofactor solve, det + 1e-16, in FP64 (a non-finite
// inverse gives d = 0).
__global__ void __launch_bounds__(256)
displacement_update_kernel(const float* __restrict__ a6, const float* __restrict__ h3, long long V,
                           int fp64, float* __restrict__ d3, long long ah_stride) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  // instance blockIdx.y: a6 / h3 ah_stride floats apart, d3 3 volumes
  a6 += (long long)blockIdx.y * ah_stride;
  h3 += (long long)blockIdx.y * ah_stride;
  d3 += (long long)blockIdx.y * 3 * V;
  if (!fp64) {
    const float a11 = a6[i], a12 = a6[V + i], a13 = a6[2 * V + i], a22 = a6[3 * V + i],
                a23 = a6[4 * V + i], a33 = a6[5 * V + i];
    const float h1 = h3[i], h2 = h3[V + i], hh3 = h3[2 * V + i];
    const float norm = 1.0f / (a11 * a22 * a33 - a11 * a23 * a23 - a12 * a12 * a33 + a12 * a23 * a13 +
                               a13 * a12 * a23 - a13 * a22 * a13 + 1e-16f);
    d3[i] = norm * ((hh3 * (a12 * a23 - a13 * a22)) - (h2 * (a12 * a33 - a13 * a23)) +
                    (h1 * (a22 * a33 - a23 * a23)));
    d3[V + i] = norm * ((h2 * (a11 * a33 - a13 * a13)) - (hh3 * (a11 * a23 - a13 * a12)) -
                        (h1 * (a12 * a33 - a23 * a13)));
    d3[2 * V + i] = norm * ((hh3 * (a11 * a22 - a12 * a12)) - (h2 * (a11 * a23 - a12 * a13)) +
                            (h1 * (a12 * a23 - a22 * a13)));
  } else {
    const double a11 = a6[i], a12 = a6[V + i], a13 = a6[2 * V + i], a22 = a6[3 * V + i],
                 a23 = a6[4 * V + i], a33 = a6[5 * V + i];
    const double h1 = h3[i], h2 = h3[V + i], hh3 = h3[2 * V + i];
    const double c11 = a22 * a33 - a23 * a23, c12 = a13 * a23 - a12 * a33, c13 = a12 * a23 - a13 * a22;
    const double c22 = a11 * a33 - a13 * a13, c23 = a12 * a13 - a11 * a23, c33 = a11 * a22 - a12 * a12;
    // the reference's regularised inverse, det + 1e-16, evaluated in double:
    // in near-singular (background) voxels the 1e-16 damps the update, and
    // the exact inverse there would be a different algorithm
    const double det = a11 * c11 + a12 * c12 + a13 * c13;
    const double r = 1.0 / (det + 1e-16);
    if (!isfinite(r)) {
      d3[i] = 0.f;
      d3[V + i] = 0.f;
      d3[2 * V + i] = 0.f;
      return;
    }
    d3[i] = (float)(r * (c11 * h1 + c12 * h2 + c13 * hh3));
    d3[V + i] = (float)(r * (c12 * h1 + c22 * h2 + c23 * hh3));
    d3[2 * V + i] = (float)(r * (c13 * h1 + c23 * h2 + c33 * hh3));
  }
}

// Structure tensor from six complex responses (used when the filter kernel
// did not fuse it): T = sum_k |q2_k| M_k (CalculateTensorComponents,
// kernelRegistration.cpp:806-845, accumulated over k = 0..5).
__global__ void __launch_bounds__(256)
tensor_components_kernel(const float2* __restrict__ q2, long long V, NonlinearConsts cst,
                         float* __restrict__ t6) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  // instance blockIdx.y: 6 complex responses in, 6 tensor volumes out
  q2 += (long long)blockIdx.y * 6 * V;
  t6 += (long long)blockIdx.y * 6 * V;
  float t[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const float2 q = __ldg(q2 + k * V + i);
    const float mag = sqrtf(q.x * q.x + q.y * q.y);
#pragma unroll
    for (int c = 0; c < 6; c++) t[c] += mag * cst.m[k][c];
  }
#pragma unroll
  for (int c = 0; c < 6; c++) t6[c * V + i] = t[c];
}

// Linear resample of `batch` volumes to a new size, scaled by `factor`
// (ChangeVolumeSize, broccoli_lib.cpp:6247-6388, followed by MultiplyVolume
// for displacement fields, :6604-6611).
__device__ __forceinline__ float sample_lin(const float* __restrict__ T, int W, int H, int D,
                                            float u, float v, float w) {
  const float uu = u - 0.5f, vv = v - 0.5f, ww = w - 0.5f;
  const float fu = floorf(uu), fv = floorf(vv), fw = floorf(ww);
  const float a = uu - fu, bb = vv - fv, c = ww - fw;
  const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
  const int xi0 = min(max(i0, 0), W - 1), xi1 = min(max(i0 + 1, 0), W - 1);
  const int yj0 = min(max(j0, 0), H - 1), yj1 = min(max(j0 + 1, 0), H - 1);
  const int zk0 = min(max(k0, 0), D - 1), zk1 = min(max(k0 + 1, 0), D - 1);
  const long long r00 = (long long)yj0 * W + (long long)zk0 * W * H;
  const long long r10 = (long long)yj1 * W + (long long)zk0 * W * H;
  const long long r01 = (long long)yj0 * W + (long long)zk1 * W * H;
  const long long r11 = (long long)yj1 * W + (long long)zk1 * W * H;
  return (1.f - a) * (1.f - bb) * (1.f - c) * __ldg(T + xi0 + r00) +
         a * (1.f - bb) * (1.f - c) * __ldg(T + xi1 + r00) +
         (1.f - a) * bb * (1.f - c) * __ldg(T + xi0 + r10) + a * bb * (1.f - c) * __ldg(T + xi1 + r10) +
         (1.f - a) * (1.f - bb) * c * __ldg(T + xi0 + r01) + a * (1.f - bb) * c * __ldg(T + xi1 + r01) +
         (1.f - a) * bb * c * __ldg(T + xi0 + r11) + a * bb * c * __ldg(T + xi1 + r11);
}

__global__ void __launch_bounds__(256)
rescale_batch_kernel(const float* __restrict__ src, int W, int H, int D, float* __restrict__ out, int W2,
                     int H2, int D2, float vx, float vy, float vz, float factor) {
  const int b = blockIdx.y;
  const long long V2 = (long long)W2 * H2 * D2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V2) return;
  const int x = (int)(i % W2), y = (int)((i / W2) % H2), z = (int)(i / ((long long)W2 * H2));
  const float v = sample_lin(src + (long long)b * W * H * D, W, H, D, x * vx + 0.5f, y * vy + 0.5f,
                             z * vz + 0.5f);
  out[(long long)b * V2 + i] = factor == 1.0f ? v : v * factor;
}

// Total = New * Old per instance with translations scaled by tscale (2 for
// the next pyramid scale) (AddAffineRegistrationParameters[NextScale],
// broccoli_lib.cpp:7252-7431), rounded to float as the reference does.
__global__ void compose_kernel(float* __restrict__ total, const float* __restrict__ add, int batch,
                               float tscale) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  float* o = total + 12 * b;
  const float* n = add + 12 * b;
  double O[16], N[16];
  const float* src[2] = {o, n};
  double* dst[2] = {O, N};
  for (int m = 0; m < 2; m++) {
    const float* p = src[m];
    double* M = dst[m];
    M[0] = (double)(p[3] + 1.0f); M[1] = (double)p[4]; M[2] = (double)p[5];
    M[3] = tscale == 1.0f ? (double)p[0] : (double)(p[0] * tscale);
    M[4] = (double)p[6]; M[5] = (double)(p[7] + 1.0f); M[6] = (double)p[8];
    M[7] = tscale == 1.0f ? (double)p[1] : (double)(p[1] * tscale);
    M[8] = (double)p[9]; M[9] = (double)p[10]; M[10] = (double)(p[11] + 1.0f);
    M[11] = tscale == 1.0f ? (double)p[2] : (double)(p[2] * tscale);
    M[12] = 0; M[13] = 0; M[14] = 0; M[15] = 1;
  }
  double T[16];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0;
      for (int k = 0; k < 4; k++) s += N[i * 4 + k] * O[k * 4 + j];
      T[i * 4 + j] = s;
    }
  o[0] = (float)T[3]; o[1] = (float)T[7]; o[2] = (float)T[11];
  o[3] = (float)(T[0] - 1.0); o[4] = (float)T[1]; o[5] = (float)T[2];
  o[6] = (float)T[4]; o[7] = (float)(T[5] - 1.0); o[8] = (float)T[6];
  o[9] = (float)T[8]; o[10] = (float)T[9]; o[11] = (float)(T[10] - 1.0);
}

// out = a + b elementwise (AddVolumes, kernelMisc.cpp:383-400).
__global__ void __launch_bounds__(256)
add_kernel(float* __restrict__ out, const float* __restrict__ a, const float* __restrict__ b, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

// Resample to new voxel sizes and centre in / crop to a new grid in one pass:
// new(xn) = interp(xi) where xi is xn shifted by the centring offsets (and
// mm_z_cut along z) and interp is the linear resample with spacing
// (N-1)/(Ni-1); uncovered voxels are 0.  ChangeVolumesResolutionAndSize,
// broccoli_lib.cpp:6950-7100, fusing RescaleVolumeLinear and
// CopyVolumeToNew (kernelRegistration.cpp:1340-1366, :1593-1678).
struct ResizeGeom {
  int Wi, Hi, Di;     // interpolated size
  int offn[3];        // added to the loop index to get the new-grid index
  int offi[3];        // added to the loop index to get the interpolated index
  float vd[3];        // (N-1)/(Ni-1)
};

__global__ void __launch_bounds__(256)
resize_to_grid_kernel(const float* __restrict__ src, int W, int H, int D, float* __restrict__ out, int W2,
                      int H2, int D2, ResizeGeom g) {
  const long long V2 = (long long)W2 * H2 * D2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V2) return;
  const int xn = (int)(i % W2), yn = (int)((i / W2) % H2), zn = (int)(i / ((long long)W2 * H2));
  const int x = xn - g.offn[0], y = yn - g.offn[1], z = zn - g.offn[2];
  const int xi = x + g.offi[0], yi = y + g.offi[1], zi = z + g.offi[2];
  float v = 0.f;
  if (x >= 0 && y >= 0 && z >= 0 && xi >= 0 && yi >= 0 && zi >= 0 && xi < g.Wi && yi < g.Hi && zi < g.Di)
    v = sample_lin(src, W, H, D, xi * g.vd[0] + 0.5f, yi * g.vd[1] + 0.5f, zi * g.vd[2] + 0.5f);
  out[i] = v;
}

// One subject of a ragged batch: its own source volume and size, resampled
// onto the shared new grid (same arithmetic as resize_to_grid_kernel).
struct ResizeJob {
  const float* src;
  int W, H, D;
  ResizeGeom g;
};

__global__ void __launch_bounds__(256)
resize_to_grid_ragged_kernel(const ResizeJob* __restrict__ jobs, float* __restrict__ out, int W2, int H2,
                             int D2) {
  const long long V2 = (long long)W2 * H2 * D2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V2) return;
  const ResizeJob& j = jobs[blockIdx.y];
  const int xn = (int)(i % W2), yn = (int)((i / W2) % H2), zn = (int)(i / ((long long)W2 * H2));
  const int x = xn - j.g.offn[0], y = yn - j.g.offn[1], z = zn - j.g.offn[2];
  const int xi = x + j.g.offi[0], yi = y + j.g.offi[1], zi = z + j.g.offi[2];
  float v = 0.f;
  if (x >= 0 && y >= 0 && z >= 0 && xi >= 0 && yi >= 0 && zi >= 0 && xi < j.g.Wi && yi < j.g.Hi && zi < j.g.Di)
    v = sample_lin(j.src, j.W, j.H, j.D, xi * j.g.vd[0] + 0.5f, yi * j.g.vd[1] + 0.5f, zi * j.g.vd[2] + 0.5f);
  out[(long long)blockIdx.y * V2 + i] = v;
}

// Sums of m, m x, m y, m z over the volume in FP64 (centre of mass;
// CalculateCenterOfMass, broccoli_lib.cpp:6763-6800, accumulates in float
// on the host after a full device-to-host copy).
__global__ void __launch_bounds__(256)
mass_moments_kernel(const float* __restrict__ vol, int W, int H, int D, double* __restrict__ sums) {
  const long long V = (long long)W * H * D;
  double m = 0, mx = 0, my = 0, mz = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = vol[i];
    const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
    m += v;
    mx += v * x;
    my += v * y;
    mz += v * z;
  }
  double s[4] = {m, mx, my, mz};
  __shared__ double red[8][4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_down_sync(0xffffffffu, s[k], o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = s[k];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w][threadIdx.x];
    atomicAdd(sums + threadIdx.x, t);
  }
}

// field += t + (A - I)(x - c) (AddLinearAndNonLinearDisplacement,
// kernelRegistration.cpp:1142-1178).
struct Params12 {
  float p[12];
};

__global__ void __launch_bounds__(256)
add_affine_to_field_kernel(float* __restrict__ field, int W, int H, int D, Params12 prm) {
  const long long V = (long long)W * H * D;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
  const float* p = prm.p;
  const float xf = (float)x - ((float)W - 1.0f) * 0.5f;
  const float yf = (float)y - ((float)H - 1.0f) * 0.5f;
  const float zf = (float)z - ((float)D - 1.0f) * 0.5f;
  field[i] += p[0] + p[3] * xf + p[4] * yf + p[5] * zf;
  field[V + i] += p[1] + p[6] * xf + p[7] * yf + p[8] * zf;
  field[2 * V + i] += p[2] + p[9] * xf + p[10] * yf + p[11] * zf;
}

// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Transforms of 4D data with NEAREST (0) or LINEAR (1) interpolation
// (TransformVolumesLinear / NonLinear, broccoli_lib.cpp:8267-8451,
// ChangeVolumesResolutionAndSize :6950-7100, CreateCombinedDisplacementField
// :8115-8143).  Coordinates and weights are computed in the reference's
// operation order with every product and sum rounded (no contraction into
// FMAs), so that nearest sampling picks the reference's voxel and linear
// sampling reproduces its arithmetic.
// ---------------------------------------------------------------------------

// OpenCL 1.2 section 8.2 nearest filtering, unnormalised coordinates,
// clamp-to-edge: i = floor(u) (volume_sampler_nearest,
// kernelRegistration.cpp:992).
__device__ __forceinline__ float sample_near(const float* __restrict__ T, int W, int H, int D, float u, float v,
                                             float w) {
  const int i = min(max((int)floorf(u), 0), W - 1);
  const int j = min(max((int)floorf(v), 0), H - 1);
  const int k = min(max((int)floorf(w), 0), D - 1);
  return __ldg(T + i + (long long)j * W + (long long)k * W * H);
}

// Linear filtering with the 8 weights formed and summed as in the
// reference's sampler, each operation rounded.
__device__ __forceinline__ float sample_lin_exact(const float* __restrict__ T, int W, int H, int D, float u,
                                                  float v, float w) {
  const float uu = __fsub_rn(u, 0.5f), vv = __fsub_rn(v, 0.5f), ww = __fsub_rn(w, 0.5f);
  const float fu = floorf(uu), fv = floorf(vv), fw = floorf(ww);
  const float a = __fsub_rn(uu, fu), b = __fsub_rn(vv, fv), c = __fsub_rn(ww, fw);
  const float a0 = __fsub_rn(1.f, a), b0 = __fsub_rn(1.f, b), c0 = __fsub_rn(1.f, c);
  const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
  const int x0 = min(max(i0, 0), W - 1), x1 = min(max(i0 + 1, 0), W - 1);
  const int y0 = min(max(j0, 0), H - 1), y1 = min(max(j0 + 1, 0), H - 1);
  const int z0 = min(max(k0, 0), D - 1), z1 = min(max(k0 + 1, 0), D - 1);
  const long long WH = (long long)W * H;
#define TX(i, j, k) __ldg(T + (i) + (long long)(j) * W + (long long)(k) * WH)
  float r = __fmul_rn(__fmul_rn(__fmul_rn(a0, b0), c0), TX(x0, y0, z0));
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(__fmul_rn(a, b0), c0), TX(x1, y0, z0)));
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(__fmul_rn(a0, b), c0), TX(x0, y1, z0)));
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(__fmul_rn(a, b), c0), TX(x1, y1, z0)));
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(__fmul_rn(a0, b0), c), TX(x0, y0, z1)));
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(__fmul_rn(a, b0), c), TX(x1, y0, z1)));
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(__fmul_rn(a0, b), c), TX(x0, y1, z1)));
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(__fmul_rn(a, b), c), TX(x1, y1, z1)));
#undef TX
  return r;
}

template <int MODE>
__device__ __forceinline__ float sample_mode(const float* __restrict__ T, int W, int H, int D, float u, float v,
                                             float w) {
  return MODE == 0 ? sample_near(T, W, H, D, u, v, w) : sample_lin_exact(T, W, H, D, u, v, w);
}

// pos + t + a xf + b yf + c zf, left to right, each operation rounded
__device__ __forceinline__ float affine_sum(float pos, float t, float a, float b, float c, float xf, float yf,
                                            float zf) {
  float r = __fadd_rn(pos, t);
  r = __fadd_rn(r, __fmul_rn(a, xf));
  r = __fadd_rn(r, __fmul_rn(b, yf));
  return __fadd_rn(r, __fmul_rn(c, zf));
}

// Volume t = blockIdx.y of the batch: out_t(x) = src_t(x + t + (A - I)(x - c))
// (InterpolateVolumeNearestLinear / LinearLinear, kernelRegistration.cpp:
// 995-1031, :1066-1101).
template <int MODE>
__global__ void __launch_bounds__(256)
transform_affine_kernel(const float* __restrict__ src, int W, int H, int D, Params12 prm,
                        float* __restrict__ out) {
  const long long V = (long long)W * H * D;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
  const float* p = prm.p;
  const float xf = (float)x - ((float)W - 1.0f) * 0.5f;
  const float yf = (float)y - ((float)H - 1.0f) * 0.5f;
  const float zf = (float)z - ((float)D - 1.0f) * 0.5f;
  const float u = __fadd_rn(affine_sum((float)x, p[0], p[3], p[4], p[5], xf, yf, zf), 0.5f);
  const float v = __fadd_rn(affine_sum((float)y, p[1], p[6], p[7], p[8], xf, yf, zf), 0.5f);
  const float w = __fadd_rn(affine_sum((float)z, p[2], p[9], p[10], p[11], xf, yf, zf), 0.5f);
  const long long t = blockIdx.y;
  out[t * V + i] = sample_mode<MODE>(src + t * V, W, H, D, u, v, w);
}

// Volume t = blockIdx.y warped by one displacement field
// (InterpolateVolumeNearestNonLinear / LinearNonLinear,
// kernelRegistration.cpp:1032-1061, :1111-1140).
template <int MODE>
__global__ void __launch_bounds__(256)
transform_field_kernel(const float* __restrict__ src, int W, int H, int D, const float* __restrict__ dx,
                       const float* __restrict__ dy, const float* __restrict__ dz, float* __restrict__ out) {
  const long long V = (long long)W * H * D;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
  const float u = __fadd_rn(__fadd_rn((float)x, __ldg(dx + i)), 0.5f);
  const float v = __fadd_rn(__fadd_rn((float)y, __ldg(dy + i)), 0.5f);
  const float w = __fadd_rn(__fadd_rn((float)z, __ldg(dz + i)), 0.5f);
  const long long t = blockIdx.y;
  out[t * V + i] = sample_mode<MODE>(src + t * V, W, H, D, u, v, w);
}

// (dx, dy, dz) += t + (A - I)(x - c) (AddLinearAndNonLinearDisplacement,
// kernelRegistration.cpp:1142-1178), each operation rounded.
__global__ void __launch_bounds__(256)
combine_field_kernel(float* __restrict__ dx, float* __restrict__ dy, float* __restrict__ dz, int W, int H, int D,
                     Params12 prm) {
  const long long V = (long long)W * H * D;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
  const float* p = prm.p;
  const float xf = (float)x - ((float)W - 1.0f) * 0.5f;
  const float yf = (float)y - ((float)H - 1.0f) * 0.5f;
  const float zf = (float)z - ((float)D - 1.0f) * 0.5f;
  dx[i] = __fadd_rn(dx[i], affine_sum(p[0], 0.f, p[3], p[4], p[5], xf, yf, zf));
  dy[i] = __fadd_rn(dy[i], affine_sum(p[1], 0.f, p[6], p[7], p[8], xf, yf, zf));
  dz[i] = __fadd_rn(dz[i], affine_sum(p[2], 0.f, p[9], p[10], p[11], xf, yf, zf));
}

// Volume t = blockIdx.y of a batch resampled as resize_to_grid_kernel does,
// with NEAREST (0) or LINEAR (1) interpolation and the reference's rounding
// (RescaleVolumeNearest / Linear, kernelRegistration.cpp:1312-1366, then
// CopyVolumeToNew, :1593-1678).
template <int MODE>
__global__ void __launch_bounds__(256)
resize_to_grid_mode_kernel(const float* __restrict__ src, int W, int H, int D, float* __restrict__ out, int W2,
                           int H2, int D2, ResizeGeom g) {
  const long long V2 = (long long)W2 * H2 * D2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V2) return;
  const long long t = blockIdx.y;
  const int xn = (int)(i % W2), yn = (int)((i / W2) % H2), zn = (int)(i / ((long long)W2 * H2));
  const int x = xn - g.offn[0], y = yn - g.offn[1], z = zn - g.offn[2];
  const int xi = x + g.offi[0], yi = y + g.offi[1], zi = z + g.offi[2];
  float v = 0.f;
  if (x >= 0 && y >= 0 && z >= 0 && xi >= 0 && yi >= 0 && zi >= 0 && xi < g.Wi && yi < g.Hi && zi < g.Di)
    v = sample_mode<MODE>(src + t * W * H * D, W, H, D, __fadd_rn(__fmul_rn((float)xi, g.vd[0]), 0.5f),
                          __fadd_rn(__fmul_rn((float)yi, g.vd[1]), 0.5f),
                          __fadd_rn(__fmul_rn((float)zi, g.vd[2]), 0.5f));
  out[t * V2 + i] = v;
}

static unsigned grid1(long long n) { return (unsigned)((n + 255) / 256); }

static int round_half_away(float v) { return (int)roundf(v); }

// Geometry of ChangeVolumesResolutionAndSize for one volume; false if the
// interpolated size is below 2 voxels along an axis.
static bool resize_geom(int W, int H, int D, float vx, float vy, float vz, int W2, int H2, int D2, float nvx,
                        float nvy, float nvz, int mm_z_cut, ResizeGeom& g) {
  g.Wi = (int)floorf((float)W * vx / nvx + 0.5f);
  g.Hi = (int)floorf((float)H * vy / nvy + 0.5f);
  g.Di = (int)floorf((float)D * vz / nvz + 0.5f);
  if (g.Wi < 2 || g.Hi < 2 || g.Di < 2) return false;
  const int diff[3] = {g.Wi - W2, g.Hi - H2, g.Di - D2};
  const int zcut = (int)round((float)mm_z_cut / nvz);
  for (int a = 0; a < 3; a++) {
    const int half = round_half_away((float)(diff[a] > 0 ? diff[a] : -diff[a]) / 2.0f);
    if (diff[a] > 0) {
      g.offn[a] = 0;
      g.offi[a] = half;
    } else {
      g.offn[a] = half;
      g.offi[a] = 0;
    }
  }
  g.offi[2] += zcut;
  g.vd[0] = (float)(W - 1) / (float)(g.Wi - 1);
  g.vd[1] = (float)(H - 1) / (float)(g.Hi - 1);
  g.vd[2] = (float)(D - 1) / (float)(g.Di - 1);
  return true;
}

cudaError_t resize_to_grid(const float* src, int W, int H, int D, float vx, float vy, float vz, float* out,
                           int W2, int H2, int D2, float nvx, float nvy, float nvz, int mm_z_cut,
                           cudaStream_t st) {
  ResizeGeom g;
  if (!resize_geom(W, H, D, vx, vy, vz, W2, H2, D2, nvx, nvy, nvz, mm_z_cut, g)) return cudaErrorInvalidValue;
  resize_to_grid_kernel<<<grid1((long long)W2 * H2 * D2), 256, 0, st>>>(src, W, H, D, out, W2, H2, D2, g);
  return cudaGetLastError();
}

cudaError_t resize_to_grid_batch(const float* src, int W, int H, int D, int T, float vx, float vy, float vz,
                                 float* out, int W2, int H2, int D2, float nvx, float nvy, float nvz, int mm_z_cut,
                                 int interp, cudaStream_t st) {
  ResizeGeom g;
  if (T <= 0 || T > 65535 || (interp != 0 && interp != 1)) return cudaErrorInvalidValue;
  if (!resize_geom(W, H, D, vx, vy, vz, W2, H2, D2, nvx, nvy, nvz, mm_z_cut, g)) return cudaErrorInvalidValue;
  const dim3 grid(grid1((long long)W2 * H2 * D2), (unsigned)T);
  if (interp == 0)
    resize_to_grid_mode_kernel<0><<<grid, 256, 0, st>>>(src, W, H, D, out, W2, H2, D2, g);
  else
    resize_to_grid_mode_kernel<1><<<grid, 256, 0, st>>>(src, W, H, D, out, W2, H2, D2, g);
  return cudaGetLastError();
}

cudaError_t transform_affine(const float* src, int W, int H, int D, int T, const float* p12, int interp,
                             float* out, cudaStream_t st) {
  if (T <= 0 || T > 65535 || (interp != 0 && interp != 1)) return cudaErrorInvalidValue;
  Params12 prm;
  for (int i = 0; i < 12; i++) prm.p[i] = p12[i];
  const dim3 grid(grid1((long long)W * H * D), (unsigned)T);
  if (interp == 0)
    transform_affine_kernel<0><<<grid, 256, 0, st>>>(src, W, H, D, prm, out);
  else
    transform_affine_kernel<1><<<grid, 256, 0, st>>>(src, W, H, D, prm, out);
  return cudaGetLastError();
}

cudaError_t transform_field(const float* src, int W, int H, int D, int T, const float* dx, const float* dy,
                            const float* dz, int interp, float* out, cudaStream_t st) {
  if (T <= 0 || T > 65535 || (interp != 0 && interp != 1)) return cudaErrorInvalidValue;
  const dim3 grid(grid1((long long)W * H * D), (unsigned)T);
  if (interp == 0)
    transform_field_kernel<0><<<grid, 256, 0, st>>>(src, W, H, D, dx, dy, dz, out);
  else
    transform_field_kernel<1><<<grid, 256, 0, st>>>(src, W, H, D, dx, dy, dz, out);
  return cudaGetLastError();
}

cudaError_t combine_field(float* dx, float* dy, float* dz, int W, int H, int D, const float* p12, cudaStream_t st) {
  Params12 prm;
  for (int i = 0; i < 12; i++) prm.p[i] = p12[i];
  combine_field_kernel<<<grid1((long long)W * H * D), 256, 0, st>>>(dx, dy, dz, W, H, D, prm);
  return cudaGetLastError();
}

size_t resize_job_bytes() { return sizeof(ResizeJob); }

cudaError_t resize_to_grid_ragged(int n, const float* const* srcs, const int* dims3n, const float* vox3n,
                                  void* h_jobs, void* d_jobs, float* out, int W2, int H2, int D2,
                                  const float* new_vox3, int mm_z_cut, cudaStream_t st) {
  ResizeJob* jobs = static_cast<ResizeJob*>(h_jobs);
  for (int b = 0; b < n; b++) {
    ResizeJob& j = jobs[b];
    j.src = srcs[b];
    j.W = dims3n[3 * b];
    j.H = dims3n[3 * b + 1];
    j.D = dims3n[3 * b + 2];
    if (!resize_geom(j.W, j.H, j.D, vox3n[3 * b], vox3n[3 * b + 1], vox3n[3 * b + 2], W2, H2, D2, new_vox3[0],
                     new_vox3[1], new_vox3[2], mm_z_cut, j.g))
      return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaMemcpyAsync(d_jobs, jobs, sizeof(ResizeJob) * n, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  dim3 grid(grid1((long long)W2 * H2 * D2), n);
  resize_to_grid_ragged_kernel<<<grid, 256, 0, st>>>(static_cast<const ResizeJob*>(d_jobs), out, W2, H2, D2);
  return cudaGetLastError();
}

cudaError_t mass_moments(const float* vol, int W, int H, int D, double* sums, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(sums, 0, 4 * sizeof(double), st);
  if (e != cudaSuccess) return e;
  long long blocks = ((long long)W * H * D + 255) / 256;
  if (blocks > 148 * 4) blocks = 148 * 4;
  mass_moments_kernel<<<(unsigned)blocks, 256, 0, st>>>(vol, W, H, D, sums);
  return cudaGetLastError();
}

cudaError_t add_affine_to_field(float* field, int W, int H, int D, const float* p12, cudaStream_t st) {
  Params12 prm;
  for (int i = 0; i < 12; i++) prm.p[i] = p12[i];
  add_affine_to_field_kernel<<<grid1((long long)W * H * D), 256, 0, st>>>(field, W, H, D, prm);
  return cudaGetLastError();
}

cudaError_t tensor_norm_max(const float* t6, long long V, float* a11, unsigned int* maxbits, cudaStream_t st,
                            int batch, long long t_stride, long long a_stride) {
  if (batch <= 0 || batch > 65535) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(maxbits, 0, sizeof(unsigned int) * batch, st);
  if (e != cudaSuccess) return e;
  long long blocks = (V + 255) / 256;
  const long long cap = (148 * 8 + batch - 1) / batch;
  if (blocks > cap) blocks = cap;
  tensor_norm_max_kernel<<<dim3((unsigned)blocks, (unsigned)batch), 256, 0, st>>>(t6, V, a11, maxbits, t_stride,
                                                                                  a_stride);
  return cudaGetLastError();
}

cudaError_t nonlinear_ah(const float* q1, const float* q2, float* t6, long long V, const unsigned int* maxbits,
                         const float* m36, const float* dirs18, float* a6, float* h3, cudaStream_t st, int batch,
                         long long ah_stride) {
  if (batch <= 0 || batch > 65535) return cudaErrorInvalidValue;
  NonlinearConsts c;
  for (int k = 0; k < 6; k++)
    for (int j = 0; j < 6; j++) c.m[k][j] = m36[6 * k + j];
  for (int a = 0; a < 3; a++)
    for (int k = 0; k < 6; k++) c.dir[a][k] = dirs18[6 * a + k];
  nonlinear_ah_kernel<<<dim3(grid1(V), (unsigned)batch), 256, 0, st>>>(reinterpret_cast<const float2*>(q1),
                                                                        reinterpret_cast<const float2*>(q2), t6, V,
                                                                        maxbits, c, a6, h3, ah_stride);
  return cudaGetLastError();
}

cudaError_t tensor_components(const float* q2, long long V, const float* m36, float* t6, cudaStream_t st,
                              int batch) {
  if (batch <= 0 || batch > 65535) return cudaErrorInvalidValue;
  NonlinearConsts c;
  for (int k = 0; k < 6; k++)
    for (int j = 0; j < 6; j++) c.m[k][j] = m36[6 * k + j];
  tensor_components_kernel<<<dim3(grid1(V), (unsigned)batch), 256, 0, st>>>(reinterpret_cast<const float2*>(q2),
                                                                             V, c, t6);
  return cudaGetLastError();
}

cudaError_t displacement_update(const float* a6, const float* h3, long long V, int fp64, float* d3,
                                cudaStream_t st, int batch, long long ah_stride) {
  if (batch <= 0 || batch > 65535) return cudaErrorInvalidValue;
  displacement_update_kernel<<<dim3(grid1(V), (unsigned)batch), 256, 0, st>>>(a6, h3, V, fp64, d3, ah_stride);
  return cudaGetLastError();
}

cudaError_t rescale_batch(const float* src, int W, int H, int D, int batch, float* out, int W2, int H2,
                          int D2, float factor, cudaStream_t st) {
  const float vx = (float)(W - 1) / (float)(W2 - 1);
  const float vy = (float)(H - 1) / (float)(H2 - 1);
  const float vz = (float)(D - 1) / (float)(D2 - 1);
  dim3 grid(grid1((long long)W2 * H2 * D2), batch);
  rescale_batch_kernel<<<grid, 256, 0, st>>>(src, W, H, D, out, W2, H2, D2, vx, vy, vz, factor);
  return cudaGetLastError();
}

cudaError_t compose(float* total, const float* add, int batch, float tscale, cudaStream_t st) {
  compose_kernel<<<(batch + 63) / 64, 64, 0, st>>>(total, add, batch, tscale);
  return cudaGetLastError();
}

cudaError_t add_volumes(float* out, const float* a, const float* b, long long n, cudaStream_t st) {
  add_kernel<<<grid1(n), 256, 0, st>>>(out, a, b, n);
  return cudaGetLastError();
}

}  // namespace brc
