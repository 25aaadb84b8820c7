// adjoint.cu -- adjoint (backward) kernels of the differentiable pieces of
// the path: the 7^3 complex filtering, the affine and displacement-field
// trilinear warps.  The separable smoothing is its own adjoint up to
// reversing the taps (smooth3d with reversed taps).
//
// Filtering: q_k(x) = sum_d V(x+d) W_k(d), W_k(d) = F_k[3-d].  With
// g_k = dL/dq_k (re, im as two real channels),
//   dL/dV(y) = sum_k sum_e [g_re,k(y+e) W_re,k(-e) + g_im,k(y+e) W_im,k(-e)],
// a correlation of the 2*NF gradient channels with the unflipped filters.
//
// Warps: out(x) = S(c(x)), c = x + t + (A-I)(x-centre) (affine) or x + u(x)
// (field); dL/dc(x) = g(x) grad S(c(x)) with the exact derivative of the
// clamp-to-edge trilinear interpolant, dL/du = dL/dc, dL/dp = sum_x dL/dc
// d c/d p, and dL/dS is scattered with atomics onto the 8 clamped corners.
#include "common.cuh"

namespace brc {

constexpr int kAdjTX = 32, kAdjTY = 8, kAdjTZ = 4, kAdjR = 8, kAdjRowPad = 44;
constexpr int kAdjThreads = (kAdjTX / kAdjR) * kAdjTY * kAdjTZ;  // 128

template <int NF>
struct AdjBank {
  float w[2 * NF][kTaps];  // channel c = 2k + (0 re, 1 im); index (ex+3) + 7(ey+3) + 49(ez+3)
};

template <int NF>
__global__ void __launch_bounds__(kAdjThreads)
filter3d_adjoint_kernel(const float* __restrict__ grad, int W, int H, int D,
                        const __grid_constant__ AdjBank<NF> bank, float* __restrict__ out) {
  constexpr int kRows = kAdjTY + 6, kSlices = kAdjTZ + 6;
  __shared__ __align__(16) float s_vol[kSlices * kRows * kAdjRowPad];
  __shared__ __align__(16) float s_w[kTaps];
  const int b = blockIdx.z;
  const int z_tiles = (D + kAdjTZ - 1) / kAdjTZ;
  const int tile_x0 = blockIdx.x * kAdjTX;
  const int tile_y0 = (blockIdx.y / z_tiles) * kAdjTY;
  const int tile_z0 = (blockIdx.y % z_tiles) * kAdjTZ;
  const long long V = (long long)W * H * D;
  const int tx = threadIdx.x % (kAdjTX / kAdjR);
  const int ty = (threadIdx.x / (kAdjTX / kAdjR)) % kAdjTY;
  const int tz = threadIdx.x / ((kAdjTX / kAdjR) * kAdjTY);
  float acc[kAdjR];
#pragma unroll
  for (int r = 0; r < kAdjR; r++) acc[r] = 0.f;

#pragma unroll 1
  for (int c = 0; c < 2 * NF; c++) {
    const float* g = grad + ((long long)b * NF + (c >> 1)) * 2 * V + (c & 1);
    __syncthreads();
    for (int i = threadIdx.x; i < kTaps; i += kAdjThreads) s_w[i] = bank.w[c][i];
    for (int i = threadIdx.x; i < kSlices * kRows * kAdjRowPad; i += kAdjThreads) {
      const int xs = i % kAdjRowPad, ys = (i / kAdjRowPad) % kRows, zs = i / (kAdjRowPad * kRows);
      const int x = tile_x0 - 4 + xs, y = tile_y0 - 3 + ys, z = tile_z0 - 3 + zs;
      float v = 0.f;
      if (x >= 0 && x < W && y >= 0 && y < H && z >= 0 && z < D)
        v = __ldg(g + 2 * (x + (long long)y * W + (long long)z * W * H));
      s_vol[i] = v;
    }
    __syncthreads();
#pragma unroll 1
    for (int dz = 0; dz < 7; dz++) {
#pragma unroll 1
      for (int dy = 0; dy < 7; dy++) {
        const float4* row = reinterpret_cast<const float4*>(
            s_vol + ((tz + dz) * kRows + (ty + dy)) * kAdjRowPad + kAdjR * tx);
        float d[16];
#pragma unroll
        for (int s = 0; s < 4; s++) {
          const float4 q = row[s];
          d[4 * s] = q.x;
          d[4 * s + 1] = q.y;
          d[4 * s + 2] = q.z;
          d[4 * s + 3] = q.w;
        }
        const float* wr = s_w + dy * 7 + dz * 49;
#pragma unroll
        for (int dx = 0; dx < 7; dx++) {
          const float w = wr[dx];
#pragma unroll
          for (int r = 0; r < kAdjR; r++) acc[r] = fmaf(d[1 + r + dx], w, acc[r]);
        }
      }
    }
  }
  const int x0 = tile_x0 + kAdjR * tx, y = tile_y0 + ty, z = tile_z0 + tz;
  if (y >= H || z >= D) return;
  float* o = out + (long long)b * V + x0 + (long long)y * W + (long long)z * W * H;
#pragma unroll
  for (int r = 0; r < kAdjR; r++)
    if (x0 + r < W) o[r] = acc[r];
}

// Value and gradient (d/du, d/dv, d/dw) of the clamp-to-edge trilinear
// interpolant at (u, v, w) (with the +0.5 texel convention).
__device__ __forceinline__ void sample_grad(const float* __restrict__ T, int W, int H, int D, float u, float v,
                                            float w, float& gx, float& gy, float& gz, long long* idx,
                                            float* wt) {
  const float uu = u - 0.5f, vv = v - 0.5f, ww = w - 0.5f;
  const float fu = floorf(uu), fv = floorf(vv), fw = floorf(ww);
  const float a = uu - fu, bb = vv - fv, c = ww - fw;
  const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
  const int xi0 = min(max(i0, 0), W - 1), xi1 = min(max(i0 + 1, 0), W - 1);
  const int yj0 = min(max(j0, 0), H - 1), yj1 = min(max(j0 + 1, 0), H - 1);
  const int zk0 = min(max(k0, 0), D - 1), zk1 = min(max(k0 + 1, 0), D - 1);
  const long long WH = (long long)W * H;
  idx[0] = xi0 + yj0 * (long long)W + zk0 * WH;
  idx[1] = xi1 + yj0 * (long long)W + zk0 * WH;
  idx[2] = xi0 + yj1 * (long long)W + zk0 * WH;
  idx[3] = xi1 + yj1 * (long long)W + zk0 * WH;
  idx[4] = xi0 + yj0 * (long long)W + zk1 * WH;
  idx[5] = xi1 + yj0 * (long long)W + zk1 * WH;
  idx[6] = xi0 + yj1 * (long long)W + zk1 * WH;
  idx[7] = xi1 + yj1 * (long long)W + zk1 * WH;
  float t[8];
#pragma unroll
  for (int k = 0; k < 8; k++) t[k] = __ldg(T + idx[k]);
  wt[0] = (1.f - a) * (1.f - bb) * (1.f - c);
  wt[1] = a * (1.f - bb) * (1.f - c);
  wt[2] = (1.f - a) * bb * (1.f - c);
  wt[3] = a * bb * (1.f - c);
  wt[4] = (1.f - a) * (1.f - bb) * c;
  wt[5] = a * (1.f - bb) * c;
  wt[6] = (1.f - a) * bb * c;
  wt[7] = a * bb * c;
  gx = (1.f - bb) * (1.f - c) * (t[1] - t[0]) + bb * (1.f - c) * (t[3] - t[2]) + (1.f - bb) * c * (t[5] - t[4]) +
       bb * c * (t[7] - t[6]);
  gy = (1.f - a) * (1.f - c) * (t[2] - t[0]) + a * (1.f - c) * (t[3] - t[1]) + (1.f - a) * c * (t[6] - t[4]) +
       a * c * (t[7] - t[5]);
  gz = (1.f - a) * (1.f - bb) * (t[4] - t[0]) + a * (1.f - bb) * (t[5] - t[1]) + (1.f - a) * bb * (t[6] - t[2]) +
       a * bb * (t[7] - t[3]);
}

constexpr int kWBThreads = 256;

// Affine warp backward: per-CTA FP64 partial sums of dL/dp (12 per
// instance) and, optionally, dL/dsrc scattered with atomics.
__global__ void __launch_bounds__(kWBThreads)
warp_affine_backward_kernel(const float* __restrict__ src, int W, int H, int D,
                            const float* __restrict__ params, const float* __restrict__ gout,
                            double* __restrict__ partials, float* __restrict__ gsrc) {
  const int b = blockIdx.y;
  const long long V = (long long)W * H * D;
  const float* S = src + (long long)b * V;
  const float* p = params + (long long)b * 12;
  double acc[12];
#pragma unroll
  for (int j = 0; j < 12; j++) acc[j] = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
    const float xf = (float)x - ((float)W - 1.0f) * 0.5f;
    const float yf = (float)y - ((float)H - 1.0f) * 0.5f;
    const float zf = (float)z - ((float)D - 1.0f) * 0.5f;
    const float u = (float)x + p[0] + p[3] * xf + p[4] * yf + p[5] * zf + 0.5f;
    const float v = (float)y + p[1] + p[6] * xf + p[7] * yf + p[8] * zf + 0.5f;
    const float w = (float)z + p[2] + p[9] * xf + p[10] * yf + p[11] * zf + 0.5f;
    float gx, gy, gz, wt[8];
    long long idx[8];
    sample_grad(S, W, H, D, u, v, w, gx, gy, gz, idx, wt);
    const float g = gout[(long long)b * V + i];
    const double cx = (double)g * gx, cy = (double)g * gy, cz = (double)g * gz;
    acc[0] += cx;
    acc[1] += cy;
    acc[2] += cz;
    acc[3] += cx * xf;
    acc[4] += cx * yf;
    acc[5] += cx * zf;
    acc[6] += cy * xf;
    acc[7] += cy * yf;
    acc[8] += cy * zf;
    acc[9] += cz * xf;
    acc[10] += cz * yf;
    acc[11] += cz * zf;
    if (gsrc != nullptr) {
      float* gs = gsrc + (long long)b * V;
#pragma unroll
      for (int k = 0; k < 8; k++) atomicAdd(gs + idx[k], g * wt[k]);
    }
  }
  __shared__ double red[kWBThreads / 32][12];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 12; j++) {
    double v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    double v = 0.0;
    for (int k = 0; k < kWBThreads / 32; k++) v += red[k][threadIdx.x];
    partials[((long long)b * gridDim.x + blockIdx.x) * 12 + threadIdx.x] = v;
  }
}

__global__ void reduce12_kernel(const double* __restrict__ partials, int nblk, double* __restrict__ out) {
  const int b = blockIdx.x, j = threadIdx.x;
  if (j >= 12) return;
  double v = 0.0;
  for (int r = 0; r < nblk; r++) v += partials[((long long)b * nblk + r) * 12 + j];
  out[(long long)b * 12 + j] = v;
}

// Field warp backward: dL/du per voxel and optionally dL/dsrc.
__global__ void __launch_bounds__(256)
warp_field_backward_kernel(const float* __restrict__ src, int W, int H, int D, const float* __restrict__ dx,
                           const float* __restrict__ dy, const float* __restrict__ dz,
                           const float* __restrict__ gout, float* __restrict__ gfield,
                           float* __restrict__ gsrc) {
  const long long V = (long long)W * H * D;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
  float gx, gy, gz, wt[8];
  long long idx[8];
  sample_grad(src, W, H, D, (float)x + dx[i] + 0.5f, (float)y + dy[i] + 0.5f, (float)z + dz[i] + 0.5f, gx, gy,
              gz, idx, wt);
  const float g = gout[i];
  if (gfield != nullptr) {
    gfield[i] = g * gx;
    gfield[V + i] = g * gy;
    gfield[2 * V + i] = g * gz;
  }
  if (gsrc != nullptr) {
#pragma unroll
    for (int k = 0; k < 8; k++) atomicAdd(gsrc + idx[k], g * wt[k]);
  }
}

// ---------------------------------------------------------------------------

template <int NF>
static cudaError_t launch_adjoint(const float* grad, int W, int H, int D, int batch, const float* h_filters,
                                  float* out, cudaStream_t st) {
  AdjBank<NF> bank;
  for (int k = 0; k < NF; k++)
    for (int c = 0; c < 2; c++)
      for (int ez = -3; ez <= 3; ez++)
        for (int ey = -3; ey <= 3; ey++)
          for (int ex = -3; ex <= 3; ex++)
            // weight W(-e) = F[3 + e]
            bank.w[2 * k + c][(ex + 3) + 7 * (ey + 3) + 49 * (ez + 3)] =
                h_filters[k * kFilterFloats + c * kTaps + (3 + ex) + 7 * (3 + ey) + 49 * (3 + ez)];
  const int z_tiles = (D + kAdjTZ - 1) / kAdjTZ;
  dim3 grid((W + kAdjTX - 1) / kAdjTX, ((H + kAdjTY - 1) / kAdjTY) * z_tiles, batch);
  filter3d_adjoint_kernel<NF><<<grid, kAdjThreads, 0, st>>>(grad, W, H, D, bank, out);
  return cudaGetLastError();
}

cudaError_t filter3d_adjoint(const float* grad, int W, int H, int D, int batch, const float* h_filters, int nfilt,
                             float* out, cudaStream_t st) {
  if (nfilt == 3) return launch_adjoint<3>(grad, W, H, D, batch, h_filters, out, st);
  if (nfilt == 6) return launch_adjoint<6>(grad, W, H, D, batch, h_filters, out, st);
  return cudaErrorInvalidValue;
}

int warp_affine_backward_blocks(long long V) {
  long long n = (V + kWBThreads - 1) / kWBThreads;
  return (int)(n < 148 * 4 ? n : 148 * 4);
}

cudaError_t warp_affine_backward(const float* src, int W, int H, int D, int batch, const float* params,
                                 const float* gout, double* partials, int nblk, double* gparams, float* gsrc,
                                 cudaStream_t st) {
  dim3 grid(nblk, batch);
  warp_affine_backward_kernel<<<grid, kWBThreads, 0, st>>>(src, W, H, D, params, gout, partials, gsrc);
  reduce12_kernel<<<batch, 32, 0, st>>>(partials, nblk, gparams);
  return cudaGetLastError();
}

cudaError_t warp_field_backward(const float* src, int W, int H, int D, const float* dx, const float* dy,
                                const float* dz, const float* gout, float* gfield, float* gsrc,
                                cudaStream_t st) {
  const long long V = (long long)W * H * D;
  warp_field_backward_kernel<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(src, W, H, D, dx, dy, dz, gout,
                                                                          gfield, gsrc);
  return cudaGetLastError();
}

}  // namespace brc
