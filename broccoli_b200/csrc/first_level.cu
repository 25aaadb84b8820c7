// first_level.cu -- the preprocessing stages of a first-level fMRI analysis
// on the C-ABI: Gaussian filters from a FWHM, tensor magnitudes, the EPI
// brain mask, and the chain of registrations, motion correction and
// normalised smoothing that runs before the statistics.  Host code plus
// the three small kernels of the mask; the registrations and resampling
// run on the kernels of filter3d*.cu / registration.cu / nonlinear.cu
// through the library's own entry points.
#include <math.h>
#include <string.h>

#include <utility>
#include <vector>

#include "../../include/broccoli_b200.h"
#include "capi_ctx.h"
#include "common.cuh"
#include "internal.h"

namespace {

// Sum over x of every (y, z) row in x order, one thread per row
// (CalculateColumnSums, kernelMisc.cpp:193-212).  The serial order keeps
// the float sum identical to the reference's; the volume is read once.
__global__ void __launch_bounds__(128) column_sums_kernel(const float* __restrict__ vol, int W, int rows,
                                                          float* __restrict__ sums) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float* p = vol + (long long)r * W;
  float s = 0.0f;
  for (int x = 0; x < W; x++) s += p[x];
  sums[r] = s;
}

// Sum over y of the row sums of every plane (CalculateRowSums,
// kernelMisc.cpp:214-231).
__global__ void __launch_bounds__(128) row_sums_kernel(const float* __restrict__ colsums, int H, int D,
                                                       float* __restrict__ sums) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= D) return;
  float s = 0.0f;
  for (int y = 0; y < H; y++) s += colsums[y + (long long)z * H];
  sums[z] = s;
}

// 1 above the threshold, 0.001 elsewhere (ThresholdVolume,
// kernelMisc.cpp:305-327).
__global__ void __launch_bounds__(256) threshold_kernel(const float* __restrict__ vol, long long V, float thr,
                                                        float* __restrict__ mask) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < V) mask[i] = vol[i] > thr ? 1.0f : 0.001f;
}

int myround(float a) { return (int)floorf(a + 0.5f); }

bool bad_size(int W, int H, int D) { return W <= 0 || H <= 0 || D <= 0; }

}  // namespace

#define FL_TRY(expr)            \
  do {                          \
    const int _st = (expr);     \
    if (_st != BRC_OK) return _st; \
  } while (0)

extern "C" void brc_smoothing_filters_fwhm(float fwhm, const float* vox, float* fx, float* fy, float* fz) {
  if (!vox || !fx || !fy || !fz) return;
  float* f[3] = {fx, fy, fz};
  for (int a = 0; a < 3; a++) {
    const double sigma = (double)fwhm / 2.354 / (double)vox[a];
    const double s2 = 2.0 * sigma * sigma;
    float sum = 0.0f;
    for (int i = 0; i < 9; i++) {
      const double u = (double)(i - 4);
      f[a][i] = (float)exp(-pow(u, 2.0) / s2);
      sum += f[a][i];
    }
    for (int i = 0; i < 9; i++) f[a][i] /= sum;
  }
}

extern "C" int brc_tensor_magnitude(brc_ctx* ctx, const float* d_vol, int W, int H, int D, const float* h_filters6,
                                    const float* h_tensors, int precision, float* d_out) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_vol || !h_filters6 || !h_tensors || !d_out || bad_size(W, H, D))
    return ctx->fail(BRC_ERR_INVALID, "brc_tensor_magnitude: bad argument");
  if (!brc_precision_valid(precision))
    return ctx->fail(BRC_ERR_UNSUPPORTED, "brc_tensor_magnitude: unknown precision");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream();
  const long long V = (long long)W * H * D;
  DevBuf q, t;
  BRC_TRY(ctx, q.ensure(sizeof(float) * 12 * V), "alloc");
  BRC_TRY(ctx, t.ensure(sizeof(float) * 6 * V + 64), "alloc");
  FilterPath fp;
  FL_TRY(make_filter_path(ctx, h_filters6, 6, precision, W, H, D, &fp));
  BRC_TRY(ctx, run_filter(fp, d_vol, W, H, D, 1, V, q.as<float>(), brc::all_instances(), st), "filter");
  float* t6 = t.as<float>();
  BRC_TRY(ctx, brc::tensor_components(q.as<float>(), V, h_tensors, t6, st), "tensor_components");
  BRC_TRY(ctx, brc::tensor_norm_max(t6, V, d_out, reinterpret_cast<unsigned int*>(t6 + 6 * V), st),
          "tensor_norm");
  ctx->launches += filter_launches(fp) + 2;
  // the temporaries are freed when this returns: finish with them first
  BRC_TRY(ctx, cudaStreamSynchronize(st), "sync");
  return BRC_OK;
}

extern "C" int brc_segment_epi(brc_ctx* ctx, const float* d_vol, int W, int H, int D, const float* voxel_size3,
                               float* d_mask) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_vol || !voxel_size3 || !d_mask || bad_size(W, H, D) || d_vol == d_mask)
    return ctx->fail(BRC_ERR_INVALID, "brc_segment_epi: bad argument");
  for (int a = 0; a < 3; a++)
    if (!(voxel_size3[a] > 0))
      return ctx->fail(BRC_ERR_INVALID, "brc_segment_epi: voxel sizes must be positive");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream();
  const long long V = (long long)W * H * D;
  const int rows = H * D;
  DevBuf sm, sums;
  BRC_TRY(ctx, sm.ensure(sizeof(float) * V), "alloc");
  BRC_TRY(ctx, sums.ensure(sizeof(float) * ((size_t)rows + D)), "alloc");
  float fx[9], fy[9], fz[9];
  brc_smoothing_filters_fwhm(4.0f, voxel_size3, fx, fy, fz);
  FL_TRY(brc_smooth3d(ctx, d_vol, W, H, D, 1, fx, fy, fz, nullptr, nullptr, sm.as<float>()));
  float* colsums = sums.as<float>();
  float* zsums = colsums + rows;
  column_sums_kernel<<<(rows + 127) / 128, 128, 0, st>>>(sm.as<float>(), W, rows, colsums);
  BRC_TRY(ctx, cudaGetLastError(), "column_sums");
  row_sums_kernel<<<(D + 127) / 128, 128, 0, st>>>(colsums, H, D, zsums);
  BRC_TRY(ctx, cudaGetLastError(), "row_sums");
  std::vector<float> hz(D);
  BRC_TRY(ctx, cudaMemcpyAsync(hz.data(), zsums, sizeof(float) * D, cudaMemcpyDeviceToHost, st), "D2H");
  BRC_TRY(ctx, cudaStreamSynchronize(st), "sync");
  float sum = 0.0f;
  for (int z = 0; z < D; z++) sum += hz[z];
  const float thr = 0.9f * sum / ((float)W * (float)H * (float)D);
  threshold_kernel<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(sm.as<float>(), V, thr, d_mask);
  BRC_TRY(ctx, cudaGetLastError(), "threshold");
  ctx->launches += 3;
  BRC_TRY(ctx, cudaStreamSynchronize(st), "sync");
  return BRC_OK;
}

extern "C" void brc_first_level_opts_default(brc_first_level_opts* o) {
  if (!o) return;
  o->linear_iterations = 10;
  o->nonlinear_iterations = 10;
  o->motion_iterations = 5;
  o->coarsest_scale_t1_mni = 4;
  o->coarsest_scale_epi_t1 = 4;
  o->mm_t1_z_cut = 0;
  o->apply_motion_correction = 1;
  o->apply_smoothing = 1;
  o->smoothing_fwhm = 6.0f;
  o->tsigma = 5.0f;
  o->esigma = 5.0f;
  o->dsigma = 5.0f;
  o->precision = BRC_PREC_FP32;
  o->solve_fp64 = 0;
}

namespace {

// Device helpers of the chain; every call returns a brc status.
struct Chain {
  brc_ctx* ctx;
  int precision;

  int get(float* h, const float* d, long long n) {
    return h ? brc_copy_to_host(ctx, h, d, sizeof(float) * (size_t)n) : BRC_OK;
  }
  int copy(float* dst, const float* src, long long n) {
    BRC_TRY(ctx, cudaMemcpyAsync(dst, src, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream()),
            "copy");
    return BRC_OK;
  }
  // CenterVolumeMass (broccoli_lib.cpp:6802-6837): integer translation of
  // the centre of mass to the grid centre, LINEAR resampling.
  int center(const float* src, int W, int H, int D, float* out) {
    return brc_center_volumes(ctx, src, W, H, D, 1, BRC_INTERP_LINEAR, out, nullptr);
  }
  // MatchVolumeMasses (broccoli_lib.cpp:6914-6948): v1 moved in place by
  // the rounded difference of the centres of mass; tmp is scratch.
  int match(float* v1, const float* v2, int W, int H, int D, float* tmp, float* p12) {
    float c1[3], c2[3];
    FL_TRY(brc_center_of_mass(ctx, v1, W, H, D, c1));
    FL_TRY(brc_center_of_mass(ctx, v2, W, H, D, c2));
    for (int i = 0; i < 12; i++) p12[i] = 0.0f;
    for (int k = 0; k < 3; k++) p12[k] = -(float)myround(c2[k] - c1[k]);
    FL_TRY(brc_transform_volumes_linear(ctx, v1, W, H, D, 1, p12, BRC_INTERP_LINEAR, tmp));
    return copy(v1, tmp, (long long)W * H * D);
  }
  // AlignTwoVolumesLinearSeveralScales with DO_OVERWRITE
  // (broccoli_lib.cpp:6391-6513): *moving is replaced by its aligned copy
  // (the buffers *moving and *spare swap).
  int scales(const float* ref, float** moving, float** spare, int W, int H, int D, const float* filters3,
             int iterations, int coarsest, int type, float* dparams, float* p12) {
    brc_linear_opts lo;
    brc_linear_opts_default(&lo, iterations);
    lo.type = type;
    lo.precision = precision;
    FL_TRY(brc_register_linear_scales(ctx, ref, *moving, W, H, D, 1, filters3, &lo, coarsest, dparams, *spare,
                                      nullptr));
    std::swap(*moving, *spare);
    return brc_copy_to_host(ctx, p12, dparams, sizeof(float) * 12);
  }
  // TransformVolumesLinear in place, LINEAR (broccoli_lib.cpp:8276-8330).
  int transform(float** vol, float** spare, int W, int H, int D, const float* p12) {
    FL_TRY(brc_transform_volumes_linear(ctx, *vol, W, H, D, 1, p12, BRC_INTERP_LINEAR, *spare));
    std::swap(*vol, *spare);
    return BRC_OK;
  }
};

struct Buffers {
  std::vector<DevBuf> b;
  explicit Buffers(size_t n) : b(n) {}
  float* f(size_t i) const { return b[i].as<float>(); }
};

}  // namespace

extern "C" int brc_first_level_preprocess(brc_ctx* ctx, const brc_first_level_input* in,
                                          const brc_first_level_opts* o, const brc_first_level_output* out) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!in || !o || !out || !in->fmri || !in->t1 || !in->mni || !in->filters3 ||
      bad_size(in->epi_w, in->epi_h, in->epi_d) || in->epi_t <= 0 || in->epi_t > 65535 ||
      bad_size(in->t1_w, in->t1_h, in->t1_d) || bad_size(in->mni_w, in->mni_h, in->mni_d) ||
      o->linear_iterations < 0 || o->nonlinear_iterations < 0 || o->motion_iterations < 0 ||
      o->coarsest_scale_t1_mni < 1 || o->coarsest_scale_epi_t1 < 1)
    return ctx->fail(BRC_ERR_INVALID, "brc_first_level_preprocess: bad argument");
  if (o->nonlinear_iterations > 0 && (!in->filters6 || !in->tensors || !in->dirs))
    return ctx->fail(BRC_ERR_INVALID, "brc_first_level_preprocess: the nonlinear stage needs its filters");
  if (!in->filters6 || !in->tensors)
    return ctx->fail(BRC_ERR_INVALID, "brc_first_level_preprocess: tensor magnitudes need the nonlinear filters");
  if (o->apply_smoothing && !(o->smoothing_fwhm > 0))
    return ctx->fail(BRC_ERR_INVALID, "brc_first_level_preprocess: smoothing FWHM must be positive");
  for (int a = 0; a < 3; a++)
    if (!(in->epi_voxel[a] > 0) || !(in->t1_voxel[a] > 0) || !(in->mni_voxel[a] > 0))
      return ctx->fail(BRC_ERR_INVALID, "brc_first_level_preprocess: voxel sizes must be positive");
  cudaSetDevice(ctx->device);
  const int W1 = in->epi_w, H1 = in->epi_h, D1 = in->epi_d, T = in->epi_t;
  const int W2 = in->t1_w, H2 = in->t1_h, D2 = in->t1_d;
  const int W3 = in->mni_w, H3 = in->mni_h, D3 = in->mni_d;
  const long long V1 = (long long)W1 * H1 * D1, V2 = (long long)W2 * H2 * D2, V3 = (long long)W3 * H3 * D3;
  Chain c{ctx, o->precision};
  // device volumes: template (0), resampled T1 (1), its skull-stripped copy
  // (2), template-size scratch (3, 4), field (5), EPI (6, 7), T1 (8), T1-size
  // EPI, tensor magnitudes and scratch (9-12), parameters (13)
  Buffers m(14);
  const size_t sizes[14] = {(size_t)V3, (size_t)V3, (size_t)V3, (size_t)V3, (size_t)V3, 3 * (size_t)V3,
                            (size_t)V1, (size_t)V1, (size_t)V2, (size_t)V2, (size_t)V2, (size_t)V2,
                            (size_t)V2, 16};
  for (int i = 0; i < 14; i++) BRC_TRY(ctx, m.b[i].ensure(sizeof(float) * sizes[i]), "alloc");
  float *mni = m.f(0), *mni_t1 = m.f(1), *skull = m.f(2), *s3a = m.f(3), *s3b = m.f(4), *field = m.f(5);
  float *epi0 = m.f(6), *epic = m.f(7), *t1 = m.f(8), *s2a = m.f(9), *tm_epi = m.f(10), *tm_t1 = m.f(11);
  float *s2b = m.f(12), *dp = m.f(13);
  FL_TRY(brc_copy_to_device(ctx, mni, in->mni, sizeof(float) * V3));
  FL_TRY(brc_copy_to_device(ctx, t1, in->t1, sizeof(float) * V2));
  FL_TRY(brc_copy_to_device(ctx, epi0, in->fmri, sizeof(float) * V1));
  const float* f3 = in->filters3;
  const int lin = o->linear_iterations;

  // ---- T1 to template: PerformRegistrationT1MNINoSkullstrip, :8226-8273
  float start_t1_mni[12], p_t1_mni[12], total[12];
  FL_TRY(c.center(t1, W2, H2, D2, s2a));
  FL_TRY(brc_change_resolution_and_size(ctx, s2a, W2, H2, D2, in->t1_voxel, mni_t1, W3, H3, D3, in->mni_voxel,
                                        o->mm_t1_z_cut));
  FL_TRY(c.match(mni_t1, mni, W3, H3, D3, s3a, start_t1_mni));
  FL_TRY(c.copy(skull, mni_t1, V3));
  FL_TRY(c.get(out->interpolated_t1, skull, V3));
  FL_TRY(c.scales(mni, &mni_t1, &s3a, W3, H3, D3, f3, lin, o->coarsest_scale_t1_mni, BRC_AFFINE, dp, p_t1_mni));
  FL_TRY(c.get(out->aligned_t1_linear, mni_t1, V3));
  const bool nonlinear = o->nonlinear_iterations > 0;
  if (nonlinear) {
    brc_nonlinear_opts no;
    brc_nonlinear_opts_default(&no, o->nonlinear_iterations);
    no.coarsest_scale = o->coarsest_scale_t1_mni;
    no.tsigma = o->tsigma;
    no.esigma = o->esigma;
    no.dsigma = o->dsigma;
    no.precision = o->precision;
    no.solve_fp64 = o->solve_fp64;
    FL_TRY(brc_register_nonlinear(ctx, mni, mni_t1, W3, H3, D3, in->filters6, in->tensors, in->dirs, &no, field,
                                  s3a));
    FL_TRY(c.get(out->aligned_t1_nonlinear, s3a, V3));
    FL_TRY(c.get(out->field, field, 3 * V3));
  }
  brc::host_add_affine(p_t1_mni, start_t1_mni, total);  // :8510
  if (out->params_t1_mni) memcpy(out->params_t1_mni, total, sizeof(total));

  // ---- first EPI volume to the resampled T1 on the template grid:
  // PerformRegistrationEPIT1, :7853-7915 (t1_epi in mni_t1's buffer)
  float start_epi_t1[12], p_epi_t1[12], epi_t1_out[12];
  float* t1_epi = mni_t1;
  FL_TRY(c.center(epi0, W1, H1, D1, epic));
  FL_TRY(brc_change_resolution_and_size(ctx, epic, W1, H1, D1, in->epi_voxel, t1_epi, W3, H3, D3, in->mni_voxel, 0));
  FL_TRY(c.match(t1_epi, skull, W3, H3, D3, s3a, start_epi_t1));
  FL_TRY(c.scales(skull, &t1_epi, &s3a, W3, H3, D3, f3, lin, o->coarsest_scale_epi_t1, BRC_AFFINE, dp, p_epi_t1));
  FL_TRY(c.get(out->aligned_epi_t1, t1_epi, V3));
  // through the T1's transforms to the template, :8544-8556
  FL_TRY(c.transform(&t1_epi, &s3a, W3, H3, D3, p_t1_mni));
  FL_TRY(c.get(out->aligned_epi_mni_linear, t1_epi, V3));
  if (nonlinear && out->aligned_epi_mni_nonlinear) {
    FL_TRY(brc_transform_volumes_nonlinear(ctx, t1_epi, W3, H3, D3, 1, field, field + V3, field + 2 * V3,
                                           BRC_INTERP_LINEAR, s3b));
    FL_TRY(c.get(out->aligned_epi_mni_nonlinear, s3b, V3));
  }
  brc::host_add_affine(p_epi_t1, start_epi_t1, epi_t1_out);  // :8574-8575
  brc::host_add_affine(p_t1_mni, epi_t1_out, total);
  if (out->params_epi_mni) memcpy(out->params_epi_mni, total, sizeof(total));

  // ---- first EPI volume to the original T1: PerformRegistrationEPIT1Original,
  // :7917-7970 (the volumes first, then their tensor magnitudes)
  float start_o[12], p[12], aff[12] = {0};
  float* t1_epi_o = s2a;
  FL_TRY(brc_change_resolution_and_size(ctx, epi0, W1, H1, D1, in->epi_voxel, t1_epi_o, W2, H2, D2, in->t1_voxel,
                                        0));
  FL_TRY(c.match(t1_epi_o, t1, W2, H2, D2, s2b, start_o));
  FL_TRY(brc_tensor_magnitude(ctx, t1_epi_o, W2, H2, D2, in->filters6, in->tensors, o->precision, tm_epi));
  FL_TRY(brc_tensor_magnitude(ctx, t1, W2, H2, D2, in->filters6, in->tensors, o->precision, tm_t1));
  const int cs = o->coarsest_scale_epi_t1 * 2;
  for (int type : {BRC_TRANSLATION, BRC_RIGID}) {
    FL_TRY(c.scales(t1, &t1_epi_o, &s2b, W2, H2, D2, f3, lin, cs, type, dp, p));
    FL_TRY(c.transform(&tm_epi, &s2b, W2, H2, D2, p));
    brc::host_add_affine(aff, p, aff);
  }
  for (int type : {BRC_RIGID, BRC_AFFINE}) {
    FL_TRY(c.scales(tm_t1, &tm_epi, &s2b, W2, H2, D2, f3, lin, 2, type, dp, p));
    FL_TRY(c.transform(&t1_epi_o, &s2b, W2, H2, D2, p));
    brc::host_add_affine(aff, p, aff);
  }
  brc::host_add_affine(aff, start_o, total);  // :8601
  if (out->params_epi_t1) memcpy(out->params_epi_t1, total, sizeof(total));

  // ---- motion correction of the series in place (PerformMotionCorrectionHost,
  // :10723-10787)
  if (o->apply_motion_correction) {
    brc_linear_opts lo;
    brc_linear_opts_default(&lo, o->motion_iterations);
    lo.type = BRC_RIGID;
    lo.precision = o->precision;
    FL_TRY(brc_motion_correct(ctx, in->fmri, W1, H1, D1, T, in->epi_voxel, f3, &lo, nullptr,
                              out->motion_parameters));
    if (out->motion_corrected) memcpy(out->motion_corrected, in->fmri, sizeof(float) * (size_t)V1 * T);
  }

  // ---- EPI mask of the first (corrected) volume, :8683-8701
  FL_TRY(brc_copy_to_device(ctx, epi0, in->fmri, sizeof(float) * V1));
  FL_TRY(brc_segment_epi(ctx, epi0, W1, H1, D1, in->epi_voxel, epic));
  FL_TRY(c.get(out->epi_mask, epic, V1));

  // ---- normalised smoothing of the series with the mask
  // (PerformSmoothingNormalizedHost, :11628-11727), :8703-8733
  if (o->apply_smoothing) {
    float fx[9], fy[9], fz[9];
    brc_smoothing_filters_fwhm(o->smoothing_fwhm, in->epi_voxel, fx, fy, fz);
    DevBuf vols;
    BRC_TRY(ctx, vols.ensure(sizeof(float) * 2 * (size_t)V1 * T), "alloc");
    float* dv = vols.as<float>();
    FL_TRY(brc_copy_to_device(ctx, dv, in->fmri, sizeof(float) * (size_t)V1 * T));
    FL_TRY(brc_smooth_normalized(ctx, dv, W1, H1, D1, T, epic, fx, fy, fz, dv + V1 * T));
    FL_TRY(brc_copy_to_host(ctx, in->fmri, dv + V1 * T, sizeof(float) * (size_t)V1 * T));
    if (out->smoothed) memcpy(out->smoothed, in->fmri, sizeof(float) * (size_t)V1 * T);
  }
  BRC_TRY(ctx, cudaStreamSynchronize(ctx->stream()), "sync");
  return BRC_OK;
}
