// drivers.cu -- multi-step entry points of the C-ABI: one nonlinear update
// step, single- and multi-scale nonlinear registration, and multi-scale
// (pyramid) linear registration.  Host code: it sequences the kernels of
// filter3d.cu / registration.cu / nonlinear.cu on the context's stream;
// nothing here synchronises with the host except where stated.
#include <math.h>
#include <string.h>

#include <vector>

#include <string>

#include "../../include/broccoli_b200.h"
#include "capi_ctx.h"
#include "common.cuh"
#include "internal.h"

namespace {

// Gaussian smoothing filter of 9 taps for a sigma in voxels, normalised by
// its float sum (CreateSmoothingFilters(..., double sigma),
// broccoli_lib.cpp:11093-11121).
void smoothing_taps(double sigma, float* f) {
  const double s2 = 2.0 * sigma * sigma;
  float sum = 0.0f;
  for (int i = 0; i < 9; i++) {
    const double u = (double)(i - 4);
    f[i] = (float)exp(-pow(u, 2.0) / s2);
    sum += f[i];
  }
  for (int i = 0; i < 9; i++) f[i] /= sum;
}

int myround(float a) { return (int)floorf(a + 0.5f); }

}  // namespace

// One nonlinear update of G instances from given responses (q1, the
// reference's, shared; q2 6 complex volumes per instance): T, its
// smoothing, norm and max, A and h, their smoothing, the per-voxel solve,
// the smoothing of the update and its addition into the fields (3 volumes
// per instance) -- the AlignTwoVolumesNonLinear loop body,
// broccoli_lib.cpp:5784-6025, every launch covering all G instances.
static int nonlinear_step(brc_ctx* ctx, const float* q1, const float* q2, int G, int W, int H, int D,
                          const float* m36, const float* dirs18, const float* ft, const float* fe,
                          const float* fd, int fp64, float* field) {
  const long long V = (long long)W * H * D;
  cudaStream_t st = ctx->stream();
  float* t6 = ctx->nl.as<float>();        // [G][6][V] smoothed T
  float* ah = t6 + 6 * V * G;             // [G][9][V] smoothed a6 then h3
  float* d3 = ah + 9 * V * G;             // [G][3][V] update
  unsigned int* maxbits = reinterpret_cast<unsigned int*>(d3 + 3 * V * G);  // G words
  // the unsmoothed T ([G][6][V]) and then A, h ([G][9][V]) go to tmp2, so
  // every smoothing writes a buffer it does not read
  float* raw = ctx->tmp2.as<float>();
  BRC_TRY(ctx, brc::tensor_components(q2, V, m36, raw, st, G), "tensor_components");
  int s = ctx->smooth(raw, W, H, D, 6 * G, ft, ft, ft, nullptr, nullptr, ctx->tmp1.as<float>(), nullptr, t6, st);
  if (s != BRC_OK) return s;
  BRC_TRY(ctx, brc::tensor_norm_max(t6, V, raw, maxbits, st, G, 6 * V, 9 * V), "tensor_norm_max");
  BRC_TRY(ctx, brc::nonlinear_ah(q1, q2, t6, V, maxbits, m36, dirs18, raw, raw + 6 * V, st, G, 9 * V),
          "nonlinear_ah");
  s = ctx->smooth(raw, W, H, D, 9 * G, fe, fe, fe, nullptr, nullptr, ctx->tmp1.as<float>(), nullptr, ah, st);
  if (s != BRC_OK) return s;
  BRC_TRY(ctx, brc::displacement_update(ah, ah + 6 * V, V, fp64, d3, st, G, 9 * V), "displacement_update");
  // the unsmoothed A, h in raw are consumed: raw takes the chunk timing of
  // the accumulating smoothing
  s = ctx->smooth(d3, W, H, D, 3 * G, fd, fd, fd, nullptr, nullptr, ctx->tmp1.as<float>(), nullptr, field, st, 1,
                  raw);
  if (s != BRC_OK) return s;
  ctx->launches += 7;
  return BRC_OK;
}

static int ensure_nonlinear_ws(brc_ctx* ctx, long long V, int G = 1) {
  BRC_TRY(ctx, ctx->nl.ensure(sizeof(float) * (18 * V * G + 64 + G)), "alloc nonlinear");
  BRC_TRY(ctx, ctx->tmp1.ensure(sizeof(float) * 9 * V), "alloc tmp");
  BRC_TRY(ctx, ctx->tmp2.ensure(sizeof(float) * 9 * V * G), "alloc tmp");
  return BRC_OK;
}

extern "C" void brc_nonlinear_opts_default(brc_nonlinear_opts* o, int iterations) {
  if (!o) return;
  o->iterations = iterations;
  o->coarsest_scale = 1;
  o->tsigma = 5.0f;
  o->esigma = 5.0f;
  o->dsigma = 5.0f;
  o->precision = BRC_PREC_FP32;
  o->solve_fp64 = 0;
}

extern "C" int brc_nonlinear_step(brc_ctx* ctx, const float* d_q1, const float* d_q2, int W, int H,
                                  int D, const float* h_tensors, const float* h_dirs, float tsigma,
                                  float esigma, float dsigma, int solve_fp64, float* d_field) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_q1 || !d_q2 || !h_tensors || !h_dirs || !d_field || W <= 0 || H <= 0 || D <= 0 ||
      !(tsigma > 0) || !(esigma > 0) || !(dsigma > 0))
    return ctx->fail(BRC_ERR_INVALID, "brc_nonlinear_step: bad argument");
  cudaSetDevice(ctx->device);
  const long long V = (long long)W * H * D;
  int s = ensure_nonlinear_ws(ctx, V);
  if (s != BRC_OK) return s;
  float ft[9], fe[9], fd[9];
  smoothing_taps(tsigma, ft);
  smoothing_taps(esigma, fe);
  smoothing_taps(dsigma, fd);
  return nonlinear_step(ctx, d_q1, d_q2, 1, W, H, D, h_tensors, h_dirs, ft, fe, fd, solve_fp64, d_field);
}

// One scale of nonlinear registration of G instances: `aligned` (in: start
// volumes, out: last warps) and `original` (the volumes the fields warp), G
// volumes of W,H,D each, one shared reference; `field` (3 volumes per
// instance) receives this scale's total update (zeroed first).
static int nonlinear_scale(brc_ctx* ctx, const float* ref, float* aligned, const float* original, int G, int W,
                           int H, int D, const float* filters6, const float* m36, const float* dirs18,
                           int iterations, const brc_nonlinear_opts* o, float* field) {
  const long long V = (long long)W * H * D;
  cudaStream_t st = ctx->stream();
  int s = ensure_nonlinear_ws(ctx, V, G);
  if (s != BRC_OK) return s;
  BRC_TRY(ctx, ctx->q1.ensure(sizeof(float) * 12 * V), "alloc q1");
  BRC_TRY(ctx, ctx->q2.ensure(sizeof(float) * 12 * V * G), "alloc q2");
  float* q1 = ctx->q1.as<float>();
  float* q2 = ctx->q2.as<float>();
  float ft[9], fe[9], fd[9];
  smoothing_taps(o->tsigma, ft);
  smoothing_taps(o->esigma, fe);
  smoothing_taps(o->dsigma, fd);
  FilterPath fp;
  s = make_filter_path(ctx, filters6, 6, o->precision, W, H, D, &fp);
  if (s != BRC_OK) return s;
  BRC_TRY(ctx, run_filter(fp, ref, W, H, D, 1, V, q1, brc::all_instances(), st), "filter ref");
  ctx->launches += filter_launches(fp);
  BRC_TRY(ctx, cudaMemsetAsync(field, 0, sizeof(float) * 3 * V * G, st), "memset field");
  for (int it = 0; it < iterations; it++) {
    BRC_TRY(ctx, run_filter(fp, aligned, W, H, D, G, V, q2, brc::all_instances(), st), "filter");
    ctx->launches += filter_launches(fp);
    s = nonlinear_step(ctx, q1, q2, G, W, H, D, m36, dirs18, ft, fe, fd, o->solve_fp64, field);
    if (s != BRC_OK) return s;
    BRC_TRY(ctx, brc::warp_field(original, W, H, D, field, field + V, field + 2 * V, aligned, st, G, V, 3 * V, V),
            "warp");
    ctx->launches += 1;
  }
  return BRC_OK;
}

// AlignTwoVolumesNonLinearSeveralScales (broccoli_lib.cpp:6516-6665) for G
// moving volumes (d_moving, G volumes one after another) and one reference:
// d_field receives 3 volumes per instance, d_aligned one.  Every launch of
// the pyramid covers all G instances; per instance the arithmetic is that
// of a single registration.
static int register_nonlinear_group(brc_ctx* ctx, const float* d_ref, const float* d_moving, int G, int W, int H,
                                    int D, const float* h_filters6, const float* h_tensors, const float* h_dirs,
                                    const brc_nonlinear_opts* o, float* d_field, float* d_aligned) {
  cudaStream_t st = ctx->stream();
  const long long V = (long long)W * H * D;
  // scale buffers: reference (1), originals and aligned (G each), two field
  // sets (3G each)
  BRC_TRY(ctx, ctx->pyr.ensure(sizeof(float) * (V + 8 * V * G)), "alloc pyramid");
  float* r_s = ctx->pyr.as<float>();
  float* o_s = r_s + V;
  float* a_s = o_s + V * G;
  float* tot = a_s + V * G;       // [G][3][vs]
  float* upd = tot + 3 * V * G;   // [G][3][vs]
  int cw = myround((float)W / (float)o->coarsest_scale);
  int ch = myround((float)H / (float)o->coarsest_scale);
  int cd = myround((float)D / (float)o->coarsest_scale);
  if (cw < 2 || ch < 2 || cd < 2)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_nonlinear: coarsest scale leaves fewer than 2 voxels");
  if (o->coarsest_scale == 1) {
    BRC_TRY(ctx, cudaMemcpyAsync(o_s, d_moving, sizeof(float) * V * G, cudaMemcpyDeviceToDevice, st), "copy");
    BRC_TRY(ctx, cudaMemcpyAsync(r_s, d_ref, sizeof(float) * V, cudaMemcpyDeviceToDevice, st), "copy");
  } else {
    BRC_TRY(ctx, brc::rescale_batch(d_moving, W, H, D, G, o_s, cw, ch, cd, 1.0f, st), "rescale");
    BRC_TRY(ctx, brc::rescale_batch(d_ref, W, H, D, 1, r_s, cw, ch, cd, 1.0f, st), "rescale");
    ctx->launches += 2;
  }
  BRC_TRY(ctx, cudaMemsetAsync(tot, 0, sizeof(float) * 3 * (long long)cw * ch * cd * G, st), "memset");
  for (int scale = o->coarsest_scale; scale >= 1; scale /= 2) {
    const long long vs = (long long)cw * ch * cd;
    BRC_TRY(ctx, cudaMemcpyAsync(a_s, o_s, sizeof(float) * vs * G, cudaMemcpyDeviceToDevice, st), "copy");
    const int iters = scale == 1 ? (int)ceilf((float)o->iterations / 2.0f) : o->iterations;
    int s = nonlinear_scale(ctx, r_s, a_s, o_s, G, cw, ch, cd, h_filters6, h_tensors, h_dirs, iters, o, upd);
    if (s != BRC_OK) return s;
    BRC_TRY(ctx, brc::add_volumes(tot, tot, upd, 3 * vs * G, st), "add");
    ctx->launches += 1;
    if (scale != 1) {
      const int pw = cw, ph = ch, pd = cd;
      cw = myround((float)W / ((float)scale / 2.0f));
      ch = myround((float)H / ((float)scale / 2.0f));
      cd = myround((float)D / ((float)scale / 2.0f));
      const long long nv = (long long)cw * ch * cd;
      // fields to the finer grid, doubled (voxel units), via the upd buffer
      BRC_TRY(ctx, brc::rescale_batch(tot, pw, ph, pd, 3 * G, upd, cw, ch, cd, 2.0f, st), "rescale field");
      BRC_TRY(ctx, cudaMemcpyAsync(tot, upd, sizeof(float) * 3 * nv * G, cudaMemcpyDeviceToDevice, st), "copy");
      BRC_TRY(ctx, brc::rescale_batch(d_ref, W, H, D, 1, r_s, cw, ch, cd, 1.0f, st), "rescale");
      BRC_TRY(ctx, brc::rescale_batch(d_moving, W, H, D, G, a_s, cw, ch, cd, 1.0f, st), "rescale");
      BRC_TRY(ctx, brc::warp_field(a_s, cw, ch, cd, tot, tot + nv, tot + 2 * nv, o_s, st, G, nv, 3 * nv, nv),
              "warp");
      ctx->launches += 4;
    } else {
      BRC_TRY(ctx, cudaMemcpyAsync(d_field, tot, sizeof(float) * 3 * V * G, cudaMemcpyDeviceToDevice, st), "copy");
      BRC_TRY(ctx, brc::warp_field(d_moving, W, H, D, d_field, d_field + V, d_field + 2 * V, d_aligned, st, G, V,
                                   3 * V, V),
              "warp");
      ctx->launches += 1;
    }
  }
  if (ctx->dbg_on) {
    bool six = true;
    for (int k = 0; k < 6; k++) six = six && ctx->dbg.quadrature_responses[k] != nullptr;
    if (six) {
      // the finest scale's reference responses, still in q1 (the reads kept
      // commented out at broccoli_lib.cpp:5754-5759)
      int s = debug_capture_check(ctx, "debug outputs");
      if (s != BRC_OK) return s;
      for (int k = 0; k < 6; k++)
        BRC_TRY(ctx, cudaMemcpyAsync(ctx->dbg.quadrature_responses[k], ctx->q1.as<float>() + 2 * V * k,
                                     sizeof(float) * 2 * V, cudaMemcpyDeviceToHost, st), "debug D2H");
      BRC_TRY(ctx, cudaStreamSynchronize(st), "debug synchronize");
    }
  }
  return BRC_OK;
}

extern "C" int brc_register_nonlinear(brc_ctx* ctx, const float* d_ref, const float* d_moving, int W,
                                      int H, int D, const float* h_filters6, const float* h_tensors,
                                      const float* h_dirs, const brc_nonlinear_opts* o, float* d_field,
                                      float* d_aligned) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_ref || !d_moving || !h_filters6 || !h_tensors || !h_dirs || !o || !d_field || !d_aligned ||
      W <= 0 || H <= 0 || D <= 0 || o->iterations < 0 || o->coarsest_scale < 1 ||
      !(o->tsigma > 0) || !(o->esigma > 0) || !(o->dsigma > 0))
    return ctx->fail(BRC_ERR_INVALID, "brc_register_nonlinear: bad argument");
  if (!brc_precision_valid(o->precision))
    return ctx->fail(BRC_ERR_UNSUPPORTED, "brc_register_nonlinear: unknown precision");
  if (d_aligned == d_moving)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_nonlinear: d_aligned must not alias d_moving");
  cudaSetDevice(ctx->device);
  return register_nonlinear_group(ctx, d_ref, d_moving, 1, W, H, D, h_filters6, h_tensors, h_dirs, o, d_field,
                                  d_aligned);
}

extern "C" int brc_change_resolution_and_size(brc_ctx* ctx, const float* d_src, int W, int H, int D,
                                              const float* voxel_size3, float* d_out, int W2, int H2,
                                              int D2, const float* new_voxel_size3, int mm_z_cut) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_src || !d_out || !voxel_size3 || !new_voxel_size3 || W <= 0 || H <= 0 || D <= 0 || W2 <= 0 ||
      H2 <= 0 || D2 <= 0 || d_src == d_out)
    return ctx->fail(BRC_ERR_INVALID, "brc_change_resolution_and_size: bad argument");
  for (int a = 0; a < 3; a++)
    if (!(voxel_size3[a] > 0) || !(new_voxel_size3[a] > 0))
      return ctx->fail(BRC_ERR_INVALID, "brc_change_resolution_and_size: voxel sizes must be positive");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::resize_to_grid(d_src, W, H, D, voxel_size3[0], voxel_size3[1], voxel_size3[2], d_out, W2,
                                   H2, D2, new_voxel_size3[0], new_voxel_size3[1], new_voxel_size3[2],
                                   mm_z_cut, ctx->stream()),
          "resize");
  ctx->launches += 1;
  return BRC_OK;
}

// Interpolation modes of the transform entries: the reference's NEAREST and
// LINEAR.  Its CUBIC kernels sum into an uninitialised variable
// (kernelRegistration.cpp:1230, :1284, :1396), so CUBIC is refused.
static int check_interp(brc_ctx* ctx, int interpolation, const char* where) {
  if (interpolation == BRC_INTERP_NEAREST || interpolation == BRC_INTERP_LINEAR) return BRC_OK;
  if (interpolation == BRC_INTERP_CUBIC)
    return ctx->fail(BRC_ERR_UNSUPPORTED, std::string(where) + ": CUBIC interpolation is not supported");
  return ctx->fail(BRC_ERR_INVALID, std::string(where) + ": unknown interpolation mode");
}

extern "C" int brc_change_resolution_and_size_batch(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T,
                                                    const float* voxel_size3, float* d_out, int W2, int H2, int D2,
                                                    const float* new_voxel_size3, int mm_z_cut, int interpolation) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_src || !d_out || !voxel_size3 || !new_voxel_size3 || W <= 0 || H <= 0 || D <= 0 || W2 <= 0 ||
      H2 <= 0 || D2 <= 0 || T <= 0 || T > 65535 || d_src == d_out)
    return ctx->fail(BRC_ERR_INVALID, "brc_change_resolution_and_size_batch: bad argument");
  for (int a = 0; a < 3; a++)
    if (!(voxel_size3[a] > 0) || !(new_voxel_size3[a] > 0))
      return ctx->fail(BRC_ERR_INVALID, "brc_change_resolution_and_size_batch: voxel sizes must be positive");
  const int s = check_interp(ctx, interpolation, "brc_change_resolution_and_size_batch");
  if (s != BRC_OK) return s;
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::resize_to_grid_batch(d_src, W, H, D, T, voxel_size3[0], voxel_size3[1], voxel_size3[2], d_out,
                                         W2, H2, D2, new_voxel_size3[0], new_voxel_size3[1], new_voxel_size3[2],
                                         mm_z_cut, interpolation, ctx->stream()),
          "resize");
  ctx->launches += 1;
  return BRC_OK;
}

extern "C" int brc_transform_volumes_linear(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T,
                                            const float* h_params12, int interpolation, float* d_out) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_src || !d_out || !h_params12 || W <= 0 || H <= 0 || D <= 0 || T <= 0 || T > 65535 || d_src == d_out)
    return ctx->fail(BRC_ERR_INVALID, "brc_transform_volumes_linear: bad argument");
  const int s = check_interp(ctx, interpolation, "brc_transform_volumes_linear");
  if (s != BRC_OK) return s;
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::transform_affine(d_src, W, H, D, T, h_params12, interpolation, d_out, ctx->stream()),
          "transform_affine");
  ctx->launches += 1;
  return BRC_OK;
}

extern "C" int brc_transform_volumes_nonlinear(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T,
                                               const float* d_dx, const float* d_dy, const float* d_dz,
                                               int interpolation, float* d_out) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_src || !d_out || !d_dx || !d_dy || !d_dz || W <= 0 || H <= 0 || D <= 0 || T <= 0 || T > 65535 ||
      d_src == d_out)
    return ctx->fail(BRC_ERR_INVALID, "brc_transform_volumes_nonlinear: bad argument");
  const int s = check_interp(ctx, interpolation, "brc_transform_volumes_nonlinear");
  if (s != BRC_OK) return s;
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::transform_field(d_src, W, H, D, T, d_dx, d_dy, d_dz, interpolation, d_out, ctx->stream()),
          "transform_field");
  ctx->launches += 1;
  return BRC_OK;
}

extern "C" int brc_combine_displacement_field(brc_ctx* ctx, float* d_dx, float* d_dy, float* d_dz, int W, int H,
                                              int D, const float* h_params12) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_dx || !d_dy || !d_dz || !h_params12 || W <= 0 || H <= 0 || D <= 0)
    return ctx->fail(BRC_ERR_INVALID, "brc_combine_displacement_field: bad argument");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::combine_field(d_dx, d_dy, d_dz, W, H, D, h_params12, ctx->stream()), "combine_field");
  ctx->launches += 1;
  return BRC_OK;
}

extern "C" int brc_center_of_mass(brc_ctx* ctx, const float* d_vol, int W, int H, int D, float* h_com3) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_vol || !h_com3 || W <= 0 || H <= 0 || D <= 0)
    return ctx->fail(BRC_ERR_INVALID, "brc_center_of_mass: bad argument");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, ctx->ctl.ensure(sizeof(double) * 8), "alloc");
  double* sums = ctx->ctl.as<double>();
  BRC_TRY(ctx, brc::mass_moments(d_vol, W, H, D, sums, ctx->stream()), "mass_moments");
  ctx->launches += 1;
  double h[4];
  BRC_TRY(ctx, cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream()), "D2H");
  BRC_TRY(ctx, cudaStreamSynchronize(ctx->stream()), "sync");
  for (int a = 0; a < 3; a++) h_com3[a] = (float)(h[a + 1] / h[0]);
  return BRC_OK;
}

extern "C" int brc_center_volumes(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T, int interpolation,
                                  float* d_out, float* h_params12) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_src || !d_out || W <= 0 || H <= 0 || D <= 0 || T <= 0 || T > 65535 || d_src == d_out)
    return ctx->fail(BRC_ERR_INVALID, "brc_center_volumes: bad argument");
  int s = check_interp(ctx, interpolation, "brc_center_volumes");
  if (s != BRC_OK) return s;
  float com[3];
  if ((s = brc_center_of_mass(ctx, d_src, W, H, D, com)) != BRC_OK) return s;
  // CenterVolumeMass (broccoli_lib.cpp:6839-6874): integer translation that
  // moves the first volume's centre of mass to (W/2, H/2, D/2)
  float p[12] = {0};
  p[0] = -floorf((float)W / 2.0f - com[0] + 0.5f);
  p[1] = -floorf((float)H / 2.0f - com[1] + 0.5f);
  p[2] = -floorf((float)D / 2.0f - com[2] + 0.5f);
  if ((s = brc_transform_volumes_linear(ctx, d_src, W, H, D, T, p, interpolation, d_out)) != BRC_OK) return s;
  if (h_params12) memcpy(h_params12, p, sizeof(p));
  return BRC_OK;
}

extern "C" void brc_two_volume_opts_default(brc_two_volume_opts* o) {
  if (!o) return;
  o->linear_iterations = 10;
  o->nonlinear_iterations = 10;
  o->coarsest_scale = 4;
  o->mm_z_cut = 0;
  o->tsigma = 5.0f;
  o->esigma = 5.0f;
  o->dsigma = 5.0f;
  o->precision = BRC_PREC_FP32;
  o->solve_fp64 = 0;
  o->precenter = 0;
}

// PRECENTER_REGISTRATION (broccoli_lib.cpp:8003-8007): the input centred by
// its centre of mass at its own size, twice (the two CenterVolumeMass calls,
// both LINEAR), into `out` (a buffer of the input's size); `tmp` is a second
// such buffer.
static int precenter_volume(brc_ctx* ctx, const float* d_in, int W, int H, int D, float* tmp, float* out) {
  int s = brc_center_volumes(ctx, d_in, W, H, D, 1, BRC_INTERP_LINEAR, tmp, nullptr);
  if (s != BRC_OK) return s;
  return brc_center_volumes(ctx, tmp, W, H, D, 1, BRC_INTERP_LINEAR, out, nullptr);
}

// PerformRegistrationTwoVolumesWrapper, broccoli_lib.cpp:7973-8112 (single
// volume; the skull strip is left to the caller, which holds the mask):
// optional pre-centring of the input, resample to the template grid,
// match centres of mass, multi-scale affine, compose with the mass match,
// multi-scale nonlinear, add the affine motion to the field, resample the
// input again and warp it once by the combined field.
extern "C" int brc_register_two_volumes(brc_ctx* ctx, const float* d_in, int W, int H, int D,
                                        const float* voxel_size3, const float* d_tpl, int W2, int H2,
                                        int D2, const float* tpl_voxel_size3, const float* h_filters3,
                                        const float* h_filters6, const float* h_tensors,
                                        const float* h_dirs, const brc_two_volume_opts* o,
                                        float* h_params12, float* d_interpolated,
                                        float* d_aligned_linear, float* d_aligned_nonlinear,
                                        float* d_field) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_in || !d_tpl || !voxel_size3 || !tpl_voxel_size3 || !h_filters3 || !o || !h_params12 ||
      W <= 0 || H <= 0 || D <= 0 || W2 <= 0 || H2 <= 0 || D2 <= 0 || o->linear_iterations < 0 ||
      o->nonlinear_iterations < 0 || o->coarsest_scale < 1)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_two_volumes: bad argument");
  if (o->nonlinear_iterations > 0 && (!h_filters6 || !h_tensors || !h_dirs || !d_field))
    return ctx->fail(BRC_ERR_INVALID, "brc_register_two_volumes: nonlinear stage needs filters and a field");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream();
  const long long V2 = (long long)W2 * H2 * D2;
  // own buffers for the template-size working volumes
  DevBuf& work = ctx->r2v_work;
  DevBuf& lin = ctx->r2v_lin;
  BRC_TRY(ctx, work.ensure(sizeof(float) * V2), "alloc");
  BRC_TRY(ctx, lin.ensure(sizeof(float) * (V2 + 12)), "alloc");
  float* w = work.as<float>();
  float* a = lin.as<float>();
  float* dparams = a + V2;
  int s;
  DevBuf cen;
  if (o->precenter && o->linear_iterations > 0) {
    const long long V1 = (long long)W * H * D;
    BRC_TRY(ctx, cen.ensure(sizeof(float) * 2 * V1), "alloc");
    if ((s = precenter_volume(ctx, d_in, W, H, D, cen.as<float>() + V1, cen.as<float>())) != BRC_OK) return s;
    d_in = cen.as<float>();  // the centred input replaces the input throughout
  }
  s = brc_change_resolution_and_size(ctx, d_in, W, H, D, voxel_size3, w, W2, H2, D2, tpl_voxel_size3,
                                     o->mm_z_cut);
  if (s != BRC_OK) return s;
  float c1[3], c2[3];
  if ((s = brc_center_of_mass(ctx, w, W2, H2, D2, c1)) != BRC_OK) return s;
  if ((s = brc_center_of_mass(ctx, d_tpl, W2, H2, D2, c2)) != BRC_OK) return s;
  float match[12] = {0};
  for (int k = 0; k < 3; k++) match[k] = -(float)myround(c2[k] - c1[k]);
  BRC_TRY(ctx, cudaMemcpyAsync(dparams, match, sizeof(match), cudaMemcpyHostToDevice, st), "H2D");
  BRC_TRY(ctx, brc::warp_affine(w, V2, W2, H2, D2, 1, dparams, a, V2, brc::all_instances(), st), "match");
  ctx->launches += 1;
  if (d_interpolated)
    BRC_TRY(ctx, cudaMemcpyAsync(d_interpolated, a, sizeof(float) * V2, cudaMemcpyDeviceToDevice, st), "copy");
  float total[12] = {0};
  if (o->linear_iterations > 0) {
    brc_linear_opts lo;
    brc_linear_opts_default(&lo, o->linear_iterations);
    lo.type = BRC_AFFINE;
    lo.precision = o->precision;
    DevBuf& prm = ctx->r2v_prm;
    BRC_TRY(ctx, prm.ensure(sizeof(float) * 12), "alloc");
    s = brc_register_linear_scales(ctx, d_tpl, a, W2, H2, D2, 1, h_filters3, &lo, o->coarsest_scale,
                                   prm.as<float>(), w, nullptr);
    if (s != BRC_OK) return s;
    BRC_TRY(ctx, cudaMemcpyAsync(total, prm.as<float>(), sizeof(total), cudaMemcpyDeviceToHost, st), "D2H");
    BRC_TRY(ctx, cudaStreamSynchronize(st), "sync");
  } else {
    BRC_TRY(ctx, cudaMemcpyAsync(w, a, sizeof(float) * V2, cudaMemcpyDeviceToDevice, st), "copy");
  }
  if (d_aligned_linear)
    BRC_TRY(ctx, cudaMemcpyAsync(d_aligned_linear, w, sizeof(float) * V2, cudaMemcpyDeviceToDevice, st), "copy");
  // total = match * linear (AddAffineRegistrationParameters(total, match))
  {
    double O[16] = {0}, N[16] = {0}, T[16];
    const float* src[2] = {total, match};
    double* dst[2] = {O, N};
    for (int m = 0; m < 2; m++) {
      const float* p = src[m];
      double* M = dst[m];
      M[0] = (double)(p[3] + 1.0f); M[1] = p[4]; M[2] = p[5]; M[3] = p[0];
      M[4] = p[6]; M[5] = (double)(p[7] + 1.0f); M[6] = p[8]; M[7] = p[1];
      M[8] = p[9]; M[9] = p[10]; M[10] = (double)(p[11] + 1.0f); M[11] = p[2];
      M[15] = 1.0;
    }
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        double acc = 0;
        for (int k = 0; k < 4; k++) acc += N[i * 4 + k] * O[k * 4 + j];
        T[i * 4 + j] = acc;
      }
    total[0] = (float)T[3]; total[1] = (float)T[7]; total[2] = (float)T[11];
    total[3] = (float)(T[0] - 1.0); total[4] = (float)T[1]; total[5] = (float)T[2];
    total[6] = (float)T[4]; total[7] = (float)(T[5] - 1.0); total[8] = (float)T[6];
    total[9] = (float)T[8]; total[10] = (float)T[9]; total[11] = (float)(T[10] - 1.0);
  }
  for (int i = 0; i < 12; i++) h_params12[i] = total[i];
  if (o->nonlinear_iterations > 0) {
    brc_nonlinear_opts no;
    brc_nonlinear_opts_default(&no, o->nonlinear_iterations);
    no.coarsest_scale = o->coarsest_scale;
    no.tsigma = o->tsigma;
    no.esigma = o->esigma;
    no.dsigma = o->dsigma;
    no.precision = o->precision;
    no.solve_fp64 = o->solve_fp64;
    s = brc_register_nonlinear(ctx, d_tpl, w, W2, H2, D2, h_filters6, h_tensors, h_dirs, &no, d_field, a);
    if (s != BRC_OK) return s;
    if (o->linear_iterations > 0) {
      BRC_TRY(ctx, brc::add_affine_to_field(d_field, W2, H2, D2, total, st), "field");
      ctx->launches += 1;
      s = brc_change_resolution_and_size(ctx, d_in, W, H, D, voxel_size3, w, W2, H2, D2, tpl_voxel_size3,
                                         o->mm_z_cut);
      if (s != BRC_OK) return s;
      BRC_TRY(ctx, brc::warp_field(w, W2, H2, D2, d_field, d_field + V2, d_field + 2 * V2, a, st), "warp");
      ctx->launches += 1;
    }
    if (d_aligned_nonlinear)
      BRC_TRY(ctx, cudaMemcpyAsync(d_aligned_nonlinear, a, sizeof(float) * V2, cudaMemcpyDeviceToDevice, st),
              "copy");
  }
  BRC_TRY(ctx, cudaStreamSynchronize(st), "sync");
  return BRC_OK;
}

// Composition of two parameter vectors in double, total = new * old as 4x4
// affine matrices (AddAffineRegistrationParameters, broccoli_lib.cpp:
// 7252-7340 and :7433-7520).  `total` may alias `old12`.
void brc::host_add_affine(const float* old12, const float* new12, float* total) {
  double O[16] = {0}, N[16] = {0}, T[16];
  const float* src[2] = {old12, new12};
  double* dst[2] = {O, N};
  for (int m = 0; m < 2; m++) {
    const float* p = src[m];
    double* M = dst[m];
    M[0] = (double)(p[3] + 1.0f); M[1] = p[4]; M[2] = p[5]; M[3] = p[0];
    M[4] = p[6]; M[5] = (double)(p[7] + 1.0f); M[6] = p[8]; M[7] = p[1];
    M[8] = p[9]; M[9] = p[10]; M[10] = (double)(p[11] + 1.0f); M[11] = p[2];
    M[15] = 1.0;
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double acc = 0;
      for (int k = 0; k < 4; k++) acc += N[i * 4 + k] * O[k * 4 + j];
      T[i * 4 + j] = acc;
    }
  total[0] = (float)T[3]; total[1] = (float)T[7]; total[2] = (float)T[11];
  total[3] = (float)(T[0] - 1.0); total[4] = (float)T[1]; total[5] = (float)T[2];
  total[6] = (float)T[4]; total[7] = (float)(T[5] - 1.0); total[8] = (float)T[6];
  total[9] = (float)T[8]; total[10] = (float)T[9]; total[11] = (float)(T[10] - 1.0);
}

// 4x4 inverse of a parameter vector's affine matrix in double by
// Gauss-Jordan elimination with partial pivoting, rounded to float
// (InvertAffineRegistrationParameters, broccoli_lib.cpp:7186-7250).
void brc::host_invert_affine(const float* p, float* inv) {
  double M[4][8] = {{(double)(p[3] + 1.0f), p[4], p[5], p[0]},
                    {p[6], (double)(p[7] + 1.0f), p[8], p[1]},
                    {p[9], p[10], (double)(p[11] + 1.0f), p[2]},
                    {0.0, 0.0, 0.0, 1.0}};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) M[i][4 + j] = i == j ? 1.0 : 0.0;
  for (int c = 0; c < 4; c++) {
    int piv = c;
    for (int r = c + 1; r < 4; r++)
      if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
    if (piv != c)
      for (int j = 0; j < 8; j++) {
        const double t = M[c][j];
        M[c][j] = M[piv][j];
        M[piv][j] = t;
      }
    const double d = M[c][c];
    for (int j = 0; j < 8; j++) M[c][j] /= d;
    for (int r = 0; r < 4; r++)
      if (r != c) {
        const double f = M[r][c];
        if (f != 0.0)
          for (int j = 0; j < 8; j++) M[r][j] -= f * M[c][j];
      }
  }
  double I[4][4];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) I[i][j] = M[i][4 + j];
  inv[0] = (float)I[0][3];
  inv[1] = (float)I[1][3];
  inv[2] = (float)I[2][3];
  inv[3] = (float)(I[0][0] - 1.0);
  inv[4] = (float)I[0][1];
  inv[5] = (float)I[0][2];
  inv[6] = (float)I[1][0];
  inv[7] = (float)(I[1][1] - 1.0);
  inv[8] = (float)I[1][2];
  inv[9] = (float)I[2][0];
  inv[10] = (float)I[2][1];
  inv[11] = (float)(I[2][2] - 1.0);
}

extern "C" void brc_invert_affine_parameters(const float* h_params12, float* h_inverse12) {
  if (!h_params12 || !h_inverse12) return;
  float tmp[12];
  brc::host_invert_affine(h_params12, tmp);
  memcpy(h_inverse12, tmp, sizeof(tmp));
}

extern "C" int brc_register_cohort(brc_ctx* ctx, int n, const float* const* d_subjects, const int* sizes3n,
                                   const float* voxel_sizes3n, const float* d_tpl, int W2, int H2, int D2,
                                   const float* tpl_voxel_size3, const float* h_filters3, const float* h_filters6,
                                   const float* h_tensors, const float* h_dirs, const brc_two_volume_opts* o,
                                   float* h_params12n, float* d_aligned_linear, float* d_aligned_nonlinear,
                                   float* d_fields) {
  if (!ctx) return BRC_ERR_INVALID;
  if (n <= 0 || n > 65535 || !d_subjects || !sizes3n || !voxel_sizes3n || !d_tpl || !tpl_voxel_size3 ||
      !h_filters3 || !o || !h_params12n || W2 <= 0 || H2 <= 0 || D2 <= 0 || o->linear_iterations < 0 ||
      o->nonlinear_iterations < 0 || o->coarsest_scale < 1)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_cohort: bad argument");
  if (o->nonlinear_iterations > 0 && (!h_filters6 || !h_tensors || !h_dirs || !d_fields))
    return ctx->fail(BRC_ERR_INVALID, "brc_register_cohort: nonlinear stage needs filters and fields");
  for (int b = 0; b < n; b++) {
    if (!d_subjects[b] || sizes3n[3 * b] <= 0 || sizes3n[3 * b + 1] <= 0 || sizes3n[3 * b + 2] <= 0)
      return ctx->fail(BRC_ERR_INVALID, "brc_register_cohort: bad subject pointer or size");
    for (int a = 0; a < 3; a++)
      if (!(voxel_sizes3n[3 * b + a] > 0) || !(tpl_voxel_size3[a] > 0))
        return ctx->fail(BRC_ERR_INVALID, "brc_register_cohort: voxel sizes must be positive");
  }
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream();
  const long long V2 = (long long)W2 * H2 * D2;
  // template-grid working volumes of all subjects: resampled originals,
  // centred copies, linear results; parameters; resample descriptors
  DevBuf& res = ctx->coh_res;
  DevBuf& mat = ctx->coh_mat;
  DevBuf& lin = ctx->coh_lin;
  DevBuf& prm = ctx->coh_prm;
  DevBuf& jobs = ctx->coh_jobs;
  BRC_TRY(ctx, res.ensure(sizeof(float) * V2 * n), "alloc");
  BRC_TRY(ctx, mat.ensure(sizeof(float) * V2 * n), "alloc");
  BRC_TRY(ctx, lin.ensure(sizeof(float) * V2 * n), "alloc");
  BRC_TRY(ctx, prm.ensure(sizeof(float) * 12 * n), "alloc");
  BRC_TRY(ctx, jobs.ensure(brc::resize_job_bytes() * n), "alloc");
  std::vector<unsigned char> h_jobs(brc::resize_job_bytes() * n);
  // 0. optional pre-centring of every subject at its own size
  std::vector<const float*> srcs(d_subjects, d_subjects + n);
  std::vector<std::unique_ptr<DevBuf>> centred;
  if (o->precenter && o->linear_iterations > 0) {
    for (int b = 0; b < n; b++) {
      const long long V1 = (long long)sizes3n[3 * b] * sizes3n[3 * b + 1] * sizes3n[3 * b + 2];
      centred.emplace_back(new DevBuf());
      BRC_TRY(ctx, centred.back()->ensure(sizeof(float) * 2 * V1), "alloc");
      float* c = centred.back()->as<float>();
      int s0 = precenter_volume(ctx, d_subjects[b], sizes3n[3 * b], sizes3n[3 * b + 1], sizes3n[3 * b + 2], c + V1, c);
      if (s0 != BRC_OK) return s0;
      srcs[b] = c;
    }
  }
  d_subjects = srcs.data();
  // 1. every subject onto the template grid in one ragged launch
  BRC_TRY(ctx, brc::resize_to_grid_ragged(n, d_subjects, sizes3n, voxel_sizes3n, h_jobs.data(), jobs.ptr,
                                          res.as<float>(), W2, H2, D2, tpl_voxel_size3, o->mm_z_cut, st),
          "resize");
  ctx->launches += 1;
  // 2. centre of mass matching (MatchVolumeMasses), one batched warp
  float ct[3];
  int s = brc_center_of_mass(ctx, d_tpl, W2, H2, D2, ct);
  if (s != BRC_OK) return s;
  std::vector<float> match(12 * (size_t)n, 0.f);
  for (int b = 0; b < n; b++) {
    float cs[3];
    if ((s = brc_center_of_mass(ctx, res.as<float>() + V2 * b, W2, H2, D2, cs)) != BRC_OK) return s;
    for (int k = 0; k < 3; k++) match[12 * b + k] = -(float)myround(ct[k] - cs[k]);
  }
  BRC_TRY(ctx, cudaMemcpyAsync(prm.ptr, match.data(), sizeof(float) * 12 * n, cudaMemcpyHostToDevice, st), "H2D");
  BRC_TRY(ctx, brc::warp_affine(res.as<float>(), V2, W2, H2, D2, n, prm.as<float>(), mat.as<float>(), V2, brc::all_instances(), st),
          "match");
  ctx->launches += 1;
  // 3. affine stage of all subjects as one batched multi-scale registration
  std::vector<float> total(12 * (size_t)n, 0.f), linp(12 * (size_t)n, 0.f);
  if (o->linear_iterations > 0) {
    brc_linear_opts lo;
    brc_linear_opts_default(&lo, o->linear_iterations);
    lo.type = BRC_AFFINE;
    lo.precision = o->precision;
    s = brc_register_linear_scales(ctx, d_tpl, mat.as<float>(), W2, H2, D2, n, h_filters3, &lo, o->coarsest_scale,
                                   prm.as<float>(), lin.as<float>(), nullptr);
    if (s != BRC_OK) return s;
    BRC_TRY(ctx, cudaMemcpyAsync(linp.data(), prm.ptr, sizeof(float) * 12 * n, cudaMemcpyDeviceToHost, st), "D2H");
    BRC_TRY(ctx, cudaStreamSynchronize(st), "sync");
  } else {
    BRC_TRY(ctx, cudaMemcpyAsync(lin.ptr, mat.ptr, sizeof(float) * V2 * n, cudaMemcpyDeviceToDevice, st), "copy");
  }
  for (int b = 0; b < n; b++)
    brc::host_add_affine(&linp[12 * (size_t)b], &match[12 * (size_t)b], &total[12 * (size_t)b]);
  memcpy(h_params12n, total.data(), sizeof(float) * 12 * n);
  if (d_aligned_linear)
    BRC_TRY(ctx, cudaMemcpyAsync(d_aligned_linear, lin.ptr, sizeof(float) * V2 * n, cudaMemcpyDeviceToDevice, st),
            "copy");
  // 4. nonlinear stage in groups of subjects (each at template size): every
  // launch of the pyramid covers the whole group
  if (o->nonlinear_iterations > 0) {
    brc_nonlinear_opts no;
    brc_nonlinear_opts_default(&no, o->nonlinear_iterations);
    no.coarsest_scale = o->coarsest_scale;
    no.tsigma = o->tsigma;
    no.esigma = o->esigma;
    no.dsigma = o->dsigma;
    no.precision = o->precision;
    no.solve_fp64 = o->solve_fp64;
    // group size: about half the free device memory for the group's
    // workspace (~190 bytes per voxel and subject), at most 16 subjects
    size_t freeb = 0, totalb = 0;
    BRC_TRY(ctx, cudaMemGetInfo(&freeb, &totalb), "memory info");
    const double per = 190.0 * (double)V2;
    int G = (int)((0.5 * (double)freeb) / per);
    G = G < 1 ? 1 : (G > 16 ? 16 : G);
    if (G > n) G = n;
    for (int g0 = 0; g0 < n; g0 += G) {
      const int g = n - g0 < G ? n - g0 : G;
      float* fields = d_fields + 3 * V2 * g0;
      float* outs = mat.as<float>() + V2 * g0;  // the centred copies are no longer needed
      s = register_nonlinear_group(ctx, d_tpl, lin.as<float>() + V2 * g0, g, W2, H2, D2, h_filters6, h_tensors,
                                   h_dirs, &no, fields, outs);
      if (s != BRC_OK) return s;
      if (o->linear_iterations > 0) {
        for (int b = 0; b < g; b++)
          BRC_TRY(ctx, brc::add_affine_to_field(fields + 3 * V2 * b, W2, H2, D2, &total[12 * (size_t)(g0 + b)], st),
                  "field");
        BRC_TRY(ctx, brc::warp_field(res.as<float>() + V2 * g0, W2, H2, D2, fields, fields + V2, fields + 2 * V2, outs,
                                     st, g, V2, 3 * V2, V2),
                "warp");
        ctx->launches += g + 1;
      }
      if (d_aligned_nonlinear)
        BRC_TRY(ctx, cudaMemcpyAsync(d_aligned_nonlinear + V2 * g0, outs, sizeof(float) * V2 * g,
                                     cudaMemcpyDeviceToDevice, st),
                "copy");
    }
  }
  BRC_TRY(ctx, cudaStreamSynchronize(st), "sync");
  return BRC_OK;
}

extern "C" int brc_register_linear_scales(brc_ctx* ctx, const float* d_ref, const float* d_moving, int W,
                                          int H, int D, int batch, const float* h_filters,
                                          const brc_linear_opts* opts, int coarsest_scale,
                                          float* d_params, float* d_aligned, float* d_rotations) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_ref || !d_moving || !h_filters || !opts || !d_params || !d_aligned || W <= 0 || H <= 0 ||
      D <= 0 || batch <= 0 || batch > 65535 || coarsest_scale < 1)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_linear_scales: bad argument");
  if (d_aligned == d_moving)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_linear_scales: d_aligned must not alias d_moving");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream();
  const long long V = (long long)W * H * D;
  int cw = myround((float)W / (float)coarsest_scale);
  int ch = myround((float)H / (float)coarsest_scale);
  int cd = myround((float)D / (float)coarsest_scale);
  if (cw < 2 || ch < 2 || cd < 2)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_linear_scales: coarsest scale leaves fewer than 2 voxels");
  // per scale: ref (1), resampled moving (B), pre-warped moving (B), scale
  // result (B), scale params (12B) and rotations (3B)
  BRC_TRY(ctx, ctx->pyr.ensure(sizeof(float) * ((1 + 3 * (size_t)batch) * V + 15 * (size_t)batch)), "alloc");
  float* r_s = ctx->pyr.as<float>();
  float* m_s = r_s + V;
  float* o_s = m_s + V * batch;
  float* a_s = o_s + V * batch;
  float* tmp = a_s + V * batch;
  float* rt = tmp + 12 * batch;
  BRC_TRY(ctx, cudaMemsetAsync(d_params, 0, sizeof(float) * 12 * batch, st), "memset");
  if (d_rotations) BRC_TRY(ctx, cudaMemsetAsync(d_rotations, 0, sizeof(float) * 3 * batch, st), "memset");
  brc_linear_opts so = *opts;
  so.use_graph = 0;
  for (int scale = coarsest_scale; scale >= 1; scale /= 2) {
    const long long vs = (long long)cw * ch * cd;
    BRC_TRY(ctx, brc::rescale_batch(d_ref, W, H, D, 1, r_s, cw, ch, cd, 1.0f, st), "rescale");
    if (scale == coarsest_scale) {
      BRC_TRY(ctx, brc::rescale_batch(d_moving, W, H, D, batch, o_s, cw, ch, cd, 1.0f, st), "rescale");
    } else {
      BRC_TRY(ctx, brc::rescale_batch(d_moving, W, H, D, batch, m_s, cw, ch, cd, 1.0f, st), "rescale");
      BRC_TRY(ctx, brc::warp_affine(m_s, vs, cw, ch, cd, batch, d_params, o_s, vs, brc::all_instances(), st), "prewarp");
      ctx->launches += 1;
    }
    ctx->launches += 2;
    so.iterations = scale == 1 ? (int)ceilf((float)opts->iterations / 5.0f) : opts->iterations;
    int s = brc_register_linear_batched(ctx, r_s, 0, o_s, cw, ch, cd, batch, h_filters, &so, tmp, a_s,
                                        rt, nullptr);
    if (s != BRC_OK) return s;
    BRC_TRY(ctx, brc::compose(d_params, tmp, batch, scale == 1 ? 1.0f : 2.0f, st), "compose");
    ctx->launches += 1;
    if (d_rotations && so.type == BRC_RIGID) {
      BRC_TRY(ctx, brc::add_volumes(d_rotations, d_rotations, rt, 3 * batch, st), "rotations");
      ctx->launches += 1;
    }
    if (scale != 1) {
      cw = myround((float)W / ((float)scale / 2.0f));
      ch = myround((float)H / ((float)scale / 2.0f));
      cd = myround((float)D / ((float)scale / 2.0f));
    }
  }
  BRC_TRY(ctx, brc::warp_affine(d_moving, V, W, H, D, batch, d_params, d_aligned, V, brc::all_instances(), st), "warp");
  ctx->launches += 1;
  return BRC_OK;
}

// ---------------------------------------------------------------------------
// Adjoints (differentiable registration)
// ---------------------------------------------------------------------------

extern "C" int brc_filter3d_adjoint(brc_ctx* ctx, const float* d_grad, int W, int H, int D, int batch,
                                    const float* h_filters, int nfilt, float* d_out) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_grad || !d_out || !h_filters || W <= 0 || H <= 0 || D <= 0 || batch <= 0 || batch > 65535 ||
      (nfilt != 3 && nfilt != 6))
    return ctx->fail(BRC_ERR_INVALID, "brc_filter3d_adjoint: bad argument");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::filter3d_adjoint(d_grad, W, H, D, batch, h_filters, nfilt, d_out, ctx->stream()),
          "filter3d_adjoint");
  ctx->launches += 1;
  return BRC_OK;
}

extern "C" int brc_warp_affine_backward(brc_ctx* ctx, const float* d_src, int W, int H, int D, int batch,
                                        const float* d_params, const float* d_grad_out, double* d_grad_params,
                                        float* d_grad_src) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_src || !d_params || !d_grad_out || !d_grad_params || W <= 0 || H <= 0 || D <= 0 || batch <= 0 ||
      batch > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_warp_affine_backward: bad argument");
  cudaSetDevice(ctx->device);
  const long long V = (long long)W * H * D;
  const int nblk = brc::warp_affine_backward_blocks(V);
  BRC_TRY(ctx, ctx->partials.ensure(sizeof(double) * 12 * nblk * (size_t)batch), "alloc");
  if (d_grad_src)
    BRC_TRY(ctx, cudaMemsetAsync(d_grad_src, 0, sizeof(float) * V * batch, ctx->stream()), "memset");
  BRC_TRY(ctx, brc::warp_affine_backward(d_src, W, H, D, batch, d_params, d_grad_out, ctx->partials.as<double>(),
                                         nblk, d_grad_params, d_grad_src, ctx->stream()),
          "warp_affine_backward");
  ctx->launches += 2;
  return BRC_OK;
}

extern "C" int brc_warp_field_backward(brc_ctx* ctx, const float* d_src, int W, int H, int D, const float* d_dx,
                                       const float* d_dy, const float* d_dz, const float* d_grad_out,
                                       float* d_grad_field, float* d_grad_src) {
  if (!ctx) return BRC_ERR_INVALID;
  if (!d_src || !d_dx || !d_dy || !d_dz || !d_grad_out || (!d_grad_field && !d_grad_src) || W <= 0 || H <= 0 ||
      D <= 0)
    return ctx->fail(BRC_ERR_INVALID, "brc_warp_field_backward: bad argument");
  cudaSetDevice(ctx->device);
  if (d_grad_src)
    BRC_TRY(ctx, cudaMemsetAsync(d_grad_src, 0, sizeof(float) * W * (size_t)H * D, ctx->stream()), "memset");
  BRC_TRY(ctx, brc::warp_field_backward(d_src, W, H, D, d_dx, d_dy, d_dz, d_grad_out, d_grad_field, d_grad_src,
                                        ctx->stream()),
          "warp_field_backward");
  ctx->launches += 1;
  return BRC_OK;
}
