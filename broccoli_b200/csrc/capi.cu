// capi.cu -- the C-ABI of libbroccoli_b200 (include/broccoli_b200.h):
// context and workspace management, argument checking, the batched
// registration driver (optionally captured once into a CUDA graph and
// replayed) and the host-buffer motion-correction entry point.
#include <cuda_runtime.h>
#include <limits.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/broccoli_b200.h"
#include "common.cuh"

#include "capi_ctx.h"
#include "internal.h"

namespace {

uint64_t fnv1a(const void* data, size_t n, uint64_t h = 1469598103934665603ull) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

// Interior slices per CTA of the normal-equation reduction: about 4k
// interior voxels per CTA.
int pick_zpb(int W, int H) {
  const long long plane = (long long)(W > 6 ? W - 6 : 1) * (H > 6 ? H - 6 : 1);
  long long z = 4096 / (plane > 0 ? plane : 1);
  if (z < 1) z = 1;
  if (z > 64) z = 64;
  return (int)z;
}

}  // namespace

static bool bad_dims(int W, int H, int D) {
  return W <= 0 || H <= 0 || D <= 0 || (long long)W * H * D > (1ll << 31);
}

int brc_ctx::taps_for(const float* h_filters, int nfilt, bool tf32, const uint16_t** d_taps) {
  const uint64_t key = fnv1a(h_filters, sizeof(float) * brc::kFilterFloats * (size_t)nfilt,
                             1469598103934665603ull ^ (uint64_t)nfilt ^ (tf32 ? 0x100ull : 0ull));
  auto it = tc_taps.find(key);
  if (it == tc_taps.end()) {
    if (tc_taps.size() >= 16) {
      graphs.clear();  // graphs may hold the pointers released here
      tc_taps.clear();
    }
    std::vector<uint16_t> packed(brc::tc::packed_tap_bytes(nfilt, tf32) / 2);
    brc::tc::pack_taps(h_filters, nfilt, packed.data(), tf32);
    std::unique_ptr<DevBuf> buf(new DevBuf());
    BRC_TRY(this, buf->ensure(packed.size() * 2), "alloc taps");
    BRC_TRY(this, cudaMemcpy(buf->ptr, packed.data(), packed.size() * 2, cudaMemcpyHostToDevice), "upload taps");
    it = tc_taps.emplace(key, std::move(buf)).first;
  }
  *d_taps = it->second->as<uint16_t>();
  return BRC_OK;
}

int brc_ctx::check_tc_err() {
  int flag = 0;
  BRC_TRY(this, cudaMemcpy(&flag, tc_err.ptr, sizeof(int), cudaMemcpyDeviceToHost), "read wait flag");
  if (flag == 0) return BRC_OK;
  BRC_TRY(this, cudaMemset(tc_err.ptr, 0, sizeof(int)), "clear wait flag");
  return fail(BRC_ERR_TIMEOUT, "a bounded wait of the tensor-core filtering kernel gave up");
}

int brc_ctx::tune_tc(int nfilt, int W, int H, int D, const uint16_t* d_taps, bool tf32, int* ty) {
  const auto key = std::make_tuple(nfilt + (tf32 ? 100 : 0), W, H, D);
  auto it = tc_tuned.find(key);
  if (it != tc_tuned.end()) {
    *ty = it->second;
    return BRC_OK;
  }
  int tys[3];
  const int n = brc::tc::candidate_tys(nfilt, H, D, tys, 3, tf32);
  if (n <= 0) return fail(BRC_ERR_UNSUPPORTED, "volume shape not supported by the tensor-core filtering");
  *ty = tys[0];
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BRC_TRY(this, cudaStreamIsCapturing(stream(), &cap), "capture status");
  if (cap != cudaStreamCaptureStatusNone) return BRC_OK;  // no timing inside a capture
  if (n > 1) {
    // time each candidate on zero-filled scratch volumes (the kernel's
    // work does not depend on the data): one warm launch, best of three
    const long long V = (long long)W * H * D;
    long long nb = (1ll << 24) / (V > 0 ? V : 1);
    nb = nb < 1 ? 1 : (nb > 32 ? 32 : nb);
    BRC_TRY(this, cudaStreamSynchronize(stream()), "synchronize");
    BRC_TRY(this, tmp1.ensure(sizeof(float) * (size_t)(V * nb)), "alloc");
    BRC_TRY(this, tmp2.ensure(sizeof(float) * (size_t)(V * nb) * 2 * nfilt), "alloc");
    BRC_TRY(this, cudaMemsetAsync(tmp1.ptr, 0, sizeof(float) * (size_t)(V * nb), own_stream), "memset");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BRC_TRY(this, cudaEventCreate(&e0), "event");
    if (cudaEventCreate(&e1) != cudaSuccess) {
      cudaEventDestroy(e0);
      return fail(BRC_ERR_CUDA, "event");
    }
    float best = -1.f;
    cudaError_t err = cudaSuccess;
    for (int c = 0; c < n && err == cudaSuccess; c++) {
      const brc::tc::Geometry g = brc::tc::make_geometry(nfilt, H, D, tys[c], tf32);
      float ms_best = -1.f;
      for (int rep = 0; rep < 4 && err == cudaSuccess; rep++) {
        err = cudaEventRecord(e0, own_stream);
        if (err == cudaSuccess)
          err = brc::tc::launch(tmp1.as<float>(), W, H, D, (int)nb, V, d_taps, nfilt, tmp2.as<float>(),
                                brc::all_instances(), tc_err.as<int>(), g, own_stream, tf32);
        if (err == cudaSuccess) err = cudaEventRecord(e1, own_stream);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err == cudaSuccess && rep > 0 && (ms_best < 0.f || ms < ms_best)) ms_best = ms;
      }
      if (err == cudaSuccess && (best < 0.f || ms_best < best)) {
        best = ms_best;
        *ty = tys[c];
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BRC_TRY(this, err, "tile timing");
  }
  tc_tuned[key] = *ty;
  return BRC_OK;
}

int brc_ctx::smooth(const float* vol, int W, int H, int D, int batch, const float* fx, const float* fy,
                    const float* fz, const float* cert, const float* scert, float* tmp1, float* tmp2, float* out,
                    cudaStream_t st, int accumulate, float* tune_out) {
  const auto key = std::make_tuple(W, H, D, batch, (cert ? 1 : 0) + (scert ? 2 : 0));
  auto it = smooth_tuned.find(key);
  if (it != smooth_tuned.end()) {
    BRC_TRY(this, brc::smooth3d(vol, W, H, D, batch, fx, fy, fz, cert, scert, tmp1, tmp2, out, st, accumulate,
                                it->second),
            "smooth3d");
    return BRC_OK;
  }
  const long long V = (long long)W * H * D;
  const size_t bytes = sizeof(float) * (size_t)V * batch;
  // the timing runs write `dst`: the output itself, or tune_out for an
  // accumulating call
  float* dst = accumulate ? tune_out : out;
  auto overlaps = [&](const float* a, size_t na) {
    const char *o0 = reinterpret_cast<const char*>(dst), *a0 = reinterpret_cast<const char*>(a);
    return a != nullptr && o0 < a0 + na && a0 < o0 + bytes;
  };
  const bool alias = dst == nullptr || overlaps(vol, bytes) || overlaps(cert, sizeof(float) * (size_t)V) ||
                     overlaps(scert, sizeof(float) * (size_t)V) || (accumulate && overlaps(out, bytes));
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BRC_TRY(this, cudaStreamIsCapturing(st, &cap), "capture status");
  int cand[8];
  const int n = brc::smooth3d_chunk_candidates(D, cand, 8);
  if (alias || cap != cudaStreamCaptureStatusNone || n < 2) {
    BRC_TRY(this, brc::smooth3d(vol, W, H, D, batch, fx, fy, fz, cert, scert, tmp1, tmp2, out, st, accumulate),
            "smooth3d");
    return BRC_OK;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BRC_TRY(this, cudaEventCreate(&e0), "event");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(BRC_ERR_CUDA, "event");
  }
  float best = -1.f;
  int zbest = cand[0];
  cudaError_t err = cudaSuccess;
  for (int c = 0; c < n && err == cudaSuccess; c++) {
    float ms_best = -1.f;
    for (int rep = 0; rep < 3 && err == cudaSuccess; rep++) {
      err = cudaEventRecord(e0, st);
      if (err == cudaSuccess)
        err = brc::smooth3d(vol, W, H, D, batch, fx, fy, fz, cert, scert, tmp1, tmp2, dst, st, 0, cand[c]);
      if (err == cudaSuccess) err = cudaEventRecord(e1, st);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
      if (err == cudaSuccess && rep > 0 && (ms_best < 0.f || ms < ms_best)) ms_best = ms;
    }
    if (err == cudaSuccess && (best < 0.f || ms_best < best)) {
      best = ms_best;
      zbest = cand[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BRC_TRY(this, err, "z-chunk timing");
  smooth_tuned[key] = zbest;
  if (accumulate)
    BRC_TRY(this, brc::smooth3d(vol, W, H, D, batch, fx, fy, fz, cert, scert, tmp1, tmp2, out, st, accumulate, zbest),
            "smooth3d");
  return BRC_OK;
}

int brc_ctx::tune_fp32(const float* h_filters, int nfilt, bool sym, int W, int H, int D, int* tz) {
  sym = sym && brc::filter3d_bank_symmetric(h_filters, nfilt);  // the kernel the launches will take
  const auto key = std::make_tuple(nfilt + (sym ? 100 : 0), W, H, D);
  auto it = fp32_tuned.find(key);
  if (it != fp32_tuned.end()) {
    *tz = it->second;
    return BRC_OK;
  }
  *tz = brc::filter3d_default_tz(D);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BRC_TRY(this, cudaStreamIsCapturing(stream(), &cap), "capture status");
  if (cap != cudaStreamCaptureStatusNone) return BRC_OK;  // no timing inside a capture
  int cand[8];
  const int n = brc::filter3d_tz_candidates(cand, 8);
  // time each z depth on zero-filled scratch volumes (the kernels' work does
  // not depend on the data, only on the shape and on whether the bank is
  // even/odd symmetric): one warm launch, best of three
  const long long V = (long long)W * H * D;
  long long nb = (1ll << 24) / (V > 0 ? V : 1);
  nb = nb < 1 ? 1 : (nb > 32 ? 32 : nb);
  BRC_TRY(this, cudaStreamSynchronize(stream()), "synchronize");
  BRC_TRY(this, tmp1.ensure(sizeof(float) * (size_t)(V * nb)), "alloc");
  BRC_TRY(this, tmp2.ensure(sizeof(float) * (size_t)(V * nb) * 2 * nfilt), "alloc");
  BRC_TRY(this, cudaMemsetAsync(tmp1.ptr, 0, sizeof(float) * (size_t)(V * nb), own_stream), "memset");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BRC_TRY(this, cudaEventCreate(&e0), "event");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(BRC_ERR_CUDA, "event");
  }
  float best = -1.f;
  cudaError_t err = cudaSuccess;
  for (int c = 0; c < n && err == cudaSuccess; c++) {
    float ms_best = -1.f;
    for (int rep = 0; rep < 4 && err == cudaSuccess; rep++) {
      err = cudaEventRecord(e0, own_stream);
      if (err == cudaSuccess)
        err = brc::filter3d_fp32(tmp1.as<float>(), W, H, D, (int)nb, V, h_filters, nfilt, tmp2.as<float>(),
                                 brc::all_instances(), own_stream, sym, cand[c]);
      if (err == cudaSuccess) err = cudaEventRecord(e1, own_stream);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
      if (err == cudaSuccess && rep > 0 && (ms_best < 0.f || ms < ms_best)) ms_best = ms;
    }
    if (err == cudaSuccess && (best < 0.f || ms_best < best)) {
      best = ms_best;
      *tz = cand[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BRC_TRY(this, err, "z-depth timing");
  fp32_tuned[key] = *tz;
  return BRC_OK;
}

int make_filter_path(brc_ctx* ctx, const float* h_filters, int nfilt, int precision, int W, int H, int D,
                     FilterPath* fp) {
  if (nfilt != 3 && nfilt != 6) return ctx->fail(BRC_ERR_INVALID, "filtering needs 3 or 6 filters");
  fp->precision = precision;
  fp->h_filters = h_filters;
  fp->nfilt = nfilt;
  fp->d_taps = nullptr;
  fp->d_err = ctx->tc_err.as<int>();
  if (precision == BRC_PREC_FP32 || precision == BRC_PREC_FP32_GENERAL)
    return ctx->tune_fp32(h_filters, nfilt, precision == BRC_PREC_FP32, W, H, D, &fp->tz);
  if (precision != BRC_PREC_BF16X3 && precision != BRC_PREC_TF32)
    return ctx->fail(BRC_ERR_UNSUPPORTED, "unknown precision");
  const bool tf32 = precision == BRC_PREC_TF32;
  int st = ctx->taps_for(h_filters, nfilt, tf32, &fp->d_taps);
  if (st != BRC_OK) return st;
  int ty = 0;
  st = ctx->tune_tc(nfilt, W, H, D, fp->d_taps, tf32, &ty);
  if (st != BRC_OK) return st;
  fp->g = brc::tc::make_geometry(nfilt, H, D, ty, tf32);
  return BRC_OK;
}

cudaError_t run_filter(const FilterPath& fp, const float* vol, int W, int H, int D, int batch, long long stride,
                       float* out, brc::ActiveSet act, cudaStream_t st) {
  if (fp.precision == BRC_PREC_BF16X3 || fp.precision == BRC_PREC_TF32)
    return brc::tc::launch(vol, W, H, D, batch, stride, fp.d_taps, fp.nfilt, out, act, fp.d_err, fp.g, st,
                           fp.precision == BRC_PREC_TF32);
  return brc::filter3d_fp32(vol, W, H, D, batch, stride, fp.h_filters, fp.nfilt, out, act, st,
                            fp.precision == BRC_PREC_FP32, fp.tz);
}

extern "C" {

const char* brc_version(void) { return "broccoli_b200 0.1 (sm_100a)"; }

const char* brc_status_string(int s) {
  switch (s) {
    case BRC_OK: return "ok";
    case BRC_ERR_INVALID: return "invalid argument";
    case BRC_ERR_NOMEM: return "out of memory";
    case BRC_ERR_CUDA: return "CUDA error";
    case BRC_ERR_TIMEOUT: return "device-side wait timed out";
    case BRC_ERR_NODEVICE: return "no usable CUDA device";
    case BRC_ERR_UNSUPPORTED: return "unsupported option";
    case BRC_ERR_NONFINITE: return "non-finite solution";
    case BRC_ERR_SCRATCH_LIMIT: return "request exceeds the fixed scratch of the no-allocation entry point";
    default: return "unknown status";
  }
}

const char* brc_last_error(const brc_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int brc_ctx_create(int device, brc_ctx** out) {
  if (!out) return BRC_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return BRC_ERR_NODEVICE;
  if (device < 0 || device >= n) return BRC_ERR_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return BRC_ERR_NODEVICE;
  if (prop.major != 10) return BRC_ERR_NODEVICE;  // built for sm_100a only
  std::unique_ptr<brc_ctx> ctx(new brc_ctx());
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return BRC_ERR_NODEVICE;
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return BRC_ERR_CUDA;
  if (cudaEventCreateWithFlags(&ctx->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_out, cudaEventDisableTiming) != cudaSuccess)
    return BRC_ERR_CUDA;
  if (brc::filter3d_init() != cudaSuccess || brc::tc::init() != cudaSuccess) return BRC_ERR_CUDA;
  if (ctx->tc_err.ensure(16) != cudaSuccess || cudaMemset(ctx->tc_err.ptr, 0, 16) != cudaSuccess)
    return BRC_ERR_NOMEM;
  if (ctx->iters_run.ensure(16) != cudaSuccess || cudaMemset(ctx->iters_run.ptr, 0, 16) != cudaSuccess)
    return BRC_ERR_NOMEM;
  *out = ctx.release();
  return BRC_OK;
}

int brc_ctx_destroy(brc_ctx* ctx) {
  BRC_CHECK_CTX(ctx);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->own_stream);
  if (ctx->use_user_stream) cudaStreamSynchronize(ctx->user_stream);
  ctx->graphs.clear();
  if (ctx->ev_in) cudaEventDestroy(ctx->ev_in);
  if (ctx->ev_out) cudaEventDestroy(ctx->ev_out);
  for (int c = 0; c < brc_ctx::kMaxChunks; c++) {
    if (ctx->ev_chunk_in[c]) cudaEventDestroy(ctx->ev_chunk_in[c]);
    if (ctx->ev_chunk_done[c]) cudaEventDestroy(ctx->ev_chunk_done[c]);
  }
  if (ctx->copy_in) {
    cudaStreamSynchronize(ctx->copy_in);
    cudaStreamDestroy(ctx->copy_in);
  }
  if (ctx->copy_out) {
    cudaStreamSynchronize(ctx->copy_out);
    cudaStreamDestroy(ctx->copy_out);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  if (ctx->body_stream) cudaStreamDestroy(ctx->body_stream);
  delete ctx;
  return BRC_OK;
}

int brc_ctx_set_stream(brc_ctx* ctx, void* s) {
  BRC_CHECK_CTX(ctx);
  if (s == BRC_OWN_STREAM) {
    ctx->use_user_stream = false;
    ctx->user_stream = nullptr;
  } else {
    ctx->use_user_stream = true;
    ctx->user_stream = static_cast<cudaStream_t>(s);
  }
  return BRC_OK;
}

void* brc_ctx_stream(brc_ctx* ctx) { return ctx ? (void*)ctx->stream() : nullptr; }

int brc_ctx_synchronize(brc_ctx* ctx) {
  BRC_CHECK_CTX(ctx);
  BRC_TRY(ctx, cudaStreamSynchronize(ctx->stream()), "synchronize");
  return ctx->check_tc_err();
}

int brc_selftest_bounded_wait(brc_ctx* ctx, int wait_ms) {
  BRC_CHECK_CTX(ctx);
  if (wait_ms < 1 || wait_ms > 1000) return ctx->fail(BRC_ERR_INVALID, "brc_selftest_bounded_wait: 1..1000 ms");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::tc::bounded_wait_probe(wait_ms, ctx->tc_err.as<int>(), ctx->stream()), "bounded wait probe");
  ctx->launches += 1;
  return BRC_OK;
}

int brc_selftest_phase_atan2(brc_ctx* ctx, const float* d_y, const float* d_x, float* d_out, long long n) {
  BRC_CHECK_CTX(ctx);
  if (n < 0 || (n > 0 && (!d_y || !d_x || !d_out)))
    return ctx->fail(BRC_ERR_INVALID, "brc_selftest_phase_atan2: bad pointer or size");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::phase_atan2_eval(d_y, d_x, d_out, n, ctx->stream()), "phase_atan2");
  ctx->launches += n > 0 ? 1 : 0;
  return BRC_OK;
}

size_t brc_ctx_workspace_bytes(const brc_ctx* ctx) { return ctx ? ctx->workspace() : 0; }

unsigned long long brc_ctx_kernel_launches(const brc_ctx* ctx) {
  if (!ctx) return 0;
  // the kernels of the graph-run loop iterations: 5 per iteration the
  // device ran (filtering, normal equations, solve, warp, control)
  unsigned long long it = 0;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream());
  cudaStreamSynchronize(ctx->own_stream);
  if (ctx->iters_run.ptr && cudaMemcpy(&it, ctx->iters_run.ptr, sizeof(it), cudaMemcpyDeviceToHost) != cudaSuccess)
    it = 0;
  return ctx->launches + 5ull * it;
}

int brc_filter3d(brc_ctx* ctx, const float* d_vol, int W, int H, int D, int batch,
                 long long vol_stride, const float* h_filters, int nfilt, int precision,
                 float* d_out) {
  BRC_CHECK_CTX(ctx);
  if (!d_vol || !d_out || !h_filters || bad_dims(W, H, D) || batch <= 0 || batch > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_filter3d: bad pointer or size");
  if (nfilt != 3 && nfilt != 6) return ctx->fail(BRC_ERR_INVALID, "brc_filter3d: nfilt must be 3 or 6");
  if (batch > 1 && vol_stride < (long long)W * H * D)
    return ctx->fail(BRC_ERR_INVALID, "brc_filter3d: vol_stride smaller than a volume");
  cudaSetDevice(ctx->device);
  FilterPath fp;
  const int ps = make_filter_path(ctx, h_filters, nfilt, precision, W, H, D, &fp);
  if (ps != BRC_OK) return ps;
  BRC_TRY(ctx, run_filter(fp, d_vol, W, H, D, batch, vol_stride, d_out, brc::all_instances(), ctx->stream()),
          "filter3d");
  ctx->launches += filter_launches(fp);
  return BRC_OK;
}

int brc_normal_equations(brc_ctx* ctx, const float* d_q1, long long q1_stride, const float* d_q2,
                         int W, int H, int D, int batch, double* d_A, double* d_h) {
  BRC_CHECK_CTX(ctx);
  if (!d_q1 || !d_q2 || !d_A || !d_h || bad_dims(W, H, D) || batch <= 0 || batch > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_normal_equations: bad pointer or size");
  cudaSetDevice(ctx->device);
  const int zpb = pick_zpb(W, H);
  const int nint = D - 6 > 0 ? D - 6 : 1;
  const int nblk = (nint + zpb - 1) / zpb;
  BRC_TRY(ctx, ctx->partials.ensure(sizeof(double) * brc::kNSums * nblk * (size_t)batch), "alloc");
  BRC_TRY(ctx, brc::normal_eq_partials(d_q1, q1_stride, d_q2, W, H, D, batch,
                                       ctx->partials.as<double>(), nblk, zpb, ctx->stream()),
          "normal_eq_partials");
  BRC_TRY(ctx, brc::assemble_normal_eq(ctx->partials.as<double>(), nblk, batch, d_A, d_h, ctx->stream()),
          "assemble");
  ctx->launches += 2;
  return BRC_OK;
}

int brc_solve_affine_fp64(brc_ctx* ctx, const double* d_A, const double* d_h, int batch, float* d_p) {
  BRC_CHECK_CTX(ctx);
  if (!d_A || !d_h || !d_p || batch <= 0) return ctx->fail(BRC_ERR_INVALID, "brc_solve_affine_fp64: bad argument");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::solve_given(d_A, d_h, batch, d_p, ctx->stream()), "solve");
  ctx->launches += 1;
  return BRC_OK;
}

int brc_warp_affine(brc_ctx* ctx, const float* d_src, int W, int H, int D, int batch,
                    const float* d_params, float* d_out) {
  BRC_CHECK_CTX(ctx);
  if (!d_src || !d_params || !d_out || bad_dims(W, H, D) || batch <= 0 || batch > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_warp_affine: bad pointer or size");
  if (d_src == d_out) return ctx->fail(BRC_ERR_INVALID, "brc_warp_affine: in-place warp not supported");
  cudaSetDevice(ctx->device);
  const long long V = (long long)W * H * D;
  BRC_TRY(ctx, brc::warp_affine(d_src, V, W, H, D, batch, d_params, d_out, V, brc::all_instances(), ctx->stream()),
          "warp_affine");
  ctx->launches += 1;
  return BRC_OK;
}

int brc_warp_field(brc_ctx* ctx, const float* d_src, int W, int H, int D, const float* d_dx,
                   const float* d_dy, const float* d_dz, float* d_out) {
  BRC_CHECK_CTX(ctx);
  if (!d_src || !d_dx || !d_dy || !d_dz || !d_out || bad_dims(W, H, D) || d_src == d_out)
    return ctx->fail(BRC_ERR_INVALID, "brc_warp_field: bad pointer or size");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::warp_field(d_src, W, H, D, d_dx, d_dy, d_dz, d_out, ctx->stream()), "warp_field");
  ctx->launches += 1;
  return BRC_OK;
}

int brc_rescale_linear(brc_ctx* ctx, const float* d_src, int W, int H, int D, float* d_out, int W2,
                       int H2, int D2) {
  BRC_CHECK_CTX(ctx);
  if (!d_src || !d_out || bad_dims(W, H, D) || bad_dims(W2, H2, D2) || W2 < 2 || H2 < 2 || D2 < 2)
    return ctx->fail(BRC_ERR_INVALID, "brc_rescale_linear: bad pointer or size");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::rescale_linear(d_src, W, H, D, d_out, W2, H2, D2, ctx->stream()), "rescale");
  ctx->launches += 1;
  return BRC_OK;
}

int brc_smooth3d(brc_ctx* ctx, const float* d_vol, int W, int H, int D, int batch, const float* h_fx,
                 const float* h_fy, const float* h_fz, const float* d_cert, const float* d_scert,
                 float* d_out) {
  BRC_CHECK_CTX(ctx);
  if (!d_vol || !d_out || !h_fx || !h_fy || !h_fz || bad_dims(W, H, D) || batch <= 0 || batch > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_smooth3d: bad pointer or size");
  cudaSetDevice(ctx->device);
  const size_t bytes = sizeof(float) * (size_t)W * H * D * batch;
  BRC_TRY(ctx, ctx->tmp1.ensure(bytes), "alloc");
  BRC_TRY(ctx, ctx->tmp2.ensure(bytes), "alloc");
  {
    const int s = ctx->smooth(d_vol, W, H, D, batch, h_fx, h_fy, h_fz, d_cert, d_scert, ctx->tmp1.as<float>(),
                              ctx->tmp2.as<float>(), d_out, ctx->stream());
    if (s != BRC_OK) return s;
  }
  ctx->launches += 1;
  return BRC_OK;
}

int brc_smooth_normalized(brc_ctx* ctx, const float* d_vols, int W, int H, int D, int T, const float* d_mask,
                          const float* h_fx, const float* h_fy, const float* h_fz, float* d_out) {
  BRC_CHECK_CTX(ctx);
  if (!d_vols || !d_mask || !d_out || !h_fx || !h_fy || !h_fz || bad_dims(W, H, D) || T <= 0 || T > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_smooth_normalized: bad pointer or size");
  cudaSetDevice(ctx->device);
  const long long V = (long long)W * H * D;
  const size_t bytes = sizeof(float) * (size_t)V * T;
  BRC_TRY(ctx, ctx->tmp1.ensure(bytes), "alloc");
  BRC_TRY(ctx, ctx->tmp2.ensure(bytes), "alloc");
  BRC_TRY(ctx, ctx->smask.ensure(sizeof(float) * (size_t)V), "alloc");
  const cudaStream_t st = ctx->stream();
  // smoothed certainty (all-ones certainty), then the certainty-weighted
  // smoothing of every volume divided by it, then the mask product
  int s = ctx->smooth(d_mask, W, H, D, 1, h_fx, h_fy, h_fz, nullptr, nullptr, ctx->tmp1.as<float>(),
                      ctx->tmp2.as<float>(), ctx->smask.as<float>(), st);
  if (s != BRC_OK) return s;
  s = ctx->smooth(d_vols, W, H, D, T, h_fx, h_fy, h_fz, d_mask, ctx->smask.as<float>(), ctx->tmp1.as<float>(),
                  ctx->tmp2.as<float>(), d_out, st);
  if (s != BRC_OK) return s;
  BRC_TRY(ctx, brc::multiply_mask(d_out, d_mask, V, T, st), "multiply mask");
  ctx->launches += 3;
  return BRC_OK;
}

int brc_device_alloc(brc_ctx* ctx, size_t bytes, void** d_out) {
  BRC_CHECK_CTX(ctx);
  if (!d_out) return ctx->fail(BRC_ERR_INVALID, "brc_device_alloc: null output");
  *d_out = nullptr;
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, cudaMalloc(d_out, bytes ? bytes : 1), "brc_device_alloc");
  return BRC_OK;
}

int brc_device_free(brc_ctx* ctx, void* d_ptr) {
  BRC_CHECK_CTX(ctx);
  if (!d_ptr) return BRC_OK;
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, cudaStreamSynchronize(ctx->stream()), "sync");
  BRC_TRY(ctx, cudaFree(d_ptr), "brc_device_free");
  return BRC_OK;
}

int brc_copy_to_device(brc_ctx* ctx, void* d_dst, const void* h_src, size_t bytes) {
  BRC_CHECK_CTX(ctx);
  if ((!d_dst || !h_src) && bytes) return ctx->fail(BRC_ERR_INVALID, "brc_copy_to_device: null pointer");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, ctx->stream()), "H2D");
  BRC_TRY(ctx, cudaStreamSynchronize(ctx->stream()), "sync");
  return BRC_OK;
}

int brc_copy_to_host(brc_ctx* ctx, void* h_dst, const void* d_src, size_t bytes) {
  BRC_CHECK_CTX(ctx);
  if ((!d_src || !h_dst) && bytes) return ctx->fail(BRC_ERR_INVALID, "brc_copy_to_host: null pointer");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, ctx->stream()), "D2H");
  BRC_TRY(ctx, cudaStreamSynchronize(ctx->stream()), "sync");
  return BRC_OK;
}

int brc_ctx_set_debug_outputs(brc_ctx* ctx, const brc_debug_outputs* outs) {
  BRC_CHECK_CTX(ctx);
  if (outs) {
    ctx->dbg = *outs;
    ctx->dbg_on = true;
  } else {
    ctx->dbg = brc_debug_outputs{};
    ctx->dbg_on = false;
  }
  return BRC_OK;
}

int brc_phase_volumes(brc_ctx* ctx, const float* d_q1, const float* d_q2, int W, int H, int D, int axis,
                      float* d_phase_diff, float* d_cert, float* d_grad) {
  BRC_CHECK_CTX(ctx);
  if (!d_q1 || !d_q2 || bad_dims(W, H, D) || axis < 0 || axis > 2)
    return ctx->fail(BRC_ERR_INVALID, "brc_phase_volumes: bad pointer, size or axis");
  if (!d_phase_diff && !d_cert && !d_grad) return BRC_OK;
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::phase_volumes(d_q1, d_q2, W, H, D, axis, d_phase_diff, d_cert, d_grad, ctx->stream()),
          "phase_volumes");
  ctx->launches += 1;
  return BRC_OK;
}

int brc_multiply_volumes(brc_ctx* ctx, float* d_vols, int W, int H, int D, int T, const float* d_mask) {
  BRC_CHECK_CTX(ctx);
  if (!d_vols || !d_mask || bad_dims(W, H, D) || T <= 0 || T > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_multiply_volumes: bad pointer or size");
  cudaSetDevice(ctx->device);
  BRC_TRY(ctx, brc::multiply_mask(d_vols, d_mask, (long long)W * H * D, T, ctx->stream()), "multiply");
  ctx->launches += 1;
  return BRC_OK;
}

void brc_linear_opts_default(brc_linear_opts* o, int iterations) {
  if (!o) return;
  o->iterations = iterations;
  o->type = BRC_AFFINE;
  o->precision = BRC_PREC_FP32;
  o->tolerance = 0.f;
  o->use_graph = 1;
  o->certainty_sigma_x100 = 0;
}

}  // extern "C"

namespace {

struct RegPlan {
  const float* ref;
  long long ref_stride;
  const float* moving;
  int W, H, D, batch;
  const float* filters;
  brc_linear_opts opts;
  float* params;
  float* aligned;
  float* rotations;
  int* iterations;
  // workspace
  float* q1;
  float* q2;
  double* partials;
  int* conv_iter;
  int* iters_ws;
  int* status;
  int* lists;   // 3 x batch: active instances of iterations it % 3
  int* counts;  // their lengths
  const int* iter;  // the iteration being run (device counter)
  int nblk;     // partial rows per instance of the normal-equation kernel
  FilterPath fpath;
};

// Queues the whole registration on stream st; returns the number of
// kernels launched or a negative brc_status.
long long enqueue_registration(brc_ctx* ctx, const RegPlan& p, cudaStream_t st) {
  const long long V = (long long)p.W * p.H * p.D;
  const int ref_batch = p.ref_stride ? p.batch : 1;
  long long kernels = 0;
  cudaError_t e;
  if ((e = cudaMemsetAsync(p.params, 0, sizeof(float) * 12 * p.batch, st)) != cudaSuccess)
    return ctx->cuda(e, "memset params");
  if ((e = cudaMemsetAsync(p.conv_iter, 0x7f, sizeof(int) * p.batch, st)) != cudaSuccess)
    return ctx->cuda(e, "memset ctl");
  if ((e = cudaMemsetAsync(p.iters_ws, 0, sizeof(int) * p.batch, st)) != cudaSuccess)
    return ctx->cuda(e, "memset ctl");
  if ((e = cudaMemsetAsync(p.status, 0, sizeof(int) * 2, st)) != cudaSuccess) return ctx->cuda(e, "memset");
  if ((e = brc::active_init(p.lists, p.counts, p.batch, st)) != cudaSuccess) return ctx->cuda(e, "active set");
  kernels++;
  if (p.rotations && (e = cudaMemsetAsync(p.rotations, 0, sizeof(float) * 3 * p.batch, st)) != cudaSuccess)
    return ctx->cuda(e, "memset rot");
  if ((e = run_filter(p.fpath, p.ref, p.W, p.H, p.D, ref_batch, p.ref_stride ? p.ref_stride : V, p.q1,
                      brc::all_instances(), st)) != cudaSuccess)
    return ctx->cuda(e, "filter3d(ref)");
  kernels += filter_launches(p.fpath);
  if (p.opts.iterations == 0 &&
      (e = cudaMemcpyAsync(p.aligned, p.moving, sizeof(float) * V * p.batch, cudaMemcpyDeviceToDevice,
                           st)) != cudaSuccess)
    return ctx->cuda(e, "copy");
  if (p.opts.iterations > 0) {
    // one iteration: filtering (of the moving volumes themselves at
    // iteration 0, of their warps later), normal equations, solve, warp;
    // with device_iter, the kernels read the iteration from the device
    // counter p.iter and a control kernel advances it
    auto one_iteration = [&](cudaStream_t s, int it, bool device_iter, bool cond_node,
                             cudaGraphConditionalHandle h) -> long long {
      const brc::ActiveSet act{p.lists, p.counts, device_iter ? p.iter : nullptr, it, p.batch};
      const float* cur = it == 0 ? p.moving : p.aligned;
      cudaError_t ee;
      if ((ee = run_filter(p.fpath, cur, p.W, p.H, p.D, p.batch, V, p.q2, act, s)) != cudaSuccess)
        return ctx->cuda(ee, "filter3d");
      if ((ee = brc::normal_eq_march(p.q1, p.ref_stride ? 6 * V : 0, p.q2, p.W, p.H, p.D, p.batch, p.partials,
                                     p.nblk, act, s, p.opts.certainty_sigma_x100 / 100.0f)) != cudaSuccess)
        return ctx->cuda(ee, "normal_eq");
      if ((ee = brc::solve_update(p.partials, p.nblk, p.batch, p.opts.type, p.opts.tolerance, p.W, p.H, p.D,
                                  p.params, p.rotations, p.conv_iter, p.iters_ws, p.status, act, p.lists, p.counts,
                                  s)) != cudaSuccess)
        return ctx->cuda(ee, "solve");
      if ((ee = brc::warp_affine(p.moving, V, p.W, p.H, p.D, p.batch, p.params, p.aligned, V, act, s)) !=
          cudaSuccess)
        return ctx->cuda(ee, "warp");
      if (!device_iter) return 3 + filter_launches(p.fpath);
      if ((ee = brc::iteration_control(const_cast<int*>(p.iter), p.counts, p.opts.iterations, h, cond_node,
                                       ctx->iters_run.as<unsigned long long>(), s)) != cudaSuccess)
        return ctx->cuda(ee, "iteration control");
      return 4 + filter_launches(p.fpath);
    };
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &cs)) != cudaSuccess) return ctx->cuda(e, "capture status");
    if (cs == cudaStreamCaptureStatusActive && p.opts.tolerance > 0.f && p.opts.iterations > 1) {
      // a graph with early exit: iteration 0, then one conditional WHILE
      // node whose body is one iteration on the device counter (set to 1 by
      // iteration 0's control kernel), its condition set on the device by
      // the control kernel: the loop stops as soon as every instance
      // converged, with no host round trip
      const long long k0 = one_iteration(st, 0, true, false, 0);
      if (k0 < 0) return k0;
      kernels += k0;
      cudaGraph_t graph = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps)) != cudaSuccess)
        return ctx->cuda(e, "capture info");
      cudaGraphConditionalHandle h;
      if ((e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
        return ctx->cuda(e, "conditional handle");
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      if ((e = cudaGraphAddNode(&node, graph, deps, ndeps, &cp)) != cudaSuccess) return ctx->cuda(e, "while node");
      if ((e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
        return ctx->cuda(e, "capture dependencies");
      if (!ctx->body_stream &&
          (e = cudaStreamCreateWithFlags(&ctx->body_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return ctx->cuda(e, "body stream");
      if ((e = cudaStreamBeginCaptureToGraph(ctx->body_stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return ctx->cuda(e, "body capture");
      const long long kb = one_iteration(ctx->body_stream, 1, true, true, h);
      cudaGraph_t body = nullptr;
      e = cudaStreamEndCapture(ctx->body_stream, &body);
      if (kb < 0) return kb;
      if (e != cudaSuccess) return ctx->cuda(e, "end body capture");
      // the kernels the body runs are counted on the device (iters_run)
    } else {
      // every iteration enqueued with its number (a graph without early
      // exit runs all of them anyway; without a graph the host loops)
      for (int it = 0; it < p.opts.iterations; it++) {
        const long long k = one_iteration(st, it, false, false, 0);
        if (k < 0) return k;
        kernels += k;
      }
    }
  }
  if (p.iterations &&
      (e = cudaMemcpyAsync(p.iterations, p.iters_ws, sizeof(int) * p.batch, cudaMemcpyDeviceToDevice,
                           st)) != cudaSuccess)
    return ctx->cuda(e, "copy iterations");
  return kernels;
}

// The reference's DEBUG reads of one AlignTwoVolumesLinear call
// (broccoli_lib.cpp:5285-5289, :5349-5354), for the last instance of the
// batch: the reference volume's three responses, and the z-axis phase
// difference, certainty and gradient of iteration 0, whose aligned volume
// is the moving volume itself (the parameters start at 0).  Synchronises.
int debug_linear(brc_ctx* ctx, const RegPlan& p, cudaStream_t st) {
  int s = debug_capture_check(ctx, "debug outputs");
  if (s != BRC_OK) return s;
  const long long V = (long long)p.W * p.H * p.D;
  const int b = p.batch - 1;
  const float* qref = p.q1 + (p.ref_stride ? 6 * V * b : 0);
  for (int k = 0; k < 3; k++)
    if (ctx->dbg.quadrature_responses[k])
      BRC_TRY(ctx, cudaMemcpyAsync(ctx->dbg.quadrature_responses[k], qref + 2 * V * k, sizeof(float) * 2 * V,
                                   cudaMemcpyDeviceToHost, st), "debug D2H");
  float* outs[3] = {ctx->dbg.phase_differences, ctx->dbg.phase_certainties, ctx->dbg.phase_gradients};
  if (p.opts.iterations > 0 && (outs[0] || outs[1] || outs[2])) {
    BRC_TRY(ctx, ctx->dbg_q.ensure(sizeof(float) * 6 * V), "alloc debug");
    BRC_TRY(ctx, ctx->dbg_v.ensure(sizeof(float) * 3 * V), "alloc debug");
    float* q = ctx->dbg_q.as<float>();
    float* v = ctx->dbg_v.as<float>();
    BRC_TRY(ctx, run_filter(p.fpath, p.moving + V * b, p.W, p.H, p.D, 1, V, q, brc::all_instances(), st),
            "debug filter");
    BRC_TRY(ctx, brc::phase_volumes(qref + 4 * V, q + 4 * V, p.W, p.H, p.D, 2, v, v + V, v + 2 * V, st),
            "debug phase");
    ctx->launches += 1 + filter_launches(p.fpath);
    for (int k = 0; k < 3; k++)
      if (outs[k])
        BRC_TRY(ctx, cudaMemcpyAsync(outs[k], v + V * k, sizeof(float) * V, cudaMemcpyDeviceToHost, st),
                "debug D2H");
  }
  BRC_TRY(ctx, cudaStreamSynchronize(st), "debug synchronize");
  return BRC_OK;
}

}  // namespace

int debug_capture_check(brc_ctx* ctx, const char* where) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  BRC_TRY(ctx, cudaStreamIsCapturing(ctx->stream(), &cs), "capture status");
  if (cs != cudaStreamCaptureStatusNone)
    return ctx->fail(BRC_ERR_UNSUPPORTED, std::string(where) + ": not available under stream capture");
  return BRC_OK;
}

extern "C" int brc_register_linear_batched(brc_ctx* ctx, const float* d_ref, long long ref_stride,
                                           const float* d_moving, int W, int H, int D, int batch,
                                           const float* h_filters, const brc_linear_opts* opts,
                                           float* d_params, float* d_aligned, float* d_rotations,
                                           int* d_iterations) {
  BRC_CHECK_CTX(ctx);
  if (!d_ref || !d_moving || !h_filters || !opts || !d_params || bad_dims(W, H, D) || batch <= 0 ||
      batch > 65535)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_linear_batched: bad pointer or size");
  if (opts->iterations < 0 || opts->iterations > 10000 || opts->type < 0 || opts->type > 2 ||
      !(opts->tolerance >= 0.f))
    return ctx->fail(BRC_ERR_INVALID, "brc_register_linear_batched: bad options");
  if (!brc_precision_valid(opts->precision))
    return ctx->fail(BRC_ERR_UNSUPPORTED, "brc_register_linear_batched: unknown precision");
  if (opts->certainty_sigma_x100 < 0)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_linear_batched: negative certainty sigma");
  const long long V = (long long)W * H * D;
  if (ref_stride != 0 && ref_stride < V)
    return ctx->fail(BRC_ERR_INVALID, "brc_register_linear_batched: ref_stride smaller than a volume");
  cudaSetDevice(ctx->device);

  RegPlan p;
  p.ref = d_ref;
  p.ref_stride = ref_stride;
  p.moving = d_moving;
  p.W = W;
  p.H = H;
  p.D = D;
  p.batch = batch;
  p.filters = h_filters;
  p.opts = *opts;
  p.params = d_params;
  p.rotations = d_rotations;
  p.iterations = d_iterations;
  {
    int ntx, nty, zs;
    p.nblk = brc::normal_eq_march_blocks(W, H, D, &ntx, &nty, &zs);
  }

  const size_t q1n = sizeof(float) * 6 * V * (ref_stride ? batch : 1);
  const size_t q2n = sizeof(float) * 6 * V * batch;
  BRC_TRY(ctx, ctx->q1.ensure(q1n), "alloc q1");
  BRC_TRY(ctx, ctx->q2.ensure(q2n), "alloc q2");
  BRC_TRY(ctx, ctx->partials.ensure(sizeof(double) * brc::kNSums * p.nblk * (size_t)batch), "alloc");
  BRC_TRY(ctx, ctx->ctl.ensure(sizeof(int) * (5 * (size_t)batch + 8)), "alloc ctl");
  if (!d_aligned) BRC_TRY(ctx, ctx->aligned.ensure(sizeof(float) * V * batch), "alloc aligned");
  p.aligned = d_aligned ? d_aligned : ctx->aligned.as<float>();
  p.q1 = ctx->q1.as<float>();
  p.q2 = ctx->q2.as<float>();
  p.partials = ctx->partials.as<double>();
  p.conv_iter = ctx->ctl.as<int>();
  p.iters_ws = p.conv_iter + batch;
  p.status = p.iters_ws + batch;
  p.iter = p.status + 1;
  p.lists = p.status + 4;
  p.counts = p.lists + 3 * (size_t)batch;
  {
    const int ps = make_filter_path(ctx, h_filters, 3, opts->precision, W, H, D, &p.fpath);
    if (ps != BRC_OK) return ps;
  }

  const cudaStream_t user = ctx->stream();
  if (!opts->use_graph) {
    long long k = enqueue_registration(ctx, p, user);
    if (k < 0) return (int)k;
    ctx->launches += k;
  } else {
    GraphKey key;
    const uint64_t fh = fnv1a(h_filters, sizeof(float) * 3 * brc::kFilterFloats);
    key.v = {(uint64_t)d_ref, (uint64_t)ref_stride, (uint64_t)d_moving, (uint64_t)W, (uint64_t)H,
             (uint64_t)D, (uint64_t)batch, fh, (uint64_t)opts->iterations, (uint64_t)opts->type,
             (uint64_t)fnv1a(&opts->tolerance, sizeof(float)), (uint64_t)d_params,
             (uint64_t)p.aligned, (uint64_t)d_rotations, (uint64_t)d_iterations,
             (uint64_t)ctx->q1.ptr, (uint64_t)ctx->q2.ptr, (uint64_t)ctx->partials.ptr,
             (uint64_t)ctx->ctl.ptr, (uint64_t)opts->certainty_sigma_x100,
             (uint64_t)opts->precision, (uint64_t)p.fpath.d_taps};
    auto itg = ctx->graphs.find(key);
    GraphEntry* ge = nullptr;
    if (itg == ctx->graphs.end()) {
      if (ctx->graphs.size() >= 64) ctx->graphs.clear();  // a bounded cache of instantiated graphs
      std::unique_ptr<GraphEntry> ne(new GraphEntry());
      cudaStream_t cs = ctx->own_stream;
      BRC_TRY(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
      long long k = enqueue_registration(ctx, p, cs);
      cudaGraph_t g = nullptr;
      cudaError_t ee = cudaStreamEndCapture(cs, &g);
      if (k < 0) {
        if (g) cudaGraphDestroy(g);
        return (int)k;
      }
      BRC_TRY(ctx, ee, "end capture");
      ne->graph = g;
      BRC_TRY(ctx, cudaGraphInstantiate(&ne->exec, g, 0), "instantiate");
      ne->kernels = (unsigned long long)k;
      ge = ne.get();
      ctx->graphs[key] = std::move(ne);
    } else {
      ge = itg->second.get();
    }
    // Order the replay on the caller's stream: own stream waits for the
    // caller, the caller waits for the replay.
    if (user != ctx->own_stream) {
      BRC_TRY(ctx, cudaEventRecord(ctx->ev_in, user), "event");
      BRC_TRY(ctx, cudaStreamWaitEvent(ctx->own_stream, ctx->ev_in, 0), "wait");
    }
    BRC_TRY(ctx, cudaGraphLaunch(ge->exec, ctx->own_stream), "graph launch");
    if (user != ctx->own_stream) {
      BRC_TRY(ctx, cudaEventRecord(ctx->ev_out, ctx->own_stream), "event");
      BRC_TRY(ctx, cudaStreamWaitEvent(user, ctx->ev_out, 0), "wait");
    }
    ctx->launches += ge->kernels;
  }
  if (ctx->dbg_on) return debug_linear(ctx, p, user);
  return BRC_OK;
}

extern "C" int brc_motion_correct(brc_ctx* ctx, float* h_volumes, int W, int H, int D, int T,
                                  const float* voxel_size3, const float* h_filters,
                                  const brc_linear_opts* opts, const float* h_reference,
                                  float* h_motion) {
  BRC_CHECK_CTX(ctx);
  if (!h_volumes || !h_filters || !opts || bad_dims(W, H, D) || T <= 0)
    return ctx->fail(BRC_ERR_INVALID, "brc_motion_correct: bad pointer or size");
  const long long V = (long long)W * H * D;
  const int first = h_reference ? 0 : 1;
  const int batch = T - first;
  float vs[3] = {1.f, 1.f, 1.f};
  if (voxel_size3) memcpy(vs, voxel_size3, sizeof(vs));
  if (h_motion)
    for (int k = 0; k < 6; k++) h_motion[k * T] = 0.f;
  if (batch <= 0) return BRC_OK;
  cudaSetDevice(ctx->device);
  const cudaStream_t st = ctx->stream();
  BRC_TRY(ctx, ctx->series.ensure(sizeof(float) * V * (T + 1)), "alloc series");
  BRC_TRY(ctx, ctx->corrected.ensure(sizeof(float) * V * batch), "alloc corrected");
  BRC_TRY(ctx, ctx->params.ensure(sizeof(float) * 12 * batch), "alloc params");
  BRC_TRY(ctx, ctx->rot.ensure(sizeof(float) * 3 * batch), "alloc rot");
  float* d_series = ctx->series.as<float>();
  BRC_TRY(ctx, ctx->ensure_copy_streams(), "copy streams");
  // Series of 64 or more volumes are registered in three chunks, an eighth,
  // the rest and an eighth, so that only a small upload precedes the first
  // registration and a small download follows the last, while the other
  // copies run on the copy engines under registration.  (Measured per call
  // on 199 volumes of 64x64x33, TF32, with the registration loop stopping on
  // the device: one chunk 13.2 ms; 19/161/19 11.27-11.40, 22/156/21 11.10,
  // 25/150/24 10.98-11.07, 28/144/27 11.04-11.06, 32/136/31 11.23-11.28;
  // four chunks 11.37-11.74, five 12.15 -- each chunk is a registration of
  // its own, and small ones use the GPU less well.)  Chunk 0's upload
  // includes the reference (volume 0, or h_reference).
  int nchunk = 1, csz[3] = {batch, 0, 0};
  if (batch >= 64) {
    nchunk = 3;
    csz[0] = csz[2] = batch / 8;
    csz[1] = batch - 2 * csz[0];
  }
  int cst[4] = {0, 0, 0, 0};
  for (int c = 0; c < nchunk; c++) cst[c + 1] = cst[c] + csz[c];
  // the copy streams start after work the caller queued before this call
  BRC_TRY(ctx, cudaEventRecord(ctx->ev_in, st), "event");
  BRC_TRY(ctx, cudaStreamWaitEvent(ctx->copy_in, ctx->ev_in, 0), "wait");
  BRC_TRY(ctx, cudaStreamWaitEvent(ctx->copy_out, ctx->ev_in, 0), "wait");
  const float* d_ref = d_series;
  if (h_reference) {
    BRC_TRY(ctx, cudaMemcpyAsync(d_series + V * T, h_reference, sizeof(float) * V, cudaMemcpyHostToDevice,
                                 ctx->copy_in), "H2D");
    d_ref = d_series + V * T;
  }
  for (int c = 0; c < nchunk; c++) {
    const long long lo = c == 0 ? 0 : first + (long long)cst[c];
    const long long hi = first + (long long)cst[c + 1];
    if (hi > lo)
      BRC_TRY(ctx, cudaMemcpyAsync(d_series + V * lo, h_volumes + V * lo, sizeof(float) * V * (hi - lo),
                                   cudaMemcpyHostToDevice, ctx->copy_in), "H2D");
    BRC_TRY(ctx, cudaEventRecord(ctx->ev_chunk_in[c], ctx->copy_in), "event");
  }
  brc_linear_opts o = *opts;
  o.type = BRC_RIGID;
  for (int c = 0; c < nchunk; c++) {
    const int i0 = cst[c];
    const int nb = csz[c];
    BRC_TRY(ctx, cudaStreamWaitEvent(st, ctx->ev_chunk_in[c], 0), "wait");
    if (nb > 0) {
      int s = brc_register_linear_batched(ctx, d_ref, 0, d_series + V * (first + i0), W, H, D, nb, h_filters, &o,
                                          ctx->params.as<float>() + 12 * (long long)i0,
                                          ctx->corrected.as<float>() + V * i0,
                                          ctx->rot.as<float>() + 3 * (long long)i0, nullptr);
      if (s != BRC_OK) {
        cudaStreamSynchronize(ctx->copy_in);
        cudaStreamSynchronize(ctx->copy_out);
        return s;
      }
    }
    BRC_TRY(ctx, cudaEventRecord(ctx->ev_chunk_done[c], st), "event");
    BRC_TRY(ctx, cudaStreamWaitEvent(ctx->copy_out, ctx->ev_chunk_done[c], 0), "wait");
    if (nb > 0)
      BRC_TRY(ctx, cudaMemcpyAsync(h_volumes + V * (first + i0), ctx->corrected.as<float>() + V * i0,
                                   sizeof(float) * V * nb, cudaMemcpyDeviceToHost, ctx->copy_out), "D2H");
  }
  std::vector<float> prm(12 * (size_t)batch), rot(3 * (size_t)batch);
  BRC_TRY(ctx, cudaMemcpyAsync(prm.data(), ctx->params.as<float>(), sizeof(float) * 12 * batch,
                               cudaMemcpyDeviceToHost, st), "D2H");
  BRC_TRY(ctx, cudaMemcpyAsync(rot.data(), ctx->rot.as<float>(), sizeof(float) * 3 * batch,
                               cudaMemcpyDeviceToHost, st), "D2H");
  BRC_TRY(ctx, cudaStreamSynchronize(st), "synchronize");
  BRC_TRY(ctx, cudaStreamSynchronize(ctx->copy_out), "synchronize");
  if (h_motion) {
    for (int i = 0; i < batch; i++) {
      const int t = first + i;
      h_motion[t + 0 * T] = prm[12 * i + 0] * vs[0];
      h_motion[t + 1 * T] = prm[12 * i + 1] * vs[1];
      h_motion[t + 2 * T] = prm[12 * i + 2] * vs[2];
      h_motion[t + 3 * T] = rot[3 * i + 0];
      h_motion[t + 4 * T] = rot[3 * i + 1];
      h_motion[t + 5 * T] = rot[3 * i + 2];
    }
  }
  return BRC_OK;
}
