// internal.h -- host-side launchers of the kernels (namespace brc), shared by
// the C-ABI (capi.cu) and the multi-step drivers (drivers.cu).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace brc {
// filter3d.cu
cudaError_t filter3d_init();
// tz: z depth of the output block (filter3d_tz_candidates), 0 for the
// untimed choice filter3d_default_tz(D).
cudaError_t filter3d_fp32(const float* vol, int W, int H, int D, int batch, long long stride,
                          const float* h_filters, int nfilt, float* out, ActiveSet act, cudaStream_t st,
                          bool allow_symmetric = true, int tz = 0);
int filter3d_tz_candidates(int* tz, int max_n);
int filter3d_default_tz(int D);
// The bank is even/odd symmetric (the even/odd kernel can take it).
bool filter3d_bank_symmetric(const float* h_filters, int nfilt);
// registration.cu
// Normal equations of batch instances, one CTA per `zpb` interior slices of
// an instance (the single-call and allocation-free entry points).
cudaError_t normal_eq_partials(const float* q1, long long q1_stride_floats, const float* q2, int W,
                               int H, int D, int batch, double* partials, int nblk, int zpb, cudaStream_t st);
// Normal equations in the z-marching form (certainty smoothing fused in when
// cert_sigma > 0): partial rows per instance and the launch.
int normal_eq_march_blocks(int W, int H, int D, int* ntx, int* nty, int* zs);
cudaError_t normal_eq_march(const float* q1, long long q1_stride_floats, const float* q2, int W, int H, int D,
                            int batch, double* partials, int nblk, ActiveSet act, cudaStream_t st,
                            float cert_sigma);
cudaError_t assemble_normal_eq(const double* partials, int nblk, int batch, double* A, double* h,
                               cudaStream_t st);
// One iteration's solve and update of the instances in `act` (its
// iteration it; act.list not null); those whose update is not yet
// below tol are appended to list (it + 1) % 3 of `lists` / `counts` (and
// conv_iter[b] = it records the others); count (it + 2) % 3 is reset for
// the iteration after next.
cudaError_t solve_update(const double* partials, int nblk, int batch, int type, float tol, int W,
                         int H, int D, float* params, float* rotations, int* conv_iter,
                         int* iterations, int* status, ActiveSet act, int* lists, int* counts, cudaStream_t st);
// *iter += 1; with use_cond, the condition of the WHILE node that runs the
// loop is set (continue while *iter < max_it and count *iter % 3 > 0) and
// *iters_run counts the iteration.
cudaError_t iteration_control(int* iter, const int* counts, int max_it, cudaGraphConditionalHandle cond,
                              bool use_cond, unsigned long long* iters_run, cudaStream_t st);
// list0[i] = i for i < batch, counts[0] = batch, counts[1] = counts[2] = 0.
cudaError_t active_init(int* list0, int* counts, int batch, cudaStream_t st);
cudaError_t solve_given(const double* A, const double* h, int batch, float* p, cudaStream_t st);
cudaError_t warp_affine(const float* src, long long src_stride, int W, int H, int D, int batch,
                        const float* params, float* out, long long out_stride, ActiveSet act,
                        cudaStream_t st);
// batch instances blockIdx.y: src, field (dx, dy, dz) and out advance by
// their strides (floats) per instance.
cudaError_t warp_field(const float* src, int W, int H, int D, const float* dx, const float* dy,
                       const float* dz, float* out, cudaStream_t st, int batch = 1, long long src_stride = 0,
                       long long field_stride = 0, long long out_stride = 0);
cudaError_t rescale_linear(const float* src, int W, int H, int D, float* out, int W2, int H2, int D2,
                           cudaStream_t st);
// zchunk: planes per z chunk of a CTA (0: the untimed choice
// smooth3d_default_chunk); every choice gives the same result.
cudaError_t smooth3d(const float* vol, int W, int H, int D, int batch, const float* fx,
                     const float* fy, const float* fz, const float* cert, const float* scert,
                     float* tmp1, float* tmp2, float* out, cudaStream_t st, int accumulate = 0, int zchunk = 0);
int smooth3d_default_chunk(int W, int H, int D, int batch);
int smooth3d_chunk_candidates(int D, int* zc, int max_n);
// out[i] = phase_atan2(y[i], x[i]) (the arctangent of the phase kernels).
cudaError_t phase_atan2_eval(const float* y, const float* x, float* out, long long n, cudaStream_t st);
cudaError_t multiply_mask(float* vols, const float* mask, long long V, int batch, cudaStream_t st);
// Phase difference, certainty and phase gradient along `axis` of one filter
// pair (the reference's linear formulas; outputs may be null).
cudaError_t phase_volumes(const float* q1, const float* q2, int W, int H, int D, int axis, float* pd, float* cert,
                          float* grad, cudaStream_t st);
// nonlinear.cu
// The per-voxel steps of a nonlinear iteration for `batch` instances (grid
// dimension y): t6 / q2 hold 6 (complex) volumes per instance, a6 and h3
// advance by ah_stride floats per instance, d3 by 3 volumes, maxbits by one
// word; q1 (the reference's responses) is shared.
cudaError_t tensor_norm_max(const float* t6, long long V, float* a11, unsigned int* maxbits, cudaStream_t st,
                            int batch = 1, long long t_stride = 0, long long a_stride = 0);
cudaError_t nonlinear_ah(const float* q1, const float* q2, float* t6, long long V,
                         const unsigned int* maxbits, const float* m36, const float* dirs18, float* a6,
                         float* h3, cudaStream_t st, int batch = 1, long long ah_stride = 0);
cudaError_t tensor_components(const float* q2, long long V, const float* m36, float* t6, cudaStream_t st,
                              int batch = 1);
cudaError_t displacement_update(const float* a6, const float* h3, long long V, int fp64, float* d3,
                                cudaStream_t st, int batch = 1, long long ah_stride = 0);
cudaError_t rescale_batch(const float* src, int W, int H, int D, int batch, float* out, int W2, int H2,
                          int D2, float factor, cudaStream_t st);
cudaError_t compose(float* total, const float* add, int batch, float tscale, cudaStream_t st);
cudaError_t add_volumes(float* out, const float* a, const float* b, long long n, cudaStream_t st);
}  // namespace brc

namespace brc {
cudaError_t resize_to_grid(const float* src, int W, int H, int D, float vx, float vy, float vz, float* out,
                           int W2, int H2, int D2, float nvx, float nvy, float nvz, int mm_z_cut,
                           cudaStream_t st);
cudaError_t mass_moments(const float* vol, int W, int H, int D, double* sums, cudaStream_t st);
// Ragged batch of resamples onto one grid, one launch: subject b (device
// pointer srcs[b], size dims3n[3b..3b+2], voxel size vox3n[3b..3b+2]) into
// out + b W2 H2 D2.  h_jobs / d_jobs: n * resize_job_bytes() of host and
// device staging for the per-subject descriptors (pageable host memory is
// fine: the copy is staged before the call returns).
size_t resize_job_bytes();
cudaError_t resize_to_grid_ragged(int n, const float* const* srcs, const int* dims3n, const float* vox3n,
                                  void* h_jobs, void* d_jobs, float* out, int W2, int H2, int D2,
                                  const float* new_vox3, int mm_z_cut, cudaStream_t st);
// 4D transforms with interpolation 0 (NEAREST) or 1 (LINEAR), T volumes of
// W x H x D one after another; the affine parameters are host values.
cudaError_t resize_to_grid_batch(const float* src, int W, int H, int D, int T, float vx, float vy, float vz,
                                 float* out, int W2, int H2, int D2, float nvx, float nvy, float nvz, int mm_z_cut,
                                 int interp, cudaStream_t st);
cudaError_t transform_affine(const float* src, int W, int H, int D, int T, const float* p12, int interp,
                             float* out, cudaStream_t st);
cudaError_t transform_field(const float* src, int W, int H, int D, int T, const float* dx, const float* dy,
                            const float* dz, int interp, float* out, cudaStream_t st);
cudaError_t combine_field(float* dx, float* dy, float* dz, int W, int H, int D, const float* p12, cudaStream_t st);
cudaError_t add_affine_to_field(float* field, int W, int H, int D, const float* p12, cudaStream_t st);
// Host composition total = new * old of two parameter vectors (4x4 affine
// matrices in double); total may alias old12.
void host_add_affine(const float* old12, const float* new12, float* total);
// Host inverse of a parameter vector (4x4 affine matrix in double).
void host_invert_affine(const float* p12, float* inv12);
}  // namespace brc

namespace brc {
// adjoint.cu
cudaError_t filter3d_adjoint(const float* grad, int W, int H, int D, int batch, const float* h_filters, int nfilt,
                             float* out, cudaStream_t st);
int warp_affine_backward_blocks(long long V);
cudaError_t warp_affine_backward(const float* src, int W, int H, int D, int batch, const float* params,
                                 const float* gout, double* partials, int nblk, double* gparams, float* gsrc,
                                 cudaStream_t st);
cudaError_t warp_field_backward(const float* src, int W, int H, int D, const float* dx, const float* dy,
                                const float* dz, const float* gout, float* gfield, float* gsrc,
                                cudaStream_t st);
}  // namespace brc
