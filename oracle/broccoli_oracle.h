/*
 * broccoli_oracle.h -- CPU restatement of BROCCOLI's registration and
 * filtering path.  TEST INFRASTRUCTURE ONLY: the product (libbroccoli_b200)
 * never links or calls this code.  It is the checker that the CUDA path is
 * compared against, and the timed CPU baseline of bench.py.
 *
 * Every function exists twice, with suffix _f32 (float arithmetic, the
 * parity target: same operation order as the reference's OpenCL kernels) and
 * _f64 (double arithmetic, the accuracy oracle).  `real` below is float or
 * double accordingly.
 *
 * Layouts follow the reference (code/Kernels/kernelRegistration.cpp:32-40):
 *   volume index  = x + y*W + z*W*H (+ t*W*H*D)
 *   7x7x7 filters = 343 reals, x fastest; one filter is re[343] then im[343]
 *   complex response = interleaved (re, im) pairs, one volume per filter
 *   parameters    = [tx ty tz a11-1 a12 a13 a21 a22-1 a23 a31 a32 a33-1]
 */
#ifndef BROCCOLI_ORACLE_H
#define BROCCOLI_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_TRANSLATION = 0, ORC_RIGID = 1, ORC_AFFINE = 2 };

#define ORC_DECLARE(real, SFX)                                                  \
  void orc_filter3d##SFX(const real* vol, int W, int H, int D,                  \
                         const real* filters, int nfilt, real* out);            \
  void orc_phase_diff_cert##SFX(const real* q1, const real* q2, long V,         \
                                real* pd, real* cert);                          \
  void orc_phase_grad##SFX(const real* q1, const real* q2, int axis, int W,     \
                           int H, int D, real* grad);                           \
  void orc_ah_axis##SFX(const real* pd, const real* grad, const real* cert,     \
                        int axis, int W, int H, int D, int filter_size,         \
                        real* A144, real* h12);                                 \
  void orc_normal_equations##SFX(const real* q1, const real* q2, int W, int H,  \
                                 int D, real* A144, real* h12);                 \
  void orc_normal_equations_smoothcert##SFX(const real* q1, const real* q2,     \
                                            int W, int H, int D, double sigma,  \
                                            real* A144, real* h12);             \
  void orc_solve##SFX(const real* A, const real* h, int n, real* p);            \
  void orc_remove_scaling##SFX(real* p12);                                      \
  void orc_add_affine##SFX(real* old12, const real* new12);                     \
  void orc_add_affine_next_scale##SFX(real* old12, const real* new12);          \
  void orc_rotation_angles##SFX(const real* p12, real* rot3);                   \
  void orc_warp_affine##SFX(const real* src, int W, int H, int D,               \
                            const real* p12, real* out);                        \
  void orc_warp_field##SFX(const real* src, int W, int H, int D,                \
                           const real* dx, const real* dy, const real* dz,      \
                           real* out);                                          \
  void orc_align_linear##SFX(const real* ref, real* aligned,                    \
                             const real* original, int W, int H, int D,         \
                             const real* filters, int niter, int type,          \
                             real* p12, real* rot3);                            \
  void orc_align_linear_cs##SFX(const real* ref, real* aligned,                 \
                                const real* original, int W, int H, int D,      \
                                const real* filters, int niter, int type,       \
                                double cert_sigma, real* p12, real* rot3);      \
  void orc_motion_correct##SFX(real* vols, int W, int H, int D, int T,          \
                               const real* voxel_size, const real* filters,     \
                               int niter, real* motion6T);                      \
  void orc_smoothing_filter_sigma##SFX(int size, double sigma, real* f);        \
  void orc_smoothing_filter_fwhm##SFX(int size, double fwhm, double vx,         \
                                      double vy, double vz, real* fx,           \
                                      real* fy, real* fz);                      \
  void orc_smooth3d##SFX(const real* vol, const real* cert,                     \
                         const real* smoothed_cert, int W, int H, int D,        \
                         const real* fx, const real* fy, const real* fz,        \
                         real* out);                                            \
  void orc_rescale_linear##SFX(const real* src, int W, int H, int D, int W2,    \
                               int H2, int D2, real* out);                      \
  void orc_align_linear_scales##SFX(const real* ref, real* aligned, int W,      \
                                    int H, int D, int coarsest,                 \
                                    const real* filters, int niter, int type,   \
                                    real* p12, real* rot3);                     \
  void orc_tensor_components##SFX(const real* q2, long V, const real* m6,       \
                                  real* t6);                                    \
  void orc_tensor_norms##SFX(const real* t6, long V, real* norm);               \
  void orc_nonlinear_ah##SFX(const real* q1, const real* q2, const real* t6,    \
                             long V, real nx, real ny, real nz, real* a6,       \
                             real* h3);                                         \
  void orc_displacement_update##SFX(const real* a6, const real* h3, long V,     \
                                    real* d3);                                  \
  void orc_align_nonlinear##SFX(const real* ref, real* aligned,                 \
                                const real* original, int W, int H, int D,      \
                                const real* filters6, const real* tensors,      \
                                const real* dirs, int niter, double tsigma,     \
                                double esigma, double dsigma, real* field);     \
  void orc_align_nonlinear_scales##SFX(                                         \
      const real* ref, real* aligned, int W, int H, int D, int coarsest,        \
      const real* filters6, const real* tensors, const real* dirs, int niter,   \
      double tsigma, double esigma, double dsigma, real* field);                \
  void orc_change_resolution_and_size##SFX(                                     \
      const real* src, int W, int H, int D, float vx, float vy, float vz,       \
      real* out, int W2, int H2, int D2, float nvx, float nvy, float nvz,       \
      int mm_z_cut);                                                            \
  void orc_change_resolution_and_size_interp##SFX(                              \
      const real* src, int W, int H, int D, float vx, float vy, float vz,       \
      real* out, int W2, int H2, int D2, float nvx, float nvy, float nvz,       \
      int mm_z_cut, int interp);                                                \
  void orc_transform_affine##SFX(const real* src, int W, int H, int D, int T,   \
                                 const real* p, int interp, real* out);         \
  void orc_transform_field##SFX(const real* src, int W, int H, int D, int T,    \
                                const real* dx, const real* dy,                 \
                                const real* dz, int interp, real* out);         \
  void orc_center_volumes##SFX(const real* src, int W, int H, int D, int T,     \
                               int interp, real* out, real* p12);               \
  void orc_center_of_mass##SFX(const real* vol, int W, int H, int D, real* c3); \
  void orc_match_volume_masses##SFX(real* v1, const real* v2, int W, int H,     \
                                    int D, real* p12);                          \
  void orc_add_linear_nonlinear##SFX(real* field, int W, int H, int D,          \
                                     const real* p);                            \
  void orc_register_two_volumes##SFX(                                           \
      const real* in, int W, int H, int D, const float* vin, const real* tpl,   \
      int W2, int H2, int D2, const float* vtpl, int mm_z_cut, int coarsest,    \
      int lin_iter, int nl_iter, const real* filters3, const real* filters6,    \
      const real* tensors, const real* dirs, double tsigma, double esigma,      \
      double dsigma, real* p12, real* interpolated, real* aligned_linear,       \
      real* aligned_nonlinear, real* field);                                    \
  void orc_tensor_magnitude##SFX(const real* vol, int W, int H, int D,          \
                                 const real* filters6, const real* tensors,     \
                                 real* out);                                    \
  void orc_segment_epi##SFX(const real* vol, int W, int H, int D, double vx,    \
                            double vy, double vz, real* mask);

ORC_DECLARE(float, _f32)
ORC_DECLARE(double, _f64)

int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
