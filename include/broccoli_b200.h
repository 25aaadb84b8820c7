/*
 * broccoli_b200.h -- C-ABI of the B200-native registration and filtering
 * path of BROCCOLI (libbroccoli_b200.so).
 *
 * Plain C: opaque context, raw pointers, explicit sizes, int status codes.
 * Every entry point below names the reference interface it replaces
 * (file:line in the BROCCOLI source tree).  The reference exposes this path
 * through the C++ class BROCCOLI_LIB (code/BROCCOLI_LIB/broccoli_lib.h:
 * 108-467) running OpenCL kernels; the same class interface is provided on
 * top of this ABI by include/broccoli_lib.h, and the Python package binds
 * this ABI with ctypes.
 *
 * Conventions
 *   - Volumes are float32, x fastest: index = x + y*W + z*W*H (+ t*W*H*D),
 *     as in code/Kernels/kernelRegistration.cpp:32-40.
 *   - A 7x7x7 complex filter is 686 floats: re[343] then im[343], x fastest.
 *     A bank of n filters is n*686 floats.  Filters are always HOST pointers
 *     (they are passed to the kernels by value).
 *   - Complex responses are interleaved (re, im) float pairs; a bank of n
 *     filters gives n consecutive complex volumes per instance.
 *   - Registration parameters: 12 floats
 *     [tx ty tz a11-1 a12 a13 a21 a22-1 a23 a31 a32 a33-1] in voxels,
 *     origin at the volume centre ((W-1)/2, (H-1)/2, (D-1)/2).
 *   - "d_" arguments are device pointers, "h_" host pointers.  All device
 *     work is queued on the context's stream; functions that take host
 *     buffers return after the results are back on the host.
 *   - No exceptions; every function returns a brc_status.  Device-side
 *     waits are bounded and report BRC_ERR_TIMEOUT instead of spinning.
 */
#ifndef BROCCOLI_B200_H
#define BROCCOLI_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  BRC_OK = 0,
  BRC_ERR_INVALID = -1,     /* bad size, null pointer, unknown option     */
  BRC_ERR_NOMEM = -2,       /* device or pinned-host allocation failed    */
  BRC_ERR_CUDA = -3,        /* CUDA runtime error; see brc_last_error()   */
  BRC_ERR_TIMEOUT = -4,     /* a bounded device-side wait gave up         */
  BRC_ERR_NODEVICE = -5,    /* no usable sm_100 device                    */
  BRC_ERR_UNSUPPORTED = -6, /* option combination not implemented         */
  BRC_ERR_NONFINITE = -7,   /* a solve produced NaN/Inf (update dropped)  */
  BRC_ERR_SCRATCH_LIMIT = -8 /* request larger than the fixed scratch of
                               brc_normal_equations_noalloc              */
} brc_status;

/* Alignment types, same values as broccoli_constants.h:93-95. */
enum { BRC_TRANSLATION = 0, BRC_RIGID = 1, BRC_AFFINE = 2 };

/* Arithmetic of the 7^3 filtering.  FP32: fp32 FMA on the CUDA cores; a
 * bank whose filters have even real and odd imaginary parts (to 1e-6 of
 * the largest tap, true of quadrature filters) uses the half-tap even/odd
 * form.  FP32_GENERAL: fp32, always all 343 taps.  BF16X3: split-bf16
 * (hi*hi + hi*lo + lo*hi) products on the tensor cores with fp32
 * accumulation.  TF32: data and taps rounded to tf32 (10-bit mantissa), one
 * product per tap on the tensor cores (structured-sparse MMAs: the banded
 * tap matrix stores one value per sample pair), fp32 accumulation. */
enum { BRC_PREC_FP32 = 0, BRC_PREC_BF16X3 = 1, BRC_PREC_FP32_GENERAL = 2, BRC_PREC_TF32 = 3 };

typedef struct brc_ctx brc_ctx;

/* ---- context ---------------------------------------------------------- */

/* Replaces BROCCOLI_LIB::OpenCLInitiate (broccoli_lib.cpp:1181-1878):
 * binds the context to CUDA device `device` and creates its stream. */
int brc_ctx_create(int device, brc_ctx** out);
int brc_ctx_destroy(brc_ctx* ctx);
/* Queue the context's work on an existing cudaStream_t (e.g. torch's
 * current stream).  NULL is the legacy default stream (stream 0), as in the
 * CUDA runtime; BRC_OWN_STREAM returns to the context's own stream. */
#define BRC_OWN_STREAM ((void*)-1)
int brc_ctx_set_stream(brc_ctx* ctx, void* cuda_stream);
void* brc_ctx_stream(brc_ctx* ctx);
int brc_ctx_synchronize(brc_ctx* ctx);
/* Bytes of device workspace the context currently holds. */
size_t brc_ctx_workspace_bytes(const brc_ctx* ctx);
/* Number of kernels this context has launched so far (graph replays count
 * every kernel node they ran; the iterations of a registration graph's loop
 * are counted on the device, so this call first synchronises the context's
 * streams).  Used by benchmarks to report launch counts. */
unsigned long long brc_ctx_kernel_launches(const brc_ctx* ctx);
/* Replaces GetOpenCLErrorMessage / the INITIALIZATION_ERROR getters
 * (broccoli_lib.h:399-413). */
const char* brc_status_string(int status);
const char* brc_last_error(const brc_ctx* ctx);
/* Library version string. */
const char* brc_version(void);

/* ---- kernel-level entry points (device pointers, asynchronous) --------- */

/* Complex 7x7x7 filtering with zero padding (a true convolution:
 * q(x) = sum_d vol(x+d) F[3-d]) of `batch` volumes, each `vol_stride`
 * floats apart.  out: batch x nfilt complex volumes (2*W*H*D floats each).
 * nfilt is 3 (linear) or 6 (nonlinear).
 * Replaces NonseparableConvolution3D (broccoli_lib.cpp:4974-5027) and
 * Nonseparable3DConvolutionComplexThreeQuadratureFilters*
 * (kernelConvolution.cpp:2802-3693). */
int brc_filter3d(brc_ctx* ctx, const float* d_vol, int W, int H, int D, int batch,
                 long long vol_stride, const float* h_filters, int nfilt, int precision,
                 float* d_out);

/* Normal equations of the affine registration step from reference
 * responses d_q1 and aligned-volume responses d_q2 (3 complex volumes
 * each per instance; q1_stride = 0 shares one reference across the batch).
 * Outputs the full symmetric 12x12 A (column-major) and h per instance in
 * double precision.
 * Replaces CalculatePhaseDifferencesAndCertainties, CalculatePhaseGradients
 * X/Y/Z, CalculateAMatrixAndHVector2DValuesX/Y/Z, CalculateAMatrix1DValues,
 * CalculateHVector1DValues, CalculateAMatrix, CalculateHVector
 * (kernelRegistration.cpp:173-800) as driven at broccoli_lib.cpp:5315-5392. */
int brc_normal_equations(brc_ctx* ctx, const float* d_q1, long long q1_stride,
                         const float* d_q2, int W, int H, int D, int batch,
                         double* d_A, double* d_h);

/* brc_normal_equations without any device allocation.  No counterpart in
 * the reference: it is for callers that cannot let a library allocate
 * device memory -- processes whose HBM is reserved up front by a pooling
 * allocator or serving runtime, and hosts that plan all memory before they
 * start.  It takes a cudaStream_t instead of a context (NULL is the legacy
 * default stream) and keeps its per-CTA partial sums in a fixed device
 * array of BRC_NOALLOC_PARTIAL_ROWS rows x 42 doubles (about 1 MB) that
 * every GPU loading the library holds until the process exits.
 * A call needs ceil((D-6)/zpb) x batch rows, zpb = max(1, 4096 /
 * ((W-6)(H-6))) interior slices per row (64x64x33: 27 rows per volume,
 * batch <= 113); larger requests return BRC_ERR_SCRATCH_LIMIT and do
 * nothing.  The stream must belong to the current device (BRC_ERR_INVALID
 * otherwise).  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current and caches it;
 * make that first call before any stream capture.  Under lazy module loading
 * (the CUDA 12.2+ default) that lookup is also what allocates the array, so
 * a process that gives its HBM to a pool should make a set-up call first:
 * batch = 0 (other arguments ignored) only resolves the array on the current
 * device and returns; BRC_ERR_NOMEM there means the device had no room left.
 * CUDA_MODULE_LOADING=EAGER allocates it when the library loads instead.
 * After cudaDeviceReset, repeat the set-up call before the next call.  All
 * calls share the array: calls that overlap on the GPU race and must be
 * ordered by the caller.  No cudaMalloc, cudaFree or allocating library
 * routine is called. */
#define BRC_NOALLOC_PARTIAL_ROWS 3072
int brc_normal_equations_noalloc(void* cuda_stream, const float* d_q1, long long q1_stride,
                                 const float* d_q2, int W, int H, int D, int batch,
                                 double* d_A, double* d_h);

/* p = A^-1 h per instance in double, rounded to float.
 * Replaces SolveEquationSystem (broccoli_lib.cpp:17157-17186). */
int brc_solve_affine_fp64(brc_ctx* ctx, const double* d_A, const double* d_h, int batch,
                          float* d_p);

/* Trilinear (exact-weight, clamp-to-edge) warp of `batch` volumes by their
 * own 12-parameter affine transforms (d_params: batch x 12).
 * Replaces InterpolateVolumeLinearLinear (kernelRegistration.cpp:1066-1101). */
int brc_warp_affine(brc_ctx* ctx, const float* d_src, int W, int H, int D, int batch,
                    const float* d_params, float* d_out);

/* Warp by a displacement field (three volumes, voxels).
 * Replaces InterpolateVolumeLinearNonLinear (kernelRegistration.cpp:
 * 1111-1140). */
int brc_warp_field(brc_ctx* ctx, const float* d_src, int W, int H, int D,
                   const float* d_dx, const float* d_dy, const float* d_dz, float* d_out);

/* Separable 9-tap smoothing of `batch` volumes: along y of vol*cert, along
 * x, along z divided by the smoothed certainty (d_cert / d_smoothed_cert
 * may be NULL for all-ones).  Filters are host arrays of 9 taps.
 * Replaces PerformSmoothing (broccoli_lib.cpp:11274-11357, :11461-11545)
 * and SeparableConvolutionRows/Columns/Rods (kernelConvolution.cpp:
 * 52-1665). */
int brc_smooth3d(brc_ctx* ctx, const float* d_vol, int W, int H, int D, int batch,
                 const float* h_fx, const float* h_fy, const float* h_fz,
                 const float* d_cert, const float* d_smoothed_cert, float* d_out);

/* Normalised-convolution smoothing of T volumes with one certainty
 * (mask) volume: the mask is smoothed (all-ones certainty), every volume is
 * smoothed with the mask as certainty and divided by the smoothed mask along
 * the last pass, and the results are multiplied by the mask.  As in the
 * reference the division is unguarded: voxels where the smoothed mask is
 * exactly 0 come out NaN.  Filters are host arrays of 9 taps.  Replaces
 * PerformSmoothingNormalizedWrapper (broccoli_lib.cpp:11227-11272) with
 * PerformSmoothingNormalized (:11359-11450). */
int brc_smooth_normalized(brc_ctx* ctx, const float* d_vols, int W, int H, int D, int T, const float* d_mask,
                          const float* h_fx, const float* h_fy, const float* h_fz, float* d_out);

/* Linear resample to a new grid size, sample spacing (N-1)/(N'-1).
 * Replaces ChangeVolumeSize (broccoli_lib.cpp:6247-6388) with
 * RescaleVolumeLinear (kernelRegistration.cpp:1340-1366). */
int brc_rescale_linear(brc_ctx* ctx, const float* d_src, int W, int H, int D,
                       float* d_out, int W2, int H2, int D2);

/* ---- whole-path entry points ------------------------------------------ */

typedef struct {
  int iterations;        /* maximum iterations per instance               */
  int type;              /* BRC_TRANSLATION / BRC_RIGID / BRC_AFFINE       */
  int precision;         /* BRC_PREC_FP32 / BRC_PREC_BF16X3                */
  float tolerance;       /* early exit when the largest displacement of an
                            update over the volume corners is below this
                            (voxels); 0 = always run all iterations        */
  int use_graph;         /* capture the iteration loop in a CUDA graph     */
  int certainty_sigma_x100; /* >0: Gaussian smoothing (3x3x3 taps, sigma
                            = value/100 voxels) of the phase certainties
                            before the reductions; 0 = reference behaviour */
} brc_linear_opts;

/* Fill `opts` with the reference defaults (AFFINE, FP32, no early exit,
 * graph on, no certainty smoothing, `iterations` iterations). */
void brc_linear_opts_default(brc_linear_opts* opts, int iterations);

/* Batched single-scale linear registration of `batch` moving volumes to
 * reference volume(s) (ref_stride = 0: one shared reference).  All
 * instances run together; an instance whose update falls below the
 * tolerance stops updating (its convergence mask bit is set).
 * d_params (batch x 12) receives the total parameters, d_aligned (batch
 * volumes, may be NULL) the final warped volumes, d_rotations (batch x 3,
 * may be NULL; RIGID) the Euler angles in degrees, d_iterations (batch,
 * may be NULL) the iterations each instance ran.
 * Replaces AlignTwoVolumesLinear (broccoli_lib.cpp:5273-5437) called once
 * per volume, with its Setup/Cleanup (:5072-5266, :6670-6726). */
int brc_register_linear_batched(brc_ctx* ctx, const float* d_ref, long long ref_stride,
                                const float* d_moving, int W, int H, int D, int batch,
                                const float* h_filters, const brc_linear_opts* opts,
                                float* d_params, float* d_aligned, float* d_rotations,
                                int* d_iterations);

/* Rigid motion correction of a T-volume series (host buffers) to volume 0,
 * or to h_reference when it is not NULL.  h_volumes is replaced in place by
 * the corrected series (volume 0 unchanged when it is the reference);
 * h_motion (6*T, may be NULL) receives translations in mm (voxels times
 * voxel size) then rotations in degrees, laid out [t + k*T].
 * Replaces PerformMotionCorrectionWrapper (broccoli_lib.cpp:10658-10720). */
int brc_motion_correct(brc_ctx* ctx, float* h_volumes, int W, int H, int D, int T,
                       const float* voxel_size3, const float* h_filters,
                       const brc_linear_opts* opts, const float* h_reference,
                       float* h_motion);

/* Multi-scale (pyramid) linear registration of a batch to one shared
 * reference: volumes resampled to round(N/scale) for scale = coarsest,
 * coarsest/2, ..., 1; each scale registers the resampled moving volume
 * pre-warped by the total so far; totals carried with doubled translations;
 * the finest scale runs ceil(iterations/5) iterations; rotations (RIGID)
 * summed over scales.  d_aligned (batch volumes, full size) receives the
 * moving volumes warped by the total parameters.
 * Replaces AlignTwoVolumesLinearSeveralScales (broccoli_lib.cpp:6391-6513)
 * with ChangeVolumeSize (:6247-6388) and
 * AddAffineRegistrationParametersNextScale (:7344-7431). */
int brc_register_linear_scales(brc_ctx* ctx, const float* d_ref, const float* d_moving, int W, int H,
                               int D, int batch, const float* h_filters, const brc_linear_opts* opts,
                               int coarsest_scale, float* d_params, float* d_aligned,
                               float* d_rotations);

/* ---- nonlinear (displacement field) registration ----------------------- */

typedef struct {
  int iterations;      /* iterations per scale (finest: ceil(iterations/2)) */
  int coarsest_scale;  /* 1, 2, 4, 8 or 16                                  */
  float tsigma;        /* smoothing of the structure tensor (voxels)        */
  float esigma;        /* smoothing of A and h (voxels)                     */
  float dsigma;        /* smoothing of the field update (voxels)            */
  int precision;       /* BRC_PREC_FP32 / BRC_PREC_BF16X3 (filtering)        */
  int solve_fp64;      /* 0: FP32 cofactors + 1e-16 (reference); 1: the same
                          in FP64 (det + 1e-16 in double)                  */
} brc_nonlinear_opts;

/* Defaults of SetStartValues (broccoli_lib.cpp:325-355): sigmas 5,
 * coarsest scale 1, FP32, reference solve. */
void brc_nonlinear_opts_default(brc_nonlinear_opts* opts, int iterations);

/* One nonlinear update from given responses (d_q1: reference, d_q2:
 * aligned; 6 complex volumes each): structure tensor of q2 with projection
 * tensors h_tensors (6 x {m11 m12 m13 m22 m23 m33}), tensor smoothing,
 * norm (kept in a11) and max normalisation, per-voxel A and h over the six
 * filters with directions h_dirs (x[6] y[6] z[6]), their smoothing, the 3x3
 * solve, and the smoothed update ADDED to d_field (3 volumes x, y, z).
 * Replaces the loop body of AlignTwoVolumesNonLinear (broccoli_lib.cpp:
 * 5784-6025): CalculateTensorComponents, CalculateTensorNorms,
 * CalculateAMatricesAndHVectors, CalculateDisplacementUpdate
 * (kernelRegistration.cpp:806-988), CalculateMax (:10889), MultiplyVolume,
 * AddVolumes and PerformSmoothing. */
int brc_nonlinear_step(brc_ctx* ctx, const float* d_q1, const float* d_q2, int W, int H, int D,
                       const float* h_tensors, const float* h_dirs, float tsigma, float esigma,
                       float dsigma, int solve_fp64, float* d_field);

/* Multi-scale nonlinear registration of d_moving to d_ref with six filters
 * (h_filters6: 6 x 686 floats).  d_field (3 volumes) receives the total
 * displacement field, d_aligned the moving volume warped by it.
 * Replaces AlignTwoVolumesNonLinearSeveralScales (broccoli_lib.cpp:
 * 6516-6665) and AlignTwoVolumesNonLinear (:5748-6058). */
int brc_register_nonlinear(brc_ctx* ctx, const float* d_ref, const float* d_moving, int W, int H,
                           int D, const float* h_filters6, const float* h_tensors,
                           const float* h_dirs, const brc_nonlinear_opts* opts, float* d_field,
                           float* d_aligned);

/* ---- adjoints (differentiable registration) ---------------------------- */

/* Adjoint of brc_filter3d: d_out (batch volumes) = sum over the nfilt
 * filters of the correlation of the complex gradient d_grad (batch x nfilt
 * interleaved complex volumes, dL/dRe and dL/dIm) with the filters.  No
 * counterpart in the reference (its path is not differentiated); the
 * forward it inverts is NonseparableConvolution3D (broccoli_lib.cpp:
 * 4974-5027). */
int brc_filter3d_adjoint(brc_ctx* ctx, const float* d_grad, int W, int H, int D, int batch,
                         const float* h_filters, int nfilt, float* d_out);

/* Adjoint of brc_warp_affine: dL/dparams (batch x 12, double) from the
 * output gradient, with the exact derivative of the clamp-to-edge
 * trilinear interpolant; d_grad_src (may be NULL) receives dL/dsrc by
 * atomic scatter (zeroed first).  Forward: InterpolateVolumeLinearLinear
 * (kernelRegistration.cpp:1066-1101). */
int brc_warp_affine_backward(brc_ctx* ctx, const float* d_src, int W, int H, int D, int batch,
                             const float* d_params, const float* d_grad_out, double* d_grad_params,
                             float* d_grad_src);

/* Adjoint of brc_warp_field: dL/dfield (3 volumes, may be NULL) and
 * dL/dsrc (may be NULL, zeroed then scattered).  Forward:
 * InterpolateVolumeLinearNonLinear (kernelRegistration.cpp:1111-1140). */
int brc_warp_field_backward(brc_ctx* ctx, const float* d_src, int W, int H, int D, const float* d_dx,
                            const float* d_dy, const float* d_dz, const float* d_grad_out,
                            float* d_grad_field, float* d_grad_src);

/* Self-test of the failure path of the tensor-core kernels.  No counterpart
 * in the reference.  Launches one CTA that waits wait_ms (1..1000) on a
 * barrier nothing completes and then sets the context's device flag, the
 * way a CTA of the BF16X3 filtering reports a wait that ran out; the next
 * brc_ctx_synchronize returns BRC_ERR_TIMEOUT and clears the flag, and the
 * context stays usable. */
int brc_selftest_bounded_wait(brc_ctx* ctx, int wait_ms);

/* Evaluates the four-quadrant arctangent that the phase-difference and
 * phase-gradient kernels use (a polynomial fit with the hardware reciprocal
 * in place of atan2f): d_out[i] = angle of (d_x[i], d_y[i]) for n >= 0
 * device floats, so that its error can be checked against atan2.  No
 * counterpart in the reference, whose kernels call OpenCL's atan2
 * (kernelRegistration.cpp:173-382). */
int brc_selftest_phase_atan2(brc_ctx* ctx, const float* d_y, const float* d_x, float* d_out, long long n);

/* ---- device memory and host copies (for hosts without a CUDA runtime) --- */

/* cudaMalloc / cudaFree on the context's device.  Replaces the clCreateBuffer
 * / clReleaseMemObject pairs of the reference's Setup/Cleanup functions
 * (e.g. broccoli_lib.cpp:5072-5266). */
int brc_device_alloc(brc_ctx* ctx, size_t bytes, void** d_out);
int brc_device_free(brc_ctx* ctx, void* d_ptr);
/* Copies on the context's stream; both return after the copy completed.
 * Replace clEnqueueWriteBuffer / clEnqueueReadBuffer with CL_TRUE. */
int brc_copy_to_device(brc_ctx* ctx, void* d_dst, const void* h_src, size_t bytes);
int brc_copy_to_host(brc_ctx* ctx, void* h_dst, const void* d_src, size_t bytes);

/* ---- the steps either side of the registration loops -------------------- */

/* Resample d_src (voxel sizes voxel_size3, mm) to new_voxel_size3 and
 * centre it in / crop it to a W2 x H2 x D2 grid, shifted by mm_z_cut mm
 * along z; uncovered voxels are 0.
 * Replaces ChangeVolumesResolutionAndSize (broccoli_lib.cpp:6950-7100)
 * with RescaleVolumeLinear and CopyVolumeToNew (kernelRegistration.cpp:
 * 1340-1366, :1593-1678). */
int brc_change_resolution_and_size(brc_ctx* ctx, const float* d_src, int W, int H, int D,
                                   const float* voxel_size3, float* d_out, int W2, int H2, int D2,
                                   const float* new_voxel_size3, int mm_z_cut);

/* Interpolation modes of the transform and resample entries: the values of
 * the reference's INTERPOLATION_MODE (broccoli_constants.h:97-99).  CUBIC
 * is refused with BRC_ERR_UNSUPPORTED: the reference's cubic kernels sum
 * into an uninitialised variable (kernelRegistration.cpp:1230, :1284,
 * :1396), so there is no defined result to reproduce. */
#define BRC_INTERP_NEAREST 0
#define BRC_INTERP_LINEAR 1
#define BRC_INTERP_CUBIC 2

/* brc_change_resolution_and_size for T volumes (d_src: T x W x H x D one
 * after another, d_out: T x W2 x H2 x D2) with NEAREST or LINEAR
 * interpolation.  Replaces ChangeVolumesResolutionAndSize with
 * NUMBER_OF_VOLUMES = T and INTERPOLATION_MODE (broccoli_lib.cpp:6950-7100;
 * RescaleVolumeNearest / Linear and CopyVolumeToNew,
 * kernelRegistration.cpp:1312-1366, :1593-1678). */
int brc_change_resolution_and_size_batch(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T,
                                         const float* voxel_size3, float* d_out, int W2, int H2, int D2,
                                         const float* new_voxel_size3, int mm_z_cut, int interpolation);

/* One parameter vector (h_params12, host, the 12-parameter layout above)
 * applied to T volumes: out_t(x) = src_t(x + t + (A - I)(x - centre)),
 * NEAREST or LINEAR.  d_src and d_out must differ.  Replaces
 * TransformVolumesLinear (broccoli_lib.cpp:8267-8359; InterpolateVolume-
 * NearestLinear / LinearLinear, kernelRegistration.cpp:995-1031, :1066-1101). */
int brc_transform_volumes_linear(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T,
                                 const float* h_params12, int interpolation, float* d_out);

/* One displacement field (voxels, three W x H x D volumes) applied to T
 * volumes: out_t(x) = src_t(x + d(x)).  Replaces TransformVolumesNonLinear
 * (broccoli_lib.cpp:8361-8451; InterpolateVolumeNearestNonLinear /
 * LinearNonLinear, kernelRegistration.cpp:1032-1061, :1111-1140). */
int brc_transform_volumes_nonlinear(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T,
                                    const float* d_dx, const float* d_dy, const float* d_dz, int interpolation,
                                    float* d_out);

/* d += t + (A - I)(x - centre) in place: the displacement of an affine
 * parameter vector (host) added to a field.  Replaces
 * CreateCombinedDisplacementField (broccoli_lib.cpp:8115-8143;
 * AddLinearAndNonLinearDisplacement, kernelRegistration.cpp:1142-1178). */
int brc_combine_displacement_field(brc_ctx* ctx, float* d_dx, float* d_dy, float* d_dz, int W, int H, int D,
                                   const float* h_params12);

/* Centres T volumes by the first one's centre of mass: the translation
 * -round(N/2 - com) per axis (returned in h_params12 when not NULL)
 * applied to all T volumes with the given interpolation; synchronises.
 * Replaces CenterVolumesWrapper with CenterVolumeMass (broccoli_lib.cpp:
 * 8225-8245, :6839-6874). */
int brc_center_volumes(brc_ctx* ctx, const float* d_src, int W, int H, int D, int T, int interpolation,
                       float* d_out, float* h_params12);

/* Centre of mass (voxel coordinates) of a volume, FP64 reduction on the
 * device; synchronises.  Replaces CalculateCenterOfMass
 * (broccoli_lib.cpp:6763-6800, a host loop after a full device-to-host
 * copy). */
int brc_center_of_mass(brc_ctx* ctx, const float* d_vol, int W, int H, int D, float* h_com3);

typedef struct {
  int linear_iterations;     /* NUMBER_OF_ITERATIONS_FOR_LINEAR_IMAGE_REGISTRATION */
  int nonlinear_iterations;  /* ... _NONLINEAR_ ...; 0 skips the nonlinear stage   */
  int coarsest_scale;        /* COARSEST_SCALE_T1_MNI                              */
  int mm_z_cut;              /* MM_T1_Z_CUT                                        */
  float tsigma, esigma, dsigma;
  int precision;
  int solve_fp64;
  int precenter;             /* PRECENTER_REGISTRATION: centre the input by its
                                centre of mass at its own size first          */
} brc_two_volume_opts;

void brc_two_volume_opts_default(brc_two_volume_opts* opts);

/* T1-to-template normalisation of one volume: (with opts->precenter and a
 * linear stage: the input centred twice by its centre of mass at its own
 * size, as CenterVolumeMass is called twice at broccoli_lib.cpp:8003-8007;
 * the centred input then replaces the input throughout) resample onto the
 * template grid, match centres of mass, multi-scale affine registration, parameters
 * composed with the mass match (h_params12, host), multi-scale nonlinear
 * registration, affine motion added to the field, and one final warp of a
 * fresh resample by the combined field.  Output volumes are template size
 * and optional (NULL to skip); d_field (3 volumes) is required when the
 * nonlinear stage runs.  Synchronises before returning.
 * Replaces PerformRegistrationTwoVolumesWrapper (broccoli_lib.cpp:
 * 7973-8112) with MatchVolumeMasses (:6876-6948) and
 * CreateCombinedDisplacementField (:8115-8150). */
int brc_register_two_volumes(brc_ctx* ctx, const float* d_in, int W, int H, int D,
                             const float* voxel_size3, const float* d_tpl, int W2, int H2, int D2,
                             const float* tpl_voxel_size3, const float* h_filters3,
                             const float* h_filters6, const float* h_tensors, const float* h_dirs,
                             const brc_two_volume_opts* opts, float* h_params12,
                             float* d_interpolated, float* d_aligned_linear,
                             float* d_aligned_nonlinear, float* d_field);

/* T1-to-template normalisation of a cohort of n subjects of different sizes
 * (the reference normalises one subject per PerformRegistrationTwoVolumes-
 * Wrapper call, broccoli_lib.cpp:7973-8112).  d_subjects is a host array of
 * n device pointers; subject b has size sizes3n[3b..3b+2] (W, H, D) and
 * voxel size voxel_sizes3n[3b..3b+2].  All subjects are resampled onto the
 * template grid in one launch (ChangeVolumesResolutionAndSize,
 * :6950-7100), centred by their centres of mass (MatchVolumeMasses,
 * :6876-6948) with one batched warp, registered affinely as one batch
 * over the scales, then registered nonlinearly one by one (each at
 * template size).  Per subject b the results equal those of
 * brc_register_two_volumes: h_params12n[12b..] (host), d_aligned_linear +
 * b V2, d_aligned_nonlinear + b V2, d_fields + 3 b V2 (V2 = W2 H2 D2;
 * volumes optional, NULL to skip; d_fields required when the nonlinear
 * stage runs).  Synchronises before returning. */
int brc_register_cohort(brc_ctx* ctx, int n, const float* const* d_subjects, const int* sizes3n,
                        const float* voxel_sizes3n, const float* d_tpl, int W2, int H2, int D2,
                        const float* tpl_voxel_size3, const float* h_filters3, const float* h_filters6,
                        const float* h_tensors, const float* h_dirs, const brc_two_volume_opts* opts,
                        float* h_params12n, float* d_aligned_linear, float* d_aligned_nonlinear,
                        float* d_fields);

/* ---- debug outputs, masks and parameter inversion ------------------------ */

/* Host arrays the linear registration fills as the reference does with
 * DEBUG set (broccoli_lib.cpp:5285-5289, :5349-5354): every call of
 * brc_register_linear_batched (and so of the pyramid, motion-correction and
 * T1-to-template entry points built on it) writes, for its last instance,
 *   quadrature_responses[0..2]  the reference volume's three complex
 *                               responses (interleaved re, im; W H D pairs),
 *   phase_differences / phase_certainties / phase_gradients
 *                               of iteration 0 along z: arg(q1 conj q2),
 *                               |q1| |q2| cos^2(dphi/2) and the z phase
 *                               gradient of the third filter pair (the
 *                               first and last plane, which the reference
 *                               leaves unwritten, are 0 here),
 * so that after a pyramid the finest scale's values remain.  When all six
 * quadrature_responses are set, brc_register_nonlinear also writes the six
 * responses of its reference volume at the finest scale (the reads the
 * reference keeps commented out at broccoli_lib.cpp:5754-5759).  Any
 * pointer may be NULL.  Debug writes synchronise the stream and are refused
 * (BRC_ERR_UNSUPPORTED) while the context's stream is being captured.
 * outs = NULL turns them off.  No counterpart function in the reference: it
 * replaces SetDebug plus the SetOutputQuadratureFilterResponses /
 * SetOutputPhaseDifferences / Certainties / Gradients pointers
 * (broccoli_lib.h:299-304). */
typedef struct {
  void* quadrature_responses[6];
  float* phase_differences;
  float* phase_certainties;
  float* phase_gradients;
} brc_debug_outputs;
int brc_ctx_set_debug_outputs(brc_ctx* ctx, const brc_debug_outputs* outs);

/* The reference's linear phase quantities of one pair of complex responses
 * (one filter): d_phase_diff = arg(q1 conj q2), d_cert = |q1 q2| cos^2(
 * dphi/2), d_grad = the phase gradient along `axis` (0 x, 1 y, 2 z; the
 * first and last sample along the axis are 0).  Any output may be NULL.
 * Replaces CalculatePhaseDifferencesAndCertainties and CalculatePhase-
 * GradientsX/Y/Z (kernelRegistration.cpp:173-382). */
int brc_phase_volumes(brc_ctx* ctx, const float* d_q1, const float* d_q2, int W, int H, int D, int axis,
                      float* d_phase_diff, float* d_cert, float* d_grad);

/* d_vols[t][i] *= d_mask[i] for T volumes of W x H x D, in place.  Replaces
 * MultiplyVolumes (kernelMisc.cpp; the skull strip of
 * PerformRegistrationTwoVolumesWrapper, broccoli_lib.cpp:8066-8105). */
int brc_multiply_volumes(brc_ctx* ctx, float* d_vols, int W, int H, int D, int T, const float* d_mask);

/* Inverse of a 12-parameter affine transform (4x4 inverse in double, result
 * rounded to float).  Host only.  Replaces InvertAffineRegistrationParameters
 * (broccoli_lib.cpp:7186-7250). */
void brc_invert_affine_parameters(const float* h_params12, float* h_inverse12);

/* ---- first-level preprocessing ----------------------------------------- */

/* Gaussian smoothing filters of 9 taps per axis from a FWHM in mm and the
 * voxel sizes (x, y, z), each normalised by its float sum.  Host only.
 * Replaces CreateSmoothingFilters(..., FWHM, voxel sizes)
 * (broccoli_lib.cpp:11055-11091). */
void brc_smoothing_filters_fwhm(float fwhm_mm, const float* voxel_size3, float* h_fx, float* h_fy,
                                float* h_fz);

/* Tensor magnitude of one volume: its six nonlinear filter responses
 * (h_filters6: 6 x 686 floats), the structure tensor T = sum_k |q_k| M_k
 * (h_tensors: 6 x {m11 m12 m13 m22 m23 m33}) and the Frobenius norm of T
 * into d_out.  Replaces CalculateTensorMagnitude (broccoli_lib.cpp:
 * 5658-5746) with CalculateTensorComponents and CalculateTensorNorms
 * (kernelRegistration.cpp:806-875). */
int brc_tensor_magnitude(brc_ctx* ctx, const float* d_vol, int W, int H, int D, const float* h_filters6,
                         const float* h_tensors, int precision, float* d_out);

/* Brain mask of one EPI volume: smoothing with a 4 mm FWHM Gaussian, the
 * sum of the smoothed volume in the reference's order (rows over x, then
 * over y per plane, then over z on the host), and d_mask = 1 where the
 * smoothed value exceeds 0.9 x sum / (W H D), 0.001 elsewhere.
 * Synchronises.  Replaces SegmentEPIData (broccoli_lib.cpp:11008-11030)
 * with CalculateSum (:10846-10886) and ThresholdVolume (kernelMisc.cpp:
 * 305-327). */
int brc_segment_epi(brc_ctx* ctx, const float* d_vol, int W, int H, int D, const float* voxel_size3,
                    float* d_mask);

typedef struct {
  float* fmri;               /* host, T EPI volumes; replaced in place by the
                                preprocessed series                         */
  int epi_w, epi_h, epi_d, epi_t;
  float epi_voxel[3];        /* mm (x, y, z)                                 */
  const float* t1;           /* host, one T1 volume                          */
  int t1_w, t1_h, t1_d;
  float t1_voxel[3];
  const float* mni;          /* host, the template brain volume              */
  int mni_w, mni_h, mni_d;
  float mni_voxel[3];
  const float* filters3;     /* 3 x 686: linear registration filters         */
  const float* filters6;     /* 6 x 686: nonlinear registration filters      */
  const float* tensors;      /* 6 x 6 projection tensors                     */
  const float* dirs;         /* filter directions x[6] y[6] z[6]             */
} brc_first_level_input;

typedef struct {
  int linear_iterations;     /* NUMBER_OF_ITERATIONS_FOR_LINEAR_IMAGE_REGISTRATION */
  int nonlinear_iterations;  /* ... _NONLINEAR_ ...; 0 skips the nonlinear stage   */
  int motion_iterations;     /* NUMBER_OF_ITERATIONS_FOR_MOTION_CORRECTION         */
  int coarsest_scale_t1_mni; /* COARSEST_SCALE_T1_MNI                              */
  int coarsest_scale_epi_t1; /* COARSEST_SCALE_EPI_T1                              */
  int mm_t1_z_cut;           /* MM_T1_Z_CUT                                        */
  int apply_motion_correction;
  int apply_smoothing;
  float smoothing_fwhm;      /* EPI smoothing, mm                                  */
  float tsigma, esigma, dsigma;
  int precision;             /* filtering: BRC_PREC_FP32 / BRC_PREC_BF16X3         */
  int solve_fp64;
} brc_first_level_opts;

/* Defaults of the reference's FirstLevelAnalysis tool
 * (Bash_Wrapper/FirstLevelAnalysis.cpp:133-158): 10 linear and 10 nonlinear
 * iterations, 5 motion-correction iterations, coarsest scales 4, no z cut,
 * motion correction and 6 mm smoothing on, sigmas 5, FP32. */
void brc_first_level_opts_default(brc_first_level_opts* opts);

typedef struct {             /* host outputs, each may be NULL               */
  float* params_t1_mni;      /* 12 */
  float* params_epi_t1;      /* 12: EPI to the original T1                   */
  float* params_epi_mni;     /* 12 */
  float* motion_parameters;  /* 6 x T, [t + k*T]: mm then degrees            */
  float* interpolated_t1;    /* template size                                */
  float* aligned_t1_linear;
  float* aligned_t1_nonlinear;
  float* field;              /* 3 template-size volumes x, y, z              */
  float* aligned_epi_t1;     /* template size                                */
  float* aligned_epi_mni_linear;
  float* aligned_epi_mni_nonlinear;
  float* motion_corrected;   /* T EPI volumes                                */
  float* epi_mask;           /* EPI size                                     */
  float* smoothed;           /* T EPI volumes                                */
} brc_first_level_output;

/* The preprocessing stages of a first-level analysis, in the reference's
 * order: T1 to template (centring, resampling onto the template grid with
 * the z cut, mass match, multi-scale affine, multi-scale nonlinear); the
 * first EPI volume to the resampled T1 on the template grid (centring,
 * resampling, mass match, multi-scale affine) and through the T1's
 * transforms to the template; the first EPI volume to the original T1
 * (translation and rigid on the volumes, rigid and affine on their tensor
 * magnitudes); rigid motion correction of the series; the EPI mask of the
 * first corrected volume; normalised smoothing of the series with the mask.
 * Slice-timing correction and the statistics are not part of this entry.
 * Synchronises before returning.  Replaces the preprocessing of
 * PerformFirstLevelAnalysisWrapper (broccoli_lib.cpp:8480-8733) with
 * PerformRegistrationT1MNINoSkullstrip (:8226-8273),
 * PerformRegistrationEPIT1 (:7853-7915), PerformRegistrationEPIT1Original
 * (:7917-7970), PerformMotionCorrectionHost (:10723-10787), SegmentEPIData
 * (:11008-11030) and PerformSmoothingNormalizedHost (:11628-11727). */
int brc_first_level_preprocess(brc_ctx* ctx, const brc_first_level_input* in, const brc_first_level_opts* opts,
                               const brc_first_level_output* out);

#ifdef __cplusplus
}
#endif
#endif
