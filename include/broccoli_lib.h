/*
 * broccoli_lib.h -- drop-in BROCCOLI_LIB class for the registration and
 * filtering path, implemented on the C-ABI of libbroccoli_b200
 * (broccoli_b200.h) instead of OpenCL.
 *
 * It keeps the reference's class interface (code/BROCCOLI_LIB/
 * broccoli_lib.h:108-467) for the members this path uses: the same
 * constructors, OpenCLInitiate / GetOpenCLInitiated, the raw-pointer
 * setters (the caller owns every host array; setters store the pointer),
 * the Perform*Wrapper() entry points and the error getters.  No OpenCL
 * header is needed: cl_uint and cl_float2 are layout-compatible stand-ins.
 * Members of the reference outside this path (statistics, ICA, ...) are not
 * declared.
 *
 * Behaviour notes (same as the reference unless stated):
 *   - OpenCLInitiate(platform, device): platform must be 0; device is the
 *     CUDA device index.
 *   - PerformMotionCorrectionWrapper corrects h_fMRI_Volumes in place and
 *     writes 6 x T motion parameters (mm, degrees); when an output series is
 *     set with SetOutputMotionCorrectedfMRIVolumes it is filled as well.
 *   - PerformRegistrationTwoVolumesWrapper: T1 -> MNI, single volume.
 *   - PerformSmoothingWrapper: LOWPASS (from SetEPISmoothingAmount, FWHM in
 *     mm) or RANDOM (filters from SetSmoothingFilters).
 *   - PerformFirstLevelAnalysisWrapper: the preprocessing stages only
 *     (SetPreprocessingOnly(true)); outputs are written where the reference
 *     writes them: the three parameter vectors and the motion parameters
 *     always, the volumes when their SetSave* flag is on.
 *   - SetAutoMask(true): PerformSmoothingNormalizedHostWrapper makes the
 *     certainty from the first fMRI volume (SegmentEPIData) and writes it
 *     to the SetInputCertainty array.
 *   - SetDebug(true): the registrations fill the arrays of
 *     SetOutputQuadratureFilterResponses (the reference volume's responses)
 *     and SetOutputPhaseDifferences / Certainties / Gradients (iteration 0,
 *     z axis), the last AlignTwoVolumesLinear call's values, as the reference
 *     does (broccoli_lib.cpp:5285-5289, :5349-5354); the six-array form of
 *     SetOutputQuadratureFilterResponses receives instead, after a nonlinear
 *     registration, the six responses of its reference volume at the
 *     finest scale (the reads the reference keeps commented out at
 *     :5754-5759).  Gradient samples on the first and last z plane, which
 *     the reference leaves unwritten, are 0.
 *   - SetDoSkullstrip / SetDoSkullstripOriginal with SetInputMNIBrainMask
 *     and SetOutputSkullstrippedT1Volume: PerformRegistrationTwoVolumesWrapper
 *     multiplies the aligned volume by the mask, or the interpolated volume
 *     by the mask carried back by the inverse affine transform (NEAREST), as
 *     at broccoli_lib.cpp:8064-8105; a missing mask or output array is an
 *     error (BRC_ERR_INVALID), not ignored.
 *   - GetOpenCLCreateKernelErrors / GetOpenCLCreateBufferErrors: kernels are
 *     compiled into the library, so no kernel is created at run time (all
 *     zeros); element 0 of the buffer array holds BRC_ERR_NOMEM when a call
 *     failed to allocate device memory.
 *   - Extensions (new setters): SetPrecision, SetMotionCorrectionTolerance,
 *     SetSolveFP64.
 */
#ifndef BROCCOLI_LIB_B200_H
#define BROCCOLI_LIB_B200_H

#include <stddef.h>

#include <string>

#include "broccoli_b200.h"

typedef unsigned int cl_uint;
typedef union {
  float s[2];
  struct {
    float x, y;
  };
} cl_float2;

/* values of code/BROCCOLI_LIB/broccoli_constants.h used on this path */
#ifndef BROCCOLI_CONSTANTS_H
#define MATLAB 0
#define PYTHON 1
#define BASH 2
#define TRANSLATION 0
#define RIGID 1
#define AFFINE 2
#define NEAREST 0
#define LINEAR 1
#define CUBIC 2
#define DO_OVERWRITE 0
#define NO_OVERWRITE 1
#define SUCCESS 0
#define FAIL 1
#define LOWPASS 0
#define RANDOM 1
#endif

class BROCCOLI_LIB {
 public:
  BROCCOLI_LIB();
  BROCCOLI_LIB(cl_uint platform, cl_uint device);
  BROCCOLI_LIB(cl_uint platform, cl_uint device, const char* location);
  BROCCOLI_LIB(cl_uint platform, cl_uint device, int wrapper, bool verbos);
  ~BROCCOLI_LIB();

  bool OpenCLInitiate(cl_uint platform, cl_uint device);
  bool GetOpenCLInitiated();
  std::string GetOpenCLInitializationError();
  const char* GetOpenCLError();
  const char* GetOpenCLErrorMessage(int error);
  int* GetOpenCLRunKernelErrors();
  int* GetOpenCLCreateKernelErrors();
  int* GetOpenCLCreateBufferErrors();

  void SetWrapper(int wrapper);
  void SetVerbose(bool verbos);
  void SetDebug(bool debug);

  // sizes and voxel sizes
  void SetEPIWidth(size_t w);
  void SetEPIHeight(size_t h);
  void SetEPIDepth(size_t d);
  void SetEPITimepoints(size_t t);
  void SetEPIVoxelSizeX(float v);
  void SetEPIVoxelSizeY(float v);
  void SetEPIVoxelSizeZ(float v);
  void SetT1Width(size_t w);
  void SetT1Height(size_t h);
  void SetT1Depth(size_t d);
  void SetT1Timepoints(size_t t);
  void SetT1VoxelSizeX(float v);
  void SetT1VoxelSizeY(float v);
  void SetT1VoxelSizeZ(float v);
  void SetMNIWidth(size_t w);
  void SetMNIHeight(size_t h);
  void SetMNIDepth(size_t d);
  void SetMNIVoxelSizeX(float v);
  void SetMNIVoxelSizeY(float v);
  void SetMNIVoxelSizeZ(float v);

  // inputs
  void SetInputfMRIVolumes(float* input);
  void SetInputEPIVolume(float* input);
  void SetInputT1Volume(float* input);
  void SetInputMNIVolume(float* input);
  void SetInputMNIBrainVolume(float* input);

  // filters and algorithm settings
  void SetPrecenterRegistration(bool center);
  void SetDoSkullstrip(bool doskullstrip);
  void SetDoSkullstripOriginal(bool doskullstriporiginal);
  void SetInputMNIBrainMask(float* mask);
  void SetImageRegistrationFilterSize(int N);
  void SetLinearImageRegistrationFilters(float* qf1r, float* qf1i, float* qf2r, float* qf2i, float* qf3r,
                                         float* qf3i);
  void SetNonLinearImageRegistrationFilters(float* qf1r, float* qf1i, float* qf2r, float* qf2i, float* qf3r,
                                            float* qf3i, float* qf4r, float* qf4i, float* qf5r, float* qf5i,
                                            float* qf6r, float* qf6i);
  void SetProjectionTensorMatrixFirstFilter(float m11, float m12, float m13, float m22, float m23, float m33);
  void SetProjectionTensorMatrixSecondFilter(float m11, float m12, float m13, float m22, float m23, float m33);
  void SetProjectionTensorMatrixThirdFilter(float m11, float m12, float m13, float m22, float m23, float m33);
  void SetProjectionTensorMatrixFourthFilter(float m11, float m12, float m13, float m22, float m23, float m33);
  void SetProjectionTensorMatrixFifthFilter(float m11, float m12, float m13, float m22, float m23, float m33);
  void SetProjectionTensorMatrixSixthFilter(float m11, float m12, float m13, float m22, float m23, float m33);
  void SetFilterDirections(float* x, float* y, float* z);
  void SetNumberOfIterationsForLinearImageRegistration(int N);
  void SetNumberOfIterationsForNonLinearImageRegistration(int N);
  void SetNumberOfIterationsForMotionCorrection(int N);
  void SetChangeMotionCorrectionReferenceVolume(bool change);
  void SetMotionCorrectionReferenceVolume(float* reference);
  void SetCoarsestScaleT1MNI(int N);
  void SetCoarsestScaleEPIT1(int N);
  void SetApplyMotionCorrection(bool apply);
  void SetApplySmoothing(bool apply);
  void SetApplySliceTimingCorrection(bool apply);  // true is not supported
  void SetPreprocessingOnly(bool only);            // PerformFirstLevelAnalysisWrapper needs true
  void SetMMT1ZCUT(int mm);
  void SetInterpolationMode(int mode);
  void SetTsigma(float s);
  void SetEsigma(float s);
  void SetDsigma(float s);
  void SetSmoothingFilters(float* fx, float* fy, float* fz);
  void SetSmoothingType(int type);
  void SetEPISmoothingAmount(float fwhm_mm);
  void SetEPIMask(float* mask);  // certainty of PerformSmoothingNormalizedWrapper
  void SetInputCertainty(float* certainty);  // certainty of PerformSmoothingNormalizedHostWrapper
  void SetAutoMask(bool automask);  // certainty from SegmentEPIData of the first fMRI volume

  // extensions of this implementation
  void SetPrecision(int precision);             // BRC_PREC_FP32 / BRC_PREC_BF16X3
  void SetMotionCorrectionTolerance(float voxels);  // per-volume early exit (0: off)
  void SetSolveFP64(bool fp64);                 // per-voxel 3x3 solves in FP64

  // outputs (caller-allocated host arrays)
  void SetOutputMotionParameters(float* output);
  void SetOutputMotionCorrectedfMRIVolumes(float* output);
  void SetOutputT1MNIRegistrationParameters(float* output);
  void SetOutputAlignedT1VolumeLinear(float* output);
  void SetOutputAlignedT1VolumeNonLinear(float* output);
  void SetOutputInterpolatedT1Volume(float* output);
  void SetOutputDisplacementField(float* x, float* y, float* z);
  void SetOutputSmoothedfMRIVolumes(float* output);
  void SetOutputQuadratureFilterResponses(cl_float2* q1, cl_float2* q2, cl_float2* q3);
  void SetOutputQuadratureFilterResponses(cl_float2* q1, cl_float2* q2, cl_float2* q3, cl_float2* q4,
                                          cl_float2* q5, cl_float2* q6);
  void SetOutputPhaseDifferences(float* pd);
  void SetOutputPhaseCertainties(float* pc);
  void SetOutputPhaseGradients(float* pg);
  void SetOutputSkullstrippedT1Volume(float* skullstripped);
  void SetOutputEPIT1RegistrationParameters(float* output);
  void SetOutputEPIMNIRegistrationParameters(float* output);
  void SetOutputAlignedEPIVolumeT1(float* output);
  void SetOutputAlignedEPIVolumeMNILinear(float* output);
  void SetOutputAlignedEPIVolumeMNINonlinear(float* output);
  void SetOutputEPIMask(float* output);
  void SetSaveInterpolatedT1(bool save);
  void SetSaveAlignedT1MNILinear(bool save);
  void SetSaveAlignedT1MNINonLinear(bool save);
  void SetSaveAlignedEPIT1(bool save);
  void SetSaveAlignedEPIMNI(bool save);
  void SetSaveEPIMask(bool save);
  void SetSaveMotionCorrected(bool save);
  void SetSaveSmoothed(bool save);

  // entry points
  void PerformMotionCorrectionWrapper();
  void PerformRegistrationTwoVolumesWrapper();
  void PerformSmoothingWrapper();
  void PerformSmoothingNormalizedWrapper();
  void PerformSmoothingNormalizedHostWrapper();  // smooths the fMRI volumes in place
  // 4D transforms of h_T1_Volume (t1 timepoints) into the array of
  // SetOutputInterpolatedT1Volume: resampled onto the MNI grid, then the
  // parameters of SetOutputT1MNIRegistrationParameters (Linear) or the field
  // of SetOutputDisplacementField (NonLinear) applied; CenterVolumes centres
  // the T1 volumes by the first one's centre of mass at T1 size.  NEAREST or
  // LINEAR (SetInterpolationMode); CUBIC fails with BRC_ERR_UNSUPPORTED.
  void TransformVolumesLinearWrapper();
  void TransformVolumesNonLinearWrapper();
  void CenterVolumesWrapper();
  // The preprocessing of a first-level analysis (brc_first_level_preprocess):
  // T1 -> MNI, EPI -> T1, motion correction, EPI mask and normalised
  // smoothing; h_fMRI_Volumes is replaced by the preprocessed series.  The
  // statistics are not part of this library: SetPreprocessingOnly(true) is
  // required, and slice-timing correction must be off.
  void PerformFirstLevelAnalysisWrapper();
  const float* GetCenterParameters() const { return center_params_; }  // of the last CenterVolumesWrapper

  int GetLastStatus() const { return last_status_; }

 private:
  brc_ctx* ctx_ = nullptr;
  bool initiated_ = false;
  std::string init_error_;
  std::string last_error_;  // message of the last failed call (GetOpenCLError)
  int last_status_ = BRC_OK;
  int run_errors_[200] = {0};
  int create_kernel_errors_[200] = {0};
  int create_buffer_errors_[200] = {0};
  bool debug_ = false;
  bool precenter_ = false, do_skullstrip_ = false, do_skullstrip_original_ = false;
  float* h_mni_mask_ = nullptr;
  float* out_skullstripped_ = nullptr;
  float* out_pd_ = nullptr;
  float* out_pc_ = nullptr;
  float* out_pg_ = nullptr;
  int wrapper_ = BASH;
  bool verbose_ = false;

  size_t epi_w_ = 0, epi_h_ = 0, epi_d_ = 0, epi_t_ = 0;
  size_t t1_w_ = 0, t1_h_ = 0, t1_d_ = 0, t1_t_ = 1;
  size_t mni_w_ = 0, mni_h_ = 0, mni_d_ = 0;
  float epi_vox_[3] = {1, 1, 1}, t1_vox_[3] = {1, 1, 1}, mni_vox_[3] = {1, 1, 1};

  void smooth_normalized(const float* h_mask, float* h_out, const char* where);
  float* h_fmri_ = nullptr;
  float* h_epi_ = nullptr;
  float* h_t1_ = nullptr;
  float* h_mni_ = nullptr;
  float* h_mni_brain_ = nullptr;
  float* h_mc_reference_ = nullptr;

  int filter_size_ = 7;
  const float* lin_[6] = {nullptr};
  const float* nonlin_[12] = {nullptr};
  float tensors_[36] = {0};
  const float* dirs_[3] = {nullptr};
  int it_linear_ = 10, it_nonlinear_ = 10, it_mc_ = 5;
  bool change_mc_reference_ = false;
  int coarsest_ = 4, mm_z_cut_ = 0, interpolation_ = LINEAR;
  float tsigma_ = 5.0f, esigma_ = 5.0f, dsigma_ = 5.0f;
  const float* smooth_f_[3] = {nullptr};
  int smoothing_type_ = LOWPASS;
  float epi_fwhm_ = 8.0f;
  int precision_ = BRC_PREC_FP32;
  float mc_tolerance_ = 0.0f;
  bool solve_fp64_ = false;

  float* out_motion_ = nullptr;
  float* out_mc_ = nullptr;
  float* out_params_ = nullptr;
  float* out_aligned_lin_ = nullptr;
  float* out_aligned_nonlin_ = nullptr;
  float* out_interpolated_ = nullptr;
  float* out_field_[3] = {nullptr};
  float* out_smoothed_ = nullptr;
  float* h_epi_mask_ = nullptr;
  float* h_certainty_ = nullptr;
  bool auto_mask_ = false;
  cl_float2* out_q_[6] = {nullptr};

  int coarsest_epi_t1_ = 4;
  bool apply_mc_ = true, apply_smoothing_ = true, apply_slice_timing_ = false, preprocessing_only_ = false;
  float* out_params_epi_t1_ = nullptr;
  float* out_params_epi_mni_ = nullptr;
  float* out_aligned_epi_t1_ = nullptr;
  float* out_aligned_epi_mni_lin_ = nullptr;
  float* out_aligned_epi_mni_nonlin_ = nullptr;
  float* out_epi_mask_ = nullptr;
  bool save_interpolated_t1_ = false, save_t1_lin_ = false, save_t1_nonlin_ = false, save_epi_t1_ = false,
       save_epi_mni_ = false, save_epi_mask_ = false, save_mc_ = false, save_smoothed_ = false;

  float center_params_[12] = {0};
  bool t1_to_mni(const float* d_t1, float* d_out, const char* where);
  bool check(int status, const char* where);
  bool apply_debug();
  bool pack_linear(float* bank3);
  bool pack_nonlinear(float* bank6, float* dirs18);
};

#endif
