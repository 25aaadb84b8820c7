// broccoli_lib.cpp -- the BROCCOLI_LIB class (include/broccoli_lib.h) on
// the C-ABI of libbroccoli_b200.  Host code only: every device operation is
// a brc_* call; the class owns no CUDA state besides its brc_ctx.
#include "../../include/broccoli_lib.h"

#include <math.h>
#include <string.h>

#include <vector>

namespace {

// Gaussian smoothing filters from a FWHM in mm and the voxel sizes,
// normalised by their float sums (CreateSmoothingFilters,
// broccoli_lib.cpp:11055-11091).
void fwhm_filters(float fwhm, const float* vox, float* fx, float* fy, float* fz) {
  brc_smoothing_filters_fwhm(fwhm, vox, fx, fy, fz);
}

// RAII device buffer over brc_device_alloc / brc_device_free.
struct DeviceArray {
  brc_ctx* ctx;
  void* ptr = nullptr;
  int status = BRC_OK;
  DeviceArray(brc_ctx* c, size_t bytes) : ctx(c) { status = brc_device_alloc(ctx, bytes, &ptr); }
  ~DeviceArray() {
    if (ptr) brc_device_free(ctx, ptr);
  }
  float* f() const { return static_cast<float*>(ptr); }
};

}  // namespace

BROCCOLI_LIB::BROCCOLI_LIB() {}

BROCCOLI_LIB::BROCCOLI_LIB(cl_uint platform, cl_uint device) { OpenCLInitiate(platform, device); }

BROCCOLI_LIB::BROCCOLI_LIB(cl_uint platform, cl_uint device, const char* /*location*/) {
  OpenCLInitiate(platform, device);
}

BROCCOLI_LIB::BROCCOLI_LIB(cl_uint platform, cl_uint device, int wrapper, bool verbos)
    : wrapper_(wrapper), verbose_(verbos) {
  OpenCLInitiate(platform, device);
}

BROCCOLI_LIB::~BROCCOLI_LIB() {
  if (ctx_) brc_ctx_destroy(ctx_);
}

bool BROCCOLI_LIB::OpenCLInitiate(cl_uint platform, cl_uint device) {
  if (ctx_) {
    brc_ctx_destroy(ctx_);
    ctx_ = nullptr;
  }
  initiated_ = false;
  if (platform != 0) {
    init_error_ = "platform must be 0 (one CUDA platform)";
    return false;
  }
  const int s = brc_ctx_create((int)device, &ctx_);
  if (s != BRC_OK) {
    init_error_ = std::string("brc_ctx_create: ") + brc_status_string(s);
    ctx_ = nullptr;
    return false;
  }
  init_error_.clear();
  initiated_ = true;
  return true;
}

bool BROCCOLI_LIB::GetOpenCLInitiated() { return initiated_; }
std::string BROCCOLI_LIB::GetOpenCLInitializationError() { return init_error_; }
const char* BROCCOLI_LIB::GetOpenCLError() {
  if (!last_error_.empty()) return last_error_.c_str();
  return ctx_ ? brc_last_error(ctx_) : init_error_.c_str();
}
const char* BROCCOLI_LIB::GetOpenCLErrorMessage(int error) { return brc_status_string(error); }
int* BROCCOLI_LIB::GetOpenCLRunKernelErrors() { return run_errors_; }
int* BROCCOLI_LIB::GetOpenCLCreateKernelErrors() { return create_kernel_errors_; }
int* BROCCOLI_LIB::GetOpenCLCreateBufferErrors() { return create_buffer_errors_; }

void BROCCOLI_LIB::SetWrapper(int w) { wrapper_ = w; }
void BROCCOLI_LIB::SetVerbose(bool v) { verbose_ = v; }
void BROCCOLI_LIB::SetDebug(bool d) { debug_ = d; }

void BROCCOLI_LIB::SetEPIWidth(size_t w) { epi_w_ = w; }
void BROCCOLI_LIB::SetEPIHeight(size_t h) { epi_h_ = h; }
void BROCCOLI_LIB::SetEPIDepth(size_t d) { epi_d_ = d; }
void BROCCOLI_LIB::SetEPITimepoints(size_t t) { epi_t_ = t; }
void BROCCOLI_LIB::SetEPIVoxelSizeX(float v) { epi_vox_[0] = v; }
void BROCCOLI_LIB::SetEPIVoxelSizeY(float v) { epi_vox_[1] = v; }
void BROCCOLI_LIB::SetEPIVoxelSizeZ(float v) { epi_vox_[2] = v; }
void BROCCOLI_LIB::SetT1Width(size_t w) { t1_w_ = w; }
void BROCCOLI_LIB::SetT1Height(size_t h) { t1_h_ = h; }
void BROCCOLI_LIB::SetT1Depth(size_t d) { t1_d_ = d; }
void BROCCOLI_LIB::SetT1Timepoints(size_t t) { t1_t_ = t; }
void BROCCOLI_LIB::SetT1VoxelSizeX(float v) { t1_vox_[0] = v; }
void BROCCOLI_LIB::SetT1VoxelSizeY(float v) { t1_vox_[1] = v; }
void BROCCOLI_LIB::SetT1VoxelSizeZ(float v) { t1_vox_[2] = v; }
void BROCCOLI_LIB::SetMNIWidth(size_t w) { mni_w_ = w; }
void BROCCOLI_LIB::SetMNIHeight(size_t h) { mni_h_ = h; }
void BROCCOLI_LIB::SetMNIDepth(size_t d) { mni_d_ = d; }
void BROCCOLI_LIB::SetMNIVoxelSizeX(float v) { mni_vox_[0] = v; }
void BROCCOLI_LIB::SetMNIVoxelSizeY(float v) { mni_vox_[1] = v; }
void BROCCOLI_LIB::SetMNIVoxelSizeZ(float v) { mni_vox_[2] = v; }

void BROCCOLI_LIB::SetInputfMRIVolumes(float* p) { h_fmri_ = p; }
void BROCCOLI_LIB::SetInputEPIVolume(float* p) { h_epi_ = p; }
void BROCCOLI_LIB::SetInputT1Volume(float* p) { h_t1_ = p; }
void BROCCOLI_LIB::SetInputMNIVolume(float* p) { h_mni_ = p; }
void BROCCOLI_LIB::SetInputMNIBrainVolume(float* p) { h_mni_brain_ = p; }

void BROCCOLI_LIB::SetPrecenterRegistration(bool c) { precenter_ = c; }
void BROCCOLI_LIB::SetDoSkullstrip(bool b) { do_skullstrip_ = b; }
void BROCCOLI_LIB::SetDoSkullstripOriginal(bool b) { do_skullstrip_original_ = b; }
void BROCCOLI_LIB::SetInputMNIBrainMask(float* m) { h_mni_mask_ = m; }
void BROCCOLI_LIB::SetImageRegistrationFilterSize(int N) { filter_size_ = N; }
void BROCCOLI_LIB::SetLinearImageRegistrationFilters(float* a, float* b, float* c, float* d, float* e,
                                                     float* f) {
  const float* p[6] = {a, b, c, d, e, f};
  for (int i = 0; i < 6; i++) lin_[i] = p[i];
}
void BROCCOLI_LIB::SetNonLinearImageRegistrationFilters(float* a, float* b, float* c, float* d, float* e,
                                                        float* f, float* g, float* h, float* i, float* j,
                                                        float* k, float* l) {
  const float* p[12] = {a, b, c, d, e, f, g, h, i, j, k, l};
  for (int n = 0; n < 12; n++) nonlin_[n] = p[n];
}
#define BRC_SET_TENSOR(NAME, K)                                                                      \
  void BROCCOLI_LIB::NAME(float m11, float m12, float m13, float m22, float m23, float m33) {        \
    float* t = tensors_ + 6 * (K);                                                                   \
    t[0] = m11;                                                                                      \
    t[1] = m12;                                                                                      \
    t[2] = m13;                                                                                      \
    t[3] = m22;                                                                                      \
    t[4] = m23;                                                                                      \
    t[5] = m33;                                                                                      \
  }
BRC_SET_TENSOR(SetProjectionTensorMatrixFirstFilter, 0)
BRC_SET_TENSOR(SetProjectionTensorMatrixSecondFilter, 1)
BRC_SET_TENSOR(SetProjectionTensorMatrixThirdFilter, 2)
BRC_SET_TENSOR(SetProjectionTensorMatrixFourthFilter, 3)
BRC_SET_TENSOR(SetProjectionTensorMatrixFifthFilter, 4)
BRC_SET_TENSOR(SetProjectionTensorMatrixSixthFilter, 5)
#undef BRC_SET_TENSOR
void BROCCOLI_LIB::SetFilterDirections(float* x, float* y, float* z) {
  dirs_[0] = x;
  dirs_[1] = y;
  dirs_[2] = z;
}
void BROCCOLI_LIB::SetNumberOfIterationsForLinearImageRegistration(int N) { it_linear_ = N; }
void BROCCOLI_LIB::SetNumberOfIterationsForNonLinearImageRegistration(int N) { it_nonlinear_ = N; }
void BROCCOLI_LIB::SetNumberOfIterationsForMotionCorrection(int N) { it_mc_ = N; }
void BROCCOLI_LIB::SetChangeMotionCorrectionReferenceVolume(bool c) { change_mc_reference_ = c; }
void BROCCOLI_LIB::SetMotionCorrectionReferenceVolume(float* r) { h_mc_reference_ = r; }
void BROCCOLI_LIB::SetCoarsestScaleT1MNI(int N) { coarsest_ = N; }
void BROCCOLI_LIB::SetCoarsestScaleEPIT1(int N) { coarsest_epi_t1_ = N; }
void BROCCOLI_LIB::SetApplyMotionCorrection(bool b) { apply_mc_ = b; }
void BROCCOLI_LIB::SetApplySmoothing(bool b) { apply_smoothing_ = b; }
void BROCCOLI_LIB::SetApplySliceTimingCorrection(bool b) { apply_slice_timing_ = b; }
void BROCCOLI_LIB::SetPreprocessingOnly(bool b) { preprocessing_only_ = b; }
void BROCCOLI_LIB::SetMMT1ZCUT(int mm) { mm_z_cut_ = mm; }
void BROCCOLI_LIB::SetInterpolationMode(int m) { interpolation_ = m; }
void BROCCOLI_LIB::SetTsigma(float s) { tsigma_ = s; }
void BROCCOLI_LIB::SetEsigma(float s) { esigma_ = s; }
void BROCCOLI_LIB::SetDsigma(float s) { dsigma_ = s; }
void BROCCOLI_LIB::SetSmoothingFilters(float* fx, float* fy, float* fz) {
  smooth_f_[0] = fx;
  smooth_f_[1] = fy;
  smooth_f_[2] = fz;
}
void BROCCOLI_LIB::SetSmoothingType(int t) { smoothing_type_ = t; }
void BROCCOLI_LIB::SetEPISmoothingAmount(float fwhm) { epi_fwhm_ = fwhm; }
void BROCCOLI_LIB::SetEPIMask(float* m) { h_epi_mask_ = m; }
void BROCCOLI_LIB::SetInputCertainty(float* c) { h_certainty_ = c; }
void BROCCOLI_LIB::SetAutoMask(bool a) { auto_mask_ = a; }
void BROCCOLI_LIB::SetPrecision(int p) { precision_ = p; }
void BROCCOLI_LIB::SetMotionCorrectionTolerance(float v) { mc_tolerance_ = v; }
void BROCCOLI_LIB::SetSolveFP64(bool b) { solve_fp64_ = b; }

void BROCCOLI_LIB::SetOutputMotionParameters(float* o) { out_motion_ = o; }
void BROCCOLI_LIB::SetOutputMotionCorrectedfMRIVolumes(float* o) { out_mc_ = o; }
void BROCCOLI_LIB::SetOutputT1MNIRegistrationParameters(float* o) { out_params_ = o; }
void BROCCOLI_LIB::SetOutputAlignedT1VolumeLinear(float* o) { out_aligned_lin_ = o; }
void BROCCOLI_LIB::SetOutputAlignedT1VolumeNonLinear(float* o) { out_aligned_nonlin_ = o; }
void BROCCOLI_LIB::SetOutputInterpolatedT1Volume(float* o) { out_interpolated_ = o; }
void BROCCOLI_LIB::SetOutputDisplacementField(float* x, float* y, float* z) {
  out_field_[0] = x;
  out_field_[1] = y;
  out_field_[2] = z;
}
void BROCCOLI_LIB::SetOutputSmoothedfMRIVolumes(float* o) { out_smoothed_ = o; }
void BROCCOLI_LIB::SetOutputQuadratureFilterResponses(cl_float2* a, cl_float2* b, cl_float2* c) {
  out_q_[0] = a;
  out_q_[1] = b;
  out_q_[2] = c;
  out_q_[3] = out_q_[4] = out_q_[5] = nullptr;
}
void BROCCOLI_LIB::SetOutputQuadratureFilterResponses(cl_float2* a, cl_float2* b, cl_float2* c, cl_float2* d,
                                                      cl_float2* e, cl_float2* f) {
  cl_float2* q[6] = {a, b, c, d, e, f};
  for (int k = 0; k < 6; k++) out_q_[k] = q[k];
}
void BROCCOLI_LIB::SetOutputPhaseDifferences(float* p) { out_pd_ = p; }
void BROCCOLI_LIB::SetOutputPhaseCertainties(float* p) { out_pc_ = p; }
void BROCCOLI_LIB::SetOutputPhaseGradients(float* p) { out_pg_ = p; }
void BROCCOLI_LIB::SetOutputSkullstrippedT1Volume(float* p) { out_skullstripped_ = p; }
void BROCCOLI_LIB::SetOutputEPIT1RegistrationParameters(float* o) { out_params_epi_t1_ = o; }
void BROCCOLI_LIB::SetOutputEPIMNIRegistrationParameters(float* o) { out_params_epi_mni_ = o; }
void BROCCOLI_LIB::SetOutputAlignedEPIVolumeT1(float* o) { out_aligned_epi_t1_ = o; }
void BROCCOLI_LIB::SetOutputAlignedEPIVolumeMNILinear(float* o) { out_aligned_epi_mni_lin_ = o; }
void BROCCOLI_LIB::SetOutputAlignedEPIVolumeMNINonlinear(float* o) { out_aligned_epi_mni_nonlin_ = o; }
void BROCCOLI_LIB::SetOutputEPIMask(float* o) { out_epi_mask_ = o; }
void BROCCOLI_LIB::SetSaveInterpolatedT1(bool b) { save_interpolated_t1_ = b; }
void BROCCOLI_LIB::SetSaveAlignedT1MNILinear(bool b) { save_t1_lin_ = b; }
void BROCCOLI_LIB::SetSaveAlignedT1MNINonLinear(bool b) { save_t1_nonlin_ = b; }
void BROCCOLI_LIB::SetSaveAlignedEPIT1(bool b) { save_epi_t1_ = b; }
void BROCCOLI_LIB::SetSaveAlignedEPIMNI(bool b) { save_epi_mni_ = b; }
void BROCCOLI_LIB::SetSaveEPIMask(bool b) { save_epi_mask_ = b; }
void BROCCOLI_LIB::SetSaveMotionCorrected(bool b) { save_mc_ = b; }
void BROCCOLI_LIB::SetSaveSmoothed(bool b) { save_smoothed_ = b; }

bool BROCCOLI_LIB::check(int status, const char* where) {
  last_status_ = status;
  if (status == BRC_OK) {
    last_error_.clear();
    return true;
  }
  run_errors_[0] = status;
  if (status == BRC_ERR_NOMEM) create_buffer_errors_[0] = status;
  last_error_ = std::string(where) + ": " + brc_status_string(status) + (ctx_ ? std::string(" (") +
                brc_last_error(ctx_) + ")" : std::string());
  return false;
}

// The DEBUG outputs of the registrations (SetDebug, broccoli_lib.cpp:
// 5285-5289, :5349-5354) handed to the context before each entry point.
bool BROCCOLI_LIB::apply_debug() {
  if (!debug_) return check(brc_ctx_set_debug_outputs(ctx_, nullptr), "SetDebug");
  brc_debug_outputs d;
  memset(&d, 0, sizeof(d));
  for (int k = 0; k < 6; k++) d.quadrature_responses[k] = out_q_[k];
  d.phase_differences = out_pd_;
  d.phase_certainties = out_pc_;
  d.phase_gradients = out_pg_;
  return check(brc_ctx_set_debug_outputs(ctx_, &d), "SetDebug");
}

bool BROCCOLI_LIB::pack_linear(float* bank) {
  for (int i = 0; i < 6; i++)
    if (!lin_[i]) return false;
  for (int k = 0; k < 3; k++) {
    memcpy(bank + k * 686, lin_[2 * k], sizeof(float) * 343);
    memcpy(bank + k * 686 + 343, lin_[2 * k + 1], sizeof(float) * 343);
  }
  return true;
}

bool BROCCOLI_LIB::pack_nonlinear(float* bank, float* dirs) {
  for (int i = 0; i < 12; i++)
    if (!nonlin_[i]) return false;
  for (int a = 0; a < 3; a++)
    if (!dirs_[a]) return false;
  for (int k = 0; k < 6; k++) {
    memcpy(bank + k * 686, nonlin_[2 * k], sizeof(float) * 343);
    memcpy(bank + k * 686 + 343, nonlin_[2 * k + 1], sizeof(float) * 343);
  }
  for (int a = 0; a < 3; a++) memcpy(dirs + 6 * a, dirs_[a], sizeof(float) * 6);
  return true;
}

// PerformMotionCorrectionWrapper, broccoli_lib.cpp:10658-10720: all volumes
// registered to volume 0 (or the given reference) in one batched call.
void BROCCOLI_LIB::PerformMotionCorrectionWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "PerformMotionCorrectionWrapper")) return;
  float bank[3 * 686];
  if (!h_fmri_ || filter_size_ != 7 || !pack_linear(bank)) {
    check(BRC_ERR_INVALID, "PerformMotionCorrectionWrapper: inputs or filters not set");
    return;
  }
  brc_linear_opts o;
  brc_linear_opts_default(&o, it_mc_);
  o.type = BRC_RIGID;
  o.precision = precision_;
  o.tolerance = mc_tolerance_;
  if (!apply_debug()) return;
  const int W = (int)epi_w_, H = (int)epi_h_, D = (int)epi_d_, T = (int)epi_t_;
  std::vector<float> motion(6 * (size_t)T);
  const float* ref = change_mc_reference_ ? h_mc_reference_ : nullptr;
  if (!check(brc_motion_correct(ctx_, h_fmri_, W, H, D, T, epi_vox_, bank, &o, ref, motion.data()),
             "brc_motion_correct"))
    return;
  if (out_motion_) memcpy(out_motion_, motion.data(), sizeof(float) * motion.size());
  if (out_mc_ && out_mc_ != h_fmri_) memcpy(out_mc_, h_fmri_, sizeof(float) * (size_t)W * H * D * T);
}

// PerformSmoothingWrapper, broccoli_lib.cpp:11122-11210.
void BROCCOLI_LIB::PerformSmoothingWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "PerformSmoothingWrapper")) return;
  if (!h_fmri_ || !out_smoothed_) {
    check(BRC_ERR_INVALID, "PerformSmoothingWrapper: input or output not set");
    return;
  }
  float fx[9], fy[9], fz[9];
  if (smoothing_type_ == RANDOM) {
    if (!smooth_f_[0] || !smooth_f_[1] || !smooth_f_[2]) {
      check(BRC_ERR_INVALID, "PerformSmoothingWrapper: smoothing filters not set");
      return;
    }
    memcpy(fx, smooth_f_[0], sizeof(fx));
    memcpy(fy, smooth_f_[1], sizeof(fy));
    memcpy(fz, smooth_f_[2], sizeof(fz));
  } else {
    fwhm_filters(epi_fwhm_, epi_vox_, fx, fy, fz);
  }
  const size_t V = epi_w_ * epi_h_ * epi_d_, n = V * epi_t_;
  DeviceArray in(ctx_, sizeof(float) * n), out(ctx_, sizeof(float) * n);
  if (!check(in.status, "alloc") || !check(out.status, "alloc")) return;
  if (!check(brc_copy_to_device(ctx_, in.ptr, h_fmri_, sizeof(float) * n), "H2D")) return;
  if (!check(brc_smooth3d(ctx_, in.f(), (int)epi_w_, (int)epi_h_, (int)epi_d_, (int)epi_t_, fx, fy, fz,
                          nullptr, nullptr, out.f()),
             "brc_smooth3d"))
    return;
  check(brc_copy_to_host(ctx_, out_smoothed_, out.ptr, sizeof(float) * n), "D2H");
}

// PerformSmoothingNormalizedWrapper, broccoli_lib.cpp:11227-11272: the EPI
// mask is the certainty; LOWPASS filters from the FWHM or RANDOM filters.
void BROCCOLI_LIB::PerformSmoothingNormalizedWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "PerformSmoothingNormalizedWrapper")) return;
  if (!h_fmri_ || !out_smoothed_ || !h_epi_mask_) {
    check(BRC_ERR_INVALID, "PerformSmoothingNormalizedWrapper: input, mask or output not set");
    return;
  }
  smooth_normalized(h_epi_mask_, out_smoothed_, "PerformSmoothingNormalizedWrapper");
}

// PerformSmoothingNormalizedHostWrapper, broccoli_lib.cpp:11729-11850 (the
// Smoothing CLI, Bash_Wrapper/Smoothing.cpp:593-613): the certainty from
// SetInputCertainty, LOWPASS filters from the FWHM, the fMRI volumes
// smoothed in place.  The reference smooths one volume per upload; here all
// volumes go through one batched call.
void BROCCOLI_LIB::PerformSmoothingNormalizedHostWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "PerformSmoothingNormalizedHostWrapper")) return;
  if (!h_fmri_ || !h_certainty_) {
    check(BRC_ERR_INVALID, "PerformSmoothingNormalizedHostWrapper: input or certainty not set");
    return;
  }
  if (auto_mask_) {
    // the certainty is the mask of the first fMRI volume, written back to
    // the host certainty array (SegmentEPIData, broccoli_lib.cpp:11008-11030)
    const size_t V = epi_w_ * epi_h_ * epi_d_;
    DeviceArray vol(ctx_, sizeof(float) * V), mask(ctx_, sizeof(float) * V);
    if (!check(vol.status, "alloc") || !check(mask.status, "alloc")) return;
    if (!check(brc_copy_to_device(ctx_, vol.ptr, h_fmri_, sizeof(float) * V), "H2D")) return;
    if (!check(brc_segment_epi(ctx_, vol.f(), (int)epi_w_, (int)epi_h_, (int)epi_d_, epi_vox_, mask.f()),
               "brc_segment_epi"))
      return;
    if (!check(brc_copy_to_host(ctx_, h_certainty_, mask.ptr, sizeof(float) * V), "D2H")) return;
  }
  const int keep = smoothing_type_;
  smoothing_type_ = LOWPASS;
  smooth_normalized(h_certainty_, h_fmri_, "PerformSmoothingNormalizedHostWrapper");
  smoothing_type_ = keep;
}

void BROCCOLI_LIB::smooth_normalized(const float* h_mask, float* h_out, const char* where) {
  float fx[9], fy[9], fz[9];
  if (smoothing_type_ == RANDOM) {
    if (!smooth_f_[0] || !smooth_f_[1] || !smooth_f_[2]) {
      check(BRC_ERR_INVALID, (std::string(where) + ": smoothing filters not set").c_str());
      return;
    }
    memcpy(fx, smooth_f_[0], sizeof(fx));
    memcpy(fy, smooth_f_[1], sizeof(fy));
    memcpy(fz, smooth_f_[2], sizeof(fz));
  } else {
    fwhm_filters(epi_fwhm_, epi_vox_, fx, fy, fz);
  }
  const size_t V = epi_w_ * epi_h_ * epi_d_, n = V * epi_t_;
  DeviceArray in(ctx_, sizeof(float) * n), out(ctx_, sizeof(float) * n), mask(ctx_, sizeof(float) * V);
  if (!check(in.status, "alloc") || !check(out.status, "alloc") || !check(mask.status, "alloc")) return;
  if (!check(brc_copy_to_device(ctx_, in.ptr, h_fmri_, sizeof(float) * n), "H2D")) return;
  if (!check(brc_copy_to_device(ctx_, mask.ptr, h_mask, sizeof(float) * V), "H2D")) return;
  if (!check(brc_smooth_normalized(ctx_, in.f(), (int)epi_w_, (int)epi_h_, (int)epi_d_, (int)epi_t_, mask.f(), fx,
                                   fy, fz, out.f()),
             "brc_smooth_normalized"))
    return;
  check(brc_copy_to_host(ctx_, h_out, out.ptr, sizeof(float) * n), "D2H");
}

// PerformRegistrationTwoVolumesWrapper, broccoli_lib.cpp:7973-8112.
// h_T1_Volume (T1 grid, t1_t_ volumes) resampled onto the MNI grid with the
// interpolation mode (ChangeVolumesResolutionAndSize), into d_out.
bool BROCCOLI_LIB::t1_to_mni(const float* d_t1, float* d_out, const char* where) {
  return check(brc_change_resolution_and_size_batch(ctx_, d_t1, (int)t1_w_, (int)t1_h_, (int)t1_d_, (int)t1_t_,
                                                    t1_vox_, d_out, (int)mni_w_, (int)mni_h_, (int)mni_d_, mni_vox_,
                                                    mm_z_cut_, interpolation_),
               where);
}

void BROCCOLI_LIB::TransformVolumesLinearWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "TransformVolumesLinearWrapper")) return;
  if (!h_t1_ || !out_params_ || !out_interpolated_) {
    check(BRC_ERR_INVALID, "TransformVolumesLinearWrapper: T1 volumes, parameters or output not set");
    return;
  }
  const size_t V1 = t1_w_ * t1_h_ * t1_d_ * t1_t_, V2 = mni_w_ * mni_h_ * mni_d_ * t1_t_;
  DeviceArray d_in(ctx_, sizeof(float) * V1), d_mni(ctx_, sizeof(float) * V2), d_out(ctx_, sizeof(float) * V2);
  for (const DeviceArray* a : {&d_in, &d_mni, &d_out})
    if (!check(a->status, "alloc")) return;
  if (!check(brc_copy_to_device(ctx_, d_in.ptr, h_t1_, sizeof(float) * V1), "H2D")) return;
  if (!t1_to_mni(d_in.f(), d_mni.f(), "TransformVolumesLinearWrapper: resample")) return;
  // the parameters are read from the array given to
  // SetOutputT1MNIRegistrationParameters, as in the reference
  if (!check(brc_transform_volumes_linear(ctx_, d_mni.f(), (int)mni_w_, (int)mni_h_, (int)mni_d_, (int)t1_t_,
                                          out_params_, interpolation_, d_out.f()),
             "TransformVolumesLinearWrapper"))
    return;
  check(brc_copy_to_host(ctx_, out_interpolated_, d_out.ptr, sizeof(float) * V2), "D2H");
}

void BROCCOLI_LIB::TransformVolumesNonLinearWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "TransformVolumesNonLinearWrapper")) return;
  if (!h_t1_ || !out_field_[0] || !out_field_[1] || !out_field_[2] || !out_interpolated_) {
    check(BRC_ERR_INVALID, "TransformVolumesNonLinearWrapper: T1 volumes, displacement field or output not set");
    return;
  }
  const size_t V1 = t1_w_ * t1_h_ * t1_d_ * t1_t_, V3 = mni_w_ * mni_h_ * mni_d_, V2 = V3 * t1_t_;
  DeviceArray d_in(ctx_, sizeof(float) * V1), d_mni(ctx_, sizeof(float) * V2), d_out(ctx_, sizeof(float) * V2),
      d_field(ctx_, sizeof(float) * 3 * V3);
  for (const DeviceArray* a : {&d_in, &d_mni, &d_out, &d_field})
    if (!check(a->status, "alloc")) return;
  if (!check(brc_copy_to_device(ctx_, d_in.ptr, h_t1_, sizeof(float) * V1), "H2D")) return;
  // the field is read from the arrays given to SetOutputDisplacementField
  for (int a = 0; a < 3; a++)
    if (!check(brc_copy_to_device(ctx_, d_field.f() + a * V3, out_field_[a], sizeof(float) * V3), "H2D")) return;
  if (!t1_to_mni(d_in.f(), d_mni.f(), "TransformVolumesNonLinearWrapper: resample")) return;
  if (!check(brc_transform_volumes_nonlinear(ctx_, d_mni.f(), (int)mni_w_, (int)mni_h_, (int)mni_d_, (int)t1_t_,
                                             d_field.f(), d_field.f() + V3, d_field.f() + 2 * V3, interpolation_,
                                             d_out.f()),
             "TransformVolumesNonLinearWrapper"))
    return;
  check(brc_copy_to_host(ctx_, out_interpolated_, d_out.ptr, sizeof(float) * V2), "D2H");
}

void BROCCOLI_LIB::CenterVolumesWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "CenterVolumesWrapper")) return;
  if (!h_t1_ || !out_interpolated_) {
    check(BRC_ERR_INVALID, "CenterVolumesWrapper: T1 volumes or output not set");
    return;
  }
  const size_t V = t1_w_ * t1_h_ * t1_d_ * t1_t_;
  DeviceArray d_in(ctx_, sizeof(float) * V), d_out(ctx_, sizeof(float) * V);
  for (const DeviceArray* a : {&d_in, &d_out})
    if (!check(a->status, "alloc")) return;
  if (!check(brc_copy_to_device(ctx_, d_in.ptr, h_t1_, sizeof(float) * V), "H2D")) return;
  if (!check(brc_center_volumes(ctx_, d_in.f(), (int)t1_w_, (int)t1_h_, (int)t1_d_, (int)t1_t_, interpolation_,
                                d_out.f(), center_params_),
             "CenterVolumesWrapper"))
    return;
  check(brc_copy_to_host(ctx_, out_interpolated_, d_out.ptr, sizeof(float) * V), "D2H");
}

void BROCCOLI_LIB::PerformRegistrationTwoVolumesWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "PerformRegistrationTwoVolumesWrapper")) return;
  float bank3[3 * 686], bank6[6 * 686], dirs[18];
  const float* tpl = h_mni_brain_ ? h_mni_brain_ : h_mni_;
  const bool nonlinear = it_nonlinear_ > 0;
  if (!h_t1_ || !tpl || !pack_linear(bank3) || (nonlinear && !pack_nonlinear(bank6, dirs))) {
    check(BRC_ERR_INVALID, "PerformRegistrationTwoVolumesWrapper: inputs or filters not set");
    return;
  }
  const size_t V1 = t1_w_ * t1_h_ * t1_d_, V2 = mni_w_ * mni_h_ * mni_d_;
  DeviceArray d_in(ctx_, sizeof(float) * V1), d_tpl(ctx_, sizeof(float) * V2);
  DeviceArray d_interp(ctx_, sizeof(float) * V2), d_lin(ctx_, sizeof(float) * V2),
      d_nonlin(ctx_, sizeof(float) * V2), d_field(ctx_, sizeof(float) * 3 * V2);
  for (const DeviceArray* a : {&d_in, &d_tpl, &d_interp, &d_lin, &d_nonlin, &d_field})
    if (!check(a->status, "alloc")) return;
  if (!check(brc_copy_to_device(ctx_, d_in.ptr, h_t1_, sizeof(float) * V1), "H2D")) return;
  if (!check(brc_copy_to_device(ctx_, d_tpl.ptr, tpl, sizeof(float) * V2), "H2D")) return;
  brc_two_volume_opts o;
  brc_two_volume_opts_default(&o);
  o.linear_iterations = it_linear_;
  o.nonlinear_iterations = it_nonlinear_;
  o.coarsest_scale = coarsest_;
  o.mm_z_cut = mm_z_cut_;
  o.tsigma = tsigma_;
  o.esigma = esigma_;
  o.dsigma = dsigma_;
  o.precision = precision_;
  o.solve_fp64 = solve_fp64_ ? 1 : 0;
  o.precenter = precenter_ ? 1 : 0;
  const bool strip = do_skullstrip_ || (do_skullstrip_original_ && it_linear_ > 0);
  if (strip && (!h_mni_mask_ || !out_skullstripped_)) {
    check(BRC_ERR_INVALID, "PerformRegistrationTwoVolumesWrapper: skull strip needs SetInputMNIBrainMask and "
                           "SetOutputSkullstrippedT1Volume");
    return;
  }
  if (!apply_debug()) return;
  float params[12];
  if (!check(brc_register_two_volumes(ctx_, d_in.f(), (int)t1_w_, (int)t1_h_, (int)t1_d_, t1_vox_, d_tpl.f(),
                                      (int)mni_w_, (int)mni_h_, (int)mni_d_, mni_vox_, bank3,
                                      nonlinear ? bank6 : nullptr, nonlinear ? tensors_ : nullptr,
                                      nonlinear ? dirs : nullptr, &o, params, d_interp.f(), d_lin.f(),
                                      d_nonlin.f(), d_field.f()),
             "brc_register_two_volumes"))
    return;
  if (out_params_) memcpy(out_params_, params, sizeof(params));
  if (out_interpolated_ && !check(brc_copy_to_host(ctx_, out_interpolated_, d_interp.ptr, sizeof(float) * V2), "D2H"))
    return;
  if (out_aligned_lin_ && !check(brc_copy_to_host(ctx_, out_aligned_lin_, d_lin.ptr, sizeof(float) * V2), "D2H"))
    return;
  if (nonlinear) {
    if (out_aligned_nonlin_ &&
        !check(brc_copy_to_host(ctx_, out_aligned_nonlin_, d_nonlin.ptr, sizeof(float) * V2), "D2H"))
      return;
    for (int a = 0; a < 3; a++)
      if (out_field_[a] &&
          !check(brc_copy_to_host(ctx_, out_field_[a], d_field.f() + a * V2, sizeof(float) * V2), "D2H"))
        return;
  }
  if (strip) {
    // broccoli_lib.cpp:8064-8105: DO_SKULLSTRIP multiplies the last aligned
    // volume by the brain mask; DO_SKULLSTRIP_ORIGINAL carries the mask back
    // by the inverse affine transform (NEAREST) and multiplies the
    // interpolated volume by it
    DeviceArray d_mask(ctx_, sizeof(float) * V2);
    if (!check(d_mask.status, "alloc")) return;
    if (!check(brc_copy_to_device(ctx_, d_mask.ptr, h_mni_mask_, sizeof(float) * V2), "H2D")) return;
    float* vol = nonlinear ? d_nonlin.f() : d_lin.f();
    const float* mask = d_mask.f();
    if (!do_skullstrip_) {
      float inv[12];
      brc_invert_affine_parameters(params, inv);
      if (!check(brc_transform_volumes_linear(ctx_, d_mask.f(), (int)mni_w_, (int)mni_h_, (int)mni_d_, 1, inv,
                                              BRC_INTERP_NEAREST, d_field.f()),
                 "skull strip: mask to the original space"))
        return;
      vol = d_interp.f();
      mask = d_field.f();
    }
    if (!check(brc_multiply_volumes(ctx_, vol, (int)mni_w_, (int)mni_h_, (int)mni_d_, 1, mask), "skull strip"))
      return;
    check(brc_copy_to_host(ctx_, out_skullstripped_, vol, sizeof(float) * V2), "D2H");
  }
}

// PerformFirstLevelAnalysisWrapper, broccoli_lib.cpp:8466-8733, up to the
// statistics (PREPROCESSING_ONLY): one brc_first_level_preprocess call.
// The parameter vectors and motion parameters are written always, the
// volumes when their SetSave* flag is on and the array is set.
void BROCCOLI_LIB::PerformFirstLevelAnalysisWrapper() {
  if (!initiated_ && !check(BRC_ERR_NODEVICE, "PerformFirstLevelAnalysisWrapper")) return;
  if (!preprocessing_only_) {
    check(BRC_ERR_UNSUPPORTED,
          "PerformFirstLevelAnalysisWrapper: the statistical analysis is not part of this library; "
          "call SetPreprocessingOnly(true)");
    return;
  }
  if (apply_slice_timing_) {
    check(BRC_ERR_UNSUPPORTED, "PerformFirstLevelAnalysisWrapper: slice-timing correction is not supported");
    return;
  }
  float bank3[3 * 686], bank6[6 * 686], dirs[18];
  const float* tpl = h_mni_brain_ ? h_mni_brain_ : h_mni_;
  if (!h_fmri_ || !h_t1_ || !tpl || !pack_linear(bank3) || !pack_nonlinear(bank6, dirs)) {
    check(BRC_ERR_INVALID, "PerformFirstLevelAnalysisWrapper: inputs or filters not set");
    return;
  }
  brc_first_level_input in;
  in.fmri = h_fmri_;
  in.epi_w = (int)epi_w_;
  in.epi_h = (int)epi_h_;
  in.epi_d = (int)epi_d_;
  in.epi_t = (int)epi_t_;
  in.t1 = h_t1_;
  in.t1_w = (int)t1_w_;
  in.t1_h = (int)t1_h_;
  in.t1_d = (int)t1_d_;
  in.mni = tpl;
  in.mni_w = (int)mni_w_;
  in.mni_h = (int)mni_h_;
  in.mni_d = (int)mni_d_;
  for (int a = 0; a < 3; a++) {
    in.epi_voxel[a] = epi_vox_[a];
    in.t1_voxel[a] = t1_vox_[a];
    in.mni_voxel[a] = mni_vox_[a];
  }
  in.filters3 = bank3;
  in.filters6 = bank6;
  in.tensors = tensors_;
  in.dirs = dirs;
  brc_first_level_opts o;
  brc_first_level_opts_default(&o);
  o.linear_iterations = it_linear_;
  o.nonlinear_iterations = it_nonlinear_;
  o.motion_iterations = it_mc_;
  o.coarsest_scale_t1_mni = coarsest_;
  o.coarsest_scale_epi_t1 = coarsest_epi_t1_;
  o.mm_t1_z_cut = mm_z_cut_;
  o.apply_motion_correction = apply_mc_ ? 1 : 0;
  o.apply_smoothing = apply_smoothing_ ? 1 : 0;
  o.smoothing_fwhm = epi_fwhm_;
  o.tsigma = tsigma_;
  o.esigma = esigma_;
  o.dsigma = dsigma_;
  o.precision = precision_;
  o.solve_fp64 = solve_fp64_ ? 1 : 0;
  brc_first_level_output out;
  memset(&out, 0, sizeof(out));
  out.params_t1_mni = out_params_;
  out.params_epi_t1 = out_params_epi_t1_;
  out.params_epi_mni = out_params_epi_mni_;
  out.motion_parameters = apply_mc_ ? out_motion_ : nullptr;
  out.interpolated_t1 = save_interpolated_t1_ ? out_interpolated_ : nullptr;
  out.aligned_t1_linear = save_t1_lin_ ? out_aligned_lin_ : nullptr;
  out.aligned_t1_nonlinear = save_t1_nonlin_ ? out_aligned_nonlin_ : nullptr;
  out.aligned_epi_t1 = save_epi_t1_ ? out_aligned_epi_t1_ : nullptr;
  out.aligned_epi_mni_linear = save_epi_mni_ ? out_aligned_epi_mni_lin_ : nullptr;
  out.aligned_epi_mni_nonlinear = save_epi_mni_ ? out_aligned_epi_mni_nonlin_ : nullptr;
  out.motion_corrected = save_mc_ && out_mc_ != h_fmri_ ? out_mc_ : nullptr;
  out.epi_mask = save_epi_mask_ ? out_epi_mask_ : nullptr;
  out.smoothed = save_smoothed_ && out_smoothed_ != h_fmri_ ? out_smoothed_ : nullptr;
  if (!apply_debug()) return;
  check(brc_first_level_preprocess(ctx_, &in, &o, &out), "brc_first_level_preprocess");
}
