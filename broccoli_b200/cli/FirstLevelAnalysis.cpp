// FirstLevelAnalysis -preprocessingonly -- the preprocessing of a
// first-level fMRI analysis on libbroccoli_b200 through the BROCCOLI_LIB
// class: T1 to template, EPI to T1, motion correction, EPI mask and
// normalised smoothing.  Arguments, options and output names follow the
// reference's tool in its -preprocessingonly mode
// (code/Bash_Wrapper/FirstLevelAnalysis.cpp: usage :236-307, the fourth
// argument :339-362, outputs :3034-3311); the statistics, slice-timing
// correction and multiple runs are not part of this library.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "broccoli_lib.h"
#include "cli_common.h"

static void usage() {
  printf("Usage:\n\n");
  printf("FirstLevelAnalysis fMRI.nii T1.nii MNI_brain.nii -preprocessingonly [options]\n\n");
  printf("Options:\n\n");
  printf(" -device                    CUDA device to use (default 0)\n");
  printf(" -iterationslinear          Iterations of the linear registrations (default 10)\n");
  printf(" -iterationsnonlinear       Iterations of the nonlinear registration (default 10, 0: none)\n");
  printf(" -zcutt1                    mm to cut from the bottom of the T1 volume (default 0)\n");
  printf(" -sigma                     Gaussian smoothing (voxels) regularising the displacement field (default 5.0)\n");
  printf(" -noslicetimingcorrection   Do not apply slice timing correction (it is never applied here)\n");
  printf(" -nomotioncorrection        Do not apply motion correction\n");
  printf(" -nosmoothing               Do not apply any smoothing\n");
  printf(" -iterationsmc              Iterations of motion correction (default 5)\n");
  printf(" -smoothing                 Smoothing of the fMRI data, FWHM in mm (default 6.0)\n");
  printf(" -savetransformations       Save the affine matrices (T1-MNI, EPI-T1, EPI-MNI)\n");
  printf(" -savet1interpolated, -savet1alignedlinear, -savet1alignednonlinear, -saveepialignedt1,\n");
  printf(" -saveepialignedmni, -saveepimask, -savemotioncorrected, -savemotionparameters, -savesmoothed,\n");
  printf(" -saveallaligned, -saveallpreprocessed, -saveall\n");
  printf(" -output                    Base name of the outputs\n");
  printf(" -filters                   Directory of the filter files (default $BROCCOLI_DIR/filters)\n");
  printf(" -precision                 fp32 (default), bf16x3 or tf32 (tensor-core filtering)\n");
  printf(" -quiet                     Print nothing\n");
  printf(" -verbose                   Print extra information\n\n");
}

namespace {

bool write_matrix(const std::string& path, const float* p, bool quiet) {
  std::ofstream m(path.c_str());
  if (!m.good()) {
    fprintf(stderr, "Could not open %s for writing\n", path.c_str());
    return false;
  }
  m.precision(6);
  m << p[3] + 1.0f << std::setw(2) << " " << p[4] << std::setw(2) << " " << p[5] << std::setw(2) << " " << p[0]
    << std::endl;
  m << p[6] << std::setw(2) << " " << p[7] + 1.0f << std::setw(2) << " " << p[8] << std::setw(2) << " " << p[1]
    << std::endl;
  m << p[9] << std::setw(2) << " " << p[10] << std::setw(2) << " " << p[11] + 1.0f << std::setw(2) << " " << p[2]
    << std::endl;
  m << 0.0f << std::setw(2) << " " << 0.0f << std::setw(2) << " " << 0.0f << std::setw(2) << " " << 1.0f
    << std::endl;
  if (!quiet) printf("Wrote %s\n", path.c_str());
  return true;
}

// name of an output: the input's name plus `plain`, or the -output base
// plus `renamed` (the reference's two naming schemes)
std::string out_name(const char* input, const char* base, const char* plain, const char* renamed,
                     const char* ext = nullptr) {
  return base ? cli::with_suffix(base, renamed, ext) : cli::with_suffix(input, plain, ext);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    usage();
    return EXIT_SUCCESS;
  }
  if (argc < 5 || strcmp(argv[4], "-preprocessingonly") != 0) {
    fprintf(stderr, "Only -preprocessingonly is supported: the statistical analysis is not part of this library\n");
    return EXIT_FAILURE;
  }
  int device = 0, it_lin = 10, it_nonlin = 10, it_mc = 5, zcut = 0, precision = BRC_PREC_FP32;
  float sigma = 5.0f, fwhm = 6.0f;
  bool mc = true, smoothing = true, quiet = false, verbose = false;
  bool s_mat = false, s_interp = false, s_t1lin = false, s_t1nonlin = false, s_epit1 = false, s_epimni = false,
       s_mask = false, s_mc = false, s_motion = false, s_smoothed = false;
  const char* out_base = nullptr;
  const char* filters_opt = nullptr;
  for (int i = 5; i < argc; i++) {
    const std::string o = argv[i];
    if (o == "-quiet") quiet = true;
    else if (o == "-verbose") verbose = true;
    else if (o == "-noslicetimingcorrection") {
    } else if (o == "-nomotioncorrection") mc = false;
    else if (o == "-nosmoothing") smoothing = false;
    else if (o == "-savetransformations") s_mat = true;
    else if (o == "-savet1interpolated") s_interp = true;
    else if (o == "-savet1alignedlinear") s_t1lin = true;
    else if (o == "-savet1alignednonlinear") s_t1nonlin = true;
    else if (o == "-saveepialignedt1") s_epit1 = true;
    else if (o == "-saveepialignedmni") s_epimni = true;
    else if (o == "-saveepimask") s_mask = true;
    else if (o == "-savemotioncorrected") s_mc = true;
    else if (o == "-savemotionparameters") s_motion = true;
    else if (o == "-savesmoothed") s_smoothed = true;
    else if (o == "-saveallaligned") s_interp = s_t1lin = s_t1nonlin = s_epit1 = s_epimni = true;
    else if (o == "-saveallpreprocessed") s_mc = s_smoothed = true;
    else if (o == "-saveall")
      s_mat = s_interp = s_t1lin = s_t1nonlin = s_epit1 = s_epimni = s_mask = s_mc = s_motion = s_smoothed = true;
    else if (o == "-device" || o == "-iterationslinear" || o == "-iterationsnonlinear" || o == "-zcutt1" ||
             o == "-sigma" || o == "-iterationsmc" || o == "-smoothing" || o == "-output" || o == "-filters" ||
             o == "-precision") {
      if (!cli::has_value(i, argc, argv)) return EXIT_FAILURE;
      const char* v = argv[++i];
      if (o == "-device") device = atoi(v);
      if (o == "-iterationslinear") it_lin = atoi(v);
      if (o == "-iterationsnonlinear") it_nonlin = atoi(v);
      if (o == "-zcutt1") zcut = atoi(v);
      if (o == "-sigma") sigma = (float)atof(v);
      if (o == "-iterationsmc") it_mc = atoi(v);
      if (o == "-smoothing") fwhm = (float)atof(v);
      if (o == "-output") out_base = v;
      if (o == "-filters") filters_opt = v;
      if (o == "-precision") {
        if (strcmp(v, "fp32") == 0) {
          precision = BRC_PREC_FP32;
        } else if (strcmp(v, "bf16x3") == 0) {
          precision = BRC_PREC_BF16X3;
        } else if (strcmp(v, "tf32") == 0) {
          precision = BRC_PREC_TF32;
        } else {
          fprintf(stderr, "Unknown precision %s\n", v);
          return EXIT_FAILURE;
        }
      }
    } else {
      fprintf(stderr, "Option %s is not supported (only the preprocessing is part of this library)\n", argv[i]);
      return EXIT_FAILURE;
    }
  }
  if (it_lin <= 0 || it_nonlin < 0 || it_mc <= 0 || !(sigma > 0.f) || !(fwhm > 0.f)) {
    fprintf(stderr, "Iterations, sigma and smoothing must be positive\n");
    return EXIT_FAILURE;
  }
  brc_nifti fmri, t1, mni;
  if (!cli::read_nifti(argv[1], &fmri) || !cli::read_nifti(argv[2], &t1) || !cli::read_nifti(argv[3], &mni))
    return EXIT_FAILURE;
  const int W = fmri.dim[1], H = fmri.dim[2], D = fmri.dim[3], T = fmri.dim[0] >= 4 ? fmri.dim[4] : 1;
  const int W3 = mni.dim[1], H3 = mni.dim[2], D3 = mni.dim[3];
  const size_t V = (size_t)W * H * D, V3 = (size_t)W3 * H3 * D3;
  const std::string dir = cli::filter_dir(filters_opt);
  if (dir.empty()) {
    fprintf(stderr, "Give -filters DIR or set BROCCOLI_DIR\n");
    return EXIT_FAILURE;
  }
  std::vector<std::vector<float>> fl, fn;
  std::vector<float> tens[6], dirs[3];
  if (!cli::read_filters(dir, "linear", 3, fl) || !cli::read_filters(dir, "nonlinear", 6, fn)) return EXIT_FAILURE;
  for (int k = 0; k < 6; k++)
    if (!cli::read_floats(dir + "projection_tensor" + std::to_string(k + 1) + ".bin", 6, tens[k]))
      return EXIT_FAILURE;
  const char* axes[3] = {"x", "y", "z"};
  for (int a = 0; a < 3; a++)
    if (!cli::read_floats(dir + "filter_directions_" + axes[a] + ".bin", 6, dirs[a])) return EXIT_FAILURE;
  if (!quiet)
    printf("fMRI %d x %d x %d x %d, T1 %d x %d x %d, template %d x %d x %d\n", W, H, D, T, t1.dim[1], t1.dim[2],
           t1.dim[3], W3, H3, D3);

  BROCCOLI_LIB b(0, (cl_uint)device, BASH, verbose);
  if (!b.GetOpenCLInitiated()) {
    fprintf(stderr, "Initialisation failed: %s\n", b.GetOpenCLInitializationError().c_str());
    return EXIT_FAILURE;
  }
  b.SetEPIWidth(W);
  b.SetEPIHeight(H);
  b.SetEPIDepth(D);
  b.SetEPITimepoints(T);
  b.SetEPIVoxelSizeX(fmri.pixdim[1]);
  b.SetEPIVoxelSizeY(fmri.pixdim[2]);
  b.SetEPIVoxelSizeZ(fmri.pixdim[3]);
  b.SetT1Width(t1.dim[1]);
  b.SetT1Height(t1.dim[2]);
  b.SetT1Depth(t1.dim[3]);
  b.SetT1VoxelSizeX(t1.pixdim[1]);
  b.SetT1VoxelSizeY(t1.pixdim[2]);
  b.SetT1VoxelSizeZ(t1.pixdim[3]);
  b.SetMNIWidth(W3);
  b.SetMNIHeight(H3);
  b.SetMNIDepth(D3);
  b.SetMNIVoxelSizeX(mni.pixdim[1]);
  b.SetMNIVoxelSizeY(mni.pixdim[2]);
  b.SetMNIVoxelSizeZ(mni.pixdim[3]);
  b.SetInputfMRIVolumes(fmri.data);
  b.SetInputT1Volume(t1.data);
  b.SetInputMNIBrainVolume(mni.data);
  b.SetImageRegistrationFilterSize(7);
  b.SetLinearImageRegistrationFilters(fl[0].data(), fl[1].data(), fl[2].data(), fl[3].data(), fl[4].data(),
                                      fl[5].data());
  b.SetNonLinearImageRegistrationFilters(fn[0].data(), fn[1].data(), fn[2].data(), fn[3].data(), fn[4].data(),
                                         fn[5].data(), fn[6].data(), fn[7].data(), fn[8].data(), fn[9].data(),
                                         fn[10].data(), fn[11].data());
  void (BROCCOLI_LIB::*set_tensor[6])(float, float, float, float, float, float) = {
      &BROCCOLI_LIB::SetProjectionTensorMatrixFirstFilter,  &BROCCOLI_LIB::SetProjectionTensorMatrixSecondFilter,
      &BROCCOLI_LIB::SetProjectionTensorMatrixThirdFilter,  &BROCCOLI_LIB::SetProjectionTensorMatrixFourthFilter,
      &BROCCOLI_LIB::SetProjectionTensorMatrixFifthFilter,  &BROCCOLI_LIB::SetProjectionTensorMatrixSixthFilter};
  for (int k = 0; k < 6; k++) (b.*set_tensor[k])(tens[k][0], tens[k][1], tens[k][2], tens[k][3], tens[k][4], tens[k][5]);
  b.SetFilterDirections(dirs[0].data(), dirs[1].data(), dirs[2].data());
  b.SetNumberOfIterationsForLinearImageRegistration(it_lin);
  b.SetNumberOfIterationsForNonLinearImageRegistration(it_nonlin);
  b.SetNumberOfIterationsForMotionCorrection(it_mc);
  // the coarsest scale that keeps at least 16 template voxels along every
  // axis (FirstLevelAnalysis.cpp:1668-1693)
  int coarsest = 1;
  for (int s = 16; s >= 2; s /= 2)
    if (W3 / s >= 16 && H3 / s >= 16 && D3 / s >= 16) {
      coarsest = s;
      break;
    }
  b.SetCoarsestScaleT1MNI(coarsest);
  b.SetCoarsestScaleEPIT1(coarsest);
  b.SetMMT1ZCUT(zcut);
  b.SetTsigma(sigma);
  b.SetEsigma(sigma);
  b.SetDsigma(sigma);
  b.SetEPISmoothingAmount(fwhm);
  b.SetApplyMotionCorrection(mc);
  b.SetApplySmoothing(smoothing);
  b.SetApplySliceTimingCorrection(false);
  b.SetPrecision(precision);
  b.SetPreprocessingOnly(true);
  std::vector<float> p_t1(12), p_epit1(12), p_epimni(12), motion(6 * (size_t)T), interp(V3), t1lin(V3),
      t1nonlin(V3), epit1(V3), epimni(V3), epimni_nl(V3), mcv(V * T), mask(V), sm(V * T);
  b.SetOutputT1MNIRegistrationParameters(p_t1.data());
  b.SetOutputEPIT1RegistrationParameters(p_epit1.data());
  b.SetOutputEPIMNIRegistrationParameters(p_epimni.data());
  b.SetOutputMotionParameters(motion.data());
  b.SetOutputInterpolatedT1Volume(interp.data());
  b.SetOutputAlignedT1VolumeLinear(t1lin.data());
  b.SetOutputAlignedT1VolumeNonLinear(t1nonlin.data());
  b.SetOutputAlignedEPIVolumeT1(epit1.data());
  b.SetOutputAlignedEPIVolumeMNILinear(epimni.data());
  b.SetOutputAlignedEPIVolumeMNINonlinear(epimni_nl.data());
  b.SetOutputMotionCorrectedfMRIVolumes(mcv.data());
  b.SetOutputEPIMask(mask.data());
  b.SetOutputSmoothedfMRIVolumes(sm.data());
  b.SetSaveInterpolatedT1(s_interp);
  b.SetSaveAlignedT1MNILinear(s_t1lin);
  b.SetSaveAlignedT1MNINonLinear(s_t1nonlin);
  b.SetSaveAlignedEPIT1(s_epit1);
  b.SetSaveAlignedEPIMNI(s_epimni);
  b.SetSaveEPIMask(s_mask);
  b.SetSaveMotionCorrected(s_mc && mc);
  b.SetSaveSmoothed(s_smoothed && smoothing);
  b.PerformFirstLevelAnalysisWrapper();
  if (b.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "Preprocessing failed: %s\n", b.GetOpenCLError());
    return EXIT_FAILURE;
  }

  const char* f = argv[1];
  const char* t = argv[2];
  const char* o = out_base;
  bool ok = true;
  if (s_mat) {
    ok = write_matrix(out_name(t, o, "_affinematrix_t1_mni", "_affinematrix_t1_mni", ".txt"), p_t1.data(), quiet) && ok;
    ok = write_matrix(out_name(f, o, "_affinematrix_epi_t1", "_affinematrix_epi_t1", ".txt"), p_epit1.data(), quiet) && ok;
    ok = write_matrix(out_name(f, o, "_affinematrix_epi_mni", "_affinematrix_epi_mni", ".txt"), p_epimni.data(), quiet) && ok;
  }
  if (s_motion && mc) {
    const std::string path = out_name(f, o, "_motionparameters", "_motionparameters", ".1D");
    std::ofstream m(path.c_str());
    m.precision(6);
    for (int i = 0; i < T; i++) {
      const float* p = motion.data();
      m << p[i + 4 * T] << std::setw(2) << " " << -p[i + 3 * T] << std::setw(2) << " " << p[i + 5 * T] << std::setw(2)
        << " " << -p[i + 2 * T] << std::setw(2) << " " << -p[i + 0 * T] << std::setw(2) << " " << -p[i + 1 * T]
        << std::endl;
    }
    ok = m.good() && ok;
    if (!quiet) printf("Wrote %s\n", path.c_str());
  }
  // template-space volumes under the template's header
  if (s_interp) ok = cli::write_nifti(out_name(t, o, "_interpolated", "_t1_interpolated"), &mni, interp.data(), W3, H3, D3, 1, quiet) && ok;
  if (s_t1lin) ok = cli::write_nifti(out_name(t, o, "_aligned_mni_linear", "_t1_aligned_mni_linear"), &mni, t1lin.data(), W3, H3, D3, 1, quiet) && ok;
  if (s_t1nonlin && it_nonlin > 0)
    ok = cli::write_nifti(out_name(t, o, "_aligned_mni_nonlinear", "_t1_aligned_mni_nonlinear"), &mni, t1nonlin.data(), W3, H3, D3, 1, quiet) && ok;
  if (s_epit1) ok = cli::write_nifti(out_name(f, o, "_aligned_t1", "_epi_aligned_t1"), &mni, epit1.data(), W3, H3, D3, 1, quiet) && ok;
  if (s_epimni) {
    ok = cli::write_nifti(out_name(f, o, "_aligned_mni_linear", "_epi_aligned_mni_linear"), &mni, epimni.data(), W3, H3, D3, 1, quiet) && ok;
    if (it_nonlin > 0)
      ok = cli::write_nifti(out_name(f, o, "_aligned_mni_nonlinear", "_epi_aligned_mni_nonlinear"), &mni, epimni_nl.data(), W3, H3, D3, 1, quiet) && ok;
  }
  // fMRI-space volumes under the fMRI header
  if (s_mc && mc) ok = cli::write_nifti(out_name(f, o, "_motion_corrected", "_motion_corrected"), &fmri, mcv.data(), W, H, D, T, quiet) && ok;
  if (s_smoothed && smoothing) ok = cli::write_nifti(out_name(f, o, "_smoothed", "_smoothed"), &fmri, sm.data(), W, H, D, T, quiet) && ok;
  if (s_mask) ok = cli::write_nifti(out_name(f, o, "_mask", "_epi_mask"), &fmri, mask.data(), W, H, D, 1, quiet) && ok;
  brc_nifti_free(&fmri);
  brc_nifti_free(&t1);
  brc_nifti_free(&mni);
  return ok ? EXIT_SUCCESS : EXIT_FAILURE;
}
