// Drives the drop-in BROCCOLI_LIB class through the preprocessing of a
// first-level analysis the way the reference's FirstLevelAnalysis CLI sets
// it up (Bash_Wrapper/FirstLevelAnalysis.cpp:2840-2900: data, sizes, filters,
// iterations, scales, smoothing, outputs), with SetPreprocessingOnly(true)
// and every SetSave* flag on.  Test program: reads raw float32 inputs from a
// directory and writes the outputs there.
//   broccoli_lib_first_level <dir> epiW epiH epiD T t1W t1H t1D mniW mniH mniD
//       evx evy evz tvx tvy tvz mvx mvy mvz lin nonlin mc coarsestT1 coarsestEPI fwhm
// inputs:  fmri.f32 t1.f32 mni.f32 filters3.f32 (3 x 686) filters6.f32 (6 x 686)
//          tensors.f32 (36) dirs.f32 (18)
// outputs: params_t1_mni.f32 params_epi_t1.f32 params_epi_mni.f32 motion.f32
//          interpolated_t1.f32 aligned_t1_linear.f32 aligned_t1_nonlinear.f32
//          aligned_epi_t1.f32 aligned_epi_mni_linear.f32 aligned_epi_mni_nonlinear.f32
//          motion_corrected.f32 epi_mask.f32 smoothed.f32 fmri.f32
#include <stdio.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "broccoli_lib.h"

static std::string dir;

static std::vector<float> read_floats(const char* name, size_t n) {
  std::vector<float> v(n);
  const std::string path = dir + "/" + name;
  FILE* f = fopen(path.c_str(), "rb");
  if (!f || fread(v.data(), sizeof(float), n, f) != n) {
    fprintf(stderr, "cannot read %zu floats from %s\n", n, path.c_str());
    exit(2);
  }
  fclose(f);
  return v;
}

static void write_floats(const char* name, const std::vector<float>& v) {
  const std::string path = dir + "/" + name;
  FILE* f = fopen(path.c_str(), "wb");
  if (!f || fwrite(v.data(), sizeof(float), v.size(), f) != v.size()) {
    fprintf(stderr, "cannot write %s\n", path.c_str());
    exit(2);
  }
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc != 27) {
    fprintf(stderr, "usage: %s dir epiW epiH epiD T t1W t1H t1D mniW mniH mniD evx evy evz tvx tvy tvz "
                    "mvx mvy mvz lin nonlin mc coarsestT1 coarsestEPI fwhm\n", argv[0]);
    return 2;
  }
  dir = argv[1];
  int a[10];
  for (int i = 0; i < 10; i++) a[i] = atoi(argv[2 + i]);
  float v[9];
  for (int i = 0; i < 9; i++) v[i] = (float)atof(argv[12 + i]);
  const int W = a[0], H = a[1], D = a[2], T = a[3];
  const size_t V1 = (size_t)W * H * D, V2 = (size_t)a[4] * a[5] * a[6], V3 = (size_t)a[7] * a[8] * a[9];
  std::vector<float> fmri = read_floats("fmri.f32", V1 * T), t1 = read_floats("t1.f32", V2),
                     mni = read_floats("mni.f32", V3), f3 = read_floats("filters3.f32", 3 * 686),
                     f6 = read_floats("filters6.f32", 6 * 686), m = read_floats("tensors.f32", 36),
                     dirs = read_floats("dirs.f32", 18);

  BROCCOLI_LIB broccoli(0, 0, BASH, false);
  if (!broccoli.GetOpenCLInitiated()) {
    fprintf(stderr, "initialisation failed: %s\n", broccoli.GetOpenCLInitializationError().c_str());
    return 1;
  }
  broccoli.SetEPIWidth(W);
  broccoli.SetEPIHeight(H);
  broccoli.SetEPIDepth(D);
  broccoli.SetEPITimepoints(T);
  broccoli.SetEPIVoxelSizeX(v[0]);
  broccoli.SetEPIVoxelSizeY(v[1]);
  broccoli.SetEPIVoxelSizeZ(v[2]);
  broccoli.SetT1Width(a[4]);
  broccoli.SetT1Height(a[5]);
  broccoli.SetT1Depth(a[6]);
  broccoli.SetT1VoxelSizeX(v[3]);
  broccoli.SetT1VoxelSizeY(v[4]);
  broccoli.SetT1VoxelSizeZ(v[5]);
  broccoli.SetMNIWidth(a[7]);
  broccoli.SetMNIHeight(a[8]);
  broccoli.SetMNIDepth(a[9]);
  broccoli.SetMNIVoxelSizeX(v[6]);
  broccoli.SetMNIVoxelSizeY(v[7]);
  broccoli.SetMNIVoxelSizeZ(v[8]);
  broccoli.SetInputfMRIVolumes(fmri.data());
  broccoli.SetInputT1Volume(t1.data());
  broccoli.SetInputMNIBrainVolume(mni.data());
  broccoli.SetImageRegistrationFilterSize(7);
  broccoli.SetLinearImageRegistrationFilters(&f3[0], &f3[343], &f3[686], &f3[686 + 343], &f3[2 * 686],
                                             &f3[2 * 686 + 343]);
  float* n = f6.data();
  broccoli.SetNonLinearImageRegistrationFilters(n, n + 343, n + 686, n + 686 + 343, n + 2 * 686,
                                                n + 2 * 686 + 343, n + 3 * 686, n + 3 * 686 + 343, n + 4 * 686,
                                                n + 4 * 686 + 343, n + 5 * 686, n + 5 * 686 + 343);
  const float* t = m.data();
  broccoli.SetProjectionTensorMatrixFirstFilter(t[0], t[1], t[2], t[3], t[4], t[5]);
  broccoli.SetProjectionTensorMatrixSecondFilter(t[6], t[7], t[8], t[9], t[10], t[11]);
  broccoli.SetProjectionTensorMatrixThirdFilter(t[12], t[13], t[14], t[15], t[16], t[17]);
  broccoli.SetProjectionTensorMatrixFourthFilter(t[18], t[19], t[20], t[21], t[22], t[23]);
  broccoli.SetProjectionTensorMatrixFifthFilter(t[24], t[25], t[26], t[27], t[28], t[29]);
  broccoli.SetProjectionTensorMatrixSixthFilter(t[30], t[31], t[32], t[33], t[34], t[35]);
  broccoli.SetFilterDirections(&dirs[0], &dirs[6], &dirs[12]);
  broccoli.SetNumberOfIterationsForLinearImageRegistration(atoi(argv[21]));
  broccoli.SetNumberOfIterationsForNonLinearImageRegistration(atoi(argv[22]));
  broccoli.SetNumberOfIterationsForMotionCorrection(atoi(argv[23]));
  broccoli.SetCoarsestScaleT1MNI(atoi(argv[24]));
  broccoli.SetCoarsestScaleEPIT1(atoi(argv[25]));
  broccoli.SetMMT1ZCUT(0);
  broccoli.SetEPISmoothingAmount((float)atof(argv[26]));
  broccoli.SetApplyMotionCorrection(true);
  broccoli.SetApplySmoothing(true);
  broccoli.SetApplySliceTimingCorrection(false);

  std::vector<float> p_t1(12), p_epi_t1(12), p_epi_mni(12), motion(6 * (size_t)T), interp(V3), t1_lin(V3),
      t1_nonlin(V3), epi_t1(V3), epi_mni_lin(V3), epi_mni_nonlin(V3), mc(V1 * T), mask(V1), smoothed(V1 * T);
  broccoli.SetOutputT1MNIRegistrationParameters(p_t1.data());
  broccoli.SetOutputEPIT1RegistrationParameters(p_epi_t1.data());
  broccoli.SetOutputEPIMNIRegistrationParameters(p_epi_mni.data());
  broccoli.SetOutputMotionParameters(motion.data());
  broccoli.SetOutputInterpolatedT1Volume(interp.data());
  broccoli.SetOutputAlignedT1VolumeLinear(t1_lin.data());
  broccoli.SetOutputAlignedT1VolumeNonLinear(t1_nonlin.data());
  broccoli.SetOutputAlignedEPIVolumeT1(epi_t1.data());
  broccoli.SetOutputAlignedEPIVolumeMNILinear(epi_mni_lin.data());
  broccoli.SetOutputAlignedEPIVolumeMNINonlinear(epi_mni_nonlin.data());
  broccoli.SetOutputMotionCorrectedfMRIVolumes(mc.data());
  broccoli.SetOutputEPIMask(mask.data());
  broccoli.SetOutputSmoothedfMRIVolumes(smoothed.data());
  broccoli.SetSaveInterpolatedT1(true);
  broccoli.SetSaveAlignedT1MNILinear(true);
  broccoli.SetSaveAlignedT1MNINonLinear(true);
  broccoli.SetSaveAlignedEPIT1(true);
  broccoli.SetSaveAlignedEPIMNI(true);
  broccoli.SetSaveMotionCorrected(true);
  broccoli.SetSaveEPIMask(true);
  broccoli.SetSaveSmoothed(true);

  broccoli.PerformFirstLevelAnalysisWrapper();  // not preprocessing-only: refused
  if (broccoli.GetLastStatus() != BRC_ERR_UNSUPPORTED) {
    fprintf(stderr, "the statistics were not refused\n");
    return 1;
  }
  broccoli.SetPreprocessingOnly(true);
  broccoli.PerformFirstLevelAnalysisWrapper();
  if (broccoli.GetLastStatus() != 0) {
    fprintf(stderr, "first-level preprocessing failed: %s\n", broccoli.GetOpenCLError());
    return 1;
  }
  write_floats("params_t1_mni.f32", p_t1);
  write_floats("params_epi_t1.f32", p_epi_t1);
  write_floats("params_epi_mni.f32", p_epi_mni);
  write_floats("motion.f32", motion);
  write_floats("interpolated_t1.f32", interp);
  write_floats("aligned_t1_linear.f32", t1_lin);
  write_floats("aligned_t1_nonlinear.f32", t1_nonlin);
  write_floats("aligned_epi_t1.f32", epi_t1);
  write_floats("aligned_epi_mni_linear.f32", epi_mni_lin);
  write_floats("aligned_epi_mni_nonlinear.f32", epi_mni_nonlin);
  write_floats("motion_corrected.f32", mc);
  write_floats("epi_mask.f32", mask);
  write_floats("smoothed.f32", smoothed);
  write_floats("fmri.f32", fmri);
  return 0;
}
