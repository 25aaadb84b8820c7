// Drives the BROCCOLI_LIB members beyond the registration results the way
// the reference's tools use them: SetDebug with SetOutputQuadratureFilter-
// Responses (three or six arrays) and SetOutputPhaseDifferences /
// Certainties / Gradients (Bash_Wrapper/RegisterTwoVolumes.cpp:1145-1160),
// SetPrecenterRegistration, SetDoSkullstrip / SetDoSkullstripOriginal with
// SetInputMNIBrainMask and SetOutputSkullstrippedT1Volume (:1088-1136), and
// the GetOpenCLCreateKernelErrors / CreateBufferErrors getters.
//
//   broccoli_lib_boundary mc  <series.f32> W H D T <filters3.f32> iters <outdir>
//       motion correction with debug outputs: q1..q3.c64, pd/pc/pg.f32
//   broccoli_lib_boundary r2v <subject.f32> W H D vx vy vz <template.f32> W2 H2 D2
//       <filters3.f32> <filters6.f32> <tensors.f32> <dirs.f32> lin nonlin coarsest zcut
//       precenter(0/1) strip(0 none, 1 mask, 2 mask original, 3 mask requested but not given)
//       <mask.f32 or -> debug(0/3/6) <outdir>
//       T1-to-template: params, interpolated, aligned_linear, aligned_nonlinear,
//       field, skull (when strip), q1..qN.c64 (when debug)
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "broccoli_lib.h"

static std::vector<float> read_floats(const char* path, size_t n) {
  std::vector<float> v(n);
  FILE* f = fopen(path, "rb");
  if (!f || fread(v.data(), sizeof(float), n, f) != n) {
    fprintf(stderr, "cannot read %zu floats from %s\n", n, path);
    exit(2);
  }
  fclose(f);
  return v;
}

static void write_floats(const std::string& path, const void* p, size_t n) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f || fwrite(p, sizeof(float), n, f) != n) {
    fprintf(stderr, "cannot write %s\n", path.c_str());
    exit(2);
  }
  fclose(f);
}

static bool errors_clear(BROCCOLI_LIB& b) {
  const int* k = b.GetOpenCLCreateKernelErrors();
  const int* m = b.GetOpenCLCreateBufferErrors();
  for (int i = 0; i < 200; i++)
    if (k[i] != 0 || m[i] != 0) return false;
  return true;
}

static int run_mc(int argc, char** argv) {
  if (argc != 10) return 2;
  const int W = atoi(argv[3]), H = atoi(argv[4]), D = atoi(argv[5]), T = atoi(argv[6]);
  const size_t V = (size_t)W * H * D;
  std::vector<float> series = read_floats(argv[2], V * T);
  std::vector<float> f = read_floats(argv[7], 3 * 686);
  const std::string dir = argv[9];
  BROCCOLI_LIB b(0, 0, BASH, false);
  if (!b.GetOpenCLInitiated()) return 1;
  b.SetEPIWidth(W);
  b.SetEPIHeight(H);
  b.SetEPIDepth(D);
  b.SetEPITimepoints(T);
  b.SetInputfMRIVolumes(series.data());
  b.SetImageRegistrationFilterSize(7);
  float* p = f.data();
  b.SetLinearImageRegistrationFilters(p, p + 343, p + 686, p + 1029, p + 1372, p + 1715);
  b.SetNumberOfIterationsForMotionCorrection(atoi(argv[8]));
  std::vector<float> motion(6 * (size_t)T), pd(V), pc(V), pg(V);
  std::vector<cl_float2> q[3];
  for (int k = 0; k < 3; k++) q[k].resize(V);
  b.SetOutputMotionParameters(motion.data());
  b.SetDebug(true);
  b.SetOutputQuadratureFilterResponses(q[0].data(), q[1].data(), q[2].data());
  b.SetOutputPhaseDifferences(pd.data());
  b.SetOutputPhaseCertainties(pc.data());
  b.SetOutputPhaseGradients(pg.data());
  b.PerformMotionCorrectionWrapper();
  if (b.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "motion correction failed: %s\n", b.GetOpenCLError());
    return 1;
  }
  if (!errors_clear(b)) return 3;
  for (int k = 0; k < 3; k++) write_floats(dir + "/q" + std::to_string(k + 1) + ".c64", q[k].data(), 2 * V);
  write_floats(dir + "/pd.f32", pd.data(), V);
  write_floats(dir + "/pc.f32", pc.data(), V);
  write_floats(dir + "/pg.f32", pg.data(), V);
  return 0;
}

static int run_r2v(int argc, char** argv) {
  if (argc != 26) return 2;
  const int W = atoi(argv[3]), H = atoi(argv[4]), D = atoi(argv[5]);
  const float vox[3] = {(float)atof(argv[6]), (float)atof(argv[7]), (float)atof(argv[8])};
  const int W2 = atoi(argv[10]), H2 = atoi(argv[11]), D2 = atoi(argv[12]);
  const size_t V1 = (size_t)W * H * D, V2 = (size_t)W2 * H2 * D2;
  std::vector<float> sub = read_floats(argv[2], V1), tpl = read_floats(argv[9], V2);
  std::vector<float> f3 = read_floats(argv[13], 3 * 686), f6 = read_floats(argv[14], 6 * 686);
  std::vector<float> tens = read_floats(argv[15], 36), dirs = read_floats(argv[16], 18);
  const int lin = atoi(argv[17]), nonlin = atoi(argv[18]), coarsest = atoi(argv[19]), zcut = atoi(argv[20]);
  const bool precenter = atoi(argv[21]) != 0;
  const int strip = atoi(argv[22]);
  const int debug = atoi(argv[24]);
  const std::string dir = argv[25];
  std::vector<float> mask = (strip == 1 || strip == 2) ? read_floats(argv[23], V2) : std::vector<float>();

  BROCCOLI_LIB b(0, 0, BASH, false);
  if (!b.GetOpenCLInitiated()) return 1;
  b.SetT1Width(W);
  b.SetT1Height(H);
  b.SetT1Depth(D);
  b.SetT1Timepoints(1);
  b.SetT1VoxelSizeX(vox[0]);
  b.SetT1VoxelSizeY(vox[1]);
  b.SetT1VoxelSizeZ(vox[2]);
  b.SetMNIWidth(W2);
  b.SetMNIHeight(H2);
  b.SetMNIDepth(D2);
  b.SetMNIVoxelSizeX(1.f);
  b.SetMNIVoxelSizeY(1.f);
  b.SetMNIVoxelSizeZ(1.f);
  b.SetInputT1Volume(sub.data());
  b.SetInputMNIBrainVolume(tpl.data());
  b.SetInterpolationMode(LINEAR);
  b.SetImageRegistrationFilterSize(7);
  float* p = f3.data();
  b.SetLinearImageRegistrationFilters(p, p + 343, p + 686, p + 1029, p + 1372, p + 1715);
  float* n = f6.data();
  b.SetNonLinearImageRegistrationFilters(n, n + 343, n + 686, n + 1029, n + 1372, n + 1715, n + 2058, n + 2401,
                                         n + 2744, n + 3087, n + 3430, n + 3773);
  const float* t = tens.data();
  b.SetProjectionTensorMatrixFirstFilter(t[0], t[1], t[2], t[3], t[4], t[5]);
  b.SetProjectionTensorMatrixSecondFilter(t[6], t[7], t[8], t[9], t[10], t[11]);
  b.SetProjectionTensorMatrixThirdFilter(t[12], t[13], t[14], t[15], t[16], t[17]);
  b.SetProjectionTensorMatrixFourthFilter(t[18], t[19], t[20], t[21], t[22], t[23]);
  b.SetProjectionTensorMatrixFifthFilter(t[24], t[25], t[26], t[27], t[28], t[29]);
  b.SetProjectionTensorMatrixSixthFilter(t[30], t[31], t[32], t[33], t[34], t[35]);
  b.SetFilterDirections(dirs.data(), dirs.data() + 6, dirs.data() + 12);
  b.SetNumberOfIterationsForLinearImageRegistration(lin);
  b.SetNumberOfIterationsForNonLinearImageRegistration(nonlin);
  b.SetCoarsestScaleT1MNI(coarsest);
  b.SetMMT1ZCUT(zcut);
  b.SetPrecenterRegistration(precenter);
  std::vector<float> params(12), interp(V2), al(V2), anl(V2), fx(V2), fy(V2), fz(V2), skull(V2);
  b.SetOutputT1MNIRegistrationParameters(params.data());
  b.SetOutputInterpolatedT1Volume(interp.data());
  b.SetOutputAlignedT1VolumeLinear(al.data());
  b.SetOutputAlignedT1VolumeNonLinear(anl.data());
  b.SetOutputDisplacementField(fx.data(), fy.data(), fz.data());
  if (strip) {
    if (strip != 3) b.SetInputMNIBrainMask(mask.data());
    b.SetOutputSkullstrippedT1Volume(skull.data());
    b.SetDoSkullstrip(strip == 1 || strip == 3);
    b.SetDoSkullstripOriginal(strip == 2);
  }
  std::vector<cl_float2> q[6];
  if (debug) {
    for (int k = 0; k < debug; k++) q[k].resize(V2);
    b.SetDebug(true);
    if (debug == 3)
      b.SetOutputQuadratureFilterResponses(q[0].data(), q[1].data(), q[2].data());
    else
      b.SetOutputQuadratureFilterResponses(q[0].data(), q[1].data(), q[2].data(), q[3].data(), q[4].data(),
                                           q[5].data());
  }
  b.PerformRegistrationTwoVolumesWrapper();
  if (b.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "registration failed: %s\n", b.GetOpenCLError());
    return 1;
  }
  if (!errors_clear(b)) return 3;
  write_floats(dir + "/params.f32", params.data(), 12);
  write_floats(dir + "/interpolated.f32", interp.data(), V2);
  write_floats(dir + "/aligned_linear.f32", al.data(), V2);
  write_floats(dir + "/aligned_nonlinear.f32", anl.data(), V2);
  std::vector<float> field(3 * V2);
  memcpy(field.data(), fx.data(), sizeof(float) * V2);
  memcpy(field.data() + V2, fy.data(), sizeof(float) * V2);
  memcpy(field.data() + 2 * V2, fz.data(), sizeof(float) * V2);
  write_floats(dir + "/field.f32", field.data(), 3 * V2);
  if (strip) write_floats(dir + "/skull.f32", skull.data(), V2);
  for (int k = 0; k < debug; k++) write_floats(dir + "/q" + std::to_string(k + 1) + ".c64", q[k].data(), 2 * V2);
  return 0;
}

int main(int argc, char** argv) {
  int r = 2;
  if (argc > 1 && strcmp(argv[1], "mc") == 0) r = run_mc(argc, argv);
  if (argc > 1 && strcmp(argv[1], "r2v") == 0) r = run_r2v(argc, argv);
  if (r == 2) fprintf(stderr, "usage: %s mc|r2v ...\n", argv[0]);
  if (r == 0) printf("ok\n");
  return r;
}
