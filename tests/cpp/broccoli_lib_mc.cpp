// Drives the drop-in BROCCOLI_LIB class the way the reference's
// MotionCorrection CLI does (Bash_Wrapper/MotionCorrection.cpp:584-692):
// construct, set sizes / voxel sizes / filters / iterations / outputs, call
// PerformMotionCorrectionWrapper.  Test program: reads a raw float32 series
// and the 3 linear filters from files, writes the corrected series and the
// 6 x T motion parameters.
//   broccoli_lib_mc <series.f32> W H D T vx vy vz <filters.f32> iters <out_series.f32> <out_motion.f32>
#include <stdio.h>
#include <stdlib.h>

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

static void write_floats(const char* path, const float* p, size_t n) {
  FILE* f = fopen(path, "wb");
  if (!f || fwrite(p, sizeof(float), n, f) != n) {
    fprintf(stderr, "cannot write %s\n", path);
    exit(2);
  }
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc != 13) {
    fprintf(stderr, "usage: %s series W H D T vx vy vz filters iters out_series out_motion\n", argv[0]);
    return 2;
  }
  const int W = atoi(argv[2]), H = atoi(argv[3]), D = atoi(argv[4]), T = atoi(argv[5]);
  const size_t n = (size_t)W * H * D * T;
  std::vector<float> series = read_floats(argv[1], n);
  std::vector<float> filters = read_floats(argv[9], 3 * 686);
  std::vector<float> motion(6 * (size_t)T);

  BROCCOLI_LIB broccoli(0, 0, BASH, false);
  if (!broccoli.GetOpenCLInitiated()) {
    fprintf(stderr, "initialisation failed: %s\n", broccoli.GetOpenCLInitializationError().c_str());
    return 1;
  }
  broccoli.SetEPIWidth(W);
  broccoli.SetEPIHeight(H);
  broccoli.SetEPIDepth(D);
  broccoli.SetEPITimepoints(T);
  broccoli.SetEPIVoxelSizeX((float)atof(argv[6]));
  broccoli.SetEPIVoxelSizeY((float)atof(argv[7]));
  broccoli.SetEPIVoxelSizeZ((float)atof(argv[8]));
  broccoli.SetInputfMRIVolumes(series.data());
  broccoli.SetImageRegistrationFilterSize(7);
  float* f = filters.data();
  broccoli.SetLinearImageRegistrationFilters(f, f + 343, f + 686, f + 686 + 343, f + 1372, f + 1372 + 343);
  broccoli.SetNumberOfIterationsForMotionCorrection(atoi(argv[10]));
  broccoli.SetOutputMotionParameters(motion.data());
  broccoli.PerformMotionCorrectionWrapper();
  if (broccoli.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "motion correction failed: %s\n", broccoli.GetOpenCLError());
    return 1;
  }
  write_floats(argv[11], series.data(), n);
  write_floats(argv[12], motion.data(), motion.size());
  printf("ok\n");
  return 0;
}
