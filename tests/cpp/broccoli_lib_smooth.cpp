// Drives the drop-in BROCCOLI_LIB class the way the reference's Smoothing
// CLI does (Bash_Wrapper/Smoothing.cpp:593-613): volumes, certainty, FWHM,
// sizes and voxel sizes, then PerformSmoothingNormalizedHostWrapper, which
// smooths the volumes in place.  Test program: reads a raw float32 series
// and certainty volume, writes the smoothed series.
//   broccoli_lib_smooth <series.f32> <certainty.f32 | auto> W H D T vx vy vz fwhm_mm <out.f32>
#include <stdio.h>
#include <stdlib.h>

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

int main(int argc, char** argv) {
  if (argc != 12) {
    fprintf(stderr, "usage: %s series certainty W H D T vx vy vz fwhm_mm out\n", argv[0]);
    return 2;
  }
  const int W = atoi(argv[3]), H = atoi(argv[4]), D = atoi(argv[5]), T = atoi(argv[6]);
  const size_t V = (size_t)W * H * D;
  std::vector<float> series = read_floats(argv[1], V * T);
  // certainty "auto": SetAutoMask(true), the mask of the first volume is
  // made by the library and written to <out>.mask
  const bool automask = std::string(argv[2]) == "auto";
  std::vector<float> certainty = automask ? std::vector<float>(V, 0.f) : read_floats(argv[2], V);

  BROCCOLI_LIB broccoli(0, 0, BASH, false);
  if (!broccoli.GetOpenCLInitiated()) {
    fprintf(stderr, "initialisation failed: %s\n", broccoli.GetOpenCLInitializationError().c_str());
    return 1;
  }
  broccoli.SetInputfMRIVolumes(series.data());
  broccoli.SetAutoMask(automask);
  broccoli.SetInputCertainty(certainty.data());
  broccoli.SetEPISmoothingAmount((float)atof(argv[10]));
  broccoli.SetEPIWidth(W);
  broccoli.SetEPIHeight(H);
  broccoli.SetEPIDepth(D);
  broccoli.SetEPITimepoints(T);
  broccoli.SetEPIVoxelSizeX((float)atof(argv[7]));
  broccoli.SetEPIVoxelSizeY((float)atof(argv[8]));
  broccoli.SetEPIVoxelSizeZ((float)atof(argv[9]));
  broccoli.PerformSmoothingNormalizedHostWrapper();
  if (broccoli.GetLastStatus() != 0) {
    fprintf(stderr, "smoothing failed: %s\n", broccoli.GetOpenCLError());
    return 1;
  }
  FILE* f = fopen(argv[11], "wb");
  if (!f || fwrite(series.data(), sizeof(float), series.size(), f) != series.size()) {
    fprintf(stderr, "cannot write %s\n", argv[11]);
    return 2;
  }
  fclose(f);
  if (automask) {
    const std::string mp = std::string(argv[11]) + ".mask";
    FILE* m = fopen(mp.c_str(), "wb");
    if (!m || fwrite(certainty.data(), sizeof(float), V, m) != V) {
      fprintf(stderr, "cannot write %s\n", mp.c_str());
      return 2;
    }
    fclose(m);
  }
  return 0;
}
