// Smoothing -- normalised Gaussian smoothing of an fMRI series stored as
// NIfTI, on libbroccoli_b200 through the BROCCOLI_LIB class.  Options and
// outputs follow the reference's tool (code/Bash_Wrapper/Smoothing.cpp:
// usage :102-112, class calls :593-613, outputs :652-683): the smoothed
// series (input_sm.nii, FLOAT32 under the input's header) and, with
// -automask, the mask it made (input_mask.nii, or output_mask.nii).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "broccoli_lib.h"
#include "cli_common.h"

static void usage() {
  printf("Usage:\n\n");
  printf("Smoothing input.nii [options]\n\n");
  printf("Options:\n\n");
  printf(" -device          CUDA device to use (default 0)\n");
  printf(" -fwhm            Amount of smoothing to apply (in mm, default 6 mm)\n");
  printf(" -mask            Perform smoothing inside mask (normalized convolution)\n");
  printf(" -automask        Generate a mask and perform smoothing inside mask (normalized convolution)\n");
  printf(" -output          Set output filename (default input_sm.nii)\n");
  printf(" -quiet           Print nothing\n");
  printf(" -verbose         Print extra information\n\n");
}

int main(int argc, char** argv) {
  if (argc < 2) {
    usage();
    return EXIT_SUCCESS;
  }
  int device = 0;
  float fwhm = 6.0f;
  const char* mask_path = nullptr;
  const char* out_path = nullptr;
  bool automask = false, quiet = false, verbose = false;
  for (int i = 2; i < argc; i++) {
    const std::string o = argv[i];
    if (o == "-quiet") {
      quiet = true;
    } else if (o == "-verbose") {
      verbose = true;
    } else if (o == "-automask") {
      automask = true;
    } else if (o == "-device" || o == "-fwhm" || o == "-mask" || o == "-output") {
      if (!cli::has_value(i, argc, argv)) return EXIT_FAILURE;
      const char* v = argv[++i];
      if (o == "-device") device = atoi(v);
      if (o == "-fwhm") fwhm = (float)atof(v);
      if (o == "-mask") mask_path = v;
      if (o == "-output") out_path = v;
    } else {
      fprintf(stderr, "Unknown option %s\n", argv[i]);
      return EXIT_FAILURE;
    }
  }
  if (!(fwhm > 0.0f)) {
    fprintf(stderr, "The FWHM must be positive\n");
    return EXIT_FAILURE;
  }
  if (mask_path && automask) {
    fprintf(stderr, "Give -mask or -automask, not both\n");
    return EXIT_FAILURE;
  }
  brc_nifti in;
  if (!cli::read_nifti(argv[1], &in)) return EXIT_FAILURE;
  const int W = in.dim[1], H = in.dim[2], D = in.dim[3], T = in.dim[0] >= 4 ? in.dim[4] : 1;
  const size_t V = (size_t)W * H * D;
  // the certainty: the mask, or ones (Smoothing.cpp:440-505)
  std::vector<float> certainty(V, 1.0f);
  if (mask_path) {
    brc_nifti m;
    if (!cli::read_nifti(mask_path, &m)) return EXIT_FAILURE;
    const bool same = m.dim[1] == W && m.dim[2] == H && m.dim[3] == D;
    if (same) memcpy(certainty.data(), m.data, sizeof(float) * V);
    brc_nifti_free(&m);
    if (!same) {
      fprintf(stderr, "The mask must have the size of the volumes\n");
      return EXIT_FAILURE;
    }
  }
  if (!quiet)
    printf("Smoothing %d volumes of %d x %d x %d voxels (%.3g x %.3g x %.3g mm) with %.3g mm FWHM\n", T, W, H, D,
           in.pixdim[1], in.pixdim[2], in.pixdim[3], fwhm);

  BROCCOLI_LIB broccoli(0, (cl_uint)device, BASH, verbose);
  if (!broccoli.GetOpenCLInitiated()) {
    fprintf(stderr, "Initialisation failed: %s\n", broccoli.GetOpenCLInitializationError().c_str());
    return EXIT_FAILURE;
  }
  broccoli.SetInputfMRIVolumes(in.data);
  broccoli.SetAutoMask(automask);
  broccoli.SetInputCertainty(certainty.data());
  broccoli.SetEPISmoothingAmount(fwhm);
  broccoli.SetEPIWidth(W);
  broccoli.SetEPIHeight(H);
  broccoli.SetEPIDepth(D);
  broccoli.SetEPITimepoints(T);
  broccoli.SetEPIVoxelSizeX(in.pixdim[1]);
  broccoli.SetEPIVoxelSizeY(in.pixdim[2]);
  broccoli.SetEPIVoxelSizeZ(in.pixdim[3]);
  broccoli.PerformSmoothingNormalizedHostWrapper();
  if (broccoli.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "Smoothing failed: %s\n", broccoli.GetOpenCLError());
    return EXIT_FAILURE;
  }
  const std::string base = out_path ? std::string(out_path) : cli::with_suffix(argv[1], "_sm");
  bool ok = cli::write_nifti(base, &in, in.data, W, H, D, T, quiet);
  if (automask)
    ok = cli::write_nifti(cli::with_suffix(out_path ? base : std::string(argv[1]), "_mask"), &in,
                          certainty.data(), W, H, D, 1, quiet) && ok;
  brc_nifti_free(&in);
  return ok ? EXIT_SUCCESS : EXIT_FAILURE;
}
