// MotionCorrection -- rigid motion correction of an fMRI series stored as
// NIfTI, on libbroccoli_b200 through the BROCCOLI_LIB class.  Options and
// outputs follow the reference's tool (code/Bash_Wrapper/MotionCorrection.cpp:
// usage :113-130, motion parameter file :747-775): the corrected series
// (input_mc.nii, FLOAT32 under the input's header) and
// input_motionparameters.1D (one line per volume, AFNI's column order).
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
  printf("MotionCorrection input.nii [options]\n\n");
  printf("Options:\n\n");
  printf(" -device             CUDA device to use (default 0)\n");
  printf(" -referencevolume    Align all volumes to this volume (default: the first volume)\n");
  printf(" -iterations         Iterations of the registration per volume (default 5)\n");
  printf(" -output             Output filename (default input_mc.nii)\n");
  printf(" -filters            Directory of the filter files (default $BROCCOLI_DIR/filters)\n");
  printf(" -precision          fp32 (default), bf16x3 or tf32 (tensor-core filtering)\n");
  printf(" -tolerance          Stop a volume's iterations once its update is below this many voxels (default 0: off)\n");
  printf(" -quiet              Print nothing\n");
  printf(" -verbose            Print extra information\n\n");
}

int main(int argc, char** argv) {
  if (argc < 2) {
    usage();
    return EXIT_SUCCESS;
  }
  int device = 0, iterations = 5, precision = BRC_PREC_FP32;
  float tolerance = 0.f;
  const char* ref_path = nullptr;
  const char* out_path = nullptr;
  const char* filters_opt = nullptr;
  bool quiet = false, verbose = false;
  for (int i = 2; i < argc; i++) {
    const std::string o = argv[i];
    if (o == "-quiet") {
      quiet = true;
    } else if (o == "-verbose") {
      verbose = true;
    } else if (o == "-device" || o == "-iterations" || o == "-referencevolume" || o == "-output" ||
               o == "-filters" || o == "-precision" || o == "-tolerance") {
      if (!cli::has_value(i, argc, argv)) return EXIT_FAILURE;
      const char* v = argv[++i];
      if (o == "-device") device = atoi(v);
      if (o == "-iterations") iterations = atoi(v);
      if (o == "-referencevolume") ref_path = v;
      if (o == "-output") out_path = v;
      if (o == "-filters") filters_opt = v;
      if (o == "-tolerance") tolerance = (float)atof(v);
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
      fprintf(stderr, "Unknown option %s\n", argv[i]);
      return EXIT_FAILURE;
    }
  }
  if (iterations <= 0) {
    fprintf(stderr, "The number of iterations must be positive\n");
    return EXIT_FAILURE;
  }

  brc_nifti in;
  if (!cli::read_nifti(argv[1], &in)) return EXIT_FAILURE;
  const int W = in.dim[1], H = in.dim[2], D = in.dim[3], T = in.dim[0] >= 4 ? in.dim[4] : 1;
  brc_nifti ref{};
  bool have_ref = false;
  if (ref_path) {
    if (!cli::read_nifti(ref_path, &ref)) return EXIT_FAILURE;
    have_ref = true;
    if (ref.dim[1] != W || ref.dim[2] != H || ref.dim[3] != D) {
      fprintf(stderr, "The reference volume must have the size of the series' volumes\n");
      return EXIT_FAILURE;
    }
  }
  const std::string dir = cli::filter_dir(filters_opt);
  if (dir.empty()) {
    fprintf(stderr, "Give -filters DIR or set BROCCOLI_DIR\n");
    return EXIT_FAILURE;
  }
  std::vector<std::vector<float>> f;
  if (!cli::read_filters(dir, "linear", 3, f)) return EXIT_FAILURE;
  if (!quiet)
    printf("Series of %d volumes of %d x %d x %d voxels (%.3g x %.3g x %.3g mm)\n", T, W, H, D, in.pixdim[1],
           in.pixdim[2], in.pixdim[3]);

  BROCCOLI_LIB broccoli(0, (cl_uint)device, BASH, verbose);
  if (!broccoli.GetOpenCLInitiated()) {
    fprintf(stderr, "Initialisation failed: %s\n", broccoli.GetOpenCLInitializationError().c_str());
    return EXIT_FAILURE;
  }
  std::vector<float> motion(6 * (size_t)T, 0.f);
  broccoli.SetEPIWidth(W);
  broccoli.SetEPIHeight(H);
  broccoli.SetEPIDepth(D);
  broccoli.SetEPITimepoints(T);
  broccoli.SetEPIVoxelSizeX(in.pixdim[1]);
  broccoli.SetEPIVoxelSizeY(in.pixdim[2]);
  broccoli.SetEPIVoxelSizeZ(in.pixdim[3]);
  broccoli.SetInputfMRIVolumes(in.data);
  broccoli.SetImageRegistrationFilterSize(7);
  broccoli.SetLinearImageRegistrationFilters(f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(),
                                             f[5].data());
  broccoli.SetNumberOfIterationsForMotionCorrection(iterations);
  broccoli.SetChangeMotionCorrectionReferenceVolume(have_ref);
  if (have_ref) broccoli.SetMotionCorrectionReferenceVolume(ref.data);
  broccoli.SetPrecision(precision);
  broccoli.SetMotionCorrectionTolerance(tolerance);
  broccoli.SetOutputMotionParameters(motion.data());
  broccoli.PerformMotionCorrectionWrapper();
  if (broccoli.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "Motion correction failed: %s\n", broccoli.GetOpenCLError());
    return EXIT_FAILURE;
  }

  const std::string base = out_path ? std::string(out_path) : cli::with_suffix(argv[1], "_mc");
  bool ok = cli::write_nifti(base, &in, in.data, W, H, D, T, quiet);
  // translations (mm) and rotations (degrees) as AFNI orders them: roll,
  // pitch, yaw, dS, dL, dP (the reference's column order and signs)
  const std::string mp = cli::with_suffix(out_path ? base : std::string(argv[1]), "_motionparameters", ".1D");
  std::ofstream file(mp.c_str());
  if (file.good()) {
    file.precision(6);
    for (int t = 0; t < T; t++) {
      const float* p = motion.data();
      file << p[t + 4 * T] << std::setw(2) << " " << -p[t + 3 * T] << std::setw(2) << " " << p[t + 5 * T]
           << std::setw(2) << " " << -p[t + 2 * T] << std::setw(2) << " " << -p[t + 0 * T] << std::setw(2) << " "
           << -p[t + 1 * T] << std::endl;
    }
    if (!quiet) printf("Wrote %s\n", mp.c_str());
  } else {
    fprintf(stderr, "Could not open %s for writing\n", mp.c_str());
    ok = false;
  }
  brc_nifti_free(&in);
  if (have_ref) brc_nifti_free(&ref);
  return ok ? EXIT_SUCCESS : EXIT_FAILURE;
}
