// RegisterTwoVolumes -- affine and nonlinear registration of a volume to a
// reference (template) volume stored as NIfTI, on libbroccoli_b200 through
// the BROCCOLI_LIB class.  Options and outputs follow the reference's tool
// (code/Bash_Wrapper/RegisterTwoVolumes.cpp: usage :131-157, class set-up
// :1086-1143, affine matrix file :1220-1246, volumes :1250-1302): outputs
// at the reference's size under its header, input_aligned_linear.nii,
// input_aligned_nonlinear.nii and, on request, input_interpolated.nii,
// input_displacement_{x,y,z}.nii, input_affinematrix.txt, input_masked.nii
// (-mask / -maskoriginal, :1292-1295) and the debug volumes of -debug
// (:1304-1318: phase differences, certainties and gradients, the three
// quadrature filter responses as real and imaginary volumes).
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
  printf("RegisterTwoVolumes input.nii reference.nii [options]\n\n");
  printf("Options:\n\n");
  printf(" -device                 CUDA device to use (default 0)\n");
  printf(" -iterationslinear       Iterations of the linear registration (default 10), 0: none\n");
  printf(" -iterationsnonlinear    Iterations of the nonlinear registration (default 10), 0: none\n");
  printf(" -lowestscale            Coarsest scale of the pyramid: 1, 2, 4, 8 or 16 (default 4)\n");
  printf(" -sigma                  Gaussian smoothing (voxels) regularising the displacement field (default 5.0)\n");
  printf(" -zcut                   mm to cut from the bottom of the input volume (default 0)\n");
  printf(" -savematrix             Save the affine transformation matrix (input_affinematrix.txt)\n");
  printf(" -savefield              Save the displacement field\n");
  printf(" -saveinterpolated       Save the input resampled onto the reference grid, before alignment\n");
  printf(" -output                 Output base filename (default: the input's)\n");
  printf(" -filters                Directory of the filter files (default $BROCCOLI_DIR/filters)\n");
  printf(" -precision              fp32 (default), bf16x3 or tf32 (tensor-core filtering)\n");
  printf(" -precenter              Centre the input volume by its centre of mass first (default off)\n");
  printf(" -mask                   Mask (reference size) applied after the registration, e.g. a skull strip\n");
  printf(" -maskoriginal           Mask applied to the interpolated, unregistered input through the inverse\n");
  printf("                         affine transform\n");
  printf(" -debug                  Save the phase differences, certainties, gradients and filter responses\n");
  printf(" -quiet                  Print nothing\n");
  printf(" -verbose                Print extra information\n\n");
}

int main(int argc, char** argv) {
  if (argc < 3) {
    usage();
    return EXIT_SUCCESS;
  }
  int device = 0, it_lin = 10, it_nonlin = 10, coarsest = 4, zcut = 0, precision = BRC_PREC_FP32;
  float sigma = 5.0f;
  bool save_matrix = false, save_field = false, save_interp = false, quiet = false, verbose = false;
  bool precenter = false, debug = false, mask_original = false;
  const char* mask_name = nullptr;
  const char* out_opt = nullptr;
  const char* filters_opt = nullptr;
  for (int i = 3; i < argc; i++) {
    const std::string o = argv[i];
    if (o == "-savematrix") {
      save_matrix = true;
    } else if (o == "-savefield") {
      save_field = true;
    } else if (o == "-saveinterpolated") {
      save_interp = true;
    } else if (o == "-quiet") {
      quiet = true;
    } else if (o == "-verbose") {
      verbose = true;
    } else if (o == "-device" || o == "-iterationslinear" || o == "-iterationsnonlinear" || o == "-lowestscale" ||
               o == "-sigma" || o == "-zcut" || o == "-output" || o == "-filters" || o == "-precision") {
      if (!cli::has_value(i, argc, argv)) return EXIT_FAILURE;
      const char* v = argv[++i];
      if (o == "-device") device = atoi(v);
      if (o == "-iterationslinear") it_lin = atoi(v);
      if (o == "-iterationsnonlinear") it_nonlin = atoi(v);
      if (o == "-lowestscale") coarsest = atoi(v);
      if (o == "-sigma") sigma = (float)atof(v);
      if (o == "-zcut") zcut = atoi(v);
      if (o == "-output") out_opt = v;
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
    } else if (o == "-precenter") {
      precenter = true;
    } else if (o == "-debug") {
      debug = true;
    } else if (o == "-mask" || o == "-maskoriginal") {
      if (!cli::has_value(i, argc, argv)) return EXIT_FAILURE;
      mask_name = argv[++i];
      mask_original = o == "-maskoriginal";
    } else {
      fprintf(stderr, "Unknown option %s\n", argv[i]);
      return EXIT_FAILURE;
    }
  }
  if (it_lin < 0 || it_nonlin < 0 || !(coarsest == 1 || coarsest == 2 || coarsest == 4 || coarsest == 8 ||
                                       coarsest == 16) || !(sigma > 0.f)) {
    fprintf(stderr, "Invalid iterations, lowest scale or sigma\n");
    return EXIT_FAILURE;
  }

  brc_nifti t1, mni, mask;
  memset(&mask, 0, sizeof(mask));
  if (!cli::read_nifti(argv[1], &t1) || !cli::read_nifti(argv[2], &mni)) return EXIT_FAILURE;
  const int W = t1.dim[1], H = t1.dim[2], D = t1.dim[3];
  const int W2 = mni.dim[1], H2 = mni.dim[2], D2 = mni.dim[3];
  const size_t V2 = (size_t)W2 * H2 * D2;
  if (mask_name) {
    if (!cli::read_nifti(mask_name, &mask)) return EXIT_FAILURE;
    if (mask.dim[1] != W2 || mask.dim[2] != H2 || mask.dim[3] != D2) {
      fprintf(stderr, "Reference volume has the dimensions %d x %d x %d, while the mask volume has the dimensions "
                      "%d x %d x %d. Aborting!\n", W2, H2, D2, mask.dim[1], mask.dim[2], mask.dim[3]);
      return EXIT_FAILURE;
    }
  }
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
    printf("Registering %d x %d x %d (%.3g mm) to %d x %d x %d (%.3g mm)\n", W, H, D, t1.pixdim[1], W2, H2, D2,
           mni.pixdim[1]);

  BROCCOLI_LIB broccoli(0, (cl_uint)device, BASH, verbose);
  if (!broccoli.GetOpenCLInitiated()) {
    fprintf(stderr, "Initialisation failed: %s\n", broccoli.GetOpenCLInitializationError().c_str());
    return EXIT_FAILURE;
  }
  std::vector<float> interp(V2), lin(V2), nonlin(V2), fx(V2), fy(V2), fz(V2), params(12, 0.f);
  broccoli.SetInputT1Volume(t1.data);
  broccoli.SetInputMNIBrainVolume(mni.data);
  broccoli.SetT1Width(W);
  broccoli.SetT1Height(H);
  broccoli.SetT1Depth(D);
  broccoli.SetT1Timepoints(1);
  broccoli.SetT1VoxelSizeX(t1.pixdim[1]);
  broccoli.SetT1VoxelSizeY(t1.pixdim[2]);
  broccoli.SetT1VoxelSizeZ(t1.pixdim[3]);
  broccoli.SetMNIWidth(W2);
  broccoli.SetMNIHeight(H2);
  broccoli.SetMNIDepth(D2);
  broccoli.SetMNIVoxelSizeX(mni.pixdim[1]);
  broccoli.SetMNIVoxelSizeY(mni.pixdim[2]);
  broccoli.SetMNIVoxelSizeZ(mni.pixdim[3]);
  broccoli.SetInterpolationMode(LINEAR);
  broccoli.SetNumberOfIterationsForLinearImageRegistration(it_lin);
  broccoli.SetNumberOfIterationsForNonLinearImageRegistration(it_nonlin);
  broccoli.SetImageRegistrationFilterSize(7);
  broccoli.SetLinearImageRegistrationFilters(fl[0].data(), fl[1].data(), fl[2].data(), fl[3].data(), fl[4].data(),
                                             fl[5].data());
  broccoli.SetNonLinearImageRegistrationFilters(fn[0].data(), fn[1].data(), fn[2].data(), fn[3].data(),
                                                fn[4].data(), fn[5].data(), fn[6].data(), fn[7].data(),
                                                fn[8].data(), fn[9].data(), fn[10].data(), fn[11].data());
  void (BROCCOLI_LIB::*set_tensor[6])(float, float, float, float, float, float) = {
      &BROCCOLI_LIB::SetProjectionTensorMatrixFirstFilter,  &BROCCOLI_LIB::SetProjectionTensorMatrixSecondFilter,
      &BROCCOLI_LIB::SetProjectionTensorMatrixThirdFilter,  &BROCCOLI_LIB::SetProjectionTensorMatrixFourthFilter,
      &BROCCOLI_LIB::SetProjectionTensorMatrixFifthFilter,  &BROCCOLI_LIB::SetProjectionTensorMatrixSixthFilter};
  for (int k = 0; k < 6; k++)
    (broccoli.*set_tensor[k])(tens[k][0], tens[k][1], tens[k][2], tens[k][3], tens[k][4], tens[k][5]);
  broccoli.SetFilterDirections(dirs[0].data(), dirs[1].data(), dirs[2].data());
  broccoli.SetCoarsestScaleT1MNI(coarsest);
  broccoli.SetMMT1ZCUT(zcut);
  broccoli.SetTsigma(sigma);
  broccoli.SetEsigma(sigma);
  broccoli.SetDsigma(sigma);
  broccoli.SetPrecision(precision);
  broccoli.SetOutputInterpolatedT1Volume(interp.data());
  broccoli.SetOutputAlignedT1VolumeLinear(lin.data());
  broccoli.SetOutputAlignedT1VolumeNonLinear(nonlin.data());
  broccoli.SetOutputT1MNIRegistrationParameters(params.data());
  broccoli.SetOutputDisplacementField(fx.data(), fy.data(), fz.data());
  broccoli.SetPrecenterRegistration(precenter);
  std::vector<float> masked(mask_name ? V2 : 0), pd(debug ? V2 : 0), pc(debug ? V2 : 0), pg(debug ? V2 : 0);
  std::vector<cl_float2> q[3];
  if (mask_name) {
    broccoli.SetInputMNIBrainMask(mask.data);
    broccoli.SetOutputSkullstrippedT1Volume(masked.data());
    broccoli.SetDoSkullstrip(!mask_original);
    broccoli.SetDoSkullstripOriginal(mask_original);
  }
  if (debug) {
    for (int k = 0; k < 3; k++) q[k].resize(V2);
    broccoli.SetDebug(true);
    broccoli.SetOutputQuadratureFilterResponses(q[0].data(), q[1].data(), q[2].data());
    broccoli.SetOutputPhaseDifferences(pd.data());
    broccoli.SetOutputPhaseCertainties(pc.data());
    broccoli.SetOutputPhaseGradients(pg.data());
  }
  broccoli.PerformRegistrationTwoVolumesWrapper();
  if (broccoli.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "Registration failed: %s\n", broccoli.GetOpenCLError());
    return EXIT_FAILURE;
  }

  const std::string base = out_opt ? std::string(out_opt) : std::string(argv[1]);
  bool ok = true;
  if (save_matrix && it_lin > 0) {
    const std::string mp = cli::with_suffix(base, "_affinematrix", ".txt");
    std::ofstream m(mp.c_str());
    if (m.good()) {
      const float* p = params.data();
      m.precision(6);
      m << p[3] + 1.0f << std::setw(2) << " " << p[4] << std::setw(2) << " " << p[5] << std::setw(2) << " " << p[0]
        << std::endl;
      m << p[6] << std::setw(2) << " " << p[7] + 1.0f << std::setw(2) << " " << p[8] << std::setw(2) << " " << p[1]
        << std::endl;
      m << p[9] << std::setw(2) << " " << p[10] << std::setw(2) << " " << p[11] + 1.0f << std::setw(2) << " "
        << p[2] << std::endl;
      m << 0.0f << std::setw(2) << " " << 0.0f << std::setw(2) << " " << 0.0f << std::setw(2) << " " << 1.0f
        << std::endl;
      if (!quiet) printf("Wrote %s\n", mp.c_str());
    } else {
      fprintf(stderr, "Could not open %s for writing\n", mp.c_str());
      ok = false;
    }
  }
  if (save_interp) ok = cli::write_nifti(cli::with_suffix(base, "_interpolated"), &mni, interp.data(), W2, H2, D2, 1,
                                         quiet) && ok;
  ok = cli::write_nifti(cli::with_suffix(base, "_aligned_linear"), &mni, lin.data(), W2, H2, D2, 1, quiet) && ok;
  if (it_nonlin > 0) {
    ok = cli::write_nifti(cli::with_suffix(base, "_aligned_nonlinear"), &mni, nonlin.data(), W2, H2, D2, 1, quiet) &&
         ok;
    if (save_field) {
      ok = cli::write_nifti(cli::with_suffix(base, "_displacement_x"), &mni, fx.data(), W2, H2, D2, 1, quiet) && ok;
      ok = cli::write_nifti(cli::with_suffix(base, "_displacement_y"), &mni, fy.data(), W2, H2, D2, 1, quiet) && ok;
      ok = cli::write_nifti(cli::with_suffix(base, "_displacement_z"), &mni, fz.data(), W2, H2, D2, 1, quiet) && ok;
    }
  }
  if (mask_name && (!mask_original || it_lin > 0))
    ok = cli::write_nifti(cli::with_suffix(base, "_masked"), &mni, masked.data(), W2, H2, D2, 1, quiet) && ok;
  if (debug) {
    ok = cli::write_nifti(cli::with_suffix(base, "_phase_gradients"), &mni, pg.data(), W2, H2, D2, 1, quiet) && ok;
    ok = cli::write_nifti(cli::with_suffix(base, "_phase_certainties"), &mni, pc.data(), W2, H2, D2, 1, quiet) && ok;
    ok = cli::write_nifti(cli::with_suffix(base, "_phase_differences"), &mni, pd.data(), W2, H2, D2, 1, quiet) && ok;
    std::vector<float> re(V2), im(V2);
    for (int k = 0; k < 3; k++) {
      for (size_t i = 0; i < V2; i++) {
        re[i] = q[k][i].x;
        im[i] = q[k][i].y;
      }
      const std::string n = "_quadrature_filter_response_" + std::to_string(k + 1);
      ok = cli::write_nifti(cli::with_suffix(base, n + "_real"), &mni, re.data(), W2, H2, D2, 1, quiet) && ok;
      ok = cli::write_nifti(cli::with_suffix(base, n + "_imag"), &mni, im.data(), W2, H2, D2, 1, quiet) && ok;
    }
  }
  brc_nifti_free(&t1);
  brc_nifti_free(&mni);
  if (mask_name) brc_nifti_free(&mask);
  return ok ? EXIT_SUCCESS : EXIT_FAILURE;
}
