// TransformVolume -- applies an affine matrix, a scaling, a centring or a
// displacement field to a NIfTI volume (or series) on libbroccoli_b200
// through the BROCCOLI_LIB class.  Options and outputs follow the
// reference's tool (code/Bash_Wrapper/TransformVolume.cpp: usage :109-127,
// matrix file :644-702, scaling :704-727, class calls :800-843, outputs
// :884-915): the input is resampled onto the reference volume's grid and
// transformed, and written under the reference's header as
// input_warped.nii (input_centered.nii for -centering) or the -output name.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <string>
#include <vector>

#include "broccoli_lib.h"
#include "cli_common.h"

static void usage() {
  printf("Usage, transformation matrix:\n\n");
  printf("TransformVolume volume_to_transform.nii reference_volume.nii -matrix affine_matrix.1D  [options]\n\n");
  printf("Usage, scaling:\n\n");
  printf("TransformVolume volume_to_transform.nii volume_to_transform.nii -scaling 2.3  [options]\n\n");
  printf("Usage, centering:\n\n");
  printf("TransformVolume volume_to_transform.nii volume_to_transform.nii -centering  [options]\n\n");
  printf("Usage, displacement field:\n\n");
  printf("TransformVolume volume_to_transform.nii reference_volume.nii -field displacement_field_x.nii "
         "displacement_field_y.nii displacement_field_z.nii  [options]\n\n");
  printf("Options:\n\n");
  printf(" -device                    CUDA device to use (default 0)\n");
  printf(" -matrix                    An affine transformation matrix (4 x 4) in a text file\n");
  printf(" -scaling                   A scaling to apply to each dimension\n");
  printf(" -centering                 Center the volume mass\n");
  printf(" -field                     An arbitrary deformation field in three files\n");
  printf(" -interpolation             The interpolation to use, 0 = nearest neighbour, 1 = trilinear (default 1)\n");
  printf(" -zcut                      Number of mm to cut from the bottom of the input volume (default 0)\n");
  printf(" -output                    Set output filename (default volume_to_transform_warped.nii)\n");
  printf(" -quiet                     Print nothing\n\n");
}

int main(int argc, char** argv) {
  if (argc < 3) {
    usage();
    return EXIT_SUCCESS;
  }
  int device = 0, interpolation = LINEAR, zcut = 0;
  const char* matrix_path = nullptr;
  const char* field_path[3] = {nullptr, nullptr, nullptr};
  const char* out_path = nullptr;
  float scaling = 0.0f;
  bool centering = false, quiet = false;
  for (int i = 3; i < argc; i++) {
    const std::string o = argv[i];
    if (o == "-quiet") {
      quiet = true;
    } else if (o == "-centering") {
      centering = true;
    } else if (o == "-field") {
      if (i + 3 >= argc) {
        fprintf(stderr, "Option -field needs three files\n");
        return EXIT_FAILURE;
      }
      for (int a = 0; a < 3; a++) field_path[a] = argv[++i];
    } else if (o == "-device" || o == "-matrix" || o == "-scaling" || o == "-interpolation" || o == "-zcut" ||
               o == "-output") {
      if (!cli::has_value(i, argc, argv)) return EXIT_FAILURE;
      const char* v = argv[++i];
      if (o == "-device") device = atoi(v);
      if (o == "-matrix") matrix_path = v;
      if (o == "-scaling") scaling = (float)atof(v);
      if (o == "-interpolation") interpolation = atoi(v);
      if (o == "-zcut") zcut = atoi(v);
      if (o == "-output") out_path = v;
    } else {
      fprintf(stderr, "Unknown option %s\n", argv[i]);
      return EXIT_FAILURE;
    }
  }
  const int modes = (matrix_path ? 1 : 0) + (scaling != 0.0f ? 1 : 0) + (centering ? 1 : 0) + (field_path[0] ? 1 : 0);
  if (modes != 1) {
    fprintf(stderr, "Give exactly one of -matrix, -scaling, -centering and -field\n");
    return EXIT_FAILURE;
  }
  if (scaling < 0.0f) {
    fprintf(stderr, "The scaling must be positive\n");
    return EXIT_FAILURE;
  }
  if (interpolation != NEAREST && interpolation != LINEAR) {
    fprintf(stderr, "The interpolation must be 0 (nearest) or 1 (trilinear)\n");
    return EXIT_FAILURE;
  }

  brc_nifti in, ref;
  if (!cli::read_nifti(argv[1], &in) || !cli::read_nifti(argv[2], &ref)) return EXIT_FAILURE;
  const int W = in.dim[1], H = in.dim[2], D = in.dim[3], T = in.dim[0] >= 4 ? in.dim[4] : 1;
  const int W2 = ref.dim[1], H2 = ref.dim[2], D2 = ref.dim[3];
  const size_t V2 = (size_t)W2 * H2 * D2;

  // parameters: matrix rows (a11 a12 a13 tx / ... / 0 0 0 1) into {t, A - I}
  float params[16] = {0};
  if (matrix_path) {
    std::ifstream m(matrix_path);
    if (!m.good()) {
      fprintf(stderr, "Unable to open affine matrix file %s\n", matrix_path);
      return EXIT_FAILURE;
    }
    const int idx[16] = {3, 4, 5, 0, 6, 7, 8, 1, 9, 10, 11, 2, 12, 13, 14, 15};
    for (int p = 0; p < 16; p++)
      if (!(m >> params[idx[p]])) {
        fprintf(stderr, "Could not read all values of the affine matrix file %s (stopped at value %d)\n", matrix_path,
                p);
        return EXIT_FAILURE;
      }
    params[3] -= 1.0f;
    params[7] -= 1.0f;
    params[11] -= 1.0f;
  } else if (scaling != 0.0f) {
    params[3] = params[7] = params[11] = 1.0f / scaling - 1.0f;
  }
  std::vector<std::vector<float>> field(3);
  if (field_path[0]) {
    for (int a = 0; a < 3; a++) {
      brc_nifti f;
      if (!cli::read_nifti(field_path[a], &f)) return EXIT_FAILURE;
      const bool same = f.dim[1] == W2 && f.dim[2] == H2 && f.dim[3] == D2;
      if (same) field[a].assign(f.data, f.data + V2);
      brc_nifti_free(&f);
      if (!same) {
        fprintf(stderr, "The displacement field %s does not have the size of the reference volume\n",
                field_path[a]);
        return EXIT_FAILURE;
      }
    }
  }

  BROCCOLI_LIB broccoli(0, (cl_uint)device, BASH, false);
  if (!broccoli.GetOpenCLInitiated()) {
    fprintf(stderr, "Initialisation failed: %s\n", broccoli.GetOpenCLInitializationError().c_str());
    return EXIT_FAILURE;
  }
  // the centred series keeps the input's grid
  const int oW = centering ? W : W2, oH = centering ? H : H2, oD = centering ? D : D2;
  std::vector<float> out((size_t)oW * oH * oD * T);
  broccoli.SetInputT1Volume(in.data);
  broccoli.SetT1Width(W);
  broccoli.SetT1Height(H);
  broccoli.SetT1Depth(D);
  broccoli.SetT1Timepoints(T);
  broccoli.SetT1VoxelSizeX(in.pixdim[1]);
  broccoli.SetT1VoxelSizeY(in.pixdim[2]);
  broccoli.SetT1VoxelSizeZ(in.pixdim[3]);
  broccoli.SetMNIWidth(W2);
  broccoli.SetMNIHeight(H2);
  broccoli.SetMNIDepth(D2);
  broccoli.SetMNIVoxelSizeX(ref.pixdim[1]);
  broccoli.SetMNIVoxelSizeY(ref.pixdim[2]);
  broccoli.SetMNIVoxelSizeZ(ref.pixdim[3]);
  broccoli.SetMMT1ZCUT(zcut);
  broccoli.SetInterpolationMode(interpolation);
  if (field_path[0]) broccoli.SetOutputDisplacementField(field[0].data(), field[1].data(), field[2].data());
  broccoli.SetOutputT1MNIRegistrationParameters(params);
  broccoli.SetOutputInterpolatedT1Volume(out.data());
  if (centering)
    broccoli.CenterVolumesWrapper();
  else if (field_path[0])
    broccoli.TransformVolumesNonLinearWrapper();
  else
    broccoli.TransformVolumesLinearWrapper();
  if (broccoli.GetLastStatus() != BRC_OK) {
    fprintf(stderr, "Transformation failed: %s\n", broccoli.GetOpenCLError());
    return EXIT_FAILURE;
  }
  const std::string path =
      out_path ? std::string(out_path) : cli::with_suffix(argv[1], centering ? "_centered" : "_warped");
  const bool ok = cli::write_nifti(path, centering ? &in : &ref, out.data(), oW, oH, oD, T, quiet);
  brc_nifti_free(&in);
  brc_nifti_free(&ref);
  return ok ? EXIT_SUCCESS : EXIT_FAILURE;
}
