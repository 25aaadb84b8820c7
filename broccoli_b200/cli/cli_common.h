// cli_common.h -- helpers shared by the command-line tools: the filter
// files of the reference's layout, output file names, option values.
#pragma once

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "broccoli_nifti.h"

namespace cli {

constexpr int kTaps = 7 * 7 * 7;

// The directory of the filter files: -filters DIR, else $BROCCOLI_DIR/filters
// (where the reference's tools look, Bash_Wrapper/MotionCorrection.cpp:552-563).
inline std::string filter_dir(const char* opt) {
  std::string d;
  if (opt) {
    d = opt;
  } else if (const char* b = getenv("BROCCOLI_DIR")) {
    d = std::string(b);
    if (!d.empty() && d.back() != '/') d += '/';
    d += "filters";
  }
  if (!d.empty() && d.back() != '/') d += '/';
  return d;
}

// n float32 values of a binary file (the reference's ReadBinaryFile).
inline bool read_floats(const std::string& path, size_t n, std::vector<float>& out) {
  out.assign(n, 0.f);
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) {
    fprintf(stderr, "Could not open %s\n", path.c_str());
    return false;
  }
  const size_t got = fread(out.data(), sizeof(float), n, f);
  fclose(f);
  if (got != n) {
    fprintf(stderr, "%s holds fewer than %zu floats\n", path.c_str(), n);
    return false;
  }
  return true;
}

// filter{k}_{real,imag}_{kind}_registration.bin for k = 1..count, real and
// imaginary parts in the order the class setters take them.
inline bool read_filters(const std::string& dir, const char* kind, int count, std::vector<std::vector<float>>& f) {
  f.assign(2 * count, {});
  for (int k = 0; k < count; k++)
    for (int c = 0; c < 2; c++) {
      const std::string p = dir + "filter" + std::to_string(k + 1) + (c == 0 ? "_real_" : "_imag_") + kind +
                            "_registration.bin";
      if (!read_floats(p, kTaps, f[2 * k + c])) return false;
    }
  return true;
}

// base with `suffix` inserted before a .nii / .nii.gz extension (".nii"
// added when there is none).  The reference inserts before the first dot of
// the whole path (HelpFunctions.cpp:337-352), which misplaces it for paths
// with dotted directories.
inline std::string with_suffix(const std::string& base, const std::string& suffix, const char* ext = nullptr) {
  std::string stem = base, e = ".nii";
  for (const char* x : {".nii.gz", ".nii"}) {
    const size_t n = strlen(x);
    if (stem.size() > n && stem.compare(stem.size() - n, n, x) == 0) {
      e = x;
      stem.resize(stem.size() - n);
      break;
    }
  }
  return stem + suffix + (ext ? ext : e.c_str());
}

inline bool has_value(int i, int argc, char** argv) {
  if (i + 1 < argc) return true;
  fprintf(stderr, "Option %s needs a value\n", argv[i]);
  return false;
}

inline bool read_nifti(const char* path, brc_nifti* img) {
  const int s = brc_nifti_read(path, img);
  if (s != 0) fprintf(stderr, "Could not read %s: %s\n", path, brc_nifti_error());
  return s == 0;
}

inline bool write_nifti(const std::string& path, const brc_nifti* like, const float* data, int nx, int ny, int nz,
                        int nt, bool quiet) {
  const int s = brc_nifti_write(path.c_str(), like, data, nx, ny, nz, nt);
  if (s != 0) {
    fprintf(stderr, "Could not write %s: %s\n", path.c_str(), brc_nifti_error());
    return false;
  }
  if (!quiet) printf("Wrote %s\n", path.c_str());
  return true;
}

}  // namespace cli
