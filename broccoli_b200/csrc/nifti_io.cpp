// nifti_io.cpp -- NIfTI-1 single-file reading and FLOAT32 writing for the
// command-line tools (include/broccoli_nifti.h).  Header fields are read at
// the offsets of the NIfTI-1 standard (348-byte header, magic "n+1" at 344,
// data from vox_offset); a byte-swapped sizeof_hdr marks a file of the
// other byte order, whose header is converted field by field.  zlib's gz
// stream reads plain and compressed files alike.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#include <string>
#include <vector>

#include "../../include/broccoli_b200.h"
#include "../../include/broccoli_nifti.h"

namespace {

thread_local std::string g_err;

int fail(int status, const std::string& msg) {
  g_err = msg;
  return status;
}

// NIfTI-1 datatype codes
enum {
  kUINT8 = 2,
  kINT16 = 4,
  kINT32 = 8,
  kFLOAT32 = 16,
  kFLOAT64 = 64,
  kINT8 = 256,
  kUINT16 = 512,
  kUINT32 = 768,
};

int bytes_per_voxel(int dt) {
  switch (dt) {
    case kUINT8:
    case kINT8: return 1;
    case kINT16:
    case kUINT16: return 2;
    case kINT32:
    case kUINT32:
    case kFLOAT32: return 4;
    case kFLOAT64: return 8;
    default: return 0;
  }
}

void swap_bytes(unsigned char* p, int n) {
  for (int i = 0; i < n / 2; i++) {
    const unsigned char t = p[i];
    p[i] = p[n - 1 - i];
    p[n - 1 - i] = t;
  }
}

// Converts a header of the other byte order in place: every multi-byte
// field of the NIfTI-1 layout.
void swap_header(unsigned char* h) {
  for (int off : {0, 32, 140, 144}) swap_bytes(h + off, 4);  // ints
  for (int off : {36, 68, 70, 72, 74, 120, 252, 254}) swap_bytes(h + off, 2);
  for (int k = 0; k < 8; k++) swap_bytes(h + 40 + 2 * k, 2);  // dim
  for (int off : {56, 60, 64, 108, 112, 116, 124, 128, 132, 136}) swap_bytes(h + off, 4);
  for (int k = 0; k < 8; k++) swap_bytes(h + 76 + 4 * k, 4);    // pixdim
  for (int k = 0; k < 18; k++) swap_bytes(h + 256 + 4 * k, 4);  // quatern_*, qoffset_*, srow_*
}

template <class T>
T get(const unsigned char* h, int off) {
  T v;
  memcpy(&v, h + off, sizeof(T));
  return v;
}
template <class T>
void put(unsigned char* h, int off, T v) {
  memcpy(h + off, &v, sizeof(T));
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t n = strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

template <class T>
void convert(const unsigned char* src, long long n, bool swap, float* dst) {
  for (long long i = 0; i < n; i++) {
    unsigned char b[sizeof(T)];
    memcpy(b, src + i * (long long)sizeof(T), sizeof(T));
    if (swap) swap_bytes(b, sizeof(T));
    T v;
    memcpy(&v, b, sizeof(T));
    dst[i] = (float)v;
  }
}

}  // namespace

extern "C" const char* brc_nifti_error(void) { return g_err.c_str(); }

extern "C" void brc_nifti_free(brc_nifti* img) {
  if (!img) return;
  free(img->data);
  img->data = nullptr;
}

extern "C" int brc_nifti_read(const char* path, brc_nifti* img) {
  if (!path || !img) return fail(BRC_ERR_INVALID, "brc_nifti_read: null argument");
  memset(img, 0, sizeof(*img));
  const std::string p(path);
  if (ends_with(p, ".hdr") || ends_with(p, ".img") || ends_with(p, ".hdr.gz") || ends_with(p, ".img.gz"))
    return fail(BRC_ERR_UNSUPPORTED, p + ": .hdr/.img pairs are not read, convert to .nii");
  gzFile f = gzopen(path, "rb");
  if (!f) return fail(BRC_ERR_INVALID, p + ": cannot open");
  unsigned char* h = img->header;
  if (gzread(f, h, 348) != 348) {
    gzclose(f);
    return fail(BRC_ERR_INVALID, p + ": shorter than a NIfTI-1 header");
  }
  bool swap = false;
  if (get<int32_t>(h, 0) != 348) {
    unsigned char s[4];
    memcpy(s, h, 4);
    swap_bytes(s, 4);
    int32_t v;
    memcpy(&v, s, 4);
    if (v != 348) {
      gzclose(f);
      return fail(BRC_ERR_INVALID, p + ": sizeof_hdr is not 348 (not NIfTI-1)");
    }
    swap = true;
    swap_header(h);
  }
  if (memcmp(h + 344, "n+1", 4) != 0) {
    gzclose(f);
    return fail(memcmp(h + 344, "ni1", 4) == 0 ? BRC_ERR_UNSUPPORTED : BRC_ERR_INVALID,
                p + ": magic is not \"n+1\" (single-file NIfTI-1)");
  }
  const int nd = get<int16_t>(h, 40);
  if (nd < 1 || nd > 7) {
    gzclose(f);
    return fail(BRC_ERR_INVALID, p + ": dim[0] out of range");
  }
  long long n = 1;
  img->dim[0] = nd;
  for (int k = 1; k < 8; k++) {
    const int d = get<int16_t>(h, 40 + 2 * k);
    img->dim[k] = k <= nd ? (d > 0 ? d : 1) : 1;
    if (k <= nd) n *= img->dim[k];
  }
  for (int k = 0; k < 8; k++) img->pixdim[k] = get<float>(h, 76 + 4 * k);
  img->datatype = get<int16_t>(h, 70);
  const int bpv = bytes_per_voxel(img->datatype);
  if (bpv == 0) {
    gzclose(f);
    return fail(BRC_ERR_UNSUPPORTED, p + ": datatype " + std::to_string(img->datatype) + " is not read");
  }
  const float vo = get<float>(h, 108);
  const long long off = vo >= 348.0f ? (long long)vo : 352;
  std::vector<unsigned char> skip((size_t)(off - 348));
  if (!skip.empty() && gzread(f, skip.data(), (unsigned)skip.size()) != (int)skip.size()) {
    gzclose(f);
    return fail(BRC_ERR_INVALID, p + ": truncated before vox_offset");
  }
  std::vector<unsigned char> raw;
  try {
    raw.resize((size_t)(n * bpv));
  } catch (...) {
    gzclose(f);
    return fail(BRC_ERR_NOMEM, p + ": cannot hold the voxels");
  }
  size_t got = 0;
  while (got < raw.size()) {
    const size_t want = raw.size() - got > (1u << 30) ? (1u << 30) : raw.size() - got;
    const int r = gzread(f, raw.data() + got, (unsigned)want);
    if (r <= 0) break;
    got += (size_t)r;
  }
  gzclose(f);
  if (got != raw.size()) return fail(BRC_ERR_INVALID, p + ": truncated voxel data");
  img->data = static_cast<float*>(malloc(sizeof(float) * (size_t)n));
  if (!img->data) return fail(BRC_ERR_NOMEM, p + ": cannot hold the voxels");
  switch (img->datatype) {
    case kUINT8: convert<uint8_t>(raw.data(), n, swap, img->data); break;
    case kINT8: convert<int8_t>(raw.data(), n, swap, img->data); break;
    case kINT16: convert<int16_t>(raw.data(), n, swap, img->data); break;
    case kUINT16: convert<uint16_t>(raw.data(), n, swap, img->data); break;
    case kINT32: convert<int32_t>(raw.data(), n, swap, img->data); break;
    case kUINT32: convert<uint32_t>(raw.data(), n, swap, img->data); break;
    case kFLOAT32: convert<float>(raw.data(), n, swap, img->data); break;
    case kFLOAT64: convert<double>(raw.data(), n, swap, img->data); break;
  }
  return BRC_OK;
}

extern "C" int brc_nifti_write(const char* path, const brc_nifti* like, const float* data, int nx, int ny, int nz,
                               int nt) {
  if (!path || !data || nx <= 0 || ny <= 0 || nz <= 0 || nt <= 0 || nx > 32767 || ny > 32767 || nz > 32767 ||
      nt > 32767)
    return fail(BRC_ERR_INVALID, "brc_nifti_write: bad argument");
  unsigned char h[352];
  memset(h, 0, sizeof(h));
  if (like) {
    memcpy(h, like->header, 348);
  } else {
    for (int k = 1; k < 8; k++) put<float>(h, 76 + 4 * k, 1.0f);
    put<float>(h, 112, 1.0f);  // scl_slope
  }
  put<int32_t>(h, 0, 348);
  const int nd = nt > 1 ? 4 : 3;
  const int dims[8] = {nd, nx, ny, nz, nt, 1, 1, 1};
  for (int k = 0; k < 8; k++) put<int16_t>(h, 40 + 2 * k, (int16_t)dims[k]);
  put<int16_t>(h, 70, (int16_t)kFLOAT32);
  put<int16_t>(h, 72, (int16_t)32);
  put<float>(h, 108, 352.0f);
  const long long n = (long long)nx * ny * nz * nt;
  float lo = INFINITY, hi = -INFINITY;
  for (long long i = 0; i < n; i++) {
    lo = data[i] < lo ? data[i] : lo;
    hi = data[i] > hi ? data[i] : hi;
  }
  put<float>(h, 124, hi);  // cal_max
  put<float>(h, 128, lo);  // cal_min
  memcpy(h + 344, "n+1", 4);
  // h[348..351]: the extension flag, 0 (no extensions)
  const std::string p(path);
  const bool gz = ends_with(p, ".gz");
  if (gz) {
    gzFile f = gzopen(path, "wb6");
    if (!f) return fail(BRC_ERR_INVALID, p + ": cannot create");
    bool ok = gzwrite(f, h, 352) == 352;
    const unsigned char* src = reinterpret_cast<const unsigned char*>(data);
    size_t left = (size_t)n * 4, done = 0;
    while (ok && left > 0) {
      const size_t chunk = left > (1u << 30) ? (1u << 30) : left;
      ok = gzwrite(f, src + done, (unsigned)chunk) == (int)chunk;
      done += chunk;
      left -= chunk;
    }
    if (gzclose(f) != Z_OK) ok = false;
    return ok ? BRC_OK : fail(BRC_ERR_INVALID, p + ": write failed");
  }
  FILE* f = fopen(path, "wb");
  if (!f) return fail(BRC_ERR_INVALID, p + ": cannot create");
  bool ok = fwrite(h, 1, 352, f) == 352 && fwrite(data, 4, (size_t)n, f) == (size_t)n;
  if (fclose(f) != 0) ok = false;
  return ok ? BRC_OK : fail(BRC_ERR_INVALID, p + ": write failed");
}
