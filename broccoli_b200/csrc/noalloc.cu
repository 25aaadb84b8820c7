// noalloc.cu -- normal equations of the affine step without any device
// allocation: brc_normal_equations_noalloc.
//
// Some callers cannot let a library call cudaMalloc: processes whose device
// memory is reserved up front by a pooling allocator or a serving runtime
// (a cudaMalloc there can fail once the pool holds the HBM, or bypass the
// pool's accounting), and hosts that plan all memory before they start and
// forbid allocation afterwards.  This entry point needs no context and no
// workspace: the per-CTA partial sums live in a fixed device array that
// every GPU loading this library holds until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents.  Nothing in it has to start at zero: each call's reduction CTAs
// overwrite every row that the same call's assembly step then reads.  Calls
// that overlap on the GPU (different streams, or host threads, without
// ordering between them) race on the array and must not be issued.
#include <mutex>

#include "../../include/broccoli_b200.h"
#include "common.cuh"
#include "internal.h"

namespace {

// Fixed scratch: BRC_NOALLOC_PARTIAL_ROWS rows of 42 FP64 partial sums
// (1,032,192 bytes).
static __device__ __align__(256) double g_partials[BRC_NOALLOC_PARTIAL_ROWS * brc::kNSums];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, looked up
// once per device (the host-side symbol is only a stand-in).
cudaError_t scratch_address(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_addr[device] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess) return e;
    g_addr[device] = static_cast<double*>(p);
  }
  *out = g_addr[device];
  return cudaSuccess;
}

int pick_zpb(int W, int H) {
  const long long plane = (long long)(W > 6 ? W - 6 : 1) * (H > 6 ? H - 6 : 1);
  long long z = 4096 / (plane > 0 ? plane : 1);
  if (z < 1) z = 1;
  if (z > 64) z = 64;
  return (int)z;
}

}  // namespace

extern "C" int brc_normal_equations_noalloc(void* cuda_stream, const float* d_q1, long long q1_stride,
                                            const float* d_q2, int W, int H, int D, int batch,
                                            double* d_A, double* d_h) {
  if (!d_q1 || !d_q2 || !d_A || !d_h || W <= 0 || H <= 0 || D <= 0 || batch <= 0 || batch > 65535 ||
      (long long)W * H * D > (1ll << 31))
    return BRC_ERR_INVALID;
  const int zpb = pick_zpb(W, H);
  const int nint = D - 6 > 0 ? D - 6 : 1;
  const int nblk = (nint + zpb - 1) / zpb;
  if ((long long)nblk * batch > BRC_NOALLOC_PARTIAL_ROWS) return BRC_ERR_SCRATCH_LIMIT;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return BRC_ERR_NODEVICE;
  double* partials = nullptr;
  if (scratch_address(device, &partials) != cudaSuccess) return BRC_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  if (brc::normal_eq_partials(d_q1, q1_stride, d_q2, W, H, D, batch, partials, nblk, zpb, st) !=
      cudaSuccess)
    return BRC_ERR_CUDA;
  if (brc::assemble_normal_eq(partials, nblk, batch, d_A, d_h, st) != cudaSuccess) return BRC_ERR_CUDA;
  return BRC_OK;
}
