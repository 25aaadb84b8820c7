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
//
// Under lazy module loading (the CUDA 12.2+ default) the array is allocated
// when the module is first used on a device, not when the library loads.  A
// process that hands its HBM to a pool should therefore make one set-up
// call (batch = 0) on each device before the pool reserves the memory, or
// run with CUDA_MODULE_LOADING=EAGER, which allocates the array at load
// time.  Otherwise that first call may fail with BRC_ERR_NOMEM.  The
// address is cached per device; after cudaDeviceReset make a set-up call
// again before the next call on that device.
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

// Device address of the scratch array on `device` (current), looked up once
// per device at set-up and cached; the host-side symbol is only a stand-in.
// refresh = true repeats the lookup: after cudaDeviceReset the module is
// loaded again, possibly at another address.  Under lazy module loading (the
// CUDA 12.2+ default) the first lookup on a device loads the module and
// allocates the array.
cudaError_t scratch_address(int device, bool refresh, double** out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_addr[device] == nullptr || refresh) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess) {
      g_addr[device] = nullptr;
      return e;
    }
    g_addr[device] = static_cast<double*>(p);
  }
  *out = g_addr[device];
  return cudaSuccess;
}

int status_of(cudaError_t e) {
  return e == cudaSuccess ? BRC_OK : (e == cudaErrorMemoryAllocation ? BRC_ERR_NOMEM : BRC_ERR_CUDA);
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
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return BRC_ERR_NODEVICE;
  if (st != nullptr) {
    // the scratch address belongs to the current device: a stream of another
    // device would launch the kernels against the wrong memory
    int sdev = -1;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess || sdev != device) return BRC_ERR_INVALID;
  }
  if (batch == 0) {
    // set-up only: (re)resolve the array on this device, loading the module
    // under lazy loading
    double* partials = nullptr;
    return status_of(scratch_address(device, true, &partials));
  }
  if (!d_q1 || !d_q2 || !d_A || !d_h || W <= 0 || H <= 0 || D <= 0 || batch < 0 || batch > 65535 ||
      (long long)W * H * D > (1ll << 31))
    return BRC_ERR_INVALID;
  const int zpb = pick_zpb(W, H);
  const int nint = D - 6 > 0 ? D - 6 : 1;
  const int nblk = (nint + zpb - 1) / zpb;
  if ((long long)nblk * batch > BRC_NOALLOC_PARTIAL_ROWS) return BRC_ERR_SCRATCH_LIMIT;
  double* partials = nullptr;
  const cudaError_t e = scratch_address(device, false, &partials);
  if (e != cudaSuccess) return status_of(e);
  if (brc::normal_eq_partials(d_q1, q1_stride, d_q2, W, H, D, batch, partials, nblk, zpb, st) !=
      cudaSuccess)
    return BRC_ERR_CUDA;
  if (brc::assemble_normal_eq(partials, nblk, batch, d_A, d_h, st) != cudaSuccess) return BRC_ERR_CUDA;
  return BRC_OK;
}
