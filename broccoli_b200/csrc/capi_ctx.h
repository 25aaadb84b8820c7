// capi_ctx.h -- the library context (struct brc_ctx) and the workspace and
// error helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "filter3d_tc.h"

#include "../../include/broccoli_b200.h"

// Grow-only device buffer.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
  cudaError_t ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

struct GraphKey {
  std::vector<unsigned long long> v;
  bool operator<(const GraphKey& o) const { return v < o.v; }
};

struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long kernels = 0;
  ~GraphEntry() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

struct brc_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  // stream on which the body of a registration graph's WHILE node is captured
  cudaStream_t body_stream = nullptr;
  cudaStream_t user_stream = nullptr;
  bool use_user_stream = false;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // host<->device copy streams of brc_motion_correct and their per-chunk
  // events (created on first use)
  static constexpr int kMaxChunks = 4;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_chunk_in[kMaxChunks] = {}, ev_chunk_done[kMaxChunks] = {};
  std::string last_error;
  unsigned long long launches = 0;
  DevBuf q1, q2, aligned, partials, ctl, tmp1, tmp2, series, corrected, params, rot, nl, pyr;
  // working volumes of the T1-to-template and cohort drivers, kept across
  // calls so that their addresses (and the captured graphs keyed by them)
  // stay the same from one call to the next
  DevBuf r2v_work, r2v_lin, r2v_prm, coh_res, coh_mat, coh_lin, coh_prm, coh_jobs;
  std::map<GraphKey, std::unique_ptr<GraphEntry>> graphs;
  // packed taps of the tensor-core filtering (split BF16, or the stored
  // half of TF32's structured-sparse rows), per filter bank and precision
  // (key: hash of the bank, its size and the precision); graphs may hold
  // these pointers, so an entry lives as long as the graphs do
  std::map<uint64_t, std::unique_ptr<DevBuf>> tc_taps;
  DevBuf tc_err;  // device int: a bounded wait of a tensor-core kernel gave up
  // device count of the iterations that registration graphs ran (their
  // loops stop on the device, so their kernel count is known only there)
  DevBuf iters_run;
  DevBuf smask;   // smoothed certainty of brc_smooth_normalized
  // tensor-core tile height chosen by timing, per (nfilt, W, H, D)
  std::map<std::tuple<int, int, int, int>, int> tc_tuned;
  std::map<std::tuple<int, int, int, int>, int> fp32_tuned;  // (nfilt + 100 sym, W, H, D) -> z depth
  std::map<std::tuple<int, int, int, int, int>, int> smooth_tuned;  // (W, H, D, batch, cert kind) -> z chunk
  // host arrays of the debug outputs (brc_ctx_set_debug_outputs)
  bool dbg_on = false;
  brc_debug_outputs dbg{};
  DevBuf dbg_q, dbg_v;  // device staging of the debug outputs

  cudaStream_t stream() const { return use_user_stream ? user_stream : own_stream; }

  cudaError_t ensure_copy_streams() {
    cudaError_t e = cudaSuccess;
    if (!copy_in && (e = cudaStreamCreateWithFlags(&copy_in, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if (!copy_out && (e = cudaStreamCreateWithFlags(&copy_out, cudaStreamNonBlocking)) != cudaSuccess) return e;
    for (int c = 0; c < kMaxChunks; c++) {
      if (!ev_chunk_in[c] &&
          (e = cudaEventCreateWithFlags(&ev_chunk_in[c], cudaEventDisableTiming)) != cudaSuccess)
        return e;
      if (!ev_chunk_done[c] &&
          (e = cudaEventCreateWithFlags(&ev_chunk_done[c], cudaEventDisableTiming)) != cudaSuccess)
        return e;
    }
    return e;
  }

  int fail(int status, const std::string& msg) {
    last_error = msg;
    return status;
  }
  int cuda(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return BRC_OK;
    last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? BRC_ERR_NOMEM : BRC_ERR_CUDA;
  }
  // Device copy of the packed taps of a bank (uploaded on first use; call
  // outside stream capture).
  int taps_for(const float* h_filters, int nfilt, bool tf32, const uint16_t** d_taps);
  // Reads and clears the tensor-core wait flag (synchronises the device).
  int check_tc_err();
  // Tile height of the tensor-core filtering for a shape: the fastest of the
  // cost model's candidates, timed once per shape (outside stream capture;
  // under capture the cost model's first choice).
  int tune_tc(int nfilt, int W, int H, int D, const uint16_t* d_taps, bool tf32, int* ty);
  // z depth of the FP32 filtering's output block for this shape and kind
  // of kernel (even/odd when sym and the bank is symmetric, else general):
  // the candidates timed once (outside stream capture), then cached.
  int tune_fp32(const float* h_filters, int nfilt, bool sym, int W, int H, int D, int* tz);
  // brc::smooth3d with the z chunk tuned per (shape, batch, certainty
  // kind): the first call of a key that writes a buffer it does not read
  // and does not accumulate (outside stream capture) runs every candidate
  // on its own buffers (the result is the same for each) and keeps the
  // fastest; an accumulating call given tune_out (batch volumes that
  // overlap nothing and may be overwritten) times the candidates without
  // accumulation into tune_out first.  Other calls take the tuned or the
  // untimed choice.
  int smooth(const float* vol, int W, int H, int D, int batch, const float* fx, const float* fy, const float* fz,
             const float* cert, const float* scert, float* tmp1, float* tmp2, float* out, cudaStream_t st,
             int accumulate = 0, float* tune_out = nullptr);

  size_t workspace() const {
    return q1.bytes + q2.bytes + aligned.bytes + partials.bytes + ctl.bytes + tmp1.bytes +
           tmp2.bytes + series.bytes + corrected.bytes + params.bytes + rot.bytes + nl.bytes + pyr.bytes +
           r2v_work.bytes + r2v_lin.bytes + r2v_prm.bytes + coh_res.bytes + coh_mat.bytes + coh_lin.bytes +
           coh_prm.bytes + coh_jobs.bytes;
  }
};

// The filtering kernel of one precision with what it needs, fixed before
// any stream capture (make_filter_path uploads the packed taps of the
// tensor-core path).
struct FilterPath {
  int precision = 0;
  const float* h_filters = nullptr;
  int nfilt = 3;
  const uint16_t* d_taps = nullptr;
  brc::tc::Geometry g{};
  int* d_err = nullptr;
  int tz = 0;  // FP32 filtering: z depth of the output block (0: untimed choice)
};
int make_filter_path(brc_ctx* ctx, const float* h_filters, int nfilt, int precision, int W, int H, int D,
                     FilterPath* fp);
inline bool brc_precision_valid(int p) {
  return p == BRC_PREC_FP32 || p == BRC_PREC_FP32_GENERAL || p == BRC_PREC_BF16X3 || p == BRC_PREC_TF32;
}
// Kernels one run_filter call launches.
inline int filter_launches(const FilterPath&) { return 1; }
cudaError_t run_filter(const FilterPath& fp, const float* vol, int W, int H, int D, int batch, long long stride,
                       float* out, brc::ActiveSet act, cudaStream_t st);
// Refuses debug writes while the context's stream is being captured.
int debug_capture_check(brc_ctx* ctx, const char* where);

#define BRC_CHECK_CTX(ctx) \
  do {                     \
    if (!(ctx)) return BRC_ERR_INVALID; \
  } while (0)

#define BRC_TRY(ctx, expr, where)                  \
  do {                                             \
    int _s = (ctx)->cuda((expr), (where));         \
    if (_s != BRC_OK) return _s;                   \
  } while (0)

