// filter3d_tc.h -- host interface of the tcgen05 filtering kernel (split
// BF16 or TF32; filter3d_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "common.cuh"

namespace brc {
namespace tc {

constexpr int kM = 128;    // GEMM M: (stacked plane, real filter, x offset) rows
constexpr int kK = 16;     // GEMM K: input samples along x per window
constexpr int kXo = 10;    // outputs along x per window (kK - 6)
constexpr int kMaxN = 256; // GEMM N limit (rows of one tile)
// TF32 runs structured-sparse MMAs whose metadata takes one TMEM column
// beyond both accumulators: N at most 240
constexpr int kMaxNSparse = 240;

// Tile geometry of one launch, chosen on the host.  The kernel is
// persistent (one CTA per SM over all tiles of the launch).
struct Geometry {
  int SP;      // output planes stacked along M (2 for 3 filters, 1 for 6)
  int Ty;      // output rows along y per tile
  int Hp;      // Ty + 6: input rows per plane
  int J;       // plane groups per tile (tile = SP*J output planes)
  int N;       // GEMM N, multiple of 16, >= J*Hp
  int RP;      // shared-memory rows per plane-parity array
  int NR;      // SP * RP
  int nstage;  // GEMMs per tile: (7 + SP - 1) * 7
  int smem;    // dynamic shared memory bytes of a CTA
  int maxN;    // N limit of the precision (kMaxN, or kMaxNSparse for TF32)
};

int stacked_planes(int nfilt);
int num_stages(int nfilt);
// Bytes of the packed Toeplitz taps (split BF16, or TF32: the stored half
// of the structured-sparse rows, half the bytes) of a bank of nfilt (3 or
// 6) complex filters, and the packing itself (dst holds
// packed_tap_bytes/2 16-bit words).
size_t packed_tap_bytes(int nfilt, bool tf32);
void pack_taps(const float* h_filters, int nfilt, uint16_t* dst, bool tf32);
// The 32-bit sparsity-metadata word that the TF32 kernel writes to TMEM
// lane `lane` (0..127) of its metadata column: which sample of each pair
// (P, P + 8) a packed row keeps.
uint32_t metadata_word(int lane, int SP, int nfilt);
Geometry make_geometry(int nfilt, int H, int D, int Ty, bool tf32);
bool geometry_ok(const Geometry& g);
// The max_n cheapest tile heights by the cost model, cheapest first; returns
// how many were found.  pick_ty is the cheapest.
int candidate_tys(int nfilt, int H, int D, int* tys, int max_n, bool tf32);
int pick_ty(int nfilt, int H, int D, bool tf32);
cudaError_t init();
// One CTA waits wait_ms (1..1000) on a barrier nothing completes, then sets *d_err.
cudaError_t bounded_wait_probe(int wait_ms, int* d_err, cudaStream_t st);
cudaError_t launch(const float* vol, int W, int H, int D, int batch, long long stride, const uint16_t* d_taps,
                   int nfilt, float* out, ActiveSet act, int* d_err, const Geometry& g, cudaStream_t st,
                   bool tf32);

}  // namespace tc
}  // namespace brc
