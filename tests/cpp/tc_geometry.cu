// Host check of the tensor-core filtering's tile geometries (no GPU needed;
// built with nvcc because the library's internal header holds device code,
// but only host functions run).
//
// For banks of 3 and 6 filters, both tensor-core precisions and a grid of
// volume heights and depths, every tile height the cost model offers must
// give a launchable geometry:
//   N a multiple of 16, at least the J plane groups' J (Ty + 6) rows, at
//     most the precision's limit (256; 240 for TF32, whose sparsity
//     metadata takes a TMEM column beyond both accumulators);
//   every B row a GEMM reads inside the plane-parity array (start row up to
//     qmax (Ty + 6) + 6, then N rows);
//   shared memory within the 227 KB of a CTA;
//   no more plane groups than the volume needs, and Ty <= H.
// pick_ty must be the first candidate.  Prints "ok" and exits 0, or names
// the first bad geometry and exits 1.
#include <cstdio>

#include "../../broccoli_b200/csrc/filter3d_tc.h"

int main() {
  using namespace brc::tc;
  const int hs[] = {1, 2, 3, 7, 9, 10, 12, 17, 33, 40, 64, 65, 91, 109, 128, 170, 218, 230, 234, 256, 300};
  const int ds[] = {1, 2, 3, 4, 7, 13, 33, 64, 91, 182, 256};
  long long checked = 0;
  for (int nfilt : {3, 6})
    for (bool tf32 : {false, true})
      for (int H : hs)
        for (int D : ds) {
          int tys[3];
          const int n = candidate_tys(nfilt, H, D, tys, 3, tf32);
          if (n < 1) {
            std::fprintf(stderr, "nfilt %d tf32 %d H %d D %d: no candidate\n", nfilt, (int)tf32, H, D);
            return 1;
          }
          if (pick_ty(nfilt, H, D, tf32) != tys[0]) {
            std::fprintf(stderr, "nfilt %d tf32 %d H %d D %d: pick_ty is not the first candidate\n", nfilt,
                         (int)tf32, H, D);
            return 1;
          }
          const int limit = tf32 ? kMaxNSparse : kMaxN;
          for (int c = 0; c < n; c++) {
            const Geometry g = make_geometry(nfilt, H, D, tys[c], tf32);
            const int SP = stacked_planes(nfilt);
            const int qmax = (5 + SP) / SP;
            const int jmax = (D + SP - 1) / SP;
            const bool good = geometry_ok(g) && g.SP == SP && g.maxN == limit && g.Ty >= 1 && g.Ty <= H &&
                              g.Hp == g.Ty + 6 && g.J >= 1 && g.J <= jmax && g.N % 16 == 0 &&
                              g.N >= g.J * g.Hp && g.N >= 16 && g.N <= limit &&
                              g.RP >= qmax * g.Hp + 6 + g.N && g.NR == SP * g.RP &&
                              g.nstage == num_stages(nfilt) && g.smem <= 227 * 1024;
            if (!good) {
              std::fprintf(stderr,
                           "nfilt %d tf32 %d H %d D %d Ty %d: SP %d Hp %d J %d N %d RP %d NR %d smem %d maxN %d\n",
                           nfilt, (int)tf32, H, D, tys[c], g.SP, g.Hp, g.J, g.N, g.RP, g.NR, g.smem, g.maxN);
              return 1;
            }
            checked++;
          }
        }
  std::printf("ok %lld\n", checked);
  return 0;
}
