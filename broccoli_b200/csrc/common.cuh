// common.cuh -- shared definitions of the B200 registration/filtering kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace brc {

constexpr int kTaps = 343;          // 7 x 7 x 7
constexpr int kFilterFloats = 686;  // re[343] + im[343]
constexpr int kNParam = 12;
constexpr int kNSums = 42;          // 3 axes x (10 A sums + 4 h sums)
constexpr int kMaxFilters = 6;

// Filter bank passed to kernels by value (kernel parameter space).  Stored
// tap-major with the taps already reversed, so that coef[t][2k+c] is the
// weight that the sample at offset (dx,dy,dz) = (t%7-3, t/7%7-3, t/49-3)
// contributes to filter k's component c (0 re, 1 im): the reference's
// convolution uses F[(3-dx) + 7(3-dy) + 49(3-dz)] for that sample
// (kernelConvolution.cpp:2840-2858, broccoli_lib.cpp:5016-5017).
template <int NF>
struct FilterBank {
  float coef[kTaps * 2 * NF];
};

// Per-instance iteration control for batched registration.  An instance is
// skipped by every kernel of iteration `it` once conv_iter[b] < it; the solve
// kernel sets conv_iter[b] = it when that iteration's update fell below the
// tolerance, so the warp of that iteration still runs.
struct IterCtl {
  int* conv_iter;   // [batch], INT_MAX while active
  int* iterations;  // [batch], iterations run
};

__device__ __forceinline__ bool instance_done(const int* conv_iter, int b, int it) {
  return conv_iter != nullptr && __ldg(conv_iter + b) < it;
}

}  // namespace brc
