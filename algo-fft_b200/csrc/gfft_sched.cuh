// Compile-time Stockham schedule of a power-of-two length L with EPT
// elements per thread: stage s has prefix product P (1, EPT, EPT^2, ...) and
// radix RS = EPT, except the last, which takes the remaining factor L/P.
#pragma once
#include "gfft_math.cuh"
#include "gfft_registry.h"

namespace gfft {

template <int L, int EPT>
struct Sched {
  __host__ __device__ static constexpr int radix_at(int P) { return (P * EPT <= L) ? EPT : L / P; }
  __host__ __device__ static constexpr int num_stages() {
    int s = 0;
    for (int p = 1; p < L; p *= radix_at(p)) ++s;
    return s;
  }
};

}  // namespace gfft
