// Instantiation helper for k_pow2: one registry entry per (N, EPT, DIR).
#pragma once
#include "gfft_pow2.cuh"
#include "gfft_registry.h"

namespace gfft {

template <typename C, int N, int EPT, int DIR>
cudaError_t launch_pow2(const void* src, void* dst, int64_t count, int64_t idist, int64_t odist,
                        const void* tw, double scale, cudaStream_t st) {
  using S = Pow2Shape<N, EPT, sizeof(C)>;
  const int64_t blocks = (count + S::B - 1) / S::B;
  if (blocks <= 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  // co-resident CTAs on this device: the prefetch distance
  static const int64_t resident = resident_ctas(&k_pow2<C, N, EPT, DIR>, S::TPB, S::SMEM);
  const int64_t ahead = blocks > resident ? resident : 0;
  k_pow2<C, N, EPT, DIR><<<unsigned(blocks), S::TPB, S::SMEM, st>>>(
      static_cast<const C*>(src), static_cast<C*>(dst), count, idist, odist,
      static_cast<const C*>(tw), typename RealOf<C>::type(scale), ahead);
  return cudaGetLastError();
}

template <typename C, int N, int EPT, int DIR>
Pow2Kernel make_pow2() {
  using S = Pow2Shape<N, EPT, sizeof(C)>;
  Pow2Kernel k;
  k.prec = sizeof(C) == 8 ? kC64 : kC128;
  k.n = N;
  k.ept = EPT;
  k.dir = DIR;
  k.tpb = S::TPB;
  k.per_cta = S::B;
  k.smem = S::SMEM;
  k.func = reinterpret_cast<const void*>(&k_pow2<C, N, EPT, DIR>);
  k.launch = &launch_pow2<C, N, EPT, DIR>;
  return k;
}

template <typename C, int N, int EPT>
void reg_pow2_both() {
  register_pow2(make_pow2<C, N, EPT, -1>());
  register_pow2(make_pow2<C, N, EPT, +1>());
}

}  // namespace gfft
