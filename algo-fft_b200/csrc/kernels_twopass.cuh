// Instantiation helper for k_twopass.
#pragma once
#include "gfft_registry.h"
#include "gfft_twopass.cuh"

namespace gfft {

template <typename C, int N1, int EPT1, int NC1, int N2, int EPT2, int NC2, int DIR>
cudaError_t launch_twopass(const TwoPassParams& p, int grid, cudaStream_t st) {
  using TP = TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>;
  k_twopass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR><<<grid, TP::TPB, TP::SMEM, st>>>(p);
  return cudaGetLastError();
}

template <typename C, int N1, int EPT1, int NC1, int N2, int EPT2, int NC2, int DIR>
cudaError_t launch_tp_split(const TwoPassParams& p, int pass, int64_t b0, int64_t nb, cudaStream_t st) {
  using TP = TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>;
  const int64_t blocks = nb * (pass == 1 ? TP::TILES1 : TP::TILES2);
  if (blocks <= 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  if (pass == 1)
    k_tp_split<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR, 1><<<unsigned(blocks), TP::TPB, TP::SMEM, st>>>(p, b0);
  else
    k_tp_split<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR, 2><<<unsigned(blocks), TP::TPB, TP::SMEM, st>>>(p, b0);
  return cudaGetLastError();
}

template <typename C, int N1, int EPT1, int NC1, int N2, int EPT2, int NC2, int DIR>
TwoPassKernel make_twopass() {
  using TP = TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>;
  TwoPassKernel k;
  k.prec = sizeof(C) == 8 ? kC64 : kC128;
  k.n1 = N1;
  k.n2 = N2;
  k.dir = DIR;
  k.tpb = TP::TPB;
  k.smem = TP::SMEM;
  k.nc1 = NC1;
  k.nc2 = NC2;
  k.func = reinterpret_cast<const void*>(&k_twopass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>);
  k.launch = &launch_twopass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>;
  k.split_func[0] = reinterpret_cast<const void*>(&k_tp_split<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR, 1>);
  k.split_func[1] = reinterpret_cast<const void*>(&k_tp_split<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR, 2>);
  k.split = &launch_tp_split<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>;
  return k;
}

// Tile shape rule of a variant: TE elements per tile, NC = TE / L columns
// (capped at 64, at least 2), EPT = EMAX with at least 8 threads per column.
template <int TE, int EMAX, int L>
struct TileRule {
  static constexpr int NC0 = TE / L;
  static constexpr int NC = NC0 > 64 ? 64 : (NC0 < 2 ? 2 : NC0);
  static constexpr int EPT = (L / EMAX >= 8) ? EMAX : (L / 8 >= 2 ? L / 8 : 2);
};

template <typename C, int N1, int N2, int TE, int EMAX>
void reg_twopass_both() {
  using A = TileRule<TE, EMAX, N1>;
  using B = TileRule<TE, EMAX, N2>;
  TwoPassKernel f = make_twopass<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, -1>();
  TwoPassKernel i = make_twopass<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, +1>();
  f.te = i.te = TE;
  f.emax = i.emax = EMAX;
  register_twopass(f);
  register_twopass(i);
}

}  // namespace gfft
