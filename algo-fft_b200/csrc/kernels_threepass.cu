// Three-pass kernels (N = N1 x M1 x M2, every factor <= 256) for complex64
// and complex128, N = 2^21..2^24.  Tiles: 8192 (complex64) / 4096
// (complex128) elements, columns = tile / length (2..64), 16 / 8 elements
// per thread at most.
#include "gfft_internal.h"
#include "gfft_threepass.cuh"
#include "kernels_twopass.cuh"

namespace gfft {
namespace {

template <typename C, int N1, int M1, int M2, int DIR>
struct Tp3Of {
  static constexpr int TE = sizeof(C) == 8 ? 8192 : 4096, EMAX = sizeof(C) == 8 ? 16 : 8;
  using A = TileRule<TE, EMAX, N1>;
  using B = TileRule<TE, EMAX, M1>;
  using D = TileRule<TE, EMAX, M2>;
  using TP = ThreePass<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, DIR>;
  template <int PASS>
  static const void* fn() {
    return reinterpret_cast<const void*>(&k_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, DIR, PASS>);
  }
  static cudaError_t launch(const ThreePassParams& p, int pass, int64_t b0, int64_t nb, cudaStream_t st) {
    const int64_t tiles = nb * (pass == 1 ? TP::TILES1 : pass == 2 ? TP::TILES2 : TP::TILES3);
    if (tiles <= 0) return cudaSuccess;
    if (tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const unsigned g = unsigned(tiles);
    if (pass == 1)
      k_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, DIR, 1><<<g, TP::TPB, TP::SMEM, st>>>(p, b0);
    else if (pass == 2)
      k_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, DIR, 2><<<g, TP::TPB, TP::SMEM, st>>>(p, b0);
    else
      k_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, DIR, 3><<<g, TP::TPB, TP::SMEM, st>>>(p, b0);
    return cudaGetLastError();
  }
};

template <typename C, int N1, int M1, int M2>
void reg_tp3() {
  for (int d = 0; d < 2; ++d) {
    ThreePassKernel k;
    k.prec = sizeof(C) == 8 ? kC64 : kC128;
    k.n1 = N1;
    k.m1 = M1;
    k.m2 = M2;
    k.dir = d == 0 ? -1 : 1;
    if (d == 0) {
      using T = Tp3Of<C, N1, M1, M2, -1>;
      k.tpb = T::TP::TPB;
      k.smem = T::TP::SMEM;
      k.func[0] = T::template fn<1>();
      k.func[1] = T::template fn<2>();
      k.func[2] = T::template fn<3>();
      k.launch = &T::launch;
    } else {
      using T = Tp3Of<C, N1, M1, M2, 1>;
      k.tpb = T::TP::TPB;
      k.smem = T::TP::SMEM;
      k.func[0] = T::template fn<1>();
      k.func[1] = T::template fn<2>();
      k.func[2] = T::template fn<3>();
      k.launch = &T::launch;
    }
    register_threepass(k);
  }
}

struct RegThreePass {
  RegThreePass() {
    reg_tp3<float2, 128, 128, 128>();
    reg_tp3<float2, 256, 128, 128>();
    reg_tp3<float2, 256, 256, 128>();
    reg_tp3<float2, 256, 256, 256>();
    reg_tp3<double2, 128, 128, 128>();
    reg_tp3<double2, 256, 128, 128>();
    reg_tp3<double2, 256, 256, 128>();
    reg_tp3<double2, 256, 256, 256>();
  }
} reg_threepass;

}  // namespace
}  // namespace gfft
