// TMA-staged three-pass kernels, complex64, N = 2^21..2^24: tiles of 8192
// and 4096 elements, 16 elements per thread, three stage buffers.
#include "gfft_internal.h"
#include "kernels_cols_tma.cuh"

namespace gfft {
namespace {
template <int TE, int EMAX, int NST>
void reg_shapes() {
  reg_tp3t<float2, 128, 128, 128, TE, EMAX, NST>();
  reg_tp3t<float2, 256, 128, 128, TE, EMAX, NST>();
  reg_tp3t<float2, 256, 256, 128, TE, EMAX, NST>();
  reg_tp3t<float2, 256, 256, 256, TE, EMAX, NST>();
}
struct RegThreePassTmaC64 {
  RegThreePassTmaC64() {
    reg_shapes<8192, 16, 3>();
    reg_shapes<4096, 16, 3>();
  }
} reg_threepass_tma_c64;
}  // namespace
}  // namespace gfft
