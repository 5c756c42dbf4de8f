// TMA-staged three-pass kernels, complex128, N = 2^21..2^24: tiles of 4096
// and 2048 elements, 8 elements per thread, two or three stage buffers.
#include "gfft_internal.h"
#include "kernels_cols_tma.cuh"

namespace gfft {
namespace {
template <int TE, int EMAX, int NST>
void reg_shapes() {
  reg_tp3t<double2, 128, 128, 128, TE, EMAX, NST>();
  reg_tp3t<double2, 256, 128, 128, TE, EMAX, NST>();
  reg_tp3t<double2, 256, 256, 128, TE, EMAX, NST>();
  reg_tp3t<double2, 256, 256, 256, TE, EMAX, NST>();
}
struct RegThreePassTmaC128 {
  RegThreePassTmaC128() {
    reg_shapes<4096, 8, 3>();
    reg_shapes<2048, 8, 3>();
    reg_shapes<2048, 8, 2>();
  }
} reg_threepass_tma_c128;
}  // namespace
}  // namespace gfft
