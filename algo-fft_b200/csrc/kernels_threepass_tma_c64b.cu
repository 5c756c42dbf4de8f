// TMA-staged three-pass kernels, complex64: shallower pipelines (two stage
// buffers, more CTAs per SM).
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
struct RegThreePassTmaC64b {
  RegThreePassTmaC64b() {
    reg_shapes<4096, 16, 2>();
  }
} reg_threepass_tma_c64b;
}  // namespace
}  // namespace gfft
