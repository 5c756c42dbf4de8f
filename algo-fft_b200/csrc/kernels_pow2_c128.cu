// complex128 single-pass power-of-two kernels, N = 2 .. 8192.
#include "kernels_pow2.cuh"

namespace gfft {
namespace {
struct RegPow2C128 {
  RegPow2C128() {
    reg_pow2_both<double2, 2, 2>();
    reg_pow2_both<double2, 4, 4>();
    reg_pow2_both<double2, 8, 8>();
    reg_pow2_both<double2, 8, 4>();
    reg_pow2_both<double2, 16, 4>();
    reg_pow2_both<double2, 16, 8>();
    reg_pow2_both<double2, 16, 16>();
    reg_pow2_both<double2, 32, 4>();
    reg_pow2_both<double2, 32, 8>();
    reg_pow2_both<double2, 32, 16>();
    reg_pow2_both<double2, 64, 4>();
    reg_pow2_both<double2, 64, 8>();
    reg_pow2_both<double2, 64, 16>();
    reg_pow2_both<double2, 128, 8>();
    reg_pow2_both<double2, 128, 16>();
    reg_pow2_both<double2, 256, 8>();
    reg_pow2_both<double2, 256, 16>();
    reg_pow2_both<double2, 512, 8>();
    reg_pow2_both<double2, 512, 16>();
    reg_pow2_both<double2, 1024, 8>();
    reg_pow2_both<double2, 1024, 16>();
    reg_pow2_both<double2, 2048, 8>();
    reg_pow2_both<double2, 2048, 16>();
    reg_pow2_both<double2, 4096, 8>();
    reg_pow2_both<double2, 4096, 16>();
    reg_pow2_both<double2, 8192, 8>();
    reg_pow2_both<double2, 8192, 16>();
  }
} reg_pow2_c128;
}  // namespace
}  // namespace gfft
