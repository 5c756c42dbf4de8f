// complex64 single-pass power-of-two kernels, N = 2 .. 16384.
#include "kernels_pow2.cuh"

namespace gfft {
namespace {
struct RegPow2C64 {
  RegPow2C64() {
    reg_pow2_both<float2, 2, 2>();
    reg_pow2_both<float2, 4, 4>();
    reg_pow2_both<float2, 8, 8>();
    reg_pow2_both<float2, 8, 4>();
    reg_pow2_both<float2, 16, 4>();
    reg_pow2_both<float2, 16, 8>();
    reg_pow2_both<float2, 16, 16>();
    reg_pow2_both<float2, 32, 4>();
    reg_pow2_both<float2, 32, 8>();
    reg_pow2_both<float2, 32, 16>();
    reg_pow2_both<float2, 64, 4>();
    reg_pow2_both<float2, 64, 8>();
    reg_pow2_both<float2, 64, 16>();
    reg_pow2_both<float2, 128, 8>();
    reg_pow2_both<float2, 128, 16>();
    reg_pow2_both<float2, 256, 8>();
    reg_pow2_both<float2, 256, 16>();
    reg_pow2_both<float2, 512, 8>();
    reg_pow2_both<float2, 512, 16>();
    reg_pow2_both<float2, 512, 32>();
    reg_pow2_both<float2, 1024, 8>();
    reg_pow2_both<float2, 1024, 16>();
    reg_pow2_both<float2, 1024, 32>();
    reg_pow2_both<float2, 2048, 8>();
    reg_pow2_both<float2, 2048, 16>();
    reg_pow2_both<float2, 2048, 32>();
    reg_pow2_both<float2, 4096, 8>();
    reg_pow2_both<float2, 4096, 16>();
    reg_pow2_both<float2, 4096, 32>();
    reg_pow2_both<float2, 8192, 8>();
    reg_pow2_both<float2, 8192, 16>();
    reg_pow2_both<float2, 8192, 32>();
    reg_pow2_both<float2, 16384, 16>();
    reg_pow2_both<float2, 16384, 32>();
  }
} reg_pow2_c64;
}  // namespace
}  // namespace gfft
