// complex128 two-pass kernels, N = N1*N2 with N1 = 2^floor(log2 N / 2); tile variants
// (elements per tile, max elements per thread): 4096/8, 2048/8, 4096/16.
#include "kernels_twopass.cuh"

namespace gfft {
namespace {
struct RegTwoPassc128 {
  RegTwoPassc128() {
    reg_twopass_both<double2, 32, 64, 4096, 8>();
    reg_twopass_both<double2, 64, 64, 4096, 8>();
    reg_twopass_both<double2, 64, 128, 4096, 8>();
    reg_twopass_both<double2, 128, 128, 4096, 8>();
    reg_twopass_both<double2, 128, 256, 4096, 8>();
    reg_twopass_both<double2, 256, 256, 4096, 8>();
    reg_twopass_both<double2, 256, 512, 4096, 8>();
    reg_twopass_both<double2, 512, 512, 4096, 8>();
    reg_twopass_both<double2, 512, 1024, 4096, 8>();
    reg_twopass_both<double2, 1024, 1024, 4096, 8>();
    reg_twopass_both<double2, 1024, 2048, 4096, 8>();
    reg_twopass_both<double2, 2048, 2048, 4096, 8>();
    reg_twopass_both<double2, 2048, 4096, 4096, 8>();
    reg_twopass_both<double2, 4096, 4096, 4096, 8>();
    reg_twopass_both<double2, 32, 64, 2048, 8>();
    reg_twopass_both<double2, 64, 64, 2048, 8>();
    reg_twopass_both<double2, 64, 128, 2048, 8>();
    reg_twopass_both<double2, 128, 128, 2048, 8>();
    reg_twopass_both<double2, 128, 256, 2048, 8>();
    reg_twopass_both<double2, 256, 256, 2048, 8>();
    reg_twopass_both<double2, 256, 512, 2048, 8>();
    reg_twopass_both<double2, 512, 512, 2048, 8>();
    reg_twopass_both<double2, 512, 1024, 2048, 8>();
    reg_twopass_both<double2, 1024, 1024, 2048, 8>();
    reg_twopass_both<double2, 1024, 2048, 2048, 8>();
    reg_twopass_both<double2, 2048, 2048, 2048, 8>();
    reg_twopass_both<double2, 2048, 4096, 2048, 8>();
    reg_twopass_both<double2, 4096, 4096, 2048, 8>();
    reg_twopass_both<double2, 32, 64, 4096, 16>();
    reg_twopass_both<double2, 64, 64, 4096, 16>();
    reg_twopass_both<double2, 64, 128, 4096, 16>();
    reg_twopass_both<double2, 128, 128, 4096, 16>();
    reg_twopass_both<double2, 128, 256, 4096, 16>();
    reg_twopass_both<double2, 256, 256, 4096, 16>();
    reg_twopass_both<double2, 256, 512, 4096, 16>();
    reg_twopass_both<double2, 512, 512, 4096, 16>();
    reg_twopass_both<double2, 512, 1024, 4096, 16>();
    reg_twopass_both<double2, 1024, 1024, 4096, 16>();
    reg_twopass_both<double2, 1024, 2048, 4096, 16>();
    reg_twopass_both<double2, 2048, 2048, 4096, 16>();
    reg_twopass_both<double2, 2048, 4096, 4096, 16>();
    reg_twopass_both<double2, 4096, 4096, 4096, 16>();
  }
} reg_twopass_c128;
}  // namespace
}  // namespace gfft
