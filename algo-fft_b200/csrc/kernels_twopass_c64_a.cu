// complex64 two-pass kernels, N = N1*N2 with N1 = 2^floor(log2 N / 2); tile variants
// (elements per tile, max elements per thread): 8192/16, 4096/16.
#include "kernels_twopass.cuh"

namespace gfft {
namespace {
struct RegTwoPassc64a {
  RegTwoPassc64a() {
    reg_twopass_both<float2, 32, 64, 8192, 16>();
    reg_twopass_both<float2, 64, 64, 8192, 16>();
    reg_twopass_both<float2, 64, 128, 8192, 16>();
    reg_twopass_both<float2, 128, 128, 8192, 16>();
    reg_twopass_both<float2, 128, 256, 8192, 16>();
    reg_twopass_both<float2, 256, 256, 8192, 16>();
    reg_twopass_both<float2, 256, 512, 8192, 16>();
    reg_twopass_both<float2, 512, 512, 8192, 16>();
    reg_twopass_both<float2, 512, 1024, 8192, 16>();
    reg_twopass_both<float2, 1024, 1024, 8192, 16>();
    reg_twopass_both<float2, 1024, 2048, 8192, 16>();
    reg_twopass_both<float2, 2048, 2048, 8192, 16>();
    reg_twopass_both<float2, 2048, 4096, 8192, 16>();
    reg_twopass_both<float2, 4096, 4096, 8192, 16>();
    reg_twopass_both<float2, 32, 64, 4096, 16>();
    reg_twopass_both<float2, 64, 64, 4096, 16>();
    reg_twopass_both<float2, 64, 128, 4096, 16>();
    reg_twopass_both<float2, 128, 128, 4096, 16>();
    reg_twopass_both<float2, 128, 256, 4096, 16>();
    reg_twopass_both<float2, 256, 256, 4096, 16>();
    reg_twopass_both<float2, 256, 512, 4096, 16>();
    reg_twopass_both<float2, 512, 512, 4096, 16>();
    reg_twopass_both<float2, 512, 1024, 4096, 16>();
    reg_twopass_both<float2, 1024, 1024, 4096, 16>();
    reg_twopass_both<float2, 1024, 2048, 4096, 16>();
    reg_twopass_both<float2, 2048, 2048, 4096, 16>();
    reg_twopass_both<float2, 2048, 4096, 4096, 16>();
    reg_twopass_both<float2, 4096, 4096, 4096, 16>();
  }
} reg_twopass_c64a;
}  // namespace
}  // namespace gfft
