// L2-pipelined two-pass kernels, complex64, N = 2^15..2^20: tiles of 4096
// elements (32 KB, two CTAs per SM) and 8192 elements (64 KB, one CTA per
// SM), 16 elements per thread, three stage buffers.
#include "gfft_internal.h"
#include "kernels_l2pipe.cuh"

namespace gfft {
namespace {
struct RegL2PipeC64 {
  RegL2PipeC64() {
    reg_l2p_te<float2, 128, 256, 4096, 16, 3>();
    reg_l2p_te<float2, 256, 256, 4096, 16, 3>();
    reg_l2p_te<float2, 256, 512, 4096, 16, 3>();
    reg_l2p_te<float2, 512, 512, 4096, 16, 3>();
    reg_l2p_te<float2, 128, 256, 8192, 16, 3>();
    reg_l2p_te<float2, 256, 256, 8192, 16, 3>();
    reg_l2p_te<float2, 256, 512, 8192, 16, 3>();
    reg_l2p_te<float2, 512, 512, 8192, 16, 3>();
    reg_l2p_te<float2, 512, 1024, 8192, 16, 3>();
    reg_l2p_te<float2, 1024, 1024, 8192, 16, 3>();
  }
} reg_l2pipe_c64;
}  // namespace
}  // namespace gfft
