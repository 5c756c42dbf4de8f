// Power-of-two column batches: FFTs of length L <= 4096 down columns whose
// rows are `pitch` elements apart (the strided batches of
// gfft_exec_strided_batch and every non-contiguous axis of the N-D plans,
// plan_strided.go:35-99, plan_2d.go:161-400, plan_nd.go:188-460).  A CTA
// owns a tile of NC adjacent columns of one array, so each row of the tile
// is one run of NC contiguous elements in HBM; the column FFTs run the
// compile-time register/shared-memory stages of the two-pass kernel
// (col_stage) with the pitch taken at run time, reading and writing the
// columns in place of their natural order.  Lengths that are not powers of
// two use the runtime-radix column kernel.
#include "gfft_internal.h"
#include "gfft_twopass.cuh"

namespace gfft {
namespace {

// NC = columns per tile: about 8192 (complex64) / 4096 (complex128)
// elements per tile, 4..32 columns (32-byte rows at least); EPT as the
// two-pass tile rule.
template <typename C, int L>
struct ColTile {
  static constexpr int TE = sizeof(C) == 8 ? 8192 : 4096;
  static constexpr int NC0 = TE / L < 4 ? (sizeof(C) == 8 ? 4 : 2) : (TE / L > 32 ? 32 : TE / L);
  static constexpr int NC = NC0;
  static constexpr int EPT = (L / 16 >= 8) ? 16 : (L / 8 >= 2 ? L / 8 : 2);
  using S = ColShape<L, EPT, NC, sizeof(C)>;
};

template <typename C, int L, int DIR>
__global__ void __launch_bounds__(ColTile<C, L>::S::TPB)
k_pow2_cols(const C* src, C* dst, int64_t ncols, int64_t pitch, int64_t dist, int64_t tiles_per_array,
            const C* __restrict__ tw, typename RealOf<C>::type scale) {
  using T = ColTile<C, L>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  const int64_t arr = blockIdx.x / tiles_per_array;
  const int64_t col0 = (blockIdx.x % tiles_per_array) * int64_t(T::NC);
  const int c = threadIdx.x % T::NC, t = threadIdx.x / T::NC;
  const bool active = col0 + c < ncols && threadIdx.x < T::S::TPB;
  const C* in = src + arr * dist + col0;
  C* out = dst + arr * dist + col0;
  const BigTwiddle bt{nullptr, nullptr, 0};
  C v[T::EPT];
  col_stage<C, L, T::EPT, T::NC, DIR, 1, LOAD_STREAM, OUT_COLUMNS, 0, 0>(v, in, out, sh, t, c, active, tw, scale, bt,
                                                                         0, pitch);
}

template <typename C, int L, int DIR>
cudaError_t launch_cols(const void* src, void* dst, int64_t count, int64_t dist, int64_t ncols, int64_t pitch,
                        const void* tw, double scale, cudaStream_t st) {
  using T = ColTile<C, L>;
  static const cudaError_t attr =
      T::S::SMEM > 48 * 1024
          ? cudaFuncSetAttribute(&k_pow2_cols<C, L, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, T::S::SMEM)
          : cudaSuccess;
  if (attr != cudaSuccess) return attr;
  const int64_t tpa = (ncols + T::NC - 1) / T::NC;
  const int64_t tiles = tpa * count;
  if (tiles <= 0) return cudaSuccess;
  if (tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  k_pow2_cols<C, L, DIR><<<unsigned(tiles), T::S::TPB, T::S::SMEM, st>>>(
      static_cast<const C*>(src), static_cast<C*>(dst), ncols, pitch, dist, tpa, static_cast<const C*>(tw),
      typename RealOf<C>::type(scale));
  return cudaGetLastError();
}

using ColFn = cudaError_t (*)(const void*, void*, int64_t, int64_t, int64_t, int64_t, const void*, double,
                              cudaStream_t);

template <typename C, int DIR>
ColFn pick(int64_t L) {
  switch (L) {
    case 2: return &launch_cols<C, 2, DIR>;
    case 4: return &launch_cols<C, 4, DIR>;
    case 8: return &launch_cols<C, 8, DIR>;
    case 16: return &launch_cols<C, 16, DIR>;
    case 32: return &launch_cols<C, 32, DIR>;
    case 64: return &launch_cols<C, 64, DIR>;
    case 128: return &launch_cols<C, 128, DIR>;
    case 256: return &launch_cols<C, 256, DIR>;
    case 512: return &launch_cols<C, 512, DIR>;
    case 1024: return &launch_cols<C, 1024, DIR>;
    case 2048: return &launch_cols<C, 2048, DIR>;
    case 4096: return &launch_cols<C, 4096, DIR>;
  }
  return nullptr;
}

}  // namespace

bool pow2_cols_supported(int64_t n) { return n >= 2 && n <= 4096 && (n & (n - 1)) == 0; }

cudaError_t exec_pow2_cols(int prec, int dir, void* dst, const void* src, int64_t count, int64_t dist, int64_t ncols,
                           int64_t pitch, const void* tw_n, int64_t n, cudaStream_t st) {
  ColFn f = prec == kC64 ? (dir < 0 ? pick<float2, -1>(n) : pick<float2, 1>(n))
                         : (dir < 0 ? pick<double2, -1>(n) : pick<double2, 1>(n));
  if (!f) return cudaErrorNotSupported;
  return f(src, dst, count, dist, ncols, pitch, tw_n, dir < 0 ? 1.0 : 1.0 / double(n), st);
}

}  // namespace gfft
