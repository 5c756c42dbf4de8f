// Fused Bluestein chain for FFT lengths M that one CTA transforms (M <=
// 16384 complex64, <= 8192 complex128): chirp multiply and zero pad in the
// first Stockham stage's loads, FFT_M, the filter product in shared memory,
// the inverse FFT_M, and the chirp multiply (with 1/M, and 1/n for the
// inverse) in the last stage's stores -- one launch, one read and one write
// of the n user elements per transform (plan_bluestein.go:7-58,
// internal/kernels/bluestein.go:20-77 run the same chain as five passes).
#include <vector>
#include "gfft_internal.h"
#include "gfft_pow2.cuh"

namespace gfft {
namespace {

template <typename C>
struct ChirpLoad {
  static constexpr bool kShared = false;
  const C* x;
  const C* w;
  int n;
  bool valid;
  __device__ __forceinline__ C operator()(int e) const {
    return (valid && e < n) ? cmul(ld_stream(x + e), __ldg(w + e)) : C{0, 0};
  }
};

template <typename C, int M, int EPT>
struct RowStore {
  static constexpr bool kShared = true;
  C* sh;
  __device__ __forceinline__ void operator()(int e, C v) const { sh[Pow2Shape<M, EPT, sizeof(C)>::pad(e)] = v; }
};

template <typename C, int M, int EPT>
struct RowLoad {
  static constexpr bool kShared = true;
  const C* sh;
  __device__ __forceinline__ C operator()(int e) const { return sh[Pow2Shape<M, EPT, sizeof(C)>::pad(e)]; }
};

template <typename C>
struct ChirpStore {
  static constexpr bool kShared = false;
  C* y;
  const C* w;
  int n;
  typename RealOf<C>::type scale;
  bool valid;
  __device__ __forceinline__ void operator()(int e, C v) const {
    if (valid && e < n) st_stream(y + e, cscale(cmul(v, __ldg(w + e)), scale));
  }
};

// chirp / filt: the direction's chirp (n) and filter spectrum (M);
// tw: W_M^m, m < M.
template <typename C, int M, int EPT>
__global__ void __launch_bounds__(Pow2Shape<M, EPT, sizeof(C)>::TPB)
k_bs_fused(const C* src, C* dst, int64_t count, int64_t idist, int64_t odist, int n, const C* __restrict__ chirp,
           const C* __restrict__ filt, const C* __restrict__ tw, typename RealOf<C>::type scale) {
  using S = Pow2Shape<M, EPT, sizeof(C)>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw) + (threadIdx.x / S::T) * S::STRIDE;
  const int t = threadIdx.x % S::T;
  const int64_t b = int64_t(blockIdx.x) * S::B + threadIdx.x / S::T;
  const bool valid = b < count;
  ChirpLoad<C> ld{src + (valid ? b * idist : 0), chirp, n, valid};
  RowStore<C, M, EPT> st{sh};
  pow2_fft<C, M, EPT, -1>(sh, t, tw, ld, st);
  xsync<S::T>();
#pragma unroll
  for (int i = 0; i < EPT; ++i) {  // every bin has one owner thread
    const int k = t + i * S::T;
    sh[S::pad(k)] = cmul(sh[S::pad(k)], __ldg(filt + k));
  }
  xsync<S::T>();
  RowLoad<C, M, EPT> ld2{sh};
  ChirpStore<C> st2{dst + (valid ? b * odist : 0), chirp, n, scale, valid};
  pow2_fft<C, M, EPT, +1>(sh, t, tw, ld2, st2);
}

struct FusedBs {
  int prec, m;
  cudaError_t (*launch)(const void*, void*, int64_t, int64_t, int64_t, int, const void*, const void*, const void*,
                        double, cudaStream_t);
};

std::vector<FusedBs>& table() {
  static std::vector<FusedBs> t;
  return t;
}

template <typename C, int M, int EPT>
cudaError_t launch(const void* src, void* dst, int64_t count, int64_t idist, int64_t odist, int n, const void* chirp,
                   const void* filt, const void* tw, double scale, cudaStream_t st) {
  using S = Pow2Shape<M, EPT, sizeof(C)>;
  static const cudaError_t attr =
      S::SMEM > 48 * 1024
          ? cudaFuncSetAttribute(&k_bs_fused<C, M, EPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM)
          : cudaSuccess;
  if (attr != cudaSuccess) return attr;
  const int64_t blocks = (count + S::B - 1) / S::B;
  if (blocks <= 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  k_bs_fused<C, M, EPT><<<unsigned(blocks), S::TPB, S::SMEM, st>>>(
      static_cast<const C*>(src), static_cast<C*>(dst), count, idist, odist, n, static_cast<const C*>(chirp),
      static_cast<const C*>(filt), static_cast<const C*>(tw), typename RealOf<C>::type(scale));
  return cudaGetLastError();
}

template <typename C, int M, int EPT>
void reg() {
  table().push_back(FusedBs{sizeof(C) == 8 ? kC64 : kC128, M, &launch<C, M, EPT>});
}

struct Reg {
  Reg() {
    reg<float2, 4, 4>();
    reg<float2, 8, 4>();
    reg<float2, 16, 4>();
    reg<float2, 32, 8>();
    reg<float2, 64, 8>();
    reg<float2, 128, 16>();
    reg<float2, 256, 16>();
    reg<float2, 512, 16>();
    reg<float2, 1024, 16>();
    reg<float2, 2048, 16>();
    reg<float2, 4096, 16>();
    reg<float2, 8192, 32>();
    reg<float2, 16384, 32>();
    reg<double2, 4, 4>();
    reg<double2, 8, 4>();
    reg<double2, 16, 4>();
    reg<double2, 32, 8>();
    reg<double2, 64, 8>();
    reg<double2, 128, 16>();
    reg<double2, 256, 16>();
    reg<double2, 512, 16>();
    reg<double2, 1024, 16>();
    reg<double2, 2048, 16>();
    reg<double2, 4096, 16>();
    reg<double2, 8192, 16>();
  }
} reg_bs_fused;

}  // namespace

cudaError_t exec_bluestein_fused(int prec, int64_t M, const void* src, void* dst, int64_t count, int64_t idist,
                                 int64_t odist, int64_t n, const void* chirp, const void* filt, const void* tw,
                                 double scale, cudaStream_t st) {
  for (const auto& k : table())
    if (k.prec == prec && k.m == M) return k.launch(src, dst, count, idist, odist, int(n), chirp, filt, tw, scale, st);
  return cudaErrorNotSupported;
}

bool bluestein_fused_supported(int prec, int64_t M) {
  for (const auto& k : table())
    if (k.prec == prec && k.m == M) return true;
  return false;
}

}  // namespace gfft
