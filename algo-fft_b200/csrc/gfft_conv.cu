// Convolution and correlation (K11): Convolve / Convolve128 (convolve.go),
// ConvolveReal (convolve_real.go), CrossCorrelate / AutoCorrelate
// (correlate.go), and a batched ConvolveReal with one shared kernel.
//
// Same algorithm as the reference: complex convolution at the exact length
// len(a)+len(b)-1 (so it may run Bluestein), real convolution at
// NextPow2(len(a)+len(b)-1) (at least 2) -- except for long real signals
// with a short kernel (len(b) - 1 <= L/4 for an L <= 2^15 block and more
// than two blocks of output), which run overlap-save (k_conv_os): the same
// linear convolution from single-CTA transforms of 2^12..2^15 points.  The two forward transforms run
// as one batch of two, the pointwise product is one elementwise kernel
// (internal/fft/complex_mul.go:23), the inverse writes straight into a
// padded buffer whose head is the result.  Plans come from a process-wide
// cache keyed by (precision, kind, length) instead of being rebuilt on
// every call as the reference does (convolve.go:23, convolve_real.go:30).
#include <map>
#include <mutex>
#include <tuple>
#include "gfft_internal.h"
#include "gfft_real.cuh"

namespace gfft {

namespace {

std::mutex g_cache_mu;
std::map<std::tuple<int, int, int64_t>, gfft_plan*> g_cplx;     // (device, prec, n)
std::map<std::tuple<int, int, int64_t>, gfft_plan_real*> g_real;  // (device, prec, n)

gfft_status cached_plan(int prec, int64_t n, gfft_plan** out) {
  int dev = 0;
  GFFT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_cache_mu);
  auto key = std::make_tuple(dev, prec, n);
  auto it = g_cplx.find(key);
  if (it != g_cplx.end()) {
    *out = it->second;
    return GFFT_OK;
  }
  gfft_plan_options o{};
  o.device = dev;
  gfft_status s = gfft_plan_new(out, prec, n, &o);
  if (s == GFFT_OK) g_cplx[key] = *out;
  return s;
}

gfft_status cached_real_plan(int prec, int64_t n, gfft_plan_real** out) {
  int dev = 0;
  GFFT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_cache_mu);
  auto key = std::make_tuple(dev, prec, n);
  auto it = g_real.find(key);
  if (it != g_real.end()) {
    *out = it->second;
    return GFFT_OK;
  }
  gfft_plan_options o{};
  o.device = dev;
  gfft_status s = gfft_plan_real_new(out, prec, n, &o);
  if (s == GFFT_OK) g_real[key] = *out;
  return s;
}

unsigned grid1(int64_t total) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 32))); }

// rows of `w` elements: row r = src_r padded with zeros (reverse+conj when
// `rev` is set: the correlate operand of correlate.go:26-32).
template <typename T>
__global__ void k_pad(T* dst, int64_t w, const T* src, int64_t len, int64_t sdist, int64_t rows, bool rev) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < rows * w; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / w, i = e % w;
    T v{};
    if (i < len) v = src[r * sdist + (rev ? len - 1 - i : i)];
    dst[e] = v;
  }
}

template <typename T>
__global__ void k_pad_conj(T* dst, int64_t w, const T* src, int64_t len) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < w; i += int64_t(gridDim.x) * blockDim.x)
    dst[i] = i < len ? cconj(src[len - 1 - i]) : T{0, 0};
}

// A[r][k] *= B[r*bdist + k]: each of `rows` spectra of w bins times the
// shared spectrum B (bdist = 0) or its own row of B (bdist = w).
template <typename C>
__global__ void k_cmul_rows(C* A, const C* B, int64_t w, int64_t rows, int64_t bdist) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < rows * w; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / w, k = e % w;
    A[e] = cmul(A[e], B[r * bdist + k]);
  }
}

template <typename T>
__global__ void k_take_rows(T* dst, int64_t ddist, const T* src, int64_t sdist, int64_t len, int64_t rows) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < rows * len; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / len, i = e % len;
    dst[r * ddist + i] = src[r * sdist + i];
  }
}

// ---- overlap-save for long real signals ------------------------------------
//
// Block j of a signal produces outputs [j B, j B + B) from the input window
// [j B - (nb - 1), j B - (nb - 1) + L), B = L - (nb - 1): a real transform of
// length L = 2H of the window, the product with the kernel's spectrum (L/2+1
// bins, shared by every block and signal, L2-resident), and the inverse
// real transform, whose samples from nb - 1 on are the linear convolution.
// One CTA slot per block does all of it in shared memory: the window loads
// straight into the first Stockham stage, the R2C recombination, the
// product and the C2R packing happen pairwise (k, H - k) between the two
// half-length transforms, and the last stage stores the B new samples.
// HBM sees L/B reads and one write per output sample.

template <typename R>
struct WindowLoad {
  static constexpr bool kShared = false;
  const R* x;
  int64_t pos0, len;
  bool valid;
  __device__ __forceinline__ Cx<R> operator()(int e) const {
    const int64_t p = pos0 + 2 * int64_t(e);
    Cx<R> v{R(0), R(0)};
    if (valid) {
      if (p >= 0 && p < len) v.x = x[p];
      if (p + 1 >= 0 && p + 1 < len) v.y = x[p + 1];
    }
    return v;
  }
};

template <typename C, int N, int EPT>
struct SharedLoad {
  static constexpr bool kShared = true;
  const C* sh;
  __device__ __forceinline__ C operator()(int e) const { return sh[Pow2Shape<N, EPT, sizeof(C)>::pad(e)]; }
};

template <typename R>
struct WindowStore {
  static constexpr bool kShared = false;
  R* y;
  int64_t pos0, len;  // output index of window sample 0, outputs per signal
  int skip;           // the first nb - 1 window samples are wrapped: not outputs
  R scale;
  bool valid;
  __device__ __forceinline__ void operator()(int e, Cx<R> v) const {
    if (!valid) return;
    const int w = 2 * e;
    const int64_t o = pos0 + w;
    if (w >= skip && o < len) y[o] = v.x * scale;
    if (w + 1 >= skip && o + 1 < len) y[o + 1] = v.y * scale;
  }
};

template <typename C, int H, int EPT>
__global__ void __launch_bounds__(Pow2Shape<H, EPT, sizeof(C)>::TPB)
k_conv_os(const typename RealOf<C>::type* a, typename RealOf<C>::type* dst, int64_t na, int64_t a_dist,
          int64_t dst_dist, int64_t nout, int64_t nblk, int64_t total, int nb, const C* __restrict__ tw,
          const C* __restrict__ wt, const C* __restrict__ hs) {
  using R = typename RealOf<C>::type;
  using S = Pow2Shape<H, EPT, sizeof(C)>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw) + (threadIdx.x / S::T) * S::STRIDE;
  const int t = threadIdx.x % S::T;
  const int64_t g = int64_t(blockIdx.x) * S::B + threadIdx.x / S::T;  // block over all signals
  const bool valid = g < total;
  const int64_t sig = valid ? g / nblk : 0, j = valid ? g % nblk : 0;
  const int64_t B = 2 * int64_t(H) - (nb - 1);
  const int64_t pos0 = j * B - (nb - 1);
  WindowLoad<R> ld{a + sig * a_dist, pos0, na, valid};
  PaddedStore<C, H, EPT> st{sh};
  pow2_fft<C, H, EPT, -1>(sh, t, tw, ld, st);
  xsync<S::T>();
  // Z (half-length spectrum) -> X (real spectrum) -> X * Hs -> packed Z'
  const C z0 = sh[0];
  const C x0 = cmul(C{z0.x + z0.y, R(0)}, __ldg(hs));
  const C xh = cmul(C{z0.x - z0.y, R(0)}, __ldg(hs + H));
  C zp[EPT];
#pragma unroll
  for (int i = 0; i < EPT; ++i) {
    const int k = t + i * S::T;
    const C zk = sh[S::pad(k)], zhk = sh[S::pad(k == 0 ? 0 : H - k)];
    const C xk = k == 0 ? x0 : cmul(r2c_bin(z0, zk, zhk, __ldg(wt + k), k, H), __ldg(hs + k));
    const C xhk = k == 0 ? xh : cmul(r2c_bin(z0, zhk, zk, __ldg(wt + H - k), H - k, H), __ldg(hs + H - k));
    zp[i] = c2r_packed(xk, xhk, x0, xh, __ldg(wt + k), k);
  }
  xsync<S::T>();
#pragma unroll
  for (int i = 0; i < EPT; ++i) sh[S::pad(t + i * S::T)] = zp[i];
  xsync<S::T>();
  SharedLoad<C, H, EPT> ld2{sh};
  WindowStore<R> st2{dst + sig * dst_dist, j * B - (nb - 1), nout, nb - 1, R(1.0 / double(H)), valid};
  pow2_fft<C, H, EPT, +1>(sh, t, tw, ld2, st2);
}

template <typename C, int H, int EPT>
cudaError_t launch_conv_os(const void* a, void* dst, int64_t na, int64_t a_dist, int64_t dst_dist, int64_t nout,
                           int64_t nblk, int64_t count, int nb, const void* tw, const void* wt, const void* hs,
                           cudaStream_t st) {
  using S = Pow2Shape<H, EPT, sizeof(C)>;
  static const cudaError_t attr =
      S::SMEM > 48 * 1024
          ? cudaFuncSetAttribute(&k_conv_os<C, H, EPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM)
          : cudaSuccess;
  if (attr != cudaSuccess) return attr;
  using R = typename RealOf<C>::type;
  const int64_t total = count * nblk;
  k_conv_os<C, H, EPT><<<unsigned((total + S::B - 1) / S::B), S::TPB, S::SMEM, st>>>(
      static_cast<const R*>(a), static_cast<R*>(dst), na, a_dist, dst_dist, nout, nblk, total, nb,
      static_cast<const C*>(tw), static_cast<const C*>(wt), static_cast<const C*>(hs));
  return cudaGetLastError();
}

// FFT length of the overlap-save blocks: the smallest power of two with at
// most an eighth of each window wrapped (L >= 8 (nb - 1)), else at most a
// quarter, at least 4096, at most what one CTA transforms (2 x 16384
// complex64, 2 x 8192 complex128); 0 = use one transform of the whole signal
// (short signals, long kernels).  The longer blocks cost fewer transform
// points per output and run the transform on more threads per CTA: with a
// 4097-tap kernel, 2^15-point blocks (28672 outputs each, 512 threads) took
// 0.45 ms for 64 signals of 2^20 against 0.52 for 2^14-point blocks (12288
// outputs, 256 threads).
template <typename R>
int64_t os_length(int64_t na, int64_t nb) {
  const int64_t lmax = sizeof(R) == 4 ? 32768 : 16384;
  for (const int64_t wrap : {8, 4}) {
    int64_t L = 4096;
    while (L < wrap * (nb - 1)) L <<= 1;
    if (L <= lmax && na + nb - 1 > 2 * L) return L;
  }
  return 0;
}

template <typename R>
cudaError_t dispatch_conv_os(int64_t L, const R* a, R* dst, int64_t na, int64_t a_dist, int64_t dst_dist,
                             int64_t nout, int64_t nblk, int64_t count, int nb, const void* tw, const void* wt,
                             const void* hs, cudaStream_t st) {
  using C = Cx<R>;
  if constexpr (sizeof(R) == 4) {
    switch (L) {
      case 4096: return launch_conv_os<C, 2048, 16>(a, dst, na, a_dist, dst_dist, nout, nblk, count, nb, tw, wt, hs, st);
      case 8192: return launch_conv_os<C, 4096, 16>(a, dst, na, a_dist, dst_dist, nout, nblk, count, nb, tw, wt, hs, st);
      // 512 threads (16 per thread) ran 1.08x faster than 256 threads (32)
      case 16384: return launch_conv_os<C, 8192, 16>(a, dst, na, a_dist, dst_dist, nout, nblk, count, nb, tw, wt, hs, st);
      case 32768: return launch_conv_os<C, 16384, 32>(a, dst, na, a_dist, dst_dist, nout, nblk, count, nb, tw, wt, hs, st);
    }
  } else {
    switch (L) {
      case 4096: return launch_conv_os<C, 2048, 16>(a, dst, na, a_dist, dst_dist, nout, nblk, count, nb, tw, wt, hs, st);
      case 8192: return launch_conv_os<C, 4096, 16>(a, dst, na, a_dist, dst_dist, nout, nblk, count, nb, tw, wt, hs, st);
      case 16384: return launch_conv_os<C, 8192, 16>(a, dst, na, a_dist, dst_dist, nout, nblk, count, nb, tw, wt, hs, st);
    }
  }
  return cudaErrorInvalidValue;
}

}  // namespace

// Complex: dst[0, L) = IFFT_L(FFT_L(a) * FFT_L(b)), L = na + nb - 1.
template <typename C>
static gfft_status convolve_dev(int prec, C* dst, const C* a, int64_t na, const C* b, int64_t nb, bool correlate,
                                cudaStream_t st) {
  const int64_t L = na + nb - 1;
  gfft_plan* p = nullptr;
  gfft_status s = cached_plan(prec, L, &p);
  if (s != GFFT_OK) return s;
  C* work = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&work), size_t(2 * L) * sizeof(C), st));
  k_pad<C><<<grid1(L), 256, 0, st>>>(work, L, a, na, 0, 1, false);
  if (correlate)
    k_pad_conj<C><<<grid1(L), 256, 0, st>>>(work + L, L, b, nb);
  else
    k_pad<C><<<grid1(L), 256, 0, st>>>(work + L, L, b, nb, 0, 1, false);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) s = core_exec(&p->core, -1, work, work, 2, L, L, st);
  if (e == cudaSuccess && s == GFFT_OK) {
    k_cmul_rows<C><<<grid1(L), 256, 0, st>>>(work, work + L, L, 1, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && s == GFFT_OK) s = core_exec(&p->core, +1, dst, work, 1, L, L, st);
  cudaFreeAsync(work, st);
  if (e != cudaSuccess) return cuda_status(e, "convolve");
  return s;
}

// Real: `count` signals (a_len reals, a_dist apart) convolved with one kernel
// b; outputs of a_len + b_len - 1 reals, dst_dist apart.  F = NextPow2.
template <typename R>
static gfft_status convolve_real_dev(int prec, R* dst, int64_t dst_dist, const R* a, int64_t na, int64_t a_dist,
                                     int64_t count, const R* b, int64_t nb, cudaStream_t st) {
  using C = Cx<R>;
  const int64_t L = na + nb - 1;
  // long signals: overlap-save blocks (same linear convolution, transforms
  // of 2^12..2^15 points instead of one of NextPow2(na + nb - 1))
  if (const int64_t Lb = os_length<R>(na, nb)) {
    gfft_plan_real* bp = nullptr;
    gfft_status s = cached_real_plan(prec, Lb, &bp);
    if (s != GFFT_OK) return s;
    if (bp->child.algo == Algo::Pow2Smem) {
      const int64_t hb = Lb / 2 + 1;
      R* kpad = nullptr;
      GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&kpad), size_t(Lb) * sizeof(R) + size_t(hb) * sizeof(C), st));
      C* hs = reinterpret_cast<C*>(kpad + Lb);
      k_pad<R><<<grid1(Lb), 256, 0, st>>>(kpad, Lb, b, nb, 0, 1, false);
      cudaError_t e = cudaGetLastError();
      if (e == cudaSuccess) s = real_forward(bp, 0, hs, kpad, 1, Lb, hb, st);
      if (e == cudaSuccess && s == GFFT_OK) {
        const int64_t B = Lb - (nb - 1), nblk = (L + B - 1) / B;
        e = dispatch_conv_os<R>(Lb, a, dst, na, a_dist, count == 1 ? L : dst_dist, L, nblk, count, int(nb),
                                bp->child.tw, bp->wt, hs, st);
      }
      cudaFreeAsync(kpad, st);
      if (e != cudaSuccess) return cuda_status(e, "k_conv_os");
      return s;
    }
  }
  int64_t F = 2;
  while (F < L) F <<= 1;  // convolve_real.go:23-28
  const int64_t h1 = F / 2 + 1;
  gfft_plan_real* p = nullptr;
  gfft_status s = cached_real_plan(prec, F, &p);
  if (s != GFFT_OK) return s;
  // [count + 1 padded rows of F reals | count + 1 spectra of h1 bins]
  R* pad = nullptr;
  const size_t pad_bytes = size_t(count + 1) * size_t(F) * sizeof(R);
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&pad), pad_bytes + size_t(count + 1) * size_t(h1) * sizeof(C), st));
  C* spec = reinterpret_cast<C*>(reinterpret_cast<char*>(pad) + pad_bytes);
  k_pad<R><<<grid1(count * F), 256, 0, st>>>(pad, F, a, na, a_dist, count, false);
  k_pad<R><<<grid1(F), 256, 0, st>>>(pad + count * F, F, b, nb, 0, 1, false);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) s = real_forward(p, 0, spec, pad, count + 1, F, h1, st);
  if (e == cudaSuccess && s == GFFT_OK) {
    k_cmul_rows<C><<<grid1(count * h1), 256, 0, st>>>(spec, spec + count * h1, h1, count, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && s == GFFT_OK) s = real_inverse(p, pad, spec, count, F, h1, st);
  if (e == cudaSuccess && s == GFFT_OK) {
    k_take_rows<R><<<grid1(count * L), 256, 0, st>>>(dst, dst_dist, pad, F, L, count);
    e = cudaGetLastError();
  }
  cudaFreeAsync(pad, st);
  if (e != cudaSuccess) return cuda_status(e, "convolve_real");
  return s;
}

// convolve.go:10-21 / convolve_real.go:10-22 argument checks.
static gfft_status conv_args(const void* dst, int64_t dst_len, const void* a, int64_t na, const void* b, int64_t nb) {
  if (!dst || !a || !b) return GFFT_ERR_NIL_SLICE;
  if (na <= 0 || nb <= 0) return GFFT_ERR_INVALID_LENGTH;
  if (dst_len != na + nb - 1) return GFFT_ERR_LENGTH_MISMATCH;
  return GFFT_OK;
}

static gfft_status conv_any(int prec, bool real, bool corr, void* dst, int64_t dst_len, const void* a, int64_t na,
                            const void* b, int64_t nb, cudaStream_t st) {
  gfft_status s = conv_args(dst, dst_len, a, na, b, nb);
  if (s != GFFT_OK) return s;
  if (prec != GFFT_COMPLEX64 && prec != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  if (real) {
    if (prec == kC64)
      return convolve_real_dev<float>(prec, static_cast<float*>(dst), 0, static_cast<const float*>(a), na, 0, 1,
                                      static_cast<const float*>(b), nb, st);
    return convolve_real_dev<double>(prec, static_cast<double*>(dst), 0, static_cast<const double*>(a), na, 0, 1,
                                     static_cast<const double*>(b), nb, st);
  }
  if (prec == kC64)
    return convolve_dev<float2>(prec, static_cast<float2*>(dst), static_cast<const float2*>(a), na,
                                static_cast<const float2*>(b), nb, corr, st);
  return convolve_dev<double2>(prec, static_cast<double2*>(dst), static_cast<const double2*>(a), na,
                               static_cast<const double2*>(b), nb, corr, st);
}

static gfft_status conv_host(int prec, bool real, bool corr, void* dst, int64_t dst_len, const void* a, int64_t na,
                             const void* b, int64_t nb) {
  gfft_status s = conv_args(dst, dst_len, a, na, b, nb);
  if (s != GFFT_OK) return s;
  if (prec != GFFT_COMPLEX64 && prec != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  const size_t es = elem_bytes(prec) / (real ? 2 : 1);
  cudaStream_t st = nullptr;
  GFFT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  char* buf = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&buf), size_t(na + nb + dst_len) * es, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf, a, size_t(na) * es, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf + na * es, b, size_t(nb) * es, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    s = conv_any(prec, real, corr, buf + (na + nb) * es, dst_len, buf, na, buf + na * es, nb, st);
    if (s == GFFT_OK) e = cudaMemcpyAsync(dst, buf + (na + nb) * es, size_t(dst_len) * es, cudaMemcpyDeviceToHost, st);
  }
  if (buf) cudaFreeAsync(buf, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) return cuda_status(e, "convolve host path");
  if (e2 != cudaSuccess) return cuda_status(e2, "cudaStreamSynchronize");
  return s;
}

}  // namespace gfft

using namespace gfft;

extern "C" {

gfft_status gfft_convolve(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len, const void* b,
                          int64_t b_len, void* stream) {
  clear_error();
  return conv_any(precision, false, false, dst, dst_len, a, a_len, b, b_len, static_cast<cudaStream_t>(stream));
}

gfft_status gfft_correlate(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len, const void* b,
                           int64_t b_len, void* stream) {
  clear_error();
  return conv_any(precision, false, true, dst, dst_len, a, a_len, b, b_len, static_cast<cudaStream_t>(stream));
}

gfft_status gfft_convolve_real(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                               const void* b, int64_t b_len, void* stream) {
  clear_error();
  return conv_any(precision, true, false, dst, dst_len, a, a_len, b, b_len, static_cast<cudaStream_t>(stream));
}

gfft_status gfft_convolve_host(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                               const void* b, int64_t b_len) {
  clear_error();
  return conv_host(precision, false, false, dst, dst_len, a, a_len, b, b_len);
}

gfft_status gfft_correlate_host(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                                const void* b, int64_t b_len) {
  clear_error();
  return conv_host(precision, false, true, dst, dst_len, a, a_len, b, b_len);
}

gfft_status gfft_convolve_real_host(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                                    const void* b, int64_t b_len) {
  clear_error();
  return conv_host(precision, true, false, dst, dst_len, a, a_len, b, b_len);
}

gfft_status gfft_convolve_real_batch(int32_t precision, void* dst, int64_t dst_dist, const void* a, int64_t a_len,
                                     int64_t a_dist, int64_t count, const void* b, int64_t b_len, void* stream) {
  clear_error();
  if (!dst || !a || !b) return GFFT_ERR_NIL_SLICE;
  if (a_len <= 0 || b_len <= 0 || count < 1) return GFFT_ERR_INVALID_LENGTH;
  if (a_dist < a_len || dst_dist < a_len + b_len - 1) return GFFT_ERR_INVALID_STRIDE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (precision == GFFT_COMPLEX64)
    return convolve_real_dev<float>(precision, static_cast<float*>(dst), dst_dist, static_cast<const float*>(a),
                                    a_len, a_dist, count, static_cast<const float*>(b), b_len, st);
  if (precision == GFFT_COMPLEX128)
    return convolve_real_dev<double>(precision, static_cast<double*>(dst), dst_dist, static_cast<const double*>(a),
                                     a_len, a_dist, count, static_cast<const double*>(b), b_len, st);
  return GFFT_ERR_INVALID_ARGUMENT;
}

}  // extern "C"
