// Convolution and correlation (K11): Convolve / Convolve128 (convolve.go),
// ConvolveReal (convolve_real.go), CrossCorrelate / AutoCorrelate
// (correlate.go), and a batched ConvolveReal with one shared kernel.
//
// Same algorithm as the reference: complex convolution at the exact length
// len(a)+len(b)-1 (so it may run Bluestein), real convolution at
// NextPow2(len(a)+len(b)-1) (at least 2).  The two forward transforms run
// as one batch of two, the pointwise product is one elementwise kernel
// (internal/fft/complex_mul.go:23), the inverse writes straight into a
// padded buffer whose head is the result.  Plans come from a process-wide
// cache keyed by (precision, kind, length) instead of being rebuilt on
// every call as the reference does (convolve.go:23, convolve_real.go:30).
#include <map>
#include <mutex>
#include <tuple>
#include "gfft_internal.h"

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
