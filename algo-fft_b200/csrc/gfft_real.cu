// Real-input plans (PlanReal, plan_real_generic.go) over the C ABI.
#include <algorithm>
#include <climits>
#include <cmath>
#include <mutex>
#include <new>
#include <vector>
#include "gfft_internal.h"
#include "gfft_real.cuh"

namespace gfft {

struct RealKernel {
  int prec, h, ept, tpb, per_cta, smem;
  const void* fr2c;
  const void* fc2r;
  cudaError_t (*r2c)(const void*, void*, int64_t, int64_t, int64_t, const void*, const void*, double, cudaStream_t);
  cudaError_t (*c2r)(const void*, void*, int64_t, int64_t, int64_t, const void*, const void*, double, cudaStream_t);
};

static std::vector<RealKernel>& real_table() {
  static std::vector<RealKernel> t;
  return t;
}

template <typename C, int H, int EPT>
static cudaError_t launch_r2c(const void* src, void* dst, int64_t count, int64_t idist, int64_t odist, const void* tw,
                              const void* wt, double scale, cudaStream_t st) {
  using S = Pow2Shape<H, EPT, sizeof(C)>;
  const int64_t blocks = (count + S::B - 1) / S::B;
  k_r2c_pow2<C, H, EPT><<<unsigned(blocks), S::TPB, S::B * S::STRIDE * sizeof(C), st>>>(
      static_cast<const C*>(src), static_cast<C*>(dst), count, idist, odist, static_cast<const C*>(tw),
      static_cast<const C*>(wt), typename RealOf<C>::type(scale));
  return cudaGetLastError();
}

template <typename C, int H, int EPT>
static cudaError_t launch_c2r(const void* src, void* dst, int64_t count, int64_t idist, int64_t odist, const void* tw,
                              const void* wt, double scale, cudaStream_t st) {
  using S = Pow2Shape<H, EPT, sizeof(C)>;
  const int64_t blocks = (count + S::B - 1) / S::B;
  k_c2r_pow2<C, H, EPT><<<unsigned(blocks), S::TPB, S::B * S::STRIDE * sizeof(C), st>>>(
      static_cast<const C*>(src), static_cast<C*>(dst), count, idist, odist, static_cast<const C*>(tw),
      static_cast<const C*>(wt), typename RealOf<C>::type(scale));
  return cudaGetLastError();
}

template <typename C, int H, int EPT>
static void reg_real() {
  using S = Pow2Shape<H, EPT, sizeof(C)>;
  RealKernel k;
  k.prec = sizeof(C) == 8 ? kC64 : kC128;
  k.h = H;
  k.ept = EPT;
  k.tpb = S::TPB;
  k.per_cta = S::B;
  k.smem = S::B * S::STRIDE * int(sizeof(C));
  k.fr2c = reinterpret_cast<const void*>(&k_r2c_pow2<C, H, EPT>);
  k.fc2r = reinterpret_cast<const void*>(&k_c2r_pow2<C, H, EPT>);
  k.r2c = &launch_r2c<C, H, EPT>;
  k.c2r = &launch_c2r<C, H, EPT>;
  real_table().push_back(k);
}

namespace {
struct RegReal {
  RegReal() {
    reg_real<float2, 2, 2>();
    reg_real<float2, 4, 4>();
    reg_real<float2, 8, 4>();
    reg_real<float2, 16, 4>();
    reg_real<float2, 32, 8>();
    reg_real<float2, 64, 8>();
    reg_real<float2, 128, 16>();
    reg_real<float2, 256, 16>();
    reg_real<float2, 512, 16>();
    reg_real<float2, 1024, 32>();
    reg_real<float2, 2048, 16>();
    reg_real<float2, 4096, 16>();
    reg_real<float2, 8192, 32>();
    reg_real<float2, 16384, 16>();
    reg_real<double2, 2, 2>();
    reg_real<double2, 4, 4>();
    reg_real<double2, 8, 4>();
    reg_real<double2, 16, 4>();
    reg_real<double2, 32, 8>();
    reg_real<double2, 64, 8>();
    reg_real<double2, 128, 16>();
    reg_real<double2, 256, 16>();
    reg_real<double2, 512, 8>();
    reg_real<double2, 1024, 16>();
    reg_real<double2, 2048, 8>();
    reg_real<double2, 4096, 16>();
    reg_real<double2, 8192, 16>();
  }
} reg_real_kernels;
}  // namespace

static const RealKernel* find_real(int prec, int64_t h) {
  for (const auto& k : real_table())
    if (k.prec == prec && k.h == h) return &k;
  return nullptr;
}

static cudaError_t prepare_real(const RealKernel* k) {
  static std::mutex mu;
  std::lock_guard<std::mutex> g(mu);
  if (k->smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k->fr2c, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k->fc2r, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem);
    return e;
  }
  return cudaSuccess;
}

// U[k] = 0.5*(1 + sin th) + i*0.5*cos th, th = 2*pi*k/n  (plan_real_generic.go:71-86), FP64
template <typename C>
__global__ void k_real_weights(C* w, int64_t n) {
  using Re = typename RealOf<C>::type;
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k <= n / 2; k += int64_t(gridDim.x) * blockDim.x) {
    double s, c;
    sincospi(2.0 * double(k) / double(n), &s, &c);
    w[k] = C{Re(0.5 * (1.0 + s)), Re(0.5 * c)};
  }
}

static unsigned grid1(int64_t total) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 32))); }

}  // namespace gfft

using namespace gfft;

extern "C" {

gfft_status gfft_plan_real_new(gfft_plan_real** out, int32_t precision, int64_t n, const gfft_plan_options* opts) {
  clear_error();
  if (!out) return GFFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (n < 2 || n % 2 != 0) return GFFT_ERR_INVALID_LENGTH;  // plan_real_generic.go:54
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  gfft_plan_options o{};
  if (opts) o = *opts;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GFFT_ERR_NO_DEVICE;
  if (o.device < 0 || o.device >= ndev) return GFFT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(o.device));
  auto* p = new (std::nothrow) gfft_plan_real;
  if (!p) return GFFT_ERR_OUT_OF_MEMORY;
  p->prec = precision;
  p->n = n;
  p->h = n / 2;
  p->opts = o;
  PlanHint hint;
  hint.planner = o.planner;
  hint.batch = o.batch;
  hint.real = 1;
  hint.user = true;
  gfft_status s = core_init(&p->child, precision, p->h, o.device, o.strategy, &hint);
  cudaError_t e = cudaSuccess;
  if (s == GFFT_OK) e = cudaMalloc(&p->wt, size_t(p->h + 1) * elem_bytes(precision));
  if (s == GFFT_OK && e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&p->flag), sizeof(unsigned));
  if (s == GFFT_OK && e == cudaSuccess) {
    if (precision == GFFT_COMPLEX64)
      k_real_weights<float2><<<grid1(p->h + 1), 256>>>(static_cast<float2*>(p->wt), n);
    else
      k_real_weights<double2><<<grid1(p->h + 1), 256>>>(static_cast<double2*>(p->wt), n);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  }
  // the fused kernels carry their own twiddles: they need the child's W_h
  // table, i.e. a single-pass child plan of the same length
  if (s == GFFT_OK && e == cudaSuccess && p->child.algo == Algo::Pow2Smem) {
    p->fused = find_real(precision, p->h);
    if (p->fused) e = prepare_real(p->fused);
  }
  if (s == GFFT_OK && e != cudaSuccess) s = cuda_status(e, "real plan setup");
  if (s != GFFT_OK) {
    gfft_plan_real_close(p);
    return s;
  }
  *out = p;
  return GFFT_OK;
}

void gfft_plan_real_close(gfft_plan_real* p) {
  if (!p) return;
  core_free(&p->child);
  if (p->wt) cudaFree(p->wt);
  if (p->flag) cudaFree(p->flag);
  delete p;
}

int64_t gfft_plan_real_len(const gfft_plan_real* p) { return p ? p->n : 0; }
int64_t gfft_plan_real_spectrum_len(const gfft_plan_real* p) { return p ? p->h + 1 : 0; }

}  // extern "C"

namespace gfft {

// plan_batch.go:21-42 resolveBatchStrideReal + the per-transform bound
// checks of plan_real_generic.go:115-139 (reals: stride_r, bins: stride_c).
static gfft_status real_layout(const gfft_plan_real* p, int64_t real_len, int64_t cplx_len, int64_t* batch,
                               int64_t* stride_r, int64_t* stride_c) {
  const int64_t n = p->n, h = p->h;
  if (p->opts.batch <= 1 && p->opts.stride <= 0) {
    if (real_len != n || cplx_len != h + 1) return GFFT_ERR_LENGTH_MISMATCH;
    *batch = 1;
    *stride_r = n;
    *stride_c = h + 1;
    return GFFT_OK;
  }
  const int64_t b = p->opts.batch < 1 ? 1 : p->opts.batch;
  const int64_t si = p->opts.stride <= 0 ? n : p->opts.stride;
  const int64_t so = p->opts.stride <= 0 ? h + 1 : p->opts.stride;
  if (si < n || so < h + 1) return GFFT_ERR_INVALID_STRIDE;
  if ((b - 1) * si + n > real_len || (b - 1) * so + h + 1 > cplx_len) return GFFT_ERR_LENGTH_MISMATCH;
  *batch = b;
  *stride_r = si;
  *stride_c = so;
  return GFFT_OK;
}

gfft_status real_forward(gfft_plan_real* p, int scaling, void* dst, const void* src, int64_t batch, int64_t sr,
                                int64_t sc, cudaStream_t st) {
  const size_t es = elem_bytes(p->prec);
  const double scale = scaling == 1 ? 1.0 / double(p->n) : scaling == 2 ? 1.0 / std::sqrt(double(p->n)) : 1.0;
  if (p->fused && sr % 2 == 0) {
    GFFT_CUDA(p->fused->r2c(src, dst, batch, sr / 2, sc, p->child.tw, p->wt, scale, st));
    return GFFT_OK;
  }
  void* z = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&z), size_t(batch) * size_t(p->h) * es, st));
  const unsigned g = grid1(batch * (p->h + 1));
  if (p->prec == kC64)
    k_pack_real<float2><<<g, 256, 0, st>>>(static_cast<float2*>(z), static_cast<const float*>(src), p->h, batch, sr);
  else
    k_pack_real<double2><<<g, 256, 0, st>>>(static_cast<double2*>(z), static_cast<const double*>(src), p->h, batch, sr);
  gfft_status s = GFFT_OK;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) s = core_exec(&p->child, -1, z, z, batch, p->h, p->h, st);
  if (e == cudaSuccess && s == GFFT_OK) {
    if (p->prec == kC64)
      k_r2c_post<float2><<<g, 256, 0, st>>>(static_cast<float2*>(dst), static_cast<const float2*>(z),
                                             static_cast<const float2*>(p->wt), p->h, batch, sc, float(scale));
    else
      k_r2c_post<double2><<<g, 256, 0, st>>>(static_cast<double2*>(dst), static_cast<const double2*>(z),
                                              static_cast<const double2*>(p->wt), p->h, batch, sc, scale);
    e = cudaGetLastError();
  }
  cudaFreeAsync(z, st);
  if (e != cudaSuccess) return cuda_status(e, "real forward");
  return s;
}

gfft_status real_inverse(gfft_plan_real* p, void* dst, const void* src, int64_t batch, int64_t sr, int64_t sc,
                                cudaStream_t st) {
  const size_t es = elem_bytes(p->prec);
  // DC and Nyquist must be real (plan_real_generic.go:301-316)
  GFFT_CUDA(cudaMemsetAsync(p->flag, 0, sizeof(unsigned), st));
  const double eps = p->prec == kC64 ? 1e-4 : 1e-12;
  if (p->prec == kC64)
    k_check_spectrum<float2><<<grid1(batch), 256, 0, st>>>(static_cast<const float2*>(src), p->h, batch, sc, eps, p->flag);
  else
    k_check_spectrum<double2><<<grid1(batch), 256, 0, st>>>(static_cast<const double2*>(src), p->h, batch, sc, eps, p->flag);
  GFFT_CUDA(cudaGetLastError());
  unsigned bad = 0;
  GFFT_CUDA(cudaMemcpyAsync(&bad, p->flag, sizeof bad, cudaMemcpyDeviceToHost, st));
  GFFT_CUDA(cudaStreamSynchronize(st));
  if (bad) {
    set_error("DC or Nyquist bin has a non-zero imaginary part");
    return GFFT_ERR_INVALID_SPECTRUM;
  }
  const double scale = 1.0 / double(p->h);
  if (p->fused && sr % 2 == 0) {
    GFFT_CUDA(p->fused->c2r(src, dst, batch, sc, sr / 2, p->child.tw, p->wt, scale, st));
    return GFFT_OK;
  }
  void* z = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&z), size_t(batch) * size_t(p->h) * es, st));
  const unsigned g = grid1(batch * p->h);
  if (p->prec == kC64)
    k_c2r_pre<float2><<<g, 256, 0, st>>>(static_cast<float2*>(z), static_cast<const float2*>(src),
                                          static_cast<const float2*>(p->wt), p->h, batch, sc);
  else
    k_c2r_pre<double2><<<g, 256, 0, st>>>(static_cast<double2*>(z), static_cast<const double2*>(src),
                                           static_cast<const double2*>(p->wt), p->h, batch, sc);
  gfft_status s = GFFT_OK;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) s = core_exec(&p->child, +1, z, z, batch, p->h, p->h, st);
  if (e == cudaSuccess && s == GFFT_OK) {
    if (p->prec == kC64)
      k_unpack_real<float2><<<g, 256, 0, st>>>(static_cast<float*>(dst), static_cast<const float2*>(z), p->h, batch, sr);
    else
      k_unpack_real<double2><<<g, 256, 0, st>>>(static_cast<double*>(dst), static_cast<const double2*>(z), p->h, batch, sr);
    e = cudaGetLastError();
  }
  cudaFreeAsync(z, st);
  if (e != cudaSuccess) return cuda_status(e, "real inverse");
  return s;
}

// Host-slice wrapper: copies the used span in, runs, copies the result out.
static gfft_status real_host(gfft_plan_real* p, bool inverse, int scaling, void* dst, int64_t dst_bytes,
                             const void* src, int64_t src_bytes, int64_t batch, int64_t sr, int64_t sc) {
  cudaStream_t st = nullptr;
  GFFT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  void *ds = nullptr, *dd = nullptr;
  gfft_status s = GFFT_OK;
  cudaError_t e = ws_alloc(reinterpret_cast<void**>(&ds), size_t(src_bytes), st);
  if (e == cudaSuccess) e = ws_alloc(reinterpret_cast<void**>(&dd), size_t(dst_bytes), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ds, src, size_t(src_bytes), cudaMemcpyHostToDevice, st);
  // the parts of dst outside the transforms keep the caller's values
  if (e == cudaSuccess) e = cudaMemcpyAsync(dd, dst, size_t(dst_bytes), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    s = inverse ? real_inverse(p, dd, ds, batch, sr, sc, st) : real_forward(p, scaling, dd, ds, batch, sr, sc, st);
    if (s == GFFT_OK) e = cudaMemcpyAsync(dst, dd, size_t(dst_bytes), cudaMemcpyDeviceToHost, st);
  }
  if (ds) cudaFreeAsync(ds, st);
  if (dd) cudaFreeAsync(dd, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) return cuda_status(e, "real host path");
  if (e2 != cudaSuccess) return cuda_status(e2, "cudaStreamSynchronize");
  return s;
}

}  // namespace gfft

extern "C" {

gfft_status gfft_real_forward(gfft_plan_real* p, int32_t scaling, void* dst, int64_t dst_len, const void* src,
                              int64_t src_len, void* stream) {
  clear_error();
  if (!p || scaling < 0 || scaling > 2) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  int64_t b, sr, sc;
  gfft_status s = real_layout(p, src_len, dst_len, &b, &sr, &sc);
  if (s != GFFT_OK) return s;
  return real_forward(p, scaling, dst, src, b, sr, sc, static_cast<cudaStream_t>(stream));
}

gfft_status gfft_real_inverse(gfft_plan_real* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                              void* stream) {
  clear_error();
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  int64_t b, sr, sc;
  gfft_status s = real_layout(p, dst_len, src_len, &b, &sr, &sc);
  if (s != GFFT_OK) return s;
  return real_inverse(p, dst, src, b, sr, sc, static_cast<cudaStream_t>(stream));
}

gfft_status gfft_real_forward_host(gfft_plan_real* p, int32_t scaling, void* dst, int64_t dst_len, const void* src,
                                   int64_t src_len) {
  clear_error();
  if (!p || scaling < 0 || scaling > 2) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  int64_t b, sr, sc;
  gfft_status s = real_layout(p, src_len, dst_len, &b, &sr, &sc);
  if (s != GFFT_OK) return s;
  const size_t es = elem_bytes(p->prec);
  return real_host(p, false, scaling, dst, dst_len * int64_t(es), src, src_len * int64_t(es / 2), b, sr, sc);
}

gfft_status gfft_real_inverse_host(gfft_plan_real* p, void* dst, int64_t dst_len, const void* src, int64_t src_len) {
  clear_error();
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  int64_t b, sr, sc;
  gfft_status s = real_layout(p, dst_len, src_len, &b, &sr, &sc);
  if (s != GFFT_OK) return s;
  const size_t es = elem_bytes(p->prec);
  return real_host(p, true, 0, dst, dst_len * int64_t(es / 2), src, src_len * int64_t(es), b, sr, sc);
}

}  // extern "C"
