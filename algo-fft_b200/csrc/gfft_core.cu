// Kernel registry, device twiddle generation and the 1-D schedule choice.
#include <algorithm>
#include <mutex>
#include <vector>
#include "gfft_internal.h"
#include "gfft_math.cuh"

namespace gfft {

// ---------------------------------------------------------------- registry

static std::vector<Pow2Kernel>& pow2_table() {
  static std::vector<Pow2Kernel> t;
  return t;
}

void register_pow2(const Pow2Kernel& k) { pow2_table().push_back(k); }

const Pow2Kernel* find_pow2(int prec, int n, int ept, int dir) {
  for (const auto& k : pow2_table())
    if (k.prec == prec && k.n == n && k.ept == ept && k.dir == dir) return &k;
  return nullptr;
}

std::vector<const Pow2Kernel*> pow2_variants(int prec, int n, int dir) {
  std::vector<const Pow2Kernel*> v;
  for (const auto& k : pow2_table())
    if (k.prec == prec && k.n == n && k.dir == dir) v.push_back(&k);
  std::sort(v.begin(), v.end(), [](auto a, auto b) { return a->ept < b->ept; });
  return v;
}

cudaError_t prepare_kernels() {
  static std::mutex mu;
  static std::vector<int> done;  // devices already prepared
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  if (std::find(done.begin(), done.end(), dev) != done.end()) return cudaSuccess;
  for (const auto& k : pow2_table()) {
    if (k.smem > 48 * 1024) {
      e = cudaFuncSetAttribute(k.func, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
      if (e != cudaSuccess) return e;
    }
  }
  done.push_back(dev);
  return cudaSuccess;
}

// ---------------------------------------------------------------- twiddles

// W_n^m in FP64: the angle is folded into (-1/2, 1/2] turns with integer
// arithmetic first, so sincospi sees an argument of at most 1 in magnitude
// and the result is accurate to a few ulp of double before rounding to the
// element type.
template <typename C>
__global__ void k_twiddles(C* tw, int64_t n) {
  using Re = typename RealOf<C>::type;
  for (int64_t m = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; m < n; m += int64_t(gridDim.x) * blockDim.x) {
    int64_t mm = m;
    if (2 * mm > n) mm -= n;  // exp(-2πi m/n) == exp(-2πi (m-n)/n)
    double s, c;
    sincospi(-2.0 * double(mm) / double(n), &s, &c);
    tw[m] = C{Re(c), Re(s)};
  }
}

gfft_status make_twiddles(int prec, int64_t n, void** out, cudaStream_t st) {
  *out = nullptr;
  void* p = nullptr;
  GFFT_CUDA(cudaMalloc(&p, size_t(n) * elem_bytes(prec)));
  int blocks = int(std::min<int64_t>((n + 255) / 256, 4096));
  if (prec == kC64)
    k_twiddles<float2><<<blocks, 256, 0, st>>>(static_cast<float2*>(p), n);
  else
    k_twiddles<double2><<<blocks, 256, 0, st>>>(static_cast<double2*>(p), n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFree(p);
    return cuda_status(e, "k_twiddles");
  }
  *out = p;
  return GFFT_OK;
}

// ---------------------------------------------------------------- copy kernel

template <typename C>
__global__ void k_copy_batch(C* dst, const C* src, int64_t n, int64_t count, int64_t idist, int64_t odist) {
  const int64_t total = n * count;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    int64_t b = e / n, i = e - b * n;
    dst[b * odist + i] = src[b * idist + i];
  }
}

// ---------------------------------------------------------------- schedules

static int ilog2(int64_t n) {
  int l = 0;
  while ((int64_t(1) << l) < n) ++l;
  return l;
}

// Default elements-per-thread of the single-pass kernel (the autotuner may
// override it through wisdom): enough threads per transform for coalesced
// 128-byte rows, radix-32 stages where the register budget allows.
static int default_ept(int prec, int64_t n) {
  if (n <= 4) return int(n);
  if (n == 8) return 4;
  if (n <= 64) return n == 16 ? 4 : 8;
  if (n <= 256) return 16;
  if (prec == kC64 && n == 1024) return 32;
  if (prec == kC64 && n == 16384) return 16;
  return 16;
}

gfft_status core_init(PlanCore* c, int prec, int64_t n, int device) {
  c->prec = prec;
  c->n = n;
  c->device = device;
  if (n == 1) {
    c->algo = Algo::Trivial;
    c->name = "gpu:sm100:copy:n1";
    return GFFT_OK;
  }
  GFFT_CUDA(prepare_kernels());
  const bool pow2 = (n & (n - 1)) == 0;
  const int64_t max_single = prec == kC64 ? 16384 : 8192;
  if (pow2 && n <= max_single) {
    int ept = default_ept(prec, n);
    const Pow2Kernel* f = find_pow2(prec, int(n), ept, -1);
    const Pow2Kernel* i = find_pow2(prec, int(n), ept, +1);
    if (!f || !i) {
      set_error("no compiled power-of-two kernel for this size");
      return GFFT_ERR_NOT_IMPLEMENTED;
    }
    c->algo = Algo::Pow2Smem;
    c->k[0] = f;
    c->k[1] = i;
    gfft_status s = make_twiddles(prec, n, &c->tw, 0);
    if (s != GFFT_OK) return s;
    GFFT_CUDA(cudaStreamSynchronize(0));
    c->name = "gpu:sm100:pow2:n" + std::to_string(n) + ":ept" + std::to_string(ept);
    return GFFT_OK;
  }
  set_error("length " + std::to_string(n) + " has no GPU schedule yet");
  return GFFT_ERR_NOT_IMPLEMENTED;
}

void core_free(PlanCore* c) {
  if (c->tw) cudaFree(c->tw);
  c->tw = nullptr;
}

gfft_status core_exec(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                      int64_t odist, cudaStream_t st) {
  if (count <= 0) return GFFT_OK;
  switch (c->algo) {
    case Algo::Trivial: {
      if (dst == src && idist == odist) return GFFT_OK;
      int blocks = int(std::min<int64_t>((count + 255) / 256, 65535));
      if (c->prec == kC64)
        k_copy_batch<float2><<<blocks, 256, 0, st>>>(static_cast<float2*>(dst), static_cast<const float2*>(src), 1,
                                                      count, idist, odist);
      else
        k_copy_batch<double2><<<blocks, 256, 0, st>>>(static_cast<double2*>(dst), static_cast<const double2*>(src),
                                                       1, count, idist, odist);
      GFFT_CUDA(cudaGetLastError());
      return GFFT_OK;
    }
    case Algo::Pow2Smem: {
      const Pow2Kernel* k = c->k[dir < 0 ? 0 : 1];
      const double scale = dir < 0 ? 1.0 : 1.0 / double(c->n);
      GFFT_CUDA(k->launch(src, dst, count, idist, odist, c->tw, scale, st));
      return GFFT_OK;
    }
  }
  return GFFT_ERR_NOT_IMPLEMENTED;
}

}  // namespace gfft
