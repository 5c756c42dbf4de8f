// extern "C" entry points of libgfft.so (declared in include/gfft.h).
//
// Argument validation reproduces the reference's order and sentinel errors
// so a Go wrapper behaves exactly like the CPU library on bad input:
// plan.go:504-516 (batch), plan.go:574-584 (single), plan_strided.go:101-135
// (strided).
#include <climits>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <map>
#include <mutex>
#include <tuple>
#include "gfft_internal.h"

namespace gfft {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

gfft_status cuda_status(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
  if (e == cudaErrorMemoryAllocation) return GFFT_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GFFT_ERR_NO_DEVICE;
  return GFFT_ERR_CUDA;
}

static cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace gfft

using namespace gfft;

extern "C" {

gfft_status gfft_plan_new(gfft_plan** out, int32_t precision, int64_t n, const gfft_plan_options* opts) {
  clear_error();
  if (!out) return GFFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (n < 1) {
    set_error("n < 1");
    return GFFT_ERR_INVALID_LENGTH;
  }
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  gfft_plan_options o{};
  if (opts) o = *opts;
  if (o.batch < 0 || o.stride < 0) return GFFT_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return GFFT_ERR_NO_DEVICE;
  }
  if (o.device < 0 || o.device >= ndev) return GFFT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(o.device));
  auto* p = new (std::nothrow) gfft_plan;
  if (!p) return GFFT_ERR_OUT_OF_MEMORY;
  p->opts = o;
  p->precision = precision;
  PlanHint hint;
  hint.planner = o.planner;
  hint.batch = o.batch;
  hint.user = true;
  gfft_status s = core_init(&p->core, precision, n, o.device, o.strategy, &hint);
  if (s != GFFT_OK) {
    core_free(&p->core);
    delete p;
    return s;
  }
  *out = p;
  return GFFT_OK;
}

}  // extern "C"

namespace {
// Pooled plans (NewPlanPooled, plan.go:1040-1118): closed plans wait here,
// keyed by (device, precision, n, planner, strategy), for the next request
// of the same shape, so a caller that creates and closes plans in a loop
// does not rebuild twiddle tables each time.
struct PoolKey {
  int device, prec;
  int64_t n;
  int planner, strategy;
  bool operator<(const PoolKey& o) const {
    return std::tie(device, prec, n, planner, strategy) < std::tie(o.device, o.prec, o.n, o.planner, o.strategy);
  }
};
std::mutex g_pool_mu;
std::map<PoolKey, std::vector<gfft_plan*>> g_pool;
}  // namespace

extern "C" {

gfft_status gfft_plan_new_pooled(gfft_plan** out, int32_t precision, int64_t n, const gfft_plan_options* opts) {
  clear_error();
  if (!out) return GFFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  gfft_plan_options o{};
  if (opts) o = *opts;
  if (o.batch > 1 || o.stride > 0) return gfft_plan_new(out, precision, n, opts);  // layouts are not pooled
  {
    std::lock_guard<std::mutex> g(g_pool_mu);
    auto it = g_pool.find(PoolKey{o.device, precision, n, o.planner, o.strategy});
    if (it != g_pool.end() && !it->second.empty()) {
      *out = it->second.back();
      it->second.pop_back();
      return GFFT_OK;
    }
  }
  gfft_status s = gfft_plan_new(out, precision, n, opts);
  if (s == GFFT_OK) (*out)->pooled = true;
  return s;
}

void gfft_plan_pool_clear(void) {
  std::vector<gfft_plan*> all;
  {
    std::lock_guard<std::mutex> g(g_pool_mu);
    for (auto& kv : g_pool)
      for (gfft_plan* p : kv.second) all.push_back(p);
    g_pool.clear();
  }
  for (gfft_plan* p : all) {
    core_free(&p->core);
    delete p;
  }
}

void gfft_plan_close(gfft_plan* plan) {
  if (!plan) return;
  if (plan->pooled) {
    std::lock_guard<std::mutex> g(g_pool_mu);
    g_pool[PoolKey{plan->opts.device, plan->precision, plan->core.n, plan->opts.planner, plan->opts.strategy}]
        .push_back(plan);
    return;
  }
  core_free(&plan->core);
  delete plan;
}

void gfft_set_kernel_strategy(int32_t strategy) { set_kernel_strategy(strategy); }
int32_t gfft_get_kernel_strategy(void) { return get_kernel_strategy(); }
void gfft_record_benchmark_decision(int64_t n, int32_t strategy) {
  // internal/planner/selection.go:42-60: lengths >= 1 and the four
  // schedule strategies only
  if (n <= 0) return;
  if (strategy != GFFT_KERNEL_DIT && strategy != GFFT_KERNEL_STOCKHAM && strategy != GFFT_KERNEL_SIXSTEP &&
      strategy != GFFT_KERNEL_EIGHTSTEP)
    return;
  record_decision(n, strategy);
}

gfft_status gfft_plan_clone(gfft_plan** out, const gfft_plan* src) {
  clear_error();
  if (!out || !src) return GFFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(src->core.device));
  auto* p = new (std::nothrow) gfft_plan;
  if (!p) return GFFT_ERR_OUT_OF_MEMORY;
  p->opts = src->opts;
  p->precision = src->precision;
  // the same schedule, tables rebuilt for the copy
  gfft_status s = src->core.n == 1 ? core_init(&p->core, src->precision, 1, src->core.device)
                                   : core_init_variant(&p->core, src->precision, src->core.n, src->core.device,
                                                       src->core.name);
  if (s != GFFT_OK) {
    core_free(&p->core);
    delete p;
    return s;
  }
  *out = p;
  return GFFT_OK;
}

int64_t gfft_plan_len(const gfft_plan* plan) { return plan ? plan->core.n : 0; }

gfft_status gfft_plan_algorithm(const gfft_plan* plan, char* buf, size_t cap) {
  if (!plan || !buf || cap == 0) return GFFT_ERR_INVALID_ARGUMENT;
  std::strncpy(buf, plan->core.name.c_str(), cap - 1);
  buf[cap - 1] = 0;
  return GFFT_OK;
}

// plan.go:574-584 validateSlices.
static gfft_status check_single(gfft_plan* p, const void* dst, int64_t dst_len, const void* src, int64_t src_len) {
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (dst_len != p->core.n || src_len != p->core.n) return GFFT_ERR_LENGTH_MISMATCH;
  return GFFT_OK;
}

// plan.go:505-516.
static gfft_status check_batch(gfft_plan* p, const void* dst, int64_t dst_len, const void* src, int64_t src_len,
                               int64_t count) {
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (count < 1) return GFFT_ERR_INVALID_LENGTH;
  if (count > INT64_MAX / p->core.n) return GFFT_ERR_LENGTH_MISMATCH;
  const int64_t required = count * p->core.n;
  if (dst_len < required || src_len < required) return GFFT_ERR_LENGTH_MISMATCH;
  return GFFT_OK;
}

static gfft_status do_single(gfft_plan* p, int dir, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                             void* stream) {
  clear_error();
  gfft_status s = check_single(p, dst, dst_len, src, src_len);
  if (s != GFFT_OK) return s;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(p->core.device));
  return core_exec(&p->core, dir, dst, src, 1, p->core.n, p->core.n, as_stream(stream));
}

static gfft_status do_batch(gfft_plan* p, int dir, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                            int64_t count, void* stream) {
  clear_error();
  gfft_status s = check_batch(p, dst, dst_len, src, src_len, count);
  if (s != GFFT_OK) return s;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(p->core.device));
  return core_exec(&p->core, dir, dst, src, count, p->core.n, p->core.n, as_stream(stream));
}

gfft_status gfft_forward(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len, void* stream) {
  return do_single(p, -1, dst, dst_len, src, src_len, stream);
}
gfft_status gfft_inverse(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len, void* stream) {
  return do_single(p, +1, dst, dst_len, src, src_len, stream);
}
gfft_status gfft_forward_batch(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                               int64_t count, void* stream) {
  return do_batch(p, -1, dst, dst_len, src, src_len, count, stream);
}
gfft_status gfft_inverse_batch(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                               int64_t count, void* stream) {
  return do_batch(p, +1, dst, dst_len, src, src_len, count, stream);
}

// plan_strided.go:101-135 validateStridedSlices.
static gfft_status check_strided(gfft_plan* p, const void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                 int64_t stride) {
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (stride < 1) return GFFT_ERR_INVALID_STRIDE;
  const int64_t n = p->core.n;
  if (stride == 1) {
    if (dst_len < n || src_len < n) return GFFT_ERR_LENGTH_MISMATCH;
    return GFFT_OK;
  }
  const int64_t max_index = n - 1;
  if (max_index > (INT64_MAX - 1) / stride) return GFFT_ERR_INVALID_STRIDE;
  const int64_t required = 1 + max_index * stride;
  if (dst_len < required || src_len < required) return GFFT_ERR_LENGTH_MISMATCH;
  return GFFT_OK;
}

static gfft_status do_strided(gfft_plan* p, int dir, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                              int64_t stride, void* stream) {
  clear_error();
  gfft_status s = check_strided(p, dst, dst_len, src, src_len, stride);
  if (s != GFFT_OK) return s;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(p->core.device));
  const int64_t n = p->core.n;
  if (stride == 1) return core_exec(&p->core, dir, dst, src, 1, n, n, as_stream(stream));
  // Gather the column into a contiguous buffer, transform, scatter back
  // (plan_strided.go:72-98): two strided 2-D copies around one transform.
  cudaStream_t st = as_stream(stream);
  const size_t es = elem_bytes(p->core.prec);
  void* tmp = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&tmp), size_t(n) * es, st));
  cudaError_t e = cudaMemcpy2DAsync(tmp, es, src, size_t(stride) * es, es, size_t(n), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) {
    s = core_exec(&p->core, dir, tmp, tmp, 1, n, n, st);
    if (s == GFFT_OK) {
      e = cudaMemcpy2DAsync(dst, size_t(stride) * es, tmp, es, es, size_t(n), cudaMemcpyDeviceToDevice, st);
    }
  }
  cudaFreeAsync(tmp, st);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemcpy2DAsync");
  return s;
}

gfft_status gfft_forward_strided(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                 int64_t stride, void* stream) {
  return do_strided(p, -1, dst, dst_len, src, src_len, stride, stream);
}
gfft_status gfft_inverse_strided(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                 int64_t stride, void* stream) {
  return do_strided(p, +1, dst, dst_len, src, src_len, stride, stream);
}

gfft_status gfft_forward_host(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len) {
  clear_error();
  gfft_status s = check_single(p, dst, dst_len, src, src_len);
  return s != GFFT_OK ? s : run_host(p, -1, dst, src, 1);
}
gfft_status gfft_inverse_host(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len) {
  clear_error();
  gfft_status s = check_single(p, dst, dst_len, src, src_len);
  return s != GFFT_OK ? s : run_host(p, +1, dst, src, 1);
}
gfft_status gfft_forward_batch_host(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                    int64_t count) {
  clear_error();
  gfft_status s = check_batch(p, dst, dst_len, src, src_len, count);
  return s != GFFT_OK ? s : run_host(p, -1, dst, src, count);
}
gfft_status gfft_inverse_batch_host(gfft_plan* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                    int64_t count) {
  clear_error();
  gfft_status s = check_batch(p, dst, dst_len, src, src_len, count);
  return s != GFFT_OK ? s : run_host(p, +1, dst, src, count);
}

gfft_status gfft_plan_new_variant(gfft_plan** out, int32_t precision, int64_t n, const char* token) {
  clear_error();
  if (!out || !token) return GFFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (n < 1) return GFFT_ERR_INVALID_LENGTH;
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GFFT_ERR_NO_DEVICE;
  int dev = 0;
  GFFT_CUDA(cudaGetDevice(&dev));
  auto* p = new (std::nothrow) gfft_plan;
  if (!p) return GFFT_ERR_OUT_OF_MEMORY;
  p->opts.device = dev;
  p->precision = precision;
  gfft_status s = core_init_variant(&p->core, precision, n, dev, token);
  if (s != GFFT_OK) {
    core_free(&p->core);
    delete p;
    return s;
  }
  *out = p;
  return GFFT_OK;
}

static gfft_status copy_out(const std::string& text, char* buf, size_t cap, size_t* needed) {
  if (needed) *needed = text.size() + 1;
  if (!buf) return GFFT_OK;
  if (cap < text.size() + 1) {
    set_error("buffer too small");
    return GFFT_ERR_INVALID_ARGUMENT;
  }
  std::memcpy(buf, text.c_str(), text.size() + 1);
  return GFFT_OK;
}

gfft_status gfft_plan_variants(int32_t precision, int64_t n, char* buf, size_t cap, size_t* needed) {
  clear_error();
  std::string text;
  for (const auto& t : variant_tokens(precision, n)) text += t + "\n";
  return copy_out(text, buf, cap, needed);
}

gfft_status gfft_plan_check(gfft_plan* plan) {
  clear_error();
  if (!plan) return GFFT_ERR_INVALID_ARGUMENT;
  if (core_device_status(&plan->core) != 0) {
    set_error("a bounded device wait expired in this plan's kernels");
    return GFFT_ERR_TIMEOUT;
  }
  return GFFT_OK;
}

gfft_status gfft_autotune(int32_t precision, int64_t n, int64_t count, int32_t iters, char* report, size_t cap,
                          size_t* needed) {
  clear_error();
  if (n < 1) return GFFT_ERR_INVALID_LENGTH;
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GFFT_ERR_NO_DEVICE;
  std::string best, rep;
  gfft_status s = autotune(precision, n, count, iters > 0 ? iters : 10, &best, &rep);
  if (s != GFFT_OK) return s;
  return copy_out(rep, report, cap, needed);
}

gfft_status gfft_wisdom_import_string(const char* text) {
  clear_error();
  if (!text) return GFFT_ERR_INVALID_ARGUMENT;
  return wisdom_import(text);
}

gfft_status gfft_wisdom_export_string(char* buf, size_t cap, size_t* needed) {
  clear_error();
  return copy_out(wisdom_export(), buf, cap, needed);
}

gfft_status gfft_wisdom_import_file(const char* path) {
  clear_error();
  if (!path) return GFFT_ERR_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error(std::string("failed to open wisdom file: ") + path);
    return GFFT_ERR_WISDOM;
  }
  std::string text;
  char chunk[4096];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) text.append(chunk, got);
  std::fclose(f);
  return wisdom_import(text);
}

gfft_status gfft_wisdom_export_file(const char* path) {
  clear_error();
  if (!path) return GFFT_ERR_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error(std::string("failed to create wisdom file: ") + path);
    return GFFT_ERR_WISDOM;
  }
  const std::string text = wisdom_export();
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  std::fclose(f);
  if (!ok) {
    set_error("failed to write wisdom file");
    return GFFT_ERR_WISDOM;
  }
  return GFFT_OK;
}

void gfft_wisdom_clear(void) { wisdom_clear(); }

int64_t gfft_wisdom_len(void) { return int64_t(wisdom_len()); }

const char* gfft_status_string(int32_t status) {
  switch (status) {
    case GFFT_OK: return "ok";
    case GFFT_ERR_INVALID_LENGTH: return "algo-fft: invalid FFT length";
    case GFFT_ERR_NIL_SLICE: return "algo-fft: nil slice";
    case GFFT_ERR_LENGTH_MISMATCH: return "algo-fft: slice length mismatch";
    case GFFT_ERR_INVALID_STRIDE: return "algo-fft: invalid stride";
    case GFFT_ERR_INVALID_SPECTRUM: return "algo-fft: invalid spectrum";
    case GFFT_ERR_NOT_IMPLEMENTED: return "algo-fft: not implemented";
    case GFFT_ERR_CUDA: return "gfft: CUDA error";
    case GFFT_ERR_OUT_OF_MEMORY: return "gfft: out of memory";
    case GFFT_ERR_TIMEOUT: return "gfft: device wait timed out";
    case GFFT_ERR_NO_DEVICE: return "gfft: no CUDA device";
    case GFFT_ERR_INVALID_ARGUMENT: return "gfft: invalid argument";
    case GFFT_ERR_WISDOM: return "gfft: malformed wisdom";
  }
  return "gfft: unknown status";
}

const char* gfft_last_error(void) { return g_last_error.c_str(); }

gfft_status gfft_device_count(int32_t* count) {
  if (!count) return GFFT_ERR_INVALID_ARGUMENT;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
  *count = n;
  return GFFT_OK;
}

gfft_status gfft_buffer_alloc(void** ptr, int64_t bytes) {
  clear_error();
  if (!ptr || bytes < 0) return GFFT_ERR_INVALID_ARGUMENT;
  *ptr = nullptr;
  GFFT_CUDA(cudaMalloc(ptr, size_t(bytes > 0 ? bytes : 1)));
  return GFFT_OK;
}

gfft_status gfft_buffer_free(void* ptr) {
  clear_error();
  if (ptr) GFFT_CUDA(cudaFree(ptr));
  return GFFT_OK;
}

gfft_status gfft_buffer_upload(void* dst_device, const void* src_host, int64_t bytes) {
  clear_error();
  if (!dst_device || !src_host || bytes < 0) return GFFT_ERR_INVALID_ARGUMENT;
  GFFT_CUDA(cudaMemcpy(dst_device, src_host, size_t(bytes), cudaMemcpyHostToDevice));
  return GFFT_OK;
}

gfft_status gfft_buffer_download(void* dst_host, const void* src_device, int64_t bytes) {
  clear_error();
  if (!dst_host || !src_device || bytes < 0) return GFFT_ERR_INVALID_ARGUMENT;
  GFFT_CUDA(cudaMemcpy(dst_host, src_device, size_t(bytes), cudaMemcpyDeviceToHost));
  return GFFT_OK;
}

gfft_status gfft_stream_create(void** stream) {
  clear_error();
  if (!stream) return GFFT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = nullptr;
  GFFT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  *stream = s;
  return GFFT_OK;
}

gfft_status gfft_stream_synchronize(void* stream) {
  clear_error();
  GFFT_CUDA(cudaStreamSynchronize(as_stream(stream)));
  return GFFT_OK;
}

gfft_status gfft_stream_destroy(void* stream) {
  clear_error();
  if (stream) GFFT_CUDA(cudaStreamDestroy(as_stream(stream)));
  return GFFT_OK;
}

}  // extern "C"
