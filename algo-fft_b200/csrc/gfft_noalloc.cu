// Batched transform through the large-N two-pass kernel without any
// allocation in the call.
//
// Some callers cannot call cudaMalloc (or anything that may allocate) at the
// point where they run a transform: code inside a real-time or interrupt-like
// callback, a process whose allocator is owned by another runtime (a
// framework's caching allocator, a Go program that must not block in cgo on
// an allocation), or a memory-capped service that reserves every byte up
// front.  The regular entry points take their scratch from the stream-ordered
// pool on every call; this one takes it from a fixed array compiled into the
// library instead.
//
// The array is a file-scope device variable of kNoAllocScratchBytes (64 MiB).
// Every GPU that loads libgfft.so holds it for the life of the process.
// Host code only sees a host-side stand-in for its name, so the device
// address is looked up once per device with cudaGetSymbolAddress (the first
// call on each device does that, with the plan's device current; make that
// first call before any stream capture).  The region is shared by every
// call: the call's abort word and tile counters at its start are cleared on
// the call's stream before the kernel runs, the slots after them are fully
// written before they are read, and two calls that overlap on the GPU
// (different streams, or a call still running while another starts) race on
// it.  A bounded wait that expires stops only the call it happened in; it
// also sets the plan's sticky status word, which gfft_plan_check reports.
#include <mutex>
#include "gfft_internal.h"
#include "gfft_twopass.cuh"

namespace gfft {

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr size_t kNoAllocCounterBytes = size_t(512) << 10;  // abort word, tile counter, per-group counters
constexpr size_t kNoAllocStatusBytes = 256;                   // the abort word's own line at the start
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the static scratch on the current device, looked up the
// first time a device is seen (the caller has made the plan's device current).
gfft_status noalloc_scratch(void** out) {
  int dev = 0;
  GFFT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device index out of range for the no-allocation path");
    return GFFT_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return GFFT_OK;
}

}  // namespace

}  // namespace gfft

using namespace gfft;

extern "C" gfft_status gfft_exec_batch_noalloc(gfft_plan* plan, int32_t direction, void* dst, int64_t dst_len,
                                               const void* src, int64_t src_len, int64_t count, void* stream) {
  clear_error();
  if (!plan) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (count < 1) return GFFT_ERR_INVALID_LENGTH;
  const PlanCore* c = &plan->core;
  if (count > INT64_MAX / c->n) return GFFT_ERR_LENGTH_MISMATCH;
  if (dst_len < count * c->n || src_len < count * c->n) return GFFT_ERR_LENGTH_MISMATCH;
  if (direction != -1 && direction != 1) return GFFT_ERR_INVALID_ARGUMENT;
  if (c->algo != Algo::TwoPass && c->algo != Algo::L2Pipe) {
    set_error("the no-allocation entry point runs the two-pass kernel only; plan '" + c->name +
              "' uses another schedule");
    return GFFT_ERR_NOT_IMPLEMENTED;
  }
  const size_t es = elem_bytes(c->prec);
  const size_t tbytes = size_t(c->n) * es;
  const size_t slot_space = kNoAllocScratchBytes - kNoAllocCounterBytes;
  if (2 * tbytes > slot_space) {
    set_error("a length-" + std::to_string(c->n) + " transform needs " + std::to_string(2 * tbytes) +
              " bytes of scratch; the no-allocation path has " + std::to_string(slot_space));
    return GFFT_ERR_INVALID_ARGUMENT;
  }
  // Same slot geometry as the plan when it fits, else fewer transforms per
  // group and fewer slots (at least two).
  int64_t group = std::min<int64_t>(c->group, std::max<int64_t>(1, int64_t(slot_space / (2 * tbytes))));
  int64_t slots = std::max<int64_t>(2, std::min<int64_t>(c->slots, int64_t(slot_space / (group * tbytes))));
  const int64_t groups = (count + group - 1) / group;
  const size_t ctr_bytes = size_t(1 + 2 * groups) * sizeof(unsigned);
  if (kNoAllocStatusBytes + ctr_bytes > kNoAllocCounterBytes) {
    set_error("batch of " + std::to_string(count) + " transforms needs more tile counters than the " +
              std::to_string(kNoAllocCounterBytes) + "-byte counter area of the no-allocation path holds");
    return GFFT_ERR_INVALID_ARGUMENT;
  }
  // The scratch, twiddles and status word all live on the plan's device.
  DeviceGuard dg;
  GFFT_CUDA(dg.set(c->device));
  void* base = nullptr;
  gfft_status s = noalloc_scratch(&base);
  if (s != GFFT_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GFFT_CUDA(cudaMemsetAsync(base, 0, kNoAllocStatusBytes + ctr_bytes, st));
  const TwoPassKernel* k = c->tp[direction < 0 ? 0 : 1];
  TwoPassParams p;
  p.src = src;
  p.dst = dst;
  p.scratch = static_cast<char*>(base) + kNoAllocCounterBytes;
  p.count = count;
  p.idist = c->n;
  p.odist = c->n;
  p.tw1 = c->tw1;
  p.tw2 = c->tw2;
  p.bt.lo = c->bt_lo;
  p.bt.hi = c->bt_hi;
  p.bt.shift = c->bt_shift;
  p.ctr = reinterpret_cast<unsigned*>(static_cast<char*>(base) + kNoAllocStatusBytes);
  p.status = static_cast<unsigned*>(base);
  p.report = c->status;
  p.groups = int(groups);
  p.G = int(group);
  p.S = int(slots);
  p.scale = direction < 0 ? 1.0 : 1.0 / double(c->n);
  p.spin_limit = 1u << 24;
  const int64_t tiles = groups * group * ((k->n2 / k->nc1) + (k->n1 / k->nc2));
  const int grid = int(std::min<int64_t>(tiles, c->resident));
  GFFT_CUDA(k->launch(p, grid, st));
  return GFFT_OK;
}
