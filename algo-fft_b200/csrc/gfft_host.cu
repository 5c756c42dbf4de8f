// Host-slice execution of 1-D batches (the Go-slice methods Plan.Forward /
// ForwardBatch with []complex64 arguments, plan.go:332-571).
//
// A Go slice lives in pageable memory, which the copy engines cannot read
// directly: the driver then copies through its own small staging area and
// the copies of one call neither overlap each other nor the transforms.  So
// a batch in pageable memory moves through library-owned pinned lanes:
//   host thread pool: pageable src chunk -> pinned lane buffer
//   lane stream:      pinned -> device, transforms, device -> pinned
//   host thread pool: pinned lane buffer -> pageable dst chunk
// with three lanes in flight, so the host copies of one chunk overlap the
// device copies and transforms of the other two.  Buffers that are already
// pinned (cudaHostAlloc / cudaHostRegister) skip the host copies and go
// straight through the lanes' device buffers.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>
#include "gfft_copypool.h"
#include "gfft_internal.h"

namespace gfft {
namespace {

// Pinned staging buffers kept for later calls (portable: any device may
// copy from them); one lane set per concurrent call.  At most kKeep bytes
// wait in the free list; a buffer released beyond that is freed.
class PinnedPool {
 public:
  static PinnedPool& get() {
    static PinnedPool* pool = new PinnedPool();
    return *pool;
  }
  cudaError_t acquire(size_t bytes, void** out) {
    {
      std::lock_guard<std::mutex> g(mu_);
      auto it = free_.lower_bound(bytes);
      if (it != free_.end() && it->first <= 2 * bytes) {
        *out = it->second;
        kept_ -= it->first;
        free_.erase(it);
        return cudaSuccess;
      }
    }
    cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
    if (e == cudaSuccess) {
      std::lock_guard<std::mutex> g(mu_);
      size_of_[*out] = bytes;
    }
    return e;
  }
  void release(void* p) {
    if (!p) return;
    {
      std::lock_guard<std::mutex> g(mu_);
      const size_t b = size_of_[p];
      if (kept_ + b <= kKeep) {
        free_.emplace(b, p);
        kept_ += b;
        return;
      }
      size_of_.erase(p);
    }
    cudaFreeHost(p);
  }

 private:
  static constexpr size_t kKeep = size_t(512) << 20;
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  std::map<void*, size_t> size_of_;
  size_t kept_ = 0;  // bytes in free_
};

bool host_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // older drivers report unregistered memory as an error
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

constexpr int kLanes = 3;

// Streams and events of the lanes, created once per device and reused by
// later calls (one set per concurrent call).
struct LaneSet {
  int dev = -1;
  bool busy = false;
  cudaStream_t st[kLanes] = {};
  cudaEvent_t ev[kLanes] = {};
};

class LanePool {
 public:
  static LanePool& get() {
    static LanePool* pool = new LanePool();
    return *pool;
  }
  cudaError_t acquire(int dev, LaneSet** out) {
    {
      std::lock_guard<std::mutex> g(mu_);
      for (LaneSet* l : sets_)
        if (l->dev == dev && !l->busy) {
          l->busy = true;
          *out = l;
          return cudaSuccess;
        }
    }
    auto* l = new LaneSet();
    l->dev = dev;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < kLanes && e == cudaSuccess; ++i) e = cudaStreamCreateWithFlags(&l->st[i], cudaStreamNonBlocking);
    for (int i = 0; i < kLanes && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&l->ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) {
      for (int i = 0; i < kLanes; ++i) {
        if (l->st[i]) cudaStreamDestroy(l->st[i]);
        if (l->ev[i]) cudaEventDestroy(l->ev[i]);
      }
      delete l;
      return e;
    }
    l->busy = true;
    std::lock_guard<std::mutex> g(mu_);
    sets_.push_back(l);
    *out = l;
    return cudaSuccess;
  }
  void release(LaneSet* l) {
    std::lock_guard<std::mutex> g(mu_);
    l->busy = false;
  }

 private:
  std::mutex mu_;
  std::vector<LaneSet*> sets_;
};

}  // namespace

gfft_status run_host(gfft_plan* p, int dir, void* dst, const void* src, int64_t count) {
  DeviceGuard dg;
  GFFT_CUDA(dg.set(p->core.device));
  const size_t tb = size_t(p->core.n) * elem_bytes(p->core.prec);
  const size_t total = size_t(count) * tb;
  // tiny batches (up to 64 KB) copy straight from the caller's memory (the
  // driver stages them); anything larger in pageable memory goes through
  // the pinned lanes and the copy pool
  const bool staged = total > (size_t(64) << 10) && !(host_pinned(src) && host_pinned(dst));
  // chunks of about 64 MB (pinned) / 32 MB (staged), whole transforms; a
  // smaller batch is cut into about six chunks so the lanes still overlap
  const size_t target = std::min(staged ? (size_t(32) << 20) : (size_t(64) << 20),
                                 std::max(size_t(256) << 10, total / 6));
  const int64_t per = std::max<int64_t>(1, std::min<int64_t>(count, int64_t(target / tb)));
  const int64_t nchunks = (count + per - 1) / per;
  const int lanes = int(std::min<int64_t>(kLanes, nchunks));
  LaneSet* ls = nullptr;
  GFFT_CUDA(LanePool::get().acquire(p->core.device, &ls));
  cudaStream_t* st = ls->st;
  cudaEvent_t* ev = ls->ev;
  void* d[kLanes] = {};
  void* h[kLanes] = {};
  int64_t pending[kLanes] = {-1, -1, -1};  // chunk whose result waits in lane's pinned buffer
  gfft_status s = GFFT_OK;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < lanes && e == cudaSuccess; ++i) e = ws_alloc(&d[i], size_t(per) * tb, st[i]);
  for (int i = 0; staged && i < lanes && e == cudaSuccess; ++i) e = PinnedPool::get().acquire(size_t(per) * tb, &h[i]);
  if (e != cudaSuccess) s = cuda_status(e, "host path setup");
  CopyPool& cp = CopyPool::get();
  auto chunk_bytes = [&](int64_t k) { return size_t(std::min(per, count - k * per)) * tb; };
  // copies a finished chunk from its lane's pinned buffer to dst
  auto drain = [&](int lane) -> gfft_status {
    if (pending[lane] < 0) return GFFT_OK;
    const int64_t k = pending[lane];
    pending[lane] = -1;
    cudaError_t ee = cudaEventSynchronize(ev[lane]);
    if (ee != cudaSuccess) return cuda_status(ee, "cudaEventSynchronize");
    cp.copy(static_cast<char*>(dst) + size_t(k * per) * tb, h[lane], chunk_bytes(k));
    return GFFT_OK;
  };
  for (int64_t k = 0; k < nchunks && s == GFFT_OK; ++k) {
    const int lane = int(k % lanes);
    const size_t bytes = chunk_bytes(k), off = size_t(k * per) * tb;
    const int64_t m = int64_t(bytes / tb);
    const void* in = static_cast<const char*>(src) + off;
    void* out = static_cast<char*>(dst) + off;
    if (staged) {
      s = drain(lane);
      if (s != GFFT_OK) break;
      cp.copy(h[lane], in, bytes);
      in = h[lane];
      out = h[lane];
    }
    e = cudaMemcpyAsync(d[lane], in, bytes, cudaMemcpyHostToDevice, st[lane]);
    if (e != cudaSuccess) {
      s = cuda_status(e, "cudaMemcpyAsync(H2D)");
      break;
    }
    s = core_exec(&p->core, dir, d[lane], d[lane], m, p->core.n, p->core.n, st[lane]);
    if (s != GFFT_OK) break;
    e = cudaMemcpyAsync(out, d[lane], bytes, cudaMemcpyDeviceToHost, st[lane]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[lane], st[lane]);
    if (e != cudaSuccess) {
      s = cuda_status(e, "cudaMemcpyAsync(D2H)");
      break;
    }
    if (staged) pending[lane] = k;
  }
  // results of the last chunks, oldest first
  for (int64_t k = std::max<int64_t>(0, nchunks - lanes); k < nchunks && s == GFFT_OK; ++k) s = drain(int(k % lanes));
  for (int i = 0; i < lanes; ++i) {
    if (d[i]) cudaFreeAsync(d[i], st[i]);
    e = cudaStreamSynchronize(st[i]);
    if (e != cudaSuccess && s == GFFT_OK) s = cuda_status(e, "cudaStreamSynchronize");
    PinnedPool::get().release(h[i]);
  }
  LanePool::get().release(ls);
  return s;
}

}  // namespace gfft
