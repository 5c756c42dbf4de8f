// Host copy pool of the Go-slice path: large memcpys split over persistent
// threads.  Host-only C++ (no CUDA), so the pool is unit-tested on its own.
#pragma once
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace gfft {

// Splits large memcpys over persistent threads (one call at a time; the
// calling thread takes a share too; during a host-slice call it does nothing
// else, so by default every other core helps).  A worker spins for a short while on
// the job counter before it sleeps, so the back-to-back copies of one
// host-slice call do not pay a thread wake-up each.
class CopyPool {
 public:
  // workers = -1: every core but the caller's (at most 31)
  explicit CopyPool(int workers = -1) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned n = workers >= 0 ? unsigned(workers) : std::min(31u, hw > 1 ? hw - 1 : 0u);
    for (unsigned i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
    for (auto& t : workers_) t.detach();
  }

  static CopyPool& get() {
    static CopyPool* pool = new CopyPool();  // never destroyed: workers outlive static teardown
    return *pool;
  }

  void copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPart = size_t(128) << 10;
    if (bytes <= 2 * kPart || workers_.empty()) {
      std::memcpy(dst, src, bytes);
      return;
    }
    std::lock_guard<std::mutex> one(call_mu_);
    const size_t nw = workers_.size();
    dst_ = static_cast<char*>(dst);
    src_ = static_cast<const char*>(src);
    bytes_ = bytes;
    part_ = std::max(kPart, (bytes / (nw + 1) + 4095) & ~size_t(4095));
    next_.store(0, std::memory_order_relaxed);
    busy_.store(int(nw), std::memory_order_relaxed);
    {
      std::lock_guard<std::mutex> g(mu_);
      gen_.fetch_add(1, std::memory_order_release);
    }
    cv_.notify_all();
    run_parts();
    while (busy_.load(std::memory_order_acquire) > 0) std::this_thread::yield();
  }

 private:
  void run_parts() {
    for (;;) {
      const size_t at = next_.fetch_add(part_, std::memory_order_relaxed);
      if (at >= bytes_) return;
      std::memcpy(dst_ + at, src_ + at, std::min(part_, bytes_ - at));
    }
  }

  void loop() {
    // generation 0 is the pool's own: a worker that starts late still takes
    // the first job (the caller waits for every worker on each job)
    uint64_t seen = 0;
    for (;;) {
      bool got = false;
      for (int spin = 0; spin < (1 << 16) && !got; ++spin) got = gen_.load(std::memory_order_acquire) != seen;
      if (!got) {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return gen_.load(std::memory_order_acquire) != seen; });
      }
      seen = gen_.load(std::memory_order_acquire);
      run_parts();
      busy_.fetch_sub(1, std::memory_order_release);
    }
  }

  std::vector<std::thread> workers_;
  std::mutex call_mu_, mu_;
  std::condition_variable cv_;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t bytes_ = 0, part_ = 0;
  std::atomic<size_t> next_{0};
  std::atomic<int> busy_{0};
  std::atomic<uint64_t> gen_{0};
};

}  // namespace gfft
