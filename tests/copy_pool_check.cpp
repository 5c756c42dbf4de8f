// Unit check of the host copy pool (algo-fft_b200/csrc/gfft_copypool.h),
// built and run by tests/test_copy_pool.py: copies of many sizes issued
// back to back from the first instant of a fresh pool (workers still
// starting), by one and by several calling threads in turn, each checked
// byte for byte.  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <thread>
#include <vector>
#include "gfft_copypool.h"

static std::vector<unsigned char> filled(std::mt19937_64& rng) {
  std::vector<unsigned char> v(size_t(24) << 20);
  for (auto& b : v) b = static_cast<unsigned char>(rng());
  return v;
}

static int check(gfft::CopyPool& pool, std::mt19937_64& rng, int rounds, const std::vector<unsigned char>& src) {
  std::vector<unsigned char> dst(src.size());
  std::uniform_int_distribution<size_t> len(0, src.size());
  for (int r = 0; r < rounds; ++r) {
    const size_t n = (r % 3 == 0) ? len(rng) : len(rng) / 64;  // large and small copies mixed
    const size_t off = std::min(n, src.size() - n) & ~size_t(7);
    std::fill(dst.begin(), dst.end(), 0xA5);
    pool.copy(dst.data() + off, src.data() + off, n);
    for (size_t i = 0; i < dst.size(); ++i) {
      const bool inside = i >= off && i < off + n;
      if (dst[i] != (inside ? src[i] : 0xA5)) {
        std::fprintf(stderr, "round %d: byte %zu wrong (copy of %zu at %zu)\n", r, i, n, off);
        return 1;
      }
    }
  }
  return 0;
}

int main() {
  std::mt19937_64 rng(7);
  const std::vector<unsigned char> src = filled(rng);
  // fresh pools, used at once: the first copy is large and issued before the
  // workers have had time to start
  for (int workers : {1, 3, 7, 15, 31}) {
    for (int rep = 0; rep < 4; ++rep) {
      std::vector<unsigned char> dst(src.size());
      auto* pool = new gfft::CopyPool(workers);  // pools live for the process
      pool->copy(dst.data(), src.data(), src.size());
      if (dst != src) {
        std::fprintf(stderr, "first copy of a fresh %d-worker pool wrong\n", workers);
        return 1;
      }
      if (rep == 0 && check(*pool, rng, 20, src)) return 1;
    }
  }
  // several callers in turn on one pool
  auto* shared = new gfft::CopyPool(5);
  int bad = 0;
  std::vector<std::thread> callers;
  for (int t = 0; t < 4; ++t)
    callers.emplace_back([&, t] {
      std::mt19937_64 local(100 + t);
      if (check(*shared, local, 10, src)) bad = 1;
    });
  for (auto& c : callers) c.join();
  std::puts(bad ? "copy pool: FAILED" : "copy pool: ok");
  return bad;
}
