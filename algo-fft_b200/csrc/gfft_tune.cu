// Wisdom store and autotuner.
//
// Wisdom keeps the reference's text format, one decision per line
//   size:precision:features:algorithm:unix_ts
// (internal/planner/wisdom.go:96-205).  GPU decisions use features = 100
// (the sm_100 compute capability) and an algorithm token without ':' naming
// the kernel variant, e.g. "gpu-sm100-tp-1024x1024-t8192-e16".  Unlike the
// reference, where ImportWisdom fills a store that plan creation never
// consults (plan.go:832), every plan created here looks the store up.
//
// The autotuner measures every compiled variant of a length on the device
// with CUDA events (the role of internal/fft/measure.go:89-228) and records
// the fastest in the store.
#include <dlfcn.h>
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>
#include "gfft_internal.h"
#include "gfft_math.cuh"

namespace gfft {

namespace {

struct WKey {
  int64_t size;
  int prec;
  uint64_t features;
  bool operator<(const WKey& o) const {
    if (size != o.size) return size < o.size;
    if (prec != o.prec) return prec < o.prec;
    return features < o.features;
  }
};

struct WVal {
  std::string algo;
  int64_t ts;
};

std::mutex g_wmu;
std::map<WKey, WVal>& store() {
  static std::map<WKey, WVal> s;
  return s;
}

bool parse_i64(const std::string& s, int64_t* out) {
  if (s.empty()) return false;
  char* end = nullptr;
  long long v = std::strtoll(s.c_str(), &end, 10);
  if (*end != 0) return false;
  *out = v;
  return true;
}

}  // namespace

const uint64_t kGpuFeatures = 100;

bool wisdom_lookup(int64_t n, int prec, std::string* algo) {
  std::lock_guard<std::mutex> g(g_wmu);
  auto it = store().find(WKey{n, prec, kGpuFeatures});
  if (it == store().end()) return false;
  *algo = it->second.algo;
  return true;
}

void wisdom_store(int64_t n, int prec, const std::string& algo) {
  std::lock_guard<std::mutex> g(g_wmu);
  const int64_t ts = std::chrono::duration_cast<std::chrono::seconds>(
                         std::chrono::system_clock::now().time_since_epoch()).count();
  store()[WKey{n, prec, kGpuFeatures}] = WVal{algo, ts};
}

// internal/planner/wisdom.go:130-205 Import / parseWisdomLine.
gfft_status wisdom_import(const std::string& text) {
  std::map<WKey, WVal> parsed;
  std::istringstream in(text);
  std::string line;
  int lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    size_t a = line.find_first_not_of(" \t\r");
    if (a == std::string::npos) continue;
    size_t b = line.find_last_not_of(" \t\r");
    line = line.substr(a, b - a + 1);
    if (line.empty() || line[0] == '#') continue;
    std::vector<std::string> parts;
    size_t pos = 0;
    for (;;) {
      size_t q = line.find(':', pos);
      parts.push_back(line.substr(pos, q == std::string::npos ? std::string::npos : q - pos));
      if (q == std::string::npos) break;
      pos = q + 1;
    }
    int64_t size, prec, feat, ts;
    if (parts.size() != 5) {
      set_error("wisdom line " + std::to_string(lineno) + ": expected 5 fields, got " + std::to_string(parts.size()));
      return GFFT_ERR_WISDOM;
    }
    if (!parse_i64(parts[0], &size) || !parse_i64(parts[1], &prec) || prec < 0 || prec > 255 ||
        !parse_i64(parts[2], &feat) || feat < 0 || !parse_i64(parts[4], &ts)) {
      set_error("wisdom line " + std::to_string(lineno) + ": invalid number");
      return GFFT_ERR_WISDOM;
    }
    parsed[WKey{size, int(prec), uint64_t(feat)}] = WVal{parts[3], ts};
  }
  std::lock_guard<std::mutex> g(g_wmu);
  for (auto& kv : parsed) store()[kv.first] = kv.second;
  return GFFT_OK;
}

// internal/planner/wisdom.go:96-128 Export (sorted by size, precision, features).
std::string wisdom_export() {
  std::lock_guard<std::mutex> g(g_wmu);
  std::string out;
  for (const auto& kv : store()) {
    out += std::to_string(kv.first.size) + ":" + std::to_string(kv.first.prec) + ":" +
           std::to_string(kv.first.features) + ":" + kv.second.algo + ":" + std::to_string(kv.second.ts) + "\n";
  }
  return out;
}

void wisdom_clear() {
  std::lock_guard<std::mutex> g(g_wmu);
  store().clear();
}

size_t wisdom_len() {
  std::lock_guard<std::mutex> g(g_wmu);
  return store().size();
}

// The library's tuned defaults: at load time, the file named by GFFT_WISDOM
// (if set; "off" disables) or wisdom/b200_sm100.wisdom next to libgfft.so is
// imported into the store.  A missing or malformed file is ignored.
namespace {
__attribute__((constructor)) void load_default_wisdom() {
  std::string path;
  if (const char* env = std::getenv("GFFT_WISDOM")) {
    if (std::string(env) == "off") return;
    path = env;
  } else {
    Dl_info info;
    if (!dladdr(reinterpret_cast<void*>(&load_default_wisdom), &info) || !info.dli_fname) return;
    std::string lib = info.dli_fname;
    const size_t slash = lib.find_last_of('/');
    path = (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/wisdom/b200_sm100.wisdom";
  }
  std::ifstream f(path);
  if (!f) return;
  std::stringstream ss;
  ss << f.rdbuf();
  wisdom_import(ss.str());
}
}  // namespace

// ------------------------------------------------------------ autotuner

namespace {

template <typename C>
__global__ void k_fill(C* p, int64_t count) {
  using Re = typename RealOf<C>::type;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t h = uint32_t(i) * 2654435761u ^ uint32_t(i >> 32) * 40503u;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    p[i] = C{Re(int(h & 0xffff) - 32768) * Re(1.0 / 32768), Re(int(h >> 16) - 32768) * Re(1.0 / 32768)};
  }
}

}  // namespace

gfft_status autotune(int prec, int64_t n, int64_t count, int iters, std::string* best, std::string* report) {
  std::vector<std::string> toks = variant_tokens(prec, n);
  if (toks.empty()) {
    set_error("no compiled variant for this length");
    return GFFT_ERR_NOT_IMPLEMENTED;
  }
  if (count < 1) count = std::max<int64_t>(1, (int64_t(1) << 25) / n);
  const size_t bytes = size_t(count) * size_t(n) * elem_bytes(prec);
  cudaStream_t st = nullptr;
  GFFT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  void *a = nullptr, *b = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  gfft_status s = GFFT_OK;
  cudaError_t e = cudaMalloc(&a, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&b, bytes);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) {
    const int64_t total = count * n;
    if (prec == kC64)
      k_fill<float2><<<1024, 256, 0, st>>>(static_cast<float2*>(a), total);
    else
      k_fill<double2><<<1024, 256, 0, st>>>(static_cast<double2*>(a), total);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) s = cuda_status(e, "autotune setup");
  float best_ms = 0;
  std::string rep = "{\"n\": " + std::to_string(n) + ", \"precision\": " + std::to_string(prec) +
                    ", \"count\": " + std::to_string(count) + ", \"variants\": {";
  bool first = true;
  for (const auto& tok : toks) {
    if (s != GFFT_OK) break;
    PlanCore c;
    gfft_status ps = core_init_variant(&c, prec, n, c.device, tok);
    if (ps != GFFT_OK) {
      core_free(&c);
      continue;
    }
    std::vector<float> times;
    for (int it = 0; it < iters + 2 && s == GFFT_OK; ++it) {
      cudaEventRecord(e0, st);
      s = core_exec(&c, -1, b, a, count, n, n, st);
      cudaEventRecord(e1, st);
      if (s == GFFT_OK && cudaEventSynchronize(e1) == cudaSuccess) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (it >= 2) times.push_back(ms);
      }
    }
    if (s == GFFT_OK && core_device_status(&c) != 0) s = GFFT_ERR_TIMEOUT;
    core_free(&c);
    if (s != GFFT_OK || times.empty()) break;
    std::sort(times.begin(), times.end());
    const float med = times[times.size() / 2];
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.6f", med);
    rep += std::string(first ? "" : ", ") + "\"" + tok + "\": " + buf;
    first = false;
    if (best->empty() || med < best_ms) {
      best_ms = med;
      *best = tok;
    }
  }
  rep += "}, \"best\": \"" + *best + "\"}";
  if (report) *report = rep;
  if (a) cudaFree(a);
  if (b) cudaFree(b);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  if (s == GFFT_OK && !best->empty()) wisdom_store(n, prec, *best);
  return s;
}

}  // namespace gfft
