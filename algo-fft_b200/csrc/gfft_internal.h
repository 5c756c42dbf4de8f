// Internal plan object and helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include "../../include/gfft.h"
#include "gfft_registry.h"

namespace gfft {

// Thread-local detail string behind gfft_last_error().
void set_error(const std::string& msg);
void clear_error();
gfft_status cuda_status(cudaError_t e, const char* what);

#define GFFT_CUDA(call)                                         \
  do {                                                          \
    cudaError_t e_ = (call);                                    \
    if (e_ != cudaSuccess) return ::gfft::cuda_status(e_, #call); \
  } while (0)

enum class Algo { Trivial, Pow2Smem };

// Device twiddle table W_n^m = exp(-2πi m/n), m < n, generated on the GPU in
// FP64 and rounded to the element type (internal/math/twiddle.go:8-21).
gfft_status make_twiddles(int prec, int64_t n, void** out, cudaStream_t st);

struct PlanCore {
  int prec = kC64;
  int64_t n = 0;
  int device = 0;
  Algo algo = Algo::Trivial;
  const Pow2Kernel* k[2] = {nullptr, nullptr};  // [0] forward, [1] inverse
  void* tw = nullptr;
  std::string name;
};

// Chooses and prepares the schedule of a 1-D complex transform of length n.
gfft_status core_init(PlanCore* c, int prec, int64_t n, int device);
void core_free(PlanCore* c);

// Runs `count` transforms (dir -1 forward, +1 inverse) with element strides
// idist/odist between consecutive transforms; device pointers.
gfft_status core_exec(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                      int64_t odist, cudaStream_t st);

inline size_t elem_bytes(int prec) { return prec == kC64 ? 8 : 16; }

}  // namespace gfft

struct gfft_plan {
  gfft::PlanCore core;
  gfft_plan_options opts{};
};
