// Internal plan object and helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/gfft.h"
#include "gfft_registry.h"
#include "gfft_generic.cuh"

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

// Makes a device current for the guard's scope and gives the calling thread
// its previous current device back when the scope ends, so no entry point
// leaves the caller's device changed.
class DeviceGuard {
 public:
  DeviceGuard() = default;
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
  cudaError_t set(int device) {
    cudaError_t e = cudaGetDevice(&prev_);
    if (e != cudaSuccess || prev_ == device) return e;
    e = cudaSetDevice(device);
    restore_ = e == cudaSuccess;
    return e;
  }
  ~DeviceGuard() {
    if (restore_) cudaSetDevice(prev_);
  }

 private:
  int prev_ = 0;
  bool restore_ = false;
};

enum class Algo { Trivial, Pow2Smem, TwoPass, ThreePass, Generic, GenTwoPass, Bluestein, TensorCore, L2Pipe };

// Device twiddle table W_n^m = exp(-2πi m/n), m < n, generated on the GPU in
// FP64 and rounded to the element type (internal/math/twiddle.go:8-21).
gfft_status make_twiddles(int prec, int64_t n, void** out, cudaStream_t st);

struct PlanCore {
  int prec = kC64;
  int64_t n = 0;
  int device = 0;
  Algo algo = Algo::Trivial;
  const Pow2Kernel* k[2] = {nullptr, nullptr};  // [0] forward, [1] inverse
  void* tw = nullptr;                            // twiddle tables (one allocation)
  std::string name;
  // two-pass schedule
  const TwoPassKernel* tp[2] = {nullptr, nullptr};
  // three-pass schedule: kernels, W_M2 table (tw1 = W_N1, tw2 = W_M1), split W_M
  const ThreePassKernel* t3[2] = {nullptr, nullptr};
  const void* tw3 = nullptr;
  const void* btm_lo = nullptr;
  const void* btm_hi = nullptr;
  int btm_shift = 0;
  const void* tw1 = nullptr;                     // W_N1
  const void* tw2 = nullptr;                     // W_N2
  const void* bt_lo = nullptr;
  const void* bt_hi = nullptr;
  int bt_shift = 0;
  int group = 1, slots = 2, resident = 1;
  // L2-pipelined two-pass schedule (same tables as the two-pass one; tp[]
  // holds the split kernels of the same split for buffers the copy engine
  // cannot address): kernels, group bytes in MB and scratch slots
  const L2PipeKernel* l2[2] = {nullptr, nullptr};
  int l2_gmb = 16, l2_slots = 3;
  // tensor-core form: radix of its leading FP32 stage (1: n is a power of 16)
  int tc_lead = 1;
  unsigned* status = nullptr;  // device word: nonzero once a bounded wait expired
  // runtime-schedule (7-smooth) plans
  GenSched gs{}, gs1{}, gs2{};
  int64_t gn1 = 0, gn2 = 0;
  bool mixc = false;  // two passes on the compiled mixed-radix column tiles
  bool mixr = false;  // one pass on the compiled tiles in rows mode (Algo::Generic)
  // Bluestein: chirps and filters per direction, sub-plan of length bm;
  // bsm: bm = gn1 x gn2 on the compiled mixed-radix tiles (tw1 = W_gn1,
  // tw2 = W_gn2, bt_* = W_bm split)
  PlanCore* sub = nullptr;
  int64_t bm = 0;
  bool bsm = false;
  void* bs_w[2] = {nullptr, nullptr};
  void* bs_f[2] = {nullptr, nullptr};
};

bool is_smooth7(int64_t n);
// Runtime Stockham schedule of a 7-smooth n (false when n is not 7-smooth or
// needs more than 1024 threads).
bool make_gen_sched(int64_t n, GenSched* s);
gfft_status init_generic(PlanCore* c, bool mixr = false);
// Variant tokens of the runtime-radix schedules that can serve n.
std::vector<std::string> mixed_tokens(int prec, int64_t n);
// mixc: split n into two lengths with compiled mixed-radix column tiles
// (mix_split) instead of the runtime-radix column kernel.
gfft_status init_gen_twopass(PlanCore* c, bool mixc = false);
// N1 of a split n = N1 x N2 whose factors both have compiled mixed-radix
// column tiles, N1 <= N2 and nearest sqrt n; 0 when there is none.
int64_t mix_split(int64_t n);
// Compiled mixed-radix column tiles (kernels_mixcols.cu): pass 1 / pass 2
// of the four-step over columns of length L (MIX_PASS1 / MIX_PASS2), or a
// column batch (pass 2).  cudaErrorNotSupported for other lengths.
// With p.items set (item mode) `count` is the number of CTAs of the launch.
struct MixColsParams;
bool mix_cols_supported(int64_t L);
std::vector<int64_t> mix_cols_lengths();
int mix_cols_width(int prec, int pass, int64_t L);  // columns per tile (0: not compiled)
cudaError_t exec_mix_cols(int prec, int dir, int pass, int64_t L, MixColsParams p, int64_t count, cudaStream_t st);
// Bluestein on the compiled tiles (gfft_mixbs.cuh): the smallest FFT length
// M = M1 x M2 >= 2n - 1 its column lengths build (M1 <= M2 returned in *m1;
// 0 when none), and one of its passes (BSK_IN / BSK_MID / BSK_OUT) over
// `count` transforms, or `count` CTAs in item mode.
struct MixBsParams;
// Whole contiguous transforms of a compiled length (rows mode: every
// 7-smooth length 48..1024, and the non-powers of two up to 12288 for
// complex64, 6144 for complex128).
struct MixRowsParams;
bool mix_rows_supported(int prec, int64_t L);
cudaError_t exec_mix_rows(int prec, int dir, int64_t L, const MixRowsParams& p, cudaStream_t st);
int64_t bs_mixed_length(int64_t n, int64_t* m1);
int mix_bs_width(int prec, int64_t L);
cudaError_t exec_mix_bs(int prec, int kind, int64_t L, MixBsParams p, int64_t count, cudaStream_t st);
// Bluestein's FFT length: kBsAuto takes the mixed length (a product of
// compiled column lengths) where bs_mixed_preferred says so against
// NextPow2(2n - 1), the reference's; kBsPow2 / kBsMixed force either (the
// latter where a smaller mixed length exists).  bs_mixed_choice: that
// smaller mixed length (0: none, or the one-CTA fused range).
enum { kBsAuto = 0, kBsPow2 = 1, kBsMixed = 2 };
int64_t bs_mixed_choice(int64_t n, int64_t* m1);
bool bs_mixed_preferred(int64_t mx, int64_t M);
gfft_status init_bluestein(PlanCore* c, int mode = kBsAuto);
// Tensor-core split-fp16 radix-16 form (complex64, powers of two 16 <= n <= 2^24;
// n = r * 16^s with r = 2, 4, 8 takes one leading FP32 radix-r stage).
bool tc_supported(int64_t n);
gfft_status init_tc(PlanCore* c);
gfft_status exec_tc(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                    int64_t odist, cudaStream_t st);
// Column batches through the runtime column kernel (7-smooth n that fits).
bool column_sched(int64_t n, int prec, GenSched* s);
gfft_status exec_columns(const GenSched& s, int prec, int dir, void* dst, const void* src, int64_t count,
                         int64_t dist, int64_t ncols, int64_t pitch, const void* tw_n, cudaStream_t st);
// Power-of-two column batches (n <= 4096) through the compile-time column
// tiles; cudaErrorNotSupported for other lengths.
bool pow2_cols_supported(int64_t n);
cudaError_t exec_pow2_cols(int prec, int dir, void* dst, const void* src, int64_t count, int64_t dist, int64_t ncols,
                           int64_t pitch, const void* tw_n, int64_t n, cudaStream_t st);
// Bluestein as one fused kernel when the FFT length M fits one CTA (M a
// power of two <= 16384 complex64, <= 8192 complex128).
bool bluestein_fused_supported(int prec, int64_t M);
// Bluestein through the two-pass FFT_M with the chain fused into its passes
// (M = 2^15..2^20, split N1 x M / N1 as the two-pass plans).
bool bluestein_tp_supported(int prec, int64_t M, int n1);
size_t bluestein_tp_chunk_bytes(int prec, int64_t M, int64_t count);
// Bluestein through the plain three-pass FFT_M (M = 2^21..2^24) with the
// chirp, pad, filter product and output chirp fused into its first and
// third passes; `sub` is the plain three-pass plan of length M.
bool bluestein_tp3_supported(int prec, int64_t M);
gfft_status exec_bluestein_tp3(const PlanCore* sub, const void* src, void* dst, int64_t count, int64_t idist,
                               int64_t odist, int64_t n, const void* chirp, const void* filt, double scale,
                               cudaStream_t st);
cudaError_t exec_bluestein_tp(int prec, int64_t M, const void* src, void* dst, int64_t count, int64_t idist,
                              int64_t odist, int64_t n, const void* chirp, const void* filt, const void* tw1,
                              const void* tw2, BigTwiddle bt, double scale, void* scratch, void* work,
                              cudaStream_t st);
// The same chain over the rows of an uneven batch's Bluestein group: row r
// is items[r] (offset, length, chirp and filter offsets into tab), the
// forward tables serving both directions.
struct BigItem;
cudaError_t exec_bluestein_tp_items(int prec, int64_t M, int dir, const void* src, void* dst, const BigItem* items,
                                    int64_t rows, const void* tab, const void* tw1, const void* tw2, BigTwiddle bt,
                                    void* scratch, void* work, cudaStream_t st);
// Plain FFTs of length M (two-pass, the same split) of an uneven batch's
// rows, read and written in place in the packed batch.
cudaError_t exec_twopass_items(int prec, int64_t M, int dir, const void* src, void* dst, const BigItem* items,
                               int64_t rows, const void* tw1, const void* tw2, BigTwiddle bt, void* scratch,
                               cudaStream_t st);
cudaError_t exec_bluestein_fused(int prec, int64_t M, const void* src, void* dst, int64_t count, int64_t idist,
                                 int64_t odist, int64_t n, const void* chirp, const void* filt, const void* tw,
                                 double scale, cudaStream_t st);
gfft_status exec_runtime_plan(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                              int64_t odist, cudaStream_t st);

// Fills dst[j] = W_n^{(j*step) mod n} for j < count (FP64, rounded).
// Stream-ordered workspace from the library's per-device pool (released
// with cudaFreeAsync; the pool keeps the memory for later calls).
cudaError_t ws_alloc(void** p, size_t bytes, cudaStream_t st);
gfft_status fill_twiddles(int prec, void* dst, int64_t n, int64_t count, int64_t step, cudaStream_t st);

// What plan creation knows about the calls a plan will serve; the learned
// planner's shape features (batch 0 = unknown).
struct PlanHint {
  int planner = GFFT_PLANNER_ESTIMATE;
  int64_t batch = 0;   // transforms per call
  int64_t stride = 1;  // element stride inside one transform
  int real = 0;        // 1: the complex child of a real transform of length 2n
  bool user = false;   // a plan the user asked for (not a sub-plan of another schedule)
};

// Chooses and prepares the schedule of a 1-D complex transform of length n:
// a forced strategy class, else the wisdom store's variant, else (with
// GFFT_PLANNER_LEARNED and a model loaded) the learned cost model's pick,
// else defaults.
gfft_status core_init(PlanCore* c, int prec, int64_t n, int device, int strategy = GFFT_KERNEL_AUTO,
                      const PlanHint* hint = nullptr);
// Process-wide strategy override and per-length strategy decisions.
void set_kernel_strategy(int s);
int get_kernel_strategy();
void record_decision(int64_t n, int s);
// The learned cost model's choice among variant_tokens(prec, n) for the
// hinted shape (false when no model is loaded or n has < 2 variants).
bool learned_choose(int prec, int64_t n, const PlanHint& hint, std::string* token);
// Prepares the exact kernel variant named by a wisdom token.
gfft_status core_init_variant(PlanCore* c, int prec, int64_t n, int device, const std::string& token);
void core_free(PlanCore* c);
// Nonzero once a bounded device wait of this plan expired (synchronous read).
unsigned core_device_status(const PlanCore* c);
// Tokens of every compiled variant that can compute length n.
std::vector<std::string> variant_tokens(int prec, int64_t n);

// Wisdom store (process-wide).
bool wisdom_lookup(int64_t n, int prec, std::string* algo);
void wisdom_store(int64_t n, int prec, const std::string& algo);
gfft_status wisdom_import(const std::string& text);
std::string wisdom_export();
void wisdom_clear();
size_t wisdom_len();
// Times every variant of length n on count transforms; records the fastest.
gfft_status autotune(int prec, int64_t n, int64_t count, int iters, std::string* best, std::string* report);

// Runs `count` transforms (dir -1 forward, +1 inverse) with element strides
// idist/odist between consecutive transforms; device pointers.
gfft_status core_exec(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                      int64_t odist, cudaStream_t st);

inline size_t elem_bytes(int prec) { return prec == kC64 ? 8 : 16; }

}  // namespace gfft

struct gfft_plan;
namespace gfft {
// Host-slice execution of `count` transforms of a 1-D plan: copies in,
// transforms and copies out before returning (pageable buffers are staged
// through library-owned pinned lanes).
gfft_status run_host(gfft_plan* p, int dir, void* dst, const void* src, int64_t count);
}  // namespace gfft

struct gfft_plan {
  gfft::PlanCore core;
  gfft_plan_options opts{};
  int32_t precision = 0;
  bool pooled = false;  // Close returns it to the plan pool
};

namespace gfft {
struct RealKernel;
}

struct gfft_plan_real {
  gfft::PlanCore child;  // half-length complex plan (plan_real_generic.go:64)
  int prec = 0;
  int64_t n = 0, h = 0;
  gfft_plan_options opts{};
  void* wt = nullptr;  // U[k], k <= h
  const gfft::RealKernel* fused = nullptr;
  unsigned* flag = nullptr;
};

namespace gfft {
// Batched real transforms on device buffers: `batch` transforms, reals
// `sr` apart and spectra `sc` apart (element units); scaling 0 none,
// 1 x 1/n, 2 x 1/sqrt(n).
gfft_status real_forward(gfft_plan_real* p, int scaling, void* dst, const void* src, int64_t batch, int64_t sr,
                         int64_t sc, cudaStream_t st);
gfft_status real_inverse(gfft_plan_real* p, void* dst, const void* src, int64_t batch, int64_t sr, int64_t sc,
                         cudaStream_t st);
}  // namespace gfft
