// Runtime-schedule plans: 7-smooth lengths (single CTA or two passes) and
// Bluestein for every other length.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <type_traits>
#include <vector>
#include "gfft_generic.cuh"
#include "gfft_internal.h"
#include "gfft_mixbs.cuh"
#include "gfft_mixcols.cuh"

namespace gfft {

// ------------------------------------------------------------------ schedules

static bool smooth7(int64_t n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

bool is_smooth7(int64_t n) { return smooth7(n); }

// Butterflies of radix r a thread is sized for in one stage (about 16
// elements); the threads of a transform loop past that when capped at 1024.
static int qm_of(int r) { return std::max(1, 16 / r); }

// Radix order: 16s, then the rest of the twos (8, 4, 2), then 7s, 5s, 9s
// (pairs of threes) and a last 3.
static bool make_sched(int64_t n, GenSched* s) {
  *s = GenSched{};
  if (n < 2 || n > (int64_t(1) << 30) || !smooth7(n)) return false;
  std::vector<int> rad;
  int64_t m = n;
  int e2 = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++e2;
  }
  while (e2 >= 4) {
    rad.push_back(16);
    e2 -= 4;
  }
  if (e2 == 3) rad.push_back(8);
  if (e2 == 2) rad.push_back(4);
  if (e2 == 1) rad.push_back(2);
  for (int p : {7, 5})
    while (m % p == 0) {
      rad.push_back(p);
      m /= p;
    }
  while (m % 9 == 0) {  // pairs of threes as one radix-9 stage
    rad.push_back(9);
    m /= 9;
  }
  if (m % 3 == 0) {
    rad.push_back(3);
    m /= 3;
  }
  if (int(rad.size()) > 20) return false;
  s->n = int(n);
  s->nst = int(rad.size());
  int64_t prod = 1, T = 1;
  for (int i = 0; i < s->nst; ++i) {
    s->radix[i] = rad[i];
    s->p[i] = int(prod);
    s->pinv[i] = float(1.0 / double(prod));
    prod *= rad[i];
    T = std::max<int64_t>(T, (n / rad[i] + qm_of(rad[i]) - 1) / qm_of(rad[i]));
  }
  if (T > 32) T = (T + 31) / 32 * 32;
  if (T > 1024) T = 1024;
  s->T = int(T);
  // two padded buffers per transform, an odd total (column-major tiles of
  // k_gen_cols stay bank-conflict free)
  const int64_t half = n - 1 + ((n - 1) >> 5) + 1;
  if (2 * half + 1 > (int64_t(1) << 30)) return false;
  s->half = int(half);
  s->stride = int(2 * half + 1);
  s->B = 1;
  return true;
}

static const int kSmemBudget = 200 * 1024;

bool make_gen_sched(int64_t n, GenSched* s) { return make_sched(n, s); }

// --------------------------------------------------------------- launchers

template <typename C>
static cudaError_t launch_generic(const PlanCore* c, int dir, const void* src, void* dst, int64_t count,
                                  int64_t idist, int64_t odist, cudaStream_t st) {
  using Re = typename RealOf<C>::type;
  const GenSched& s = c->gs;
  const int64_t blocks = (count + s.B - 1) / s.B;
  const size_t smem = size_t(s.B) * s.stride * sizeof(C);
  const Re scale = Re(1.0 / double(c->n));
  // co-resident CTAs: the L2 prefetch distance (none for a single wave)
  const int thr = s.B * s.T;
  auto go = [&](auto lb) {
    constexpr int LB = decltype(lb)::value;
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, &k_generic<C, -1, LB>, thr, smem);
    cudaGetLastError();
    const int64_t resident = int64_t(sms) * std::max(occ, 1);
    const int64_t ahead = blocks > resident ? resident : 0;
    if (dir < 0)
      k_generic<C, -1, LB><<<unsigned(blocks), thr, smem, st>>>(static_cast<const C*>(src), static_cast<C*>(dst),
                                                                  count, idist, odist, static_cast<const C*>(c->tw), s,
                                                                  scale, ahead);
    else
      k_generic<C, +1, LB><<<unsigned(blocks), thr, smem, st>>>(static_cast<const C*>(src), static_cast<C*>(dst),
                                                                  count, idist, odist, static_cast<const C*>(c->tw), s,
                                                                  scale, ahead);
  };
  if constexpr (sizeof(C) == 16) {
    if (thr <= 512) go(std::integral_constant<int, 512>{});
    else go(std::integral_constant<int, 1024>{});
  } else {
    go(std::integral_constant<int, 1024>{});
  }
  return cudaGetLastError();
}

template <typename C, int MODE>
static cudaError_t launch_cols(const GenSched& s, int dir, const void* src, void* dst, int64_t count, int64_t in_dist,
                               int64_t out_dist, int64_t ncols, const void* tw, BigTwiddle bt, double scale,
                               cudaStream_t st, int64_t pitch = -1) {
  if (pitch < 0) pitch = ncols;
  using Re = typename RealOf<C>::type;
  const int64_t tiles = (ncols + s.B - 1) / s.B;
  const int64_t blocks = tiles * count;
  const size_t smem = size_t(s.B) * s.stride * sizeof(C);
  if (blocks <= 0) return cudaSuccess;
  if (dir < 0)
    k_gen_cols<C, -1, MODE><<<unsigned(blocks), s.B * s.T, smem, st>>>(
        static_cast<const C*>(src), static_cast<C*>(dst), count, in_dist, out_dist, ncols, pitch,
        static_cast<const C*>(tw), s, bt, Re(scale));
  else
    k_gen_cols<C, +1, MODE><<<unsigned(blocks), s.B * s.T, smem, st>>>(
        static_cast<const C*>(src), static_cast<C*>(dst), count, in_dist, out_dist, ncols, pitch,
        static_cast<const C*>(tw), s, bt, Re(scale));
  return cudaGetLastError();
}

static cudaError_t prepare_generic_kernels() {
  static std::mutex mu;
  static std::vector<int> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  if (std::find(done.begin(), done.end(), dev) != done.end()) return cudaSuccess;
  const void* fns[] = {
      reinterpret_cast<const void*>(&k_generic<float2, -1>),
      reinterpret_cast<const void*>(&k_generic<float2, +1>),
      reinterpret_cast<const void*>(&k_generic<double2, -1>),
      reinterpret_cast<const void*>(&k_generic<double2, +1>),
      reinterpret_cast<const void*>(&k_generic<double2, -1, 512>),
      reinterpret_cast<const void*>(&k_generic<double2, +1, 512>),
      reinterpret_cast<const void*>(&k_gen_cols<float2, -1, GEN_PASS1>),
      reinterpret_cast<const void*>(&k_gen_cols<float2, +1, GEN_PASS1>),
      reinterpret_cast<const void*>(&k_gen_cols<float2, -1, GEN_PASS2>),
      reinterpret_cast<const void*>(&k_gen_cols<float2, +1, GEN_PASS2>),
      reinterpret_cast<const void*>(&k_gen_cols<double2, -1, GEN_PASS1>),
      reinterpret_cast<const void*>(&k_gen_cols<double2, +1, GEN_PASS1>),
      reinterpret_cast<const void*>(&k_gen_cols<double2, -1, GEN_PASS2>),
      reinterpret_cast<const void*>(&k_gen_cols<double2, +1, GEN_PASS2>),
  };
  for (const void* f : fns) {
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget + 16 * 1024);
    if (e != cudaSuccess) return e;
  }
  done.push_back(dev);
  return cudaSuccess;
}

// -------------------------------------------------------- 7-smooth plans

// Single-CTA schedule when one transform (T <= 1024 threads, shared memory
// within budget) fits; B transforms per CTA up to 256 threads.  mixr: the
// compiled mixed-radix schedule of the length in rows mode instead (7-smooth
// lengths 48..1024).
gfft_status init_generic(PlanCore* c, bool mixr) {
  GenSched s;
  const size_t es = elem_bytes(c->prec);
  if (mixr) {
    if (!mix_rows_supported(c->prec, c->n)) return GFFT_ERR_NOT_IMPLEMENTED;
    gfft_status st = make_twiddles(c->prec, c->n, &c->tw, 0);
    if (st != GFFT_OK) return st;
    GFFT_CUDA(cudaStreamSynchronize(0));
    c->mixr = true;
    c->algo = Algo::Generic;
    c->name = "gpu-sm100-mixr-n" + std::to_string(c->n);
    return GFFT_OK;
  }
  if (!make_sched(c->n, &s) || size_t(s.stride) * es > size_t(kSmemBudget)) return GFFT_ERR_NOT_IMPLEMENTED;
  s.B = std::max(1, std::min(256 / s.T, int(kSmemBudget / (size_t(s.stride) * es))));
  GFFT_CUDA(prepare_generic_kernels());
  gfft_status st = make_twiddles(c->prec, c->n, &c->tw, 0);
  if (st != GFFT_OK) return st;
  GFFT_CUDA(cudaStreamSynchronize(0));
  c->gs = s;
  c->algo = Algo::Generic;
  c->name = "gpu-sm100-mixed-n" + std::to_string(c->n);
  return GFFT_OK;
}

// Column-tile schedule of length L with up to `want` columns per tile.
static bool make_col_sched(int64_t L, size_t es, int want, GenSched* s) {
  if (!make_sched(L, s)) return false;
  int nc = want;
  while (nc > 1 && (size_t(nc) * s->stride * es > size_t(kSmemBudget) || nc * s->T > 1024)) nc /= 2;
  if (size_t(nc) * s->stride * es > size_t(kSmemBudget) || nc * s->T > 1024) return false;
  s->B = nc;
  return true;
}

// N1 of the runtime two-pass split: the 7-smooth divisor of n nearest below
// sqrt(n) (1 when there is none).
static int64_t gen_split(int64_t n) {
  int64_t n1 = 1;
  for (int64_t d = 1; d * d <= n; ++d)
    if (n % d == 0 && smooth7(d)) n1 = d;
  return n1;
}

int64_t mix_split(int64_t n) {
  int64_t best = 0;
  for (int64_t d : mix_cols_lengths())
    if (n % d == 0 && d * d <= n && mix_cols_supported(n / d) && d > best) best = d;
  return best;
}

std::vector<std::string> mixed_tokens(int prec, int64_t n) {
  std::vector<std::string> v;
  const size_t es = elem_bytes(prec);
  GenSched s, s1, s2;
  if (make_sched(n, &s) && size_t(s.stride) * es <= size_t(kSmemBudget)) v.push_back("gpu-sm100-mixed-n" + std::to_string(n));
  if (mix_rows_supported(prec, n)) v.push_back("gpu-sm100-mixr-n" + std::to_string(n));
  const int64_t n1 = gen_split(n), n2 = n / n1;
  const int want = prec == kC64 ? 16 : 8;
  if (n1 >= 2 && make_col_sched(n1, es, want, &s1) && make_col_sched(n2, es, want, &s2))
    v.push_back("gpu-sm100-mixed2-" + std::to_string(n1) + "x" + std::to_string(n2));
  const int64_t m1 = mix_split(n);
  if (m1 >= 2) v.push_back("gpu-sm100-mixc-" + std::to_string(m1) + "x" + std::to_string(n / m1));
  return v;
}

gfft_status init_gen_twopass(PlanCore* c, bool mixc) {
  const int64_t n = c->n;
  const size_t es = elem_bytes(c->prec);
  const int64_t n1 = mixc ? mix_split(n) : gen_split(n);
  if (n1 < 2) return GFFT_ERR_NOT_IMPLEMENTED;
  const int64_t n2 = n / n1;
  const int want = c->prec == kC64 ? 16 : 8;
  if (!mixc && (!make_col_sched(n1, es, want, &c->gs1) || !make_col_sched(n2, es, want, &c->gs2)))
    return GFFT_ERR_NOT_IMPLEMENTED;
  c->mixc = mixc;
  GFFT_CUDA(prepare_generic_kernels());
  int shift = 0;
  while ((int64_t(1) << (2 * shift)) < n) ++shift;
  const int64_t nlo = int64_t(1) << shift, nhi = (n + nlo - 1) >> shift;
  GFFT_CUDA(cudaMalloc(&c->tw, size_t(n1 + n2 + nlo + nhi) * es));
  char* base = static_cast<char*>(c->tw);
  gfft_status s = fill_twiddles(c->prec, base, n1, n1, 1, 0);
  if (s == GFFT_OK) s = fill_twiddles(c->prec, base + n1 * es, n2, n2, 1, 0);
  if (s == GFFT_OK) s = fill_twiddles(c->prec, base + (n1 + n2) * es, n, nlo, 1, 0);
  if (s == GFFT_OK) s = fill_twiddles(c->prec, base + (n1 + n2 + nlo) * es, n, nhi, nlo, 0);
  if (s != GFFT_OK) return s;
  GFFT_CUDA(cudaStreamSynchronize(0));
  c->gn1 = n1;
  c->gn2 = n2;
  c->tw1 = base;
  c->tw2 = base + n1 * es;
  c->bt_lo = base + (n1 + n2) * es;
  c->bt_hi = base + (n1 + n2 + nlo) * es;
  c->bt_shift = shift;
  c->algo = Algo::GenTwoPass;
  c->name = std::string(mixc ? "gpu-sm100-mixc-" : "gpu-sm100-mixed2-") + std::to_string(n1) + "x" + std::to_string(n2);
  return GFFT_OK;
}

// The two passes of a mixc plan over transforms [0, m) of in / out.
static cudaError_t mixc_passes(const PlanCore* c, int dir, const void* in, void* scratch, void* out, int64_t m,
                               int64_t idist, int64_t odist, BigTwiddle bt, double scale, cudaStream_t st) {
  const int64_t n = c->n;
  MixColsParams p1{in, scratch, c->gn2, c->gn2, 0, idist, n, 0, c->tw1, bt, 1.0};
  cudaError_t e = exec_mix_cols(c->prec, dir, MIX_PASS1, c->gn1, p1, m, st);
  if (e != cudaSuccess) return e;
  MixColsParams p2{scratch, out, c->gn1, c->gn1, c->gn1, n, odist, 0, c->tw2, bt, scale};
  return exec_mix_cols(c->prec, dir, MIX_PASS2, c->gn2, p2, m, st);
}

static gfft_status exec_gen_twopass(const PlanCore* c, int dir, void* dst, const void* src, int64_t count,
                                    int64_t idist, int64_t odist, cudaStream_t st) {
  const size_t es = elem_bytes(c->prec);
  const int64_t n = c->n;
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(512) << 20) / (n * int64_t(es))));
  void* scratch = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&scratch), size_t(chunk) * size_t(n) * es, st));
  BigTwiddle bt{c->bt_lo, c->bt_hi, c->bt_shift};
  const double scale = 1.0 / double(n);
  cudaError_t e = cudaSuccess;
  for (int64_t b0 = 0; b0 < count && e == cudaSuccess; b0 += chunk) {
    const int64_t m = std::min(chunk, count - b0);
    const char* in = static_cast<const char*>(src) + size_t(b0) * size_t(idist) * es;
    char* out = static_cast<char*>(dst) + size_t(b0) * size_t(odist) * es;
    if (c->mixc) {
      e = mixc_passes(c, dir, in, scratch, out, m, idist, odist, bt, scale, st);
    } else if (c->prec == kC64) {
      e = launch_cols<float2, GEN_PASS1>(c->gs1, dir, in, scratch, m, idist, n, c->gn2, c->tw1, bt, 1.0, st);
      if (e == cudaSuccess)
        e = launch_cols<float2, GEN_PASS2>(c->gs2, dir, scratch, out, m, n, odist, c->gn1, c->tw2, bt, scale, st);
    } else {
      e = launch_cols<double2, GEN_PASS1>(c->gs1, dir, in, scratch, m, idist, n, c->gn2, c->tw1, bt, 1.0, st);
      if (e == cudaSuccess)
        e = launch_cols<double2, GEN_PASS2>(c->gs2, dir, scratch, out, m, n, odist, c->gn1, c->tw2, bt, scale, st);
    }
  }
  cudaFreeAsync(scratch, st);
  if (e != cudaSuccess) return cuda_status(e, c->mixc ? "k_mix_cols" : "k_gen_cols");
  return GFFT_OK;
}

// Column batch: `count` blocks `dist` apart, each holding ncols transforms of
// length s.n laid out as columns (element j of column c at j*pitch + c).
bool column_sched(int64_t n, int prec, GenSched* s) {
  return make_col_sched(n, elem_bytes(prec), prec == kC64 ? 16 : 8, s) && (prepare_generic_kernels() == cudaSuccess);
}

gfft_status exec_columns(const GenSched& s, int prec, int dir, void* dst, const void* src, int64_t count,
                         int64_t dist, int64_t ncols, int64_t pitch, const void* tw_n, cudaStream_t st) {
  if (pow2_cols_supported(s.n)) {
    const cudaError_t e = exec_pow2_cols(prec, dir, dst, src, count, dist, ncols, pitch, tw_n, s.n, st);
    if (e != cudaSuccess) return cuda_status(e, "k_pow2_cols");
    return GFFT_OK;
  }
  BigTwiddle bt{nullptr, nullptr, 0};
  const double scale = 1.0 / double(s.n);
  if (mix_cols_supported(s.n)) {
    const MixColsParams p{src, dst, ncols, pitch, pitch, dist, dist, 0, tw_n, bt, scale};
    const cudaError_t e = exec_mix_cols(prec, dir, MIX_PASS2, s.n, p, count, st);
    if (e != cudaSuccess) return cuda_status(e, "k_mix_cols");
    return GFFT_OK;
  }
  cudaError_t e = prec == kC64
                      ? launch_cols<float2, GEN_PASS2>(s, dir, src, dst, count, dist, dist, ncols, tw_n, bt, scale, st, pitch)
                      : launch_cols<double2, GEN_PASS2>(s, dir, src, dst, count, dist, dist, ncols, tw_n, bt, scale, st, pitch);
  if (e != cudaSuccess) return cuda_status(e, "k_gen_cols");
  return GFFT_OK;
}

// ---------------------------------------------------------------- Bluestein

// work[b][m] = m < n ? x[b][m] * w[m] : 0     (plan_bluestein.go:8-16)
template <typename C>
__global__ void k_bs_pre(C* work, const C* x, const C* w, int64_t n, int64_t M, int64_t count, int64_t idist) {
  const int64_t total = count * M;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / M, m = e - b * M;
    work[e] = m < n ? cmul(ld_stream(x + b * idist + m), __ldg(w + m)) : C{0, 0};
  }
}

template <typename C>
__global__ void k_bs_mul(C* work, const C* f, int64_t M, int64_t count) {
  const int64_t total = count * M;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x)
    work[e] = cmul(work[e], __ldg(f + e % M));
}

// y[b][k] = work[b][k] * w[k] * scale          (plan_bluestein.go:18-58)
template <typename C>
__global__ void k_bs_post(C* y, const C* work, const C* w, int64_t n, int64_t M, int64_t count, int64_t odist,
                          typename RealOf<C>::type scale) {
  const int64_t total = count * n;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / n, k = e - b * n;
    st_stream(y + b * odist + k, cscale(cmul(work[b * M + k], __ldg(w + k)), scale));
  }
}

static unsigned grid_for(int64_t total) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 32))); }

int64_t bs_mixed_choice(int64_t n, int64_t* m1) {
  int64_t M = 1;
  while (M < 2 * n - 1) M <<= 1;
  const int64_t mx = bs_mixed_length(n, m1);
  return M > 16384 && mx > 0 && mx < M ? mx : 0;
}

// The mixed chain's passes cost more per FFT element than the power-of-two
// chain's, by a factor that depends on M: the two-pass chain of M = 32768
// (128 x 256 tiles) runs about 1.3x slower per element than at 2^16..2^18,
// so there the mixed length wins up to M itself; at 65536 the break-even
// ratio is near 0.88 (complex64) to above 0.9 (complex128), beyond that
// 0.70 (measured on 128 MB batches of 30 primes).
bool bs_mixed_preferred(int64_t mx, int64_t M) {
  const double r = M <= 32768 ? 1.0 : M <= 65536 ? 0.9 : 0.70;
  return mx > 0 && double(mx) <= r * double(M);
}

gfft_status init_bluestein(PlanCore* c, int mode) {
  const int64_t n = c->n;
  int64_t M = 1;
  while (M < 2 * n - 1) M <<= 1;  // plan.go:865 NextPowerOfTwo(2n-1)
  // Beyond the one-CTA fused kernel, a smaller FFT length built from two
  // compiled column lengths (the product is the same up to rounding) where
  // bs_mixed_preferred expects it to be faster.
  int64_t m1 = 0;
  const int64_t mx = bs_mixed_choice(n, &m1);
  const bool bsm = mx > 0 && (mode == kBsMixed || (mode == kBsAuto && bs_mixed_preferred(mx, M)));
  if (bsm) M = mx;
  const size_t es = elem_bytes(c->prec);
  c->sub = new PlanCore;
  gfft_status s;
  if (!bsm && bluestein_tp3_supported(c->prec, M)) {
    // the plain three-pass split, whose first and third passes the chain fuses
    const ThreePassKernel* k = find_threepass(c->prec, M, -1);
    s = core_init_variant(c->sub, c->prec, M, c->device,
                          "gpu-sm100-tp3-" + std::to_string(k->n1) + "x" + std::to_string(k->m1) + "x" +
                              std::to_string(k->m2));
  } else {
    s = core_init(c->sub, c->prec, M, c->device);
  }
  if (s != GFFT_OK) return s;
  // [chirp fwd | chirp inv | filter fwd | filter inv], then for the mixed
  // chain [W_M1 | W_M2 | W_M low | W_M high]
  int shift = 0;
  while ((int64_t(1) << (2 * shift)) < M) ++shift;
  const int64_t nlo = int64_t(1) << shift, nhi = (M + nlo - 1) >> shift;
  const int64_t m2 = bsm ? M / m1 : 0;
  const int64_t extra = bsm ? m1 + m2 + nlo + nhi : 0;
  GFFT_CUDA(cudaMalloc(&c->tw, size_t(2 * n + 2 * M + extra) * es));
  char* base = static_cast<char*>(c->tw);
  void* wf = base;
  void* wi = base + n * es;
  void* ff = base + 2 * n * es;
  void* fi = base + (2 * n + M) * es;
  if (bsm) {
    char* t = base + (2 * n + 2 * M) * es;
    s = fill_twiddles(c->prec, t, m1, m1, 1, 0);
    if (s == GFFT_OK) s = fill_twiddles(c->prec, t + m1 * es, m2, m2, 1, 0);
    if (s == GFFT_OK) s = fill_twiddles(c->prec, t + (m1 + m2) * es, M, nlo, 1, 0);
    if (s == GFFT_OK) s = fill_twiddles(c->prec, t + (m1 + m2 + nlo) * es, M, nhi, nlo, 0);
    if (s != GFFT_OK) return s;
    c->bsm = true;
    c->gn1 = m1;
    c->gn2 = m2;
    c->tw1 = t;
    c->tw2 = t + m1 * es;
    c->bt_lo = t + (m1 + m2) * es;
    c->bt_hi = t + (m1 + m2 + nlo) * es;
    c->bt_shift = shift;
  }
  const unsigned g = grid_for(std::max(n, M));
  if (c->prec == kC64) {
    k_chirp<float2><<<g, 256>>>(static_cast<float2*>(wf), n, -1);
    k_chirp<float2><<<g, 256>>>(static_cast<float2*>(wi), n, +1);
    k_bs_filter_src<float2><<<g, 256>>>(static_cast<float2*>(ff), static_cast<float2*>(wf), n, M);
    k_bs_filter_src<float2><<<g, 256>>>(static_cast<float2*>(fi), static_cast<float2*>(wi), n, M);
  } else {
    k_chirp<double2><<<g, 256>>>(static_cast<double2*>(wf), n, -1);
    k_chirp<double2><<<g, 256>>>(static_cast<double2*>(wi), n, +1);
    k_bs_filter_src<double2><<<g, 256>>>(static_cast<double2*>(ff), static_cast<double2*>(wf), n, M);
    k_bs_filter_src<double2><<<g, 256>>>(static_cast<double2*>(fi), static_cast<double2*>(wi), n, M);
  }
  GFFT_CUDA(cudaGetLastError());
  // filters: forward FFT_M of b (the reference's ditForward, bluestein.go:55)
  s = core_exec(c->sub, -1, ff, ff, 1, M, M, 0);
  if (s == GFFT_OK) s = core_exec(c->sub, -1, fi, fi, 1, M, M, 0);
  if (s != GFFT_OK) return s;
  GFFT_CUDA(cudaStreamSynchronize(0));
  c->bm = M;
  c->bs_w[0] = wf;
  c->bs_w[1] = wi;
  c->bs_f[0] = ff;
  c->bs_f[1] = fi;
  c->algo = Algo::Bluestein;
  c->name = "gpu-sm100-bluestein-n" + std::to_string(n) + (bsm ? "-mx" : mx > 0 ? "-p2" : "") + "-m" +
            std::to_string(M) + "+" + c->sub->name;
  return GFFT_OK;
}

// The Bluestein chain on the compiled mixed-radix tiles (gfft_mixbs.cuh):
// three launches per chunk of transforms (column lengths M1, M2, M1),
// scratch and work of M elements per transform each.
static gfft_status exec_bluestein_mixed(const PlanCore* c, int dir, void* dst, const void* src, int64_t count,
                                        int64_t idist, int64_t odist, cudaStream_t st) {
  const size_t es = elem_bytes(c->prec);
  const int64_t n = c->n, M = c->bm, m1 = c->gn1, m2 = c->gn2;
  const int d = dir < 0 ? 0 : 1;
  // chunks of at most 512 MB per buffer, of equal size (no short tail chunk)
  const int64_t cap = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(512) << 20) / (M * int64_t(es))));
  const int64_t nchunks = (count + cap - 1) / cap;
  const int64_t chunk = (count + nchunks - 1) / nchunks;
  void* buf = nullptr;
  GFFT_CUDA(ws_alloc(&buf, 2 * size_t(chunk) * size_t(M) * es, st));
  void* scratch = buf;
  void* work = static_cast<char*>(buf) + size_t(chunk) * size_t(M) * es;
  const BigTwiddle bt{c->bt_lo, c->bt_hi, c->bt_shift};
  cudaError_t e = cudaSuccess;
  for (int64_t b0 = 0; b0 < count && e == cudaSuccess; b0 += chunk) {
    const int64_t m = std::min(chunk, count - b0);
    MixBsParams p{};
    p.x = static_cast<const char*>(src) + size_t(b0) * size_t(idist) * es;
    p.y = static_cast<char*>(dst) + size_t(b0) * size_t(odist) * es;
    p.scratch = scratch;
    p.work = work;
    p.n = n;
    p.M = M;
    p.idist = idist;
    p.odist = odist;
    p.w = c->bs_w[d];
    p.f = c->bs_f[d];
    p.bt = bt;
    p.scale = dir < 0 ? 1.0 : 1.0 / double(n);
    p.inv = 0;
    p.tw = c->tw1;
    e = exec_mix_bs(c->prec, BSK_IN, m1, p, m, st);
    if (e != cudaSuccess) break;
    p.tw = c->tw2;
    e = exec_mix_bs(c->prec, BSK_MID, m2, p, m, st);
    if (e != cudaSuccess) break;
    p.tw = c->tw1;
    e = exec_mix_bs(c->prec, BSK_OUT, m1, p, m, st);
  }
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_status(e, "k_mix_bs");
  return GFFT_OK;
}

static gfft_status exec_bluestein(const PlanCore* c, int dir, void* dst, const void* src, int64_t count,
                                  int64_t idist, int64_t odist, cudaStream_t st) {
  const size_t es = elem_bytes(c->prec);
  const int64_t n = c->n, M = c->bm;
  const int d = dir < 0 ? 0 : 1;
  if (c->bsm) return exec_bluestein_mixed(c, dir, dst, src, count, idist, odist, st);
  // one fused launch when FFT_M fits one CTA (the sub-plan is single-pass,
  // so its W_M table serves the fused stages)
  if (c->sub->algo == Algo::Pow2Smem && bluestein_fused_supported(c->prec, M)) {
    const double fscale = (dir < 0 ? 1.0 : 1.0 / double(n)) / double(M);
    const cudaError_t fe = exec_bluestein_fused(c->prec, M, src, dst, count, idist, odist, n, c->bs_w[d], c->bs_f[d],
                                                c->sub->tw, fscale, st);
    if (fe != cudaSuccess) return cuda_status(fe, "k_bs_fused");
    return GFFT_OK;
  }
  // two-pass FFT_M: the chain fused into its four passes
  if ((c->sub->algo == Algo::TwoPass || c->sub->algo == Algo::L2Pipe) && bluestein_tp_supported(c->prec, M, c->sub->tp[0]->n1)) {
    const size_t bytes = bluestein_tp_chunk_bytes(c->prec, M, count);
    void* buf = nullptr;
    GFFT_CUDA(ws_alloc(&buf, 2 * bytes, st));
    BigTwiddle bt;
    bt.lo = c->sub->bt_lo;
    bt.hi = c->sub->bt_hi;
    bt.shift = c->sub->bt_shift;
    const cudaError_t te = exec_bluestein_tp(c->prec, M, src, dst, count, idist, odist, n, c->bs_w[d], c->bs_f[d],
                                             c->sub->tw1, c->sub->tw2, bt, dir < 0 ? 1.0 : 1.0 / double(n), buf,
                                             static_cast<char*>(buf) + bytes, st);
    cudaFreeAsync(buf, st);
    if (te != cudaSuccess) return cuda_status(te, "k_bs_tp");
    return GFFT_OK;
  }
  // three-pass FFT_M: the chain fused into its first and third passes
  if (c->sub->algo == Algo::ThreePass && !c->sub->t3[0]->tma && bluestein_tp3_supported(c->prec, M))
    return exec_bluestein_tp3(c->sub, src, dst, count, idist, odist, n, c->bs_w[d], c->bs_f[d],
                              dir < 0 ? 1.0 : 1.0 / double(n), st);
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(256) << 20) / (M * int64_t(es))));
  void* work = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&work), size_t(chunk) * size_t(M) * es, st));
  gfft_status s = GFFT_OK;
  cudaError_t e = cudaSuccess;
  const double scale = dir < 0 ? 1.0 : 1.0 / double(n);
  for (int64_t b0 = 0; b0 < count && s == GFFT_OK && e == cudaSuccess; b0 += chunk) {
    const int64_t m = std::min(chunk, count - b0);
    const char* in = static_cast<const char*>(src) + size_t(b0) * size_t(idist) * es;
    char* out = static_cast<char*>(dst) + size_t(b0) * size_t(odist) * es;
    if (c->prec == kC64) {
      k_bs_pre<float2><<<grid_for(m * M), 256, 0, st>>>(static_cast<float2*>(work), reinterpret_cast<const float2*>(in),
                                                         static_cast<const float2*>(c->bs_w[d]), n, M, m, idist);
    } else {
      k_bs_pre<double2><<<grid_for(m * M), 256, 0, st>>>(static_cast<double2*>(work), reinterpret_cast<const double2*>(in),
                                                          static_cast<const double2*>(c->bs_w[d]), n, M, m, idist);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) break;
    s = core_exec(c->sub, -1, work, work, m, M, M, st);
    if (s != GFFT_OK) break;
    if (c->prec == kC64)
      k_bs_mul<float2><<<grid_for(m * M), 256, 0, st>>>(static_cast<float2*>(work), static_cast<const float2*>(c->bs_f[d]), M, m);
    else
      k_bs_mul<double2><<<grid_for(m * M), 256, 0, st>>>(static_cast<double2*>(work), static_cast<const double2*>(c->bs_f[d]), M, m);
    e = cudaGetLastError();
    if (e != cudaSuccess) break;
    s = core_exec(c->sub, +1, work, work, m, M, M, st);  // includes 1/M (bluestein.go:76)
    if (s != GFFT_OK) break;
    if (c->prec == kC64)
      k_bs_post<float2><<<grid_for(m * n), 256, 0, st>>>(reinterpret_cast<float2*>(out), static_cast<const float2*>(work),
                                                          static_cast<const float2*>(c->bs_w[d]), n, M, m, odist, float(scale));
    else
      k_bs_post<double2><<<grid_for(m * n), 256, 0, st>>>(reinterpret_cast<double2*>(out), static_cast<const double2*>(work),
                                                           static_cast<const double2*>(c->bs_w[d]), n, M, m, odist, scale);
    e = cudaGetLastError();
  }
  cudaFreeAsync(work, st);
  if (e != cudaSuccess) return cuda_status(e, "bluestein");
  return s;
}

gfft_status exec_runtime_plan(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                              int64_t odist, cudaStream_t st) {
  switch (c->algo) {
    case Algo::Generic:
      if (c->mixr) {
        MixRowsParams p{src, dst, count, idist, odist, c->tw, dir < 0 ? 1.0 : 1.0 / double(c->n)};
        const cudaError_t e = exec_mix_rows(c->prec, dir, c->n, p, st);
        if (e != cudaSuccess) return cuda_status(e, "k_mix_rows");
        return GFFT_OK;
      }
      GFFT_CUDA(c->prec == kC64 ? launch_generic<float2>(c, dir, src, dst, count, idist, odist, st)
                                : launch_generic<double2>(c, dir, src, dst, count, idist, odist, st));
      return GFFT_OK;
    case Algo::GenTwoPass:
      return exec_gen_twopass(c, dir, dst, src, count, idist, odist, st);
    case Algo::Bluestein:
      return exec_bluestein(c, dir, dst, src, count, idist, odist, st);
    default:
      return GFFT_ERR_NOT_IMPLEMENTED;
  }
}

}  // namespace gfft
