// Tensor-core precision form (K7): radix-16 DFT stages as dense products on
// the 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM), with
// split fp16 hi + lo operands and FP32 accumulation.
//
// One radix-16 stage over 256 butterflies is two M=128 GEMM tiles
//   D[m][n] = sum_k A[m][k] B[n][k],  m: butterfly, k, n < 32,
// where row m of A holds the butterfly's 16 inputs (after the FP32 twiddle
// multiply) as [Re x_0..Re x_15, Im x_0..Im x_15], and B is the real form
// of the complex DFT-16 matrix: rows n < 16 give Re y_n, rows 16.. Im y_n.
// Each operand is split as a = a_hi + a_lo (a_hi = fp16(a), a_lo =
// fp16(a - a_hi)); D = A_hi B_hi + A_hi B_lo + A_lo B_hi (the A_lo B_lo term
// is below FP32 rounding), six tcgen05.mma (K = 16) per tile, FP32 sums.
// Rows of A are scaled by a power of two (exact) so their largest entry is
// in [2^13, 2^14): the fp16 range holds, the lo parts stay normal for the
// entries that matter, and the scale is undone exactly on the way out.
//
// Operands live in shared memory in the tensor core's canonical K-major
// layout without swizzle: 8 x 8 fp16 "core matrices" of 128 bytes, K chunks
// 128 bytes apart (leading byte offset), 8-row groups 512 bytes apart
// (stride byte offset).  One thread issues the MMAs and commits them to an
// mbarrier; every thread waits (bounded), then reads its row of D from TMEM
// with tcgen05.ld (warp w reads TMEM lanes 32 (w % 4) ..; the row is the
// thread's own butterfly, so the scale stays in a register).
//
// k_tc_fft: transforms of N = 16^s <= 4096, 4096 elements per CTA (4096/N
// transforms), all s stages in shared memory, one HBM round trip.  Larger
// N = 16^s: s - 3 decimation-in-frequency stages over HBM (k_tc_dif, same
// tensor-core butterfly, post-twiddle W_L^{r m}) leave contiguous blocks of
// 4096 whose transforms k_tc_fft finishes, writing each output to its
// natural index (block digits reversed).
//
// Powers of two that are not powers of 16, n = r 16^s (r = 2, 4, 8), first
// run one decimation-in-frequency stage of radix r in FP32 on the CUDA cores
// (k_tc_lead: block j of a transform gets sum_i x[m + i n/r] W_r^{ij} times
// W_n^{jm}), then the radix-16 tensor-core chain on each block of n/r
// points; k_tc_fft's output index then reverses the block digits in the
// mixed base (r for the leading digit, 16 for the rest).
//
// The CUDA-core FP32 path (k_pow2 / k_tp_split) stays the default; this form
// is selected per plan by its variant token "gpu-sm100-tc16-n<N>"
// (gfft_plan_new_variant; the planner never picks it on its own) and is
// compared against the default and the FP64 oracle.  No counterpart in the reference (its kernels are scalar Go
// and SIMD assembly).
#include <cuda_fp16.h>
#include <algorithm>
#include <cstdio>
#include <new>
#include "gfft_internal.h"
#include "gfft_math.cuh"

namespace gfft {
namespace tc {

constexpr int R = 16;             // radix
constexpr int KD = 2 * R;         // reals per butterfly row
constexpr int BPC = 256;          // butterflies per CTA (two M = 128 tiles)
constexpr int ELEMS = BPC * R;    // 4096 elements per CTA
constexpr int PSH = 4;            // shared-memory padding: one slot per 16 elements
constexpr int A_TILE = 128 * KD * 2;  // bytes of one fp16 A tile (8 KB)
constexpr int B_MAT = KD * KD * 2;    // bytes of one fp16 B matrix (2 KB)
constexpr int TMEM_COLS = 64;         // two tiles x 32 FP32 columns
constexpr unsigned kSpin = 1u << 22;  // bounded mbarrier wait (try_wait rounds)

// shared memory: [A: tile][hl] | [B: hl] | work array | mbarrier, tmem slot
constexpr int SM_A = 0;
constexpr int SM_B = SM_A + 4 * A_TILE;
constexpr int SM_X = SM_B + 2 * B_MAT;
constexpr int SM_BAR = SM_X + (ELEMS + (ELEMS >> PSH)) * 8;
constexpr int SM_TOTAL = SM_BAR + 16;

__device__ __forceinline__ int pad(int e) { return e + (e >> PSH); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  constexpr uint32_t LBO = 128, SBO = 512;
  return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t(LBO >> 4) << 16) | (uint64_t(SBO >> 4) << 32) |
         (uint64_t(1) << 46);
}

// Instruction descriptor, kind::f16: D f32, A and B f16, both K-major,
// N = 32, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (uint32_t(32 >> 3) << 17) | (uint32_t(128 >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(IDESC), "r"(acc));
}

__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the phase with this parity to complete.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
  for (unsigned it = 0; it < kSpin; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float* f) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) f[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) in a K-major core-matrix operand.
__device__ __forceinline__ int opnd_off(int row, int k) {
  return (row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// 2^k as a float for |k| <= 126 (built from its exponent bits: exact).
__device__ __forceinline__ float pow2f(int k) { return __int_as_float((127 + k) << 23); }

__device__ __forceinline__ uint32_t pack2(__half a, __half b) {
  return uint32_t(__half_as_ushort(a)) | (uint32_t(__half_as_ushort(b)) << 16);
}

// Splits the butterfly row (16 complex, scaled by 2^sh) into hi/lo fp16
// rows of A; returns sh.
__device__ __forceinline__ int put_row(unsigned char* sm, int row, const float2* v) {
  float mx = 0.f;
#pragma unroll
  for (int j = 0; j < R; ++j) mx = fmaxf(mx, fmaxf(fabsf(v[j].x), fabsf(v[j].y)));
  int e = 0;
  if (mx > 0.f) frexpf(mx, &e);
  // max |v| * 2^sh in [2^13, 2^14); rows below 2^-106 keep a smaller scale
  const int sh = min(max(14 - e, -120), 120);
  const float sc = pow2f(sh);
  const int tile = row >> 7, m = row & 127;
  unsigned char* hi = sm + SM_A + (tile * 2 + 0) * A_TILE;
  unsigned char* lo = sm + SM_A + (tile * 2 + 1) * A_TILE;
#pragma unroll
  for (int c = 0; c < 4; ++c) {  // chunk c: Re 0-7, Re 8-15, Im 0-7, Im 8-15
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      __half hv[2], lv[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int j = (c & 1) * 8 + q * 2 + u;
        const float x = (c < 2 ? v[j].x : v[j].y) * sc;
        hv[u] = __float2half_rn(x);
        lv[u] = __float2half_rn(x - __half2float(hv[u]));
      }
      h[q] = pack2(hv[0], hv[1]);
      l[q] = pack2(lv[0], lv[1]);
    }
    *reinterpret_cast<uint4*>(hi + opnd_off(m, c * 8)) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(lo + opnd_off(m, c * 8)) = make_uint4(l[0], l[1], l[2], l[3]);
  }
  return sh;
}

// B = the real form of the DFT-16 matrix of direction DIR, split hi/lo.
template <int DIR>
__device__ __forceinline__ void build_b(unsigned char* sm) {
  for (int t = threadIdx.x; t < KD * KD; t += blockDim.x) {
    const int n = t / KD, k = t % KD;
    const int yr = n & 15, xj = k & 15;
    double s, c;
    sincospi(double((yr * xj) & 15) / 8.0, &s, &c);  // angle 2 pi q / 16
    const double wr = c, wi = DIR < 0 ? -s : s;       // W^q = wr + i wi
    double b;
    if (n < 16) b = k < 16 ? wr : -wi;                 // Re y = sum wr xr - wi xi
    else b = k < 16 ? wi : wr;                         // Im y = sum wi xr + wr xi
    const __half h = __float2half_rn(float(b));
    const __half l = __float2half_rn(float(b - double(__half2float(h))));
    *reinterpret_cast<__half*>(sm + SM_B + opnd_off(n, k)) = h;
    *reinterpret_cast<__half*>(sm + SM_B + B_MAT + opnd_off(n, k)) = l;
  }
}

struct TcState {
  uint32_t tmem;
  uint32_t phase;
  bool ok;
};

// One tensor-core radix-16 stage over the CTA's 256 butterfly rows (already
// in A).  Returns this thread's 16 outputs, unscaled by 2^-sh.
__device__ __forceinline__ void tc_stage(unsigned char* sm, TcState& st, int sh, float2* y) {
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + SM_BAR);
  fence_proxy();
  __syncthreads();
  if (threadIdx.x == 0 && st.ok) {  // after an expired wait no new MMA is issued
    fence_after();
    const uint32_t a0 = smem_u32(sm + SM_A), b0 = smem_u32(sm + SM_B);
#pragma unroll
    for (int tile = 0; tile < 2; ++tile) {
      const uint32_t d = st.tmem + tile * 32;
      const uint32_t ah = a0 + (tile * 2) * A_TILE, al = ah + A_TILE;
      const uint32_t bh = b0, bl = b0 + B_MAT;
      uint32_t acc = 0;
#pragma unroll
      for (int pr = 0; pr < 3; ++pr) {  // hi*hi, hi*lo, lo*hi
        const uint32_t a = pr == 2 ? al : ah, b = pr == 1 ? bl : bh;
#pragma unroll
        for (int kb = 0; kb < 2; ++kb) {
          mma(d, sdesc(a + kb * 256), sdesc(b + kb * 256), acc);
          acc = 1;
        }
      }
    }
    commit(bar);
  }
  const bool ok = bar_wait(bar, st.phase & 1);
  st.phase++;
  st.ok = st.ok && ok;
  fence_after();
  float f[32];
  const int w = threadIdx.x >> 5;
  tmem_ld32(st.tmem + (uint32_t((w & 3) * 32) << 16) + uint32_t((w >> 2) * 32), f);
  const float inv = pow2f(-sh);
#pragma unroll
  for (int r = 0; r < R; ++r) y[r] = make_float2(f[r] * inv, f[16 + r] * inv);
  fence_before();
}

__device__ __forceinline__ void tmem_alloc(unsigned char* sm, TcState& st) {
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + SM_BAR + 8);
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) bar_init(reinterpret_cast<uint64_t*>(sm + SM_BAR));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_before();
  __syncthreads();
  fence_after();
  st.tmem = *slot;
  st.phase = 0;
  st.ok = true;
}

__device__ __forceinline__ void tmem_free(TcState& st, unsigned* status) {
  fence_before();
  __syncthreads();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(st.tmem), "r"(TMEM_COLS));
  if (!st.ok && threadIdx.x == 0) atomicExch(status, 1u);
}

// Transforms of length N = 16^S (S <= 3): CTA c owns elements
// [c * 4096, c * 4096 + 4096) of the batch viewed as units of N; with nb > 1
// (N finishing a larger transform of nb * N points) each unit is block
// `blk` of its transform and output k goes to blk' + nb * k, blk' the
// digit-reversed block index: blk = j * 16^dig + d with j < lead (the block
// of a leading radix-`lead` stage, 0 without one) and d of dig base-16
// digits; blk' = j + lead * reverse16(d).
template <int DIR>
__global__ void __launch_bounds__(256) k_tc_fft(const float2* __restrict__ src, float2* __restrict__ dst,
                                                 int64_t units, int N, int S, int64_t nb, int dig, int lead,
                                                 const float2* __restrict__ tw, float scale, unsigned* status) {
  extern __shared__ __align__(128) unsigned char sm[];
  float2* x = reinterpret_cast<float2*>(sm + SM_X);
  TcState st;
  build_b<DIR>(sm);
  tmem_alloc(sm, st);
  const int t = threadIdx.x;
  const int bpt = N / R;                 // butterflies per unit
  const int b = t / bpt, il = t % bpt;   // unit within the CTA, butterfly within the unit
  const int upc = ELEMS / N;             // units per CTA
  const int64_t unit = int64_t(blockIdx.x) * upc + b;
  const bool valid = unit < units;
  const float2* in = src + int64_t(blockIdx.x) * ELEMS;
  float2 v[R];
#pragma unroll
  for (int j = 0; j < R; ++j) v[j] = valid ? ld_stream(in + b * N + il + j * bpt) : make_float2(0.f, 0.f);
  int P = 1;
  for (int p = 0; p < S; ++p) {
    if (p > 0) {
      __syncthreads();
#pragma unroll
      for (int j = 0; j < R; ++j) v[j] = x[pad(b * N + il + j * bpt)];
      apply_twiddles<R, DIR>(v, __ldg(tw + (il % P) * (N / (R * P))));
    }
    const int sh = put_row(sm, t, v);
    float2 y[R];
    tc_stage(sm, st, sh, y);
    const int base = b * N + (il / P) * R * P + (il % P);
    if (p + 1 < S) {
      __syncthreads();  // every thread has read its inputs of this stage
#pragma unroll
      for (int r = 0; r < R; ++r) x[pad(base + r * P)] = y[r];
    } else if (valid) {
      if (nb == 1) {
        float2* out = dst + int64_t(blockIdx.x) * ELEMS;
#pragma unroll
        for (int r = 0; r < R; ++r) st_stream(out + base + r * P, make_float2(y[r].x * scale, y[r].y * scale));
      } else {
        const int64_t tr = unit / nb, blk = unit % nb;
        const int64_t nsub = nb / lead;  // 16^dig
        int64_t rev = 0, q = blk % nsub;
        for (int d = 0; d < dig; ++d) {
          rev = rev * R + q % R;
          q /= R;
        }
        rev = blk / nsub + lead * rev;
        float2* out = dst + tr * nb * N + rev;
#pragma unroll
        for (int r = 0; r < R; ++r)  // index within the unit times the block count
          st_stream(out + int64_t(base - b * N + r * P) * nb, make_float2(y[r].x * scale, y[r].y * scale));
      }
    }
    P *= R;
  }
  tmem_free(st, status);
}

// One decimation-in-frequency radix-16 stage over sub-blocks of length L:
// butterfly m of a block at `base` reads base + m + j L/16 and writes output
// r, times W_L^{r m}, to base + r L/16 + m.  256 butterflies per CTA.
template <int DIR>
__global__ void __launch_bounds__(256) k_tc_dif(const float2* __restrict__ src, float2* __restrict__ dst,
                                                 int64_t butterflies, int64_t L, const float2* __restrict__ twL,
                                                 unsigned* status) {
  extern __shared__ __align__(128) unsigned char sm[];
  TcState st;
  build_b<DIR>(sm);
  tmem_alloc(sm, st);
  const int64_t g = int64_t(blockIdx.x) * BPC + threadIdx.x;
  const bool valid = g < butterflies;
  const int64_t q = L / R;
  const int64_t m = g % q, base = (g / q) * L;
  float2 v[R];
#pragma unroll
  for (int j = 0; j < R; ++j) v[j] = valid ? ld_stream(src + base + m + j * q) : make_float2(0.f, 0.f);
  const int sh = put_row(sm, threadIdx.x, v);
  float2 y[R];
  tc_stage(sm, st, sh, y);
  if (valid) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 w = __ldg(twL + r * m);
      if (DIR > 0) w.y = -w.y;
      st_stream(dst + base + r * q + m, cmul(y[r], w));
    }
  }
  tmem_free(st, status);
}

// Leading decimation-in-frequency stage of radix RL (2, 4 or 8) in FP32 on
// the CUDA cores, for n = RL * Lp: output block j of a transform holds
// sum_i x[m + i Lp] W_RL^{ij} times W_n^{jm} at j Lp + m.  Consecutive
// threads take consecutive m, so every load and store is coalesced.
template <int RL, int DIR>
__global__ void k_tc_lead(const float2* __restrict__ src, float2* __restrict__ dst, int64_t total, int64_t Lp,
                          BigTwiddle bt) {
  for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x) {
    const int64_t m = g % Lp, base = (g / Lp) * Lp * RL;
    float2 v[RL];
#pragma unroll
    for (int i = 0; i < RL; ++i) v[i] = ld_stream(src + base + m + i * Lp);
    dft<RL, DIR>(v);
    st_stream(dst + base + m, v[0]);
#pragma unroll
    for (int j = 1; j < RL; ++j) st_stream(dst + base + j * Lp + m, cmul(v[j], big_twiddle<float2, DIR>(bt, j * m)));
  }
}

}  // namespace tc

// Radix of the leading FP32 stage of n in the tensor-core form (1 for a
// power of 16), 0 when the form cannot serve n.
static int tc_lead_of(int64_t n) {
  if (n < 16 || n > (int64_t(1) << 24) || (n & (n - 1))) return 0;
  int lg = 0;
  while ((int64_t(1) << lg) < n) ++lg;
  return 1 << (lg % 4);
}

bool tc_supported(int64_t n) { return tc_lead_of(n) != 0; }

gfft_status init_tc(PlanCore* c) {
  if (c->prec != kC64 || !tc_supported(c->n)) {
    set_error("the tensor-core form serves complex64 powers of two 16 <= n <= 2^24");
    return GFFT_ERR_NOT_IMPLEMENTED;
  }
  static cudaError_t attr = [] {
    cudaError_t e = cudaFuncSetAttribute(&tc::k_tc_fft<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SM_TOTAL);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(&tc::k_tc_fft<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SM_TOTAL);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(&tc::k_tc_dif<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SM_TOTAL);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(&tc::k_tc_dif<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SM_TOTAL);
    return e;
  }();
  GFFT_CUDA(attr);
  // tables: W_L for every radix-16 stage length used (L = n / lead, /16, ...,
  // and 4096 or less for the last kernel), then for a leading stage the
  // split table of W_n (hi[a] lo[b], m = a 2^shift + b)
  const int64_t n = c->n;
  const int lead = tc_lead_of(n);
  const int64_t lp = n / lead;
  int64_t total = 0;
  for (int64_t L = lp; L > 4096; L /= 16) total += L;
  const int64_t nf = std::min<int64_t>(lp, 4096);
  total += nf;
  int lg = 0;
  while ((int64_t(1) << lg) < n) ++lg;
  const int shift = (lg + 1) / 2;
  const int64_t nlo = int64_t(1) << shift, nhi = n >> shift;
  if (lead > 1) total += nlo + nhi;
  GFFT_CUDA(cudaMalloc(&c->tw, size_t(total) * 8));
  int64_t off = 0;
  for (int64_t L = lp; L > 4096; L /= 16) {
    gfft_status s = fill_twiddles(kC64, static_cast<char*>(c->tw) + off * 8, L, L, 1, 0);
    if (s != GFFT_OK) return s;
    off += L;
  }
  gfft_status s = fill_twiddles(kC64, static_cast<char*>(c->tw) + off * 8, nf, nf, 1, 0);
  if (s != GFFT_OK) return s;
  off += nf;
  if (lead > 1) {
    char* base = static_cast<char*>(c->tw);
    s = fill_twiddles(kC64, base + off * 8, n, nlo, 1, 0);
    if (s == GFFT_OK) s = fill_twiddles(kC64, base + (off + nlo) * 8, n, nhi, nlo, 0);
    if (s != GFFT_OK) return s;
    c->bt_lo = base + off * 8;
    c->bt_hi = base + (off + nlo) * 8;
    c->bt_shift = shift;
  }
  c->tc_lead = lead;
  GFFT_CUDA(cudaMalloc(&c->status, sizeof(unsigned)));
  GFFT_CUDA(cudaMemset(c->status, 0, sizeof(unsigned)));
  GFFT_CUDA(cudaStreamSynchronize(0));
  c->algo = Algo::TensorCore;
  c->name = "gpu-sm100-tc16-n" + std::to_string(n);
  return GFFT_OK;
}

template <int DIR>
static cudaError_t launch_lead(int lead, const float2* in, float2* out, int64_t total, int64_t lp, BigTwiddle bt,
                               cudaStream_t st) {
  const unsigned blocks = unsigned(std::min<int64_t>((total + 255) / 256, 148 * 32));
  if (lead == 2) tc::k_tc_lead<2, DIR><<<blocks, 256, 0, st>>>(in, out, total, lp, bt);
  else if (lead == 4) tc::k_tc_lead<4, DIR><<<blocks, 256, 0, st>>>(in, out, total, lp, bt);
  else tc::k_tc_lead<8, DIR><<<blocks, 256, 0, st>>>(in, out, total, lp, bt);
  return cudaGetLastError();
}

gfft_status exec_tc(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                    int64_t odist, cudaStream_t st) {
  const int64_t n = c->n;
  if (idist != n || odist != n) {
    set_error("the tensor-core form takes contiguous batches");
    return GFFT_ERR_NOT_IMPLEMENTED;
  }
  const int lead = c->tc_lead;
  const int64_t lp = n / lead;
  const float scale = dir < 0 ? 1.f : float(1.0 / double(n));
  const float2* in = static_cast<const float2*>(src);
  float2* out = static_cast<float2*>(dst);
  const float2* tw = static_cast<const float2*>(c->tw);
  // the last kernel's unit: blocks of 4096 points, or the whole n / lead
  const int64_t nu = std::min<int64_t>(lp, 4096);
  int S = 0;
  for (int64_t m = nu; m > 1; m /= 16) ++S;
  if (lead == 1 && n <= 4096) {
    const int64_t blocks = (count * n + tc::ELEMS - 1) / tc::ELEMS;
    if (dir < 0)
      tc::k_tc_fft<-1><<<unsigned(blocks), 256, tc::SM_TOTAL, st>>>(in, out, count, int(n), S, 1, 0, 1, tw, scale,
                                                                    c->status);
    else
      tc::k_tc_fft<1><<<unsigned(blocks), 256, tc::SM_TOTAL, st>>>(in, out, count, int(n), S, 1, 0, 1, tw, scale,
                                                                   c->status);
    GFFT_CUDA(cudaGetLastError());
    return GFFT_OK;
  }
  // stages over HBM (the leading FP32 stage, then radix-16 DIF stages down
  // to blocks of 4096), ping-pong between two scratch halves (never through
  // dst, so src == dst is safe); k_tc_fft then writes dst
  int stages = lead > 1 ? 1 : 0;
  for (int64_t L = lp; L > 4096; L /= 16) ++stages;
  const size_t half_bytes = size_t(count) * size_t(n) * 8;
  void* ws = nullptr;
  GFFT_CUDA(ws_alloc(&ws, half_bytes * (stages > 1 ? 2 : 1), st));
  float2* bufs[2] = {static_cast<float2*>(ws), reinterpret_cast<float2*>(static_cast<char*>(ws) + half_bytes)};
  const float2* cur = in;
  int which = 0, dig = 0;
  int64_t off = 0;
  cudaError_t e = cudaSuccess;
  if (lead > 1) {
    BigTwiddle bt;
    bt.lo = c->bt_lo;
    bt.hi = c->bt_hi;
    bt.shift = c->bt_shift;
    float2* nxt = bufs[which];
    e = dir < 0 ? launch_lead<-1>(lead, cur, nxt, count * lp, lp, bt, st)
                : launch_lead<1>(lead, cur, nxt, count * lp, lp, bt, st);
    cur = nxt;
    which ^= 1;
  }
  for (int64_t L = lp; L > 4096 && e == cudaSuccess; L /= 16, ++dig) {
    float2* nxt = bufs[which];
    const int64_t bf = count * (n / 16);
    const unsigned blocks = unsigned((bf + tc::BPC - 1) / tc::BPC);
    if (dir < 0)
      tc::k_tc_dif<-1><<<blocks, 256, tc::SM_TOTAL, st>>>(cur, nxt, bf, L, tw + off, c->status);
    else
      tc::k_tc_dif<1><<<blocks, 256, tc::SM_TOTAL, st>>>(cur, nxt, bf, L, tw + off, c->status);
    e = cudaGetLastError();
    off += L;
    cur = nxt;
    which ^= 1;
  }
  if (e == cudaSuccess) {
    const int64_t nb = n / nu, units = count * nb;
    const unsigned blocks = unsigned((units * nu + tc::ELEMS - 1) / tc::ELEMS);
    if (dir < 0)
      tc::k_tc_fft<-1><<<blocks, 256, tc::SM_TOTAL, st>>>(cur, out, units, int(nu), S, nb, dig, lead, tw + off, scale,
                                                          c->status);
    else
      tc::k_tc_fft<1><<<blocks, 256, tc::SM_TOTAL, st>>>(cur, out, units, int(nu), S, nb, dig, lead, tw + off, scale,
                                                         c->status);
    e = cudaGetLastError();
  }
  cudaFreeAsync(ws, st);
  if (e != cudaSuccess) return cuda_status(e, "k_tc");
  return GFFT_OK;
}

}  // namespace gfft
