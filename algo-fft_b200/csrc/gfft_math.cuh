// Complex arithmetic and in-register DFT codelets for the sm_100a kernels.
//
// Elements are interleaved (re, im) pairs: float2 for complex64 and double2
// for complex128, the memory layout of Go's complex64/complex128 slices.
// Direction DIR is -1 for the forward transform exp(-2πi jk/n) and +1 for
// the inverse, as in the reference (plan.go:320-330, 372-385).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "gfft_constants.cuh"

namespace gfft {

template <typename R> struct CxOf;
template <> struct CxOf<float> { using type = float2; };
template <> struct CxOf<double> { using type = double2; };
template <typename R> using Cx = typename CxOf<R>::type;

template <typename C> struct RealOf;
template <> struct RealOf<float2> { using type = float; };
template <> struct RealOf<double2> { using type = double; };

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return C{a.x - b.x, a.y - b.y}; }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return C{a.x, -a.y}; }
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) { return C{a.x * s, a.y * s}; }

// a * (DIR * i): forward multiplies by -i, inverse by +i.
template <int DIR, typename C> __device__ __forceinline__ C mul_di(C a) {
  if constexpr (DIR > 0) return C{-a.y, a.x};
  else return C{a.y, -a.x};
}

// cos / sin(2π m / R) from the generated tables (R | 64, or a 7-smooth
// radix up to 64).
template <int R> __host__ __device__ constexpr double root_cos(int m) {
  if constexpr (64 % R == 0) return kCos64[m * (64 / R)];
  else {
    static_assert(has_root_tab(R), "no constant table for this radix");
    return root_cos_tab(R, m);
  }
}
template <int R> __host__ __device__ constexpr double root_sin(int m) {
  if constexpr (64 % R == 0) return kSin64[m * (64 / R)];
  else {
    static_assert(has_root_tab(R), "no constant table for this radix");
    return root_sin_tab(R, m);
  }
}

// a * exp(DIR * 2πi * M / R) for a compile-time root; the quarter-turn
// cases are exact sign swaps.
template <int R, int M, int DIR, typename C> __device__ __forceinline__ C twc(C a) {
  using Re = typename RealOf<C>::type;
  constexpr int m = ((M % R) + R) % R;
  if constexpr (m == 0) return a;
  else if constexpr (2 * m == R) return C{-a.x, -a.y};
  else if constexpr (4 * m == R) return mul_di<DIR>(a);
  else if constexpr (4 * m == 3 * R) return mul_di<-DIR>(a);
  else {
    constexpr double c = root_cos<R>(m);
    constexpr double s = DIR * root_sin<R>(m);
    return C{Re(c) * a.x - Re(s) * a.y, Re(c) * a.y + Re(s) * a.x};
  }
}

// First factor R1 of a composite radix R = R1 * R2 in the in-register DFT:
// 2 for 8, 4 for the other multiples of 4 (radix-4 butterflies need no
// multiplies), else the smallest prime factor.
__host__ __device__ constexpr int dft_split(int R) {
  if (R == 8) return 2;
  if (R % 4 == 0) return 4;
  for (int p = 2; p < R; ++p)
    if (R % p == 0) return p;
  return R;
}

template <int R> __host__ __device__ constexpr double cos_r(int m) { return root_cos<R>(m); }
template <int R> __host__ __device__ constexpr double sin_r(int m) { return root_sin<R>(m); }

// Odd prime radix (3, 5, 7): pairs s_j = v_j + v_{R-j}, d_j = v_j - v_{R-j};
// X_k = v0 + sum_j cos(2*pi*j*k/R) s_j  +-  DIR*i sum_j sin(2*pi*j*k/R) d_j.
// The (j, k) loops are template recursions so every cosine/sine is a
// compile-time constant folded into the arithmetic.
template <int R, int K, int J, typename C>
__device__ __forceinline__ void odd_accum(C& a, C& b, const C* s, const C* d) {
  if constexpr (J <= (R - 1) / 2) {
    using Re = typename RealOf<C>::type;
    constexpr double c = cos_r<R>((J * K) % R);
    constexpr double sn = sin_r<R>((J * K) % R);
    a.x += Re(c) * s[J].x;
    a.y += Re(c) * s[J].y;
    b.x += Re(sn) * d[J].x;
    b.y += Re(sn) * d[J].y;
    odd_accum<R, K, J + 1>(a, b, s, d);
  }
}

template <int R, int K, int DIR, typename C>
__device__ __forceinline__ void odd_out(C* v, const C* s, const C* d, C x0) {
  if constexpr (K <= (R - 1) / 2) {
    C a = x0, b = C{0, 0};
    odd_accum<R, K, 1>(a, b, s, d);
    const C ib = mul_di<DIR>(b);
    v[K] = cadd(a, ib);
    v[R - K] = csub(a, ib);
    odd_out<R, K + 1, DIR>(v, s, d, x0);
  }
}

template <int R, int DIR, typename C> __device__ __forceinline__ void dft_odd(C* v) {
  constexpr int H = (R - 1) / 2;
  C s[H + 1], d[H + 1];
#pragma unroll
  for (int j = 1; j <= H; ++j) {
    s[j] = cadd(v[j], v[R - j]);
    d[j] = csub(v[j], v[R - j]);
  }
  const C x0 = v[0];
  C sum = x0;
#pragma unroll
  for (int j = 1; j <= H; ++j) sum = cadd(sum, s[j]);
  odd_out<R, 1, DIR>(v, s, d, x0);
  v[0] = sum;
}

template <int R, int R1, int R2, int DIR, int IDX = 0, typename C>
__device__ __forceinline__ void twiddle_block(C* a) {
  if constexpr (IDX < R) {
    constexpr int n2 = IDX / R1, k1 = IDX % R1;
    a[IDX] = twc<R, n2 * k1, DIR>(a[IDX]);
    twiddle_block<R, R1, R2, DIR, IDX + 1>(a);
  }
}

// In-register DFT of R points, natural order in and out.  Composite R
// (powers of two up to 64, and 7-smooth products with a constant table) is
// split R = R1 * R2 (n = R2 n1 + n2, k = k1 + R1 k2): R2 DFTs of size R1,
// constant twiddles W_R^{n2 k1}, R1 DFTs of size R2.
template <int R, int DIR, typename C> __device__ __forceinline__ void dft(C* v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = mul_di<DIR>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  } else if constexpr (R == 3 || R == 5 || R == 7) {
    dft_odd<R, DIR>(v);
  } else {
    constexpr int R1 = dft_split(R);
    constexpr int R2 = R / R1;
    static_assert(R1 > 1 && R2 > 1 && R <= 64, "unsupported radix");
    C a[R];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
      C t[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + n2];
      dft<R1, DIR>(t);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) a[n2 * R1 + k1] = t[k1];
    }
    // constant twiddles, unrolled through a helper so M is compile-time
    twiddle_block<R, R1, R2, DIR>(a);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C t[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) t[n2] = a[n2 * R1 + k1];
      dft<R2, DIR>(t);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
    }
  }
}

// v[r] *= w^r (r = 1..RS-1) where w = tw[m] (conjugated for the inverse).
// Up to RS = 8 the powers come from a product tree w^r = w^{r/2} w^{r-r/2};
// beyond, w^r = w^{r mod 8} * (w^8)^{r/8} from the two short tables
// {w^0..w^7} and {w^0, w^8, w^16, w^24}, which keeps ten powers live
// instead of RS.  Tree depth, and so the rounding error, stays at a few ulp.
template <int RS, int DIR, typename C>
__device__ __forceinline__ void apply_twiddles(C* v, C w1) {
  if constexpr (RS > 1) {
    if constexpr (DIR > 0) w1.y = -w1.y;
    if constexpr (RS <= 8) {
      C w[RS];
      w[1] = w1;
#pragma unroll
      for (int r = 2; r < RS; ++r) w[r] = cmul(w[r / 2], w[r - r / 2]);
#pragma unroll
      for (int r = 1; r < RS; ++r) v[r] = cmul(v[r], w[r]);
    } else {
      constexpr int NH = (RS + 7) / 8;  // w^0, w^8, ... up to w^{8 (NH - 1)}
      C lo[8], hi[NH];
      lo[1] = w1;
#pragma unroll
      for (int r = 2; r < 8; ++r) lo[r] = cmul(lo[r / 2], lo[r - r / 2]);
      hi[1] = cmul(lo[4], lo[4]);
#pragma unroll
      for (int h = 2; h < NH; ++h) hi[h] = cmul(hi[h / 2], hi[h - h / 2]);
#pragma unroll
      for (int r = 1; r < RS; ++r) {
        const int a = r % 8, b = r / 8;
        if (b == 0) v[r] = cmul(v[r], lo[a]);
        else if (a == 0) v[r] = cmul(v[r], hi[b]);
        else v[r] = cmul(v[r], cmul(lo[a], hi[b]));
      }
    }
  }
}

// W_N^m for m < N from two short tables: m = a * 2^shift + b,
// W_N^m = hi[a] * lo[b] (one extra rounding of a complex product).
struct BigTwiddle {
  const void* lo;  // W_N^j, j < 2^shift
  const void* hi;  // W_N^(j << shift), j < N >> shift
  int shift;
};

template <typename C, int DIR>
__device__ __forceinline__ C big_twiddle(const BigTwiddle& bt, int64_t m) {
  const C* lo = static_cast<const C*>(bt.lo);
  const C* hi = static_cast<const C*>(bt.hi);
  C w = cmul(__ldg(hi + (m >> bt.shift)), __ldg(lo + (m & ((int64_t(1) << bt.shift) - 1))));
  if constexpr (DIR > 0) w.y = -w.y;
  return w;
}

// The same from tables that may sit in shared memory (generic loads).
template <typename C, int DIR>
__device__ __forceinline__ C big_twiddle_any(const BigTwiddle& bt, int64_t m) {
  const C* lo = static_cast<const C*>(bt.lo);
  const C* hi = static_cast<const C*>(bt.hi);
  C w = cmul(hi[m >> bt.shift], lo[m & ((int64_t(1) << bt.shift) - 1)]);
  if constexpr (DIR > 0) w.y = -w.y;
  return w;
}

// Streaming global accesses: the batch is touched exactly once.
// Asks the TMA unit to bring [p, p + bytes) into L2 ahead of its use (no
// registers, no completion to wait for).  p and bytes must be multiples of
// 16; callers check both.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Prefetches [p, p + bytes) in runs of at most 32 KB spread over the
// calling threads (thread `lane` of `nthr`); skipped unless p and bytes are
// multiples of 16.
__device__ __forceinline__ void prefetch_range(const void* p, int64_t bytes, int lane, int nthr) {
  if ((bytes & 15) || (reinterpret_cast<uintptr_t>(p) & 15)) return;
  constexpr int64_t kRun = 32768;
  const int64_t runs = (bytes + kRun - 1) / kRun;
  for (int64_t i = lane; i < runs; i += nthr) {
    const int64_t len = bytes - i * kRun < kRun ? bytes - i * kRun : kRun;
    prefetch_l2(static_cast<const char*>(p) + i * kRun, unsigned(len));
  }
}

__device__ __forceinline__ float2 ld_stream(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(float2* p, float2 v) { __stcs(p, v); }
__device__ __forceinline__ void st_stream(double2* p, double2 v) { __stcs(p, v); }

}  // namespace gfft
