// Runtime-schedule Stockham for any 7-smooth length (K3).
//
// N = product of radices from {2, 3, 4, 5, 7, 8, 9, 16}, chosen on the host;
// every stage is Stockham's self-sorting step (see gfft_pow2.cuh) with a
// runtime radix dispatched to the in-register DFT codelets.  A transform's
// data sit in shared memory (padded one element every 32) in two buffers:
// each stage reads one and writes the other, so a thread finishes one
// butterfly (R values in registers) before it loads the next, and a stage
// needs one barrier.  T threads own a transform and loop over its
// butterflies.  (Holding all of a thread's butterflies of a stage in
// registers, to work in one buffer, spilled to local memory at every
// launch bound, and the spills reached HBM.)
//
// Replaces the reference's 2/3/4/5 mixed-radix recursion
// (internal/fft/mixedradix.go:45-420) and extends it with radix 7, which the
// reference sends to Bluestein (internal/math/factor.go:30-43).
#pragma once
#include "gfft_math.cuh"

namespace gfft {

struct GenSched {
  int n;          // transform length
  int nst;        // number of stages
  int T;          // threads per transform
  int B;          // transforms per CTA
  int stride;     // shared-memory elements reserved per transform (both buffers)
  int half;       // offset of the second buffer within a transform's region
  int radix[20];  // radix of stage s
  int p[20];      // product of the radices before stage s
  float pinv[20]; // 1 / p[s], for the quotient i / p without an integer divide
};

__device__ __forceinline__ int gpad(int e) { return e + (e >> 5); }

// Thread index handed to gen_fft by threads that own no butterfly: every
// butterfly index it yields is past the end of every stage.
constexpr int kIdleThread = 1 << 28;

// i / p by a float reciprocal (exact for i < 2^24 once corrected by one
// step either way), then k = i mod p.
__device__ __forceinline__ int gen_mod(int i, int p, float pinv, int& q) {
  q = __float2int_rz(__int2float_rn(i) * pinv);
  int k = i - q * p;
  if (k < 0) {
    k += p;
    --q;
  } else if (k >= p) {
    k -= p;
    ++q;
  }
  return k;
}

// One stage: butterflies i = t, t + T, ... of radix R from `in` to `out`
// (shared memory, padded).  GI: the stage reads the transform's global
// input `gin` instead of `in` (first stage); GO: it writes the global
// output `gout` instead of `out`, scaled for the inverse (last stage).
// Consecutive threads touch consecutive elements of both.
template <int R, int DIR, bool GI, bool GO, typename C>
__device__ __forceinline__ void gen_stage(const C* in, C* out, const C* gin, C* gout, typename RealOf<C>::type scale,
                                          int n, int p, float pinv, int T, int t, const C* __restrict__ tw) {
  const int nb = n / R;
  const int step = n / (p * R);
  for (int i = t; i < nb; i += T) {
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if constexpr (GI) v[r] = ld_stream(gin + i + r * nb);
      else v[r] = in[gpad(i + r * nb)];
    }
    int q;
    const int k = gen_mod(i, p, pinv, q);
    if (p > 1) apply_twiddles<R, DIR>(v, __ldg(tw + k * step));
    dft<R, DIR>(v);
    const int j = q * p * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if constexpr (GO) {
        C o = v[r];
        if constexpr (DIR > 0) o = cscale(o, scale);
        st_stream(gout + j + r * p, o);
      } else {
        out[gpad(j + r * p)] = v[r];
      }
    }
  }
}

template <int DIR, bool GI, bool GO, typename C>
__device__ __forceinline__ void gen_stage_any(int radix, const C* a, C* b, const C* gin, C* gout,
                                              typename RealOf<C>::type scale, int n, int p, float pi, int T, int t,
                                              const C* __restrict__ tw) {
  switch (radix) {
    case 2: gen_stage<2, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
    case 3: gen_stage<3, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
    case 4: gen_stage<4, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
    case 5: gen_stage<5, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
    case 7: gen_stage<7, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
    case 8: gen_stage<8, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
    case 9: gen_stage<9, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
    default: gen_stage<16, DIR, GI, GO>(a, b, gin, gout, scale, n, p, pi, T, t, tw); break;
  }
}

// Runs all stages for one direction, the data starting in `a` (shared
// memory, padded layout; the caller synchronises after filling it), `b`
// the other buffer.  Returns the buffer that holds the result, after a
// barrier.
template <int DIR, typename C>
__device__ __forceinline__ C* gen_fft(C* a, C* b, const GenSched& s, int t, const C* __restrict__ tw) {
  using Re = typename RealOf<C>::type;
  for (int st = 0; st < s.nst; ++st) {
    gen_stage_any<DIR, false, false>(s.radix[st], a, b, static_cast<const C*>(nullptr), static_cast<C*>(nullptr),
                                     Re(1), s.n, s.p[st], s.pinv[st], s.T, t, tw);
    __syncthreads();
    C* tmp = a;
    a = b;
    b = tmp;
  }
  return a;
}

// All stages from the transform's global input `gin` to its global output
// `gout` (scaled by `scale` for the inverse): the first stage loads its
// butterflies straight from HBM and the last stores them there, so only
// the stages between touch the shared buffers a and b.
template <int DIR, typename C>
__device__ __forceinline__ void gen_fft_io(C* a, C* b, const C* gin, C* gout, typename RealOf<C>::type scale,
                                           const GenSched& s, int t, const C* __restrict__ tw) {
  if (s.nst == 1) {
    gen_stage_any<DIR, true, true>(s.radix[0], a, b, gin, gout, scale, s.n, s.p[0], s.pinv[0], s.T, t, tw);
    return;
  }
  gen_stage_any<DIR, true, false>(s.radix[0], a, b, gin, gout, scale, s.n, s.p[0], s.pinv[0], s.T, t, tw);
  __syncthreads();
  for (int st = 1; st + 1 < s.nst; ++st) {
    C* tmp = a;
    a = b;
    b = tmp;
    gen_stage_any<DIR, false, false>(s.radix[st], a, b, gin, gout, scale, s.n, s.p[st], s.pinv[st], s.T, t, tw);
    __syncthreads();
  }
  const int last = s.nst - 1;
  gen_stage_any<DIR, false, true>(s.radix[last], b, a, gin, gout, scale, s.n, s.p[last], s.pinv[last], s.T, t, tw);
}

// Batched C2C with a runtime schedule: B transforms per CTA, T threads each.
// Every thread of the CTA reaches every barrier (idle slots included).
// With ahead > 0 each CTA first asks the copy engine to bring the input of
// CTA blockIdx + ahead into L2 (ahead = the co-resident CTAs), so loads
// find it there about one CTA lifetime later.
// LB bounds the CTA size: complex128 CTAs of up to 512 threads are compiled
// for 128 registers (at 64 a radix-16 stage's 32 doubles spill).
template <typename C, int DIR, int LB = 1024>
__global__ void __launch_bounds__(LB) k_generic(const C* src, C* dst, int64_t count, int64_t idist,
                                                  int64_t odist, const C* __restrict__ tw, GenSched s,
                                                  typename RealOf<C>::type scale, int64_t ahead) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (ahead > 0) {
    const int64_t b2 = (int64_t(blockIdx.x) + ahead) * s.B;
    if (b2 < count) {
      const int64_t nb = count - b2 < s.B ? count - b2 : s.B;
      const int64_t bytes = int64_t(s.n) * int64_t(sizeof(C));
      if (idist == s.n)
        prefetch_range(src + b2 * idist, nb * bytes, threadIdx.x, blockDim.x);
      else
        for (int64_t j = 0; j < nb; ++j) prefetch_range(src + (b2 + j) * idist, bytes, threadIdx.x, blockDim.x);
    }
  }
  const int slot = threadIdx.x / s.T, t = threadIdx.x % s.T;
  const int64_t b = int64_t(blockIdx.x) * s.B + slot;
  const bool valid = slot < s.B && b < count;
  C* x = reinterpret_cast<C*>(smem_raw) + (valid ? slot : 0) * s.stride;
  gen_fft_io<DIR>(x, x + s.half, src + (valid ? b * idist : 0), dst + (valid ? b * odist : 0), scale, s,
                  valid ? t : kIdleThread, tw);
}

}  // namespace gfft

namespace gfft {

enum { GEN_PASS1 = 0, GEN_PASS2 = 1 };

// One pass of the runtime two-pass (four-step) transform for 7-smooth
// N = N1 * N2 (index maps as in gfft_twopass.cuh).  A CTA owns NC = s.B
// adjacent columns of one transform, one column per slot of T threads,
// stored column-major in shared memory with an odd per-column stride.
//   GEN_PASS1: column n2 of x viewed as N1 x N2 (L = N1, row pitch N2),
//              times W_N^{n2*k1}, stored as row n2 of the scratch (N2 x N1).
//   GEN_PASS2: column k1 of the scratch (L = N2, row pitch N1), stored as
//              column k1 of the output viewed as N2 x N1.
// `ncols` columns (N2 in pass 1, N1 in pass 2) with rows `pitch` elements
// apart (pitch = ncols in the four-step; larger for strided column batches);
// a last partial tile masks its missing columns.
// Loads and stores walk the tile in the order that keeps NC (pass-1 load,
// pass-2 load and store) or L (pass-1 store) elements contiguous in HBM.
template <typename C, int DIR, int MODE>
__global__ void __launch_bounds__(1024) k_gen_cols(const C* src, C* dst, int64_t count, int64_t in_dist,
                                                   int64_t out_dist, int64_t ncols, int64_t pitch,
                                                   const C* __restrict__ tw, GenSched s, BigTwiddle bt,
                                                   typename RealOf<C>::type scale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  const int L = s.n, NC = s.B;
  const int64_t tiles = (ncols + NC - 1) / NC;
  const int64_t b = int64_t(blockIdx.x) / tiles;
  const int64_t col0 = (int64_t(blockIdx.x) % tiles) * NC;
  const bool valid = b < count;
  const C* in = src + (valid ? b * in_dist : 0);
  C* out = dst + (valid ? b * out_dist : 0);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int ncs = __ffs(NC) - 1;  // NC is a power of two
  for (int e = tid; e < L * NC; e += nthr) {
    const int row = e >> ncs, c = e & (NC - 1);
    C v = C{0, 0};
    if (valid && col0 + c < ncols) {
      const C* p = in + int64_t(row) * pitch + col0 + c;
      v = MODE == GEN_PASS1 ? ld_stream(p) : __ldcg(p);
    }
    base[c * s.stride + gpad(row)] = v;
  }
  __syncthreads();
  const int slot = tid / s.T, t = tid % s.T;
  C* col = base + (slot < NC ? slot : 0) * s.stride;
  gen_fft<DIR>(col, col + s.half, s, slot < NC ? t : kIdleThread, tw);
  // every column's result sits in the same buffer of its region
  const C* res = base + ((s.nst & 1) ? s.half : 0);
  if (!valid) return;
  if constexpr (MODE == GEN_PASS1) {
    const C* lo = static_cast<const C*>(bt.lo);
    const C* hi = static_cast<const C*>(bt.hi);
    const int64_t mask = (int64_t(1) << bt.shift) - 1;
    // rows k1 across the threads (each store instruction writes a run of
    // the row n2 in HBM), columns in turn; W^(n2 k1) of the next column is
    // this one's times W^(k1) (a coalesced lookup), gathered exactly every
    // fourth column so rounding grows by at most three products
    for (int k1 = tid; k1 < L; k1 += nthr) {
      const C step = cmul(__ldg(hi + (k1 >> bt.shift)), __ldg(lo + (k1 & mask)));
      C w = C{1, 0};
      for (int c = 0; c < NC; ++c) {
        const int64_t n2 = col0 + c;
        if (n2 >= ncols) break;
        if ((c & 3) == 0) {
          const int64_t m = n2 * k1;
          w = cmul(__ldg(hi + (m >> bt.shift)), __ldg(lo + (m & mask)));
        } else {
          w = cmul(w, step);
        }
        C wd = w;
        if constexpr (DIR > 0) wd.y = -wd.y;
        __stcg(out + n2 * L + k1, cmul(res[c * s.stride + gpad(k1)], wd));
      }
    }
  } else {
    for (int e = tid; e < L * NC; e += nthr) {
      const int k2 = e >> ncs, c = e & (NC - 1);
      if (col0 + c >= ncols) continue;
      C v = res[c * s.stride + gpad(k2)];
      if constexpr (DIR > 0) v = cscale(v, scale);
      st_stream(out + int64_t(k2) * pitch + col0 + c, v);
    }
  }
}

// Chirp w_k = exp(sign * i*pi * k^2 / n) with k^2 reduced mod 2n in exact
// integer arithmetic before the FP64 evaluation (the reference evaluates
// float64(k*k)/n, internal/kernels/bluestein.go:20-32, which loses
// precision as k grows).
template <typename C>
__global__ void k_chirp(C* w, int64_t n, int sign) {
  using Re = typename RealOf<C>::type;
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x) {
    int64_t m = (k * k) % (2 * n);
    if (m > n) m -= 2 * n;
    double s, c;
    sincospi(double(sign) * double(m) / double(n), &s, &c);
    w[k] = C{Re(c), Re(s)};
  }
}

// b_k = conj(w_k) for k < n, b_{M-k} = conj(w_k) for 0 < k < n, else 0
// (internal/kernels/bluestein.go:39-58).
template <typename C>
__global__ void k_bs_filter_src(C* b, const C* w, int64_t n, int64_t M) {
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < M; j += int64_t(gridDim.x) * blockDim.x) {
    C v{0, 0};
    if (j < n) v = cconj(w[j]);
    else if (M - j < n) v = cconj(w[M - j]);
    b[j] = v;
  }
}

}  // namespace gfft
