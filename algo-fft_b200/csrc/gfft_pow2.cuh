// Single-pass shared-memory Stockham kernel for power-of-two N (K1).
//
// One transform is owned by T = N/EPT threads; each thread holds EPT
// elements in registers.  Stage s (radix RS, p = product of the previous
// radices) is Stockham's self-sorting step: butterfly i reads
// x[i + r*N/RS], multiplies by W_{p*RS}^{r*k} (k = i mod p; one coalesced
// load of W_{p*RS}^k, powers by a product tree), runs DFT_RS in registers
// and writes y[(i-k)*RS + k + r*p].  The first stage reads straight from HBM and the last writes straight to HBM,
// both at unit stride across the T threads (fully coalesced), so shared
// memory carries only the exchanges in between.  Shared memory is padded by
// one element every EPT elements, which makes every exchange pattern
// bank-conflict free for EPT >= 8 (checked exhaustively on the CPU for each
// schedule), and keeps every shared address of a thread a compile-time
// offset from one base per butterfly.
//
// Replaces the reference's size-specific DIT codelets 4..16384
// (internal/kernels/codelet_init.go:60-440) and the radix-2 Stockham
// (internal/kernels/stockham.go:21) for one batch of transforms
// (plan.go:504-571).
#pragma once
#include "gfft_sched.cuh"

namespace gfft {

template <int N, int EPT, int ES>
struct Pow2Shape {
  static constexpr int T = N / EPT;                        // threads per transform
  static constexpr int TPB = T >= 256 ? T : 256;           // threads per CTA
  static constexpr int B = TPB / T;                        // transforms per CTA
  static constexpr int PSH = EPT == 2 ? 1 : EPT == 4 ? 2 : EPT == 8 ? 3 : EPT == 16 ? 4 : 5;
  static constexpr int PAD_EXTRA = (T < 16) ? 1 : 0;
  static constexpr int STRIDE = (N - 1) + ((N - 1) >> PSH) + 1 + PAD_EXTRA;  // per transform
  static constexpr int SMEM = (N == EPT) ? 0 : B * STRIDE * ES;               // bytes per CTA
  __host__ __device__ static constexpr int pad(int e) { return e + (e >> PSH); }
};

template <int T>
__device__ __forceinline__ void xsync() {
  if constexpr (T <= 32) __syncwarp();
  else __syncthreads();
}

// Stage recursion of one length-N transform owned by T threads.  The first
// stage takes its inputs from ld(e) and the last hands its outputs to
// st(e, value) (e = element index in natural order), so callers fuse their
// own prologue and epilogue (global I/O, pre-/post-twiddles, real-FFT
// repacking, Bluestein chirps) into the transform.  A policy with
// kShared = true reads or writes this transform's shared memory, and the
// stage then adds the barrier that in-place reuse needs.
template <typename C, int N, int EPT, int DIR, int P, typename LD, typename ST>
__device__ __forceinline__ void pow2_stage(C* v, C* sh, int t, const C* __restrict__ tw, LD& ld, ST& st) {
  using S = Pow2Shape<N, EPT, sizeof(C)>;
  using SC = Sched<N, EPT>;
  constexpr int T = S::T;
  constexpr int RS = SC::radix_at(P);
  constexpr int Q = EPT / RS;
  constexpr int STRIDE = N / RS;
  constexpr bool FIRST = (P == 1);
  constexpr bool LAST = (P * RS == N);

  if constexpr (FIRST) {
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
      for (int r = 0; r < RS; ++r) v[q * RS + r] = ld(t + q * T + r * STRIDE);
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if constexpr (STRIDE % EPT == 0) {
        const int pb = S::pad(t + q * T);
#pragma unroll
        for (int r = 0; r < RS; ++r) v[q * RS + r] = sh[pb + r * (STRIDE + STRIDE / EPT)];
      } else {
#pragma unroll
        for (int r = 0; r < RS; ++r) v[q * RS + r] = sh[S::pad(t + q * T + r * STRIDE)];
      }
    }
  }

#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if constexpr (P > 1) {
      const int k = (t + q * T) & (P - 1);
      apply_twiddles<RS, DIR>(v + q * RS, __ldg(tw + k * (N / (P * RS))));
    }
    dft<RS, DIR>(v + q * RS);
  }

  if constexpr (LAST) {
    // a store policy that writes back into this transform's shared memory
    // must wait until every thread has read the last stage's inputs
    if constexpr (ST::kShared && !(FIRST && !LD::kShared)) xsync<T>();
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
      for (int r = 0; r < RS; ++r) st(t + q * T + r * P, v[q * RS + r]);
  } else {
    if constexpr (!FIRST || LD::kShared) xsync<T>();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = t + q * T;
      const int k = i & (P - 1);
      const int a = i / P;
      // pad(j + r*P) with j = a*P*RS + k: every term but the last is per-butterfly.
      const int jb = a * P * RS + k + (a * P * RS) / EPT;
      if constexpr (P >= EPT) {
        const int pb = jb + (k >> S::PSH);
#pragma unroll
        for (int r = 0; r < RS; ++r) sh[pb + r * (P + P / EPT)] = v[q * RS + r];
      } else {
#pragma unroll
        for (int r = 0; r < RS; ++r) sh[jb + r * P + r / (EPT / P)] = v[q * RS + r];
      }
    }
    xsync<T>();
    pow2_stage<C, N, EPT, DIR, P * RS>(v, sh, t, tw, ld, st);
  }
}

template <typename C, int N, int EPT, int DIR, typename LD, typename ST>
__device__ __forceinline__ void pow2_fft(C* sh, int t, const C* __restrict__ tw, LD& ld, ST& st) {
  C v[EPT];
  pow2_stage<C, N, EPT, DIR, 1>(v, sh, t, tw, ld, st);
}

// L2 prefetch of the inputs of CTA blockIdx + ahead (B transforms of `len`
// elements, `idist` apart), issued by the CTA's threads before its own work;
// ahead = co-resident CTAs, so the data lands about one CTA lifetime early.
template <int B, int TPB, typename C>
__device__ __forceinline__ void prefetch_ahead(const C* src, int64_t count, int64_t idist, int64_t len,
                                               int64_t ahead) {
  if (ahead <= 0) return;
  const int64_t b2 = (int64_t(blockIdx.x) + ahead) * B;
  if (b2 >= count) return;
  const int nb = int(count - b2 < B ? count - b2 : B);
  if (idist == len)
    prefetch_range(src + b2 * idist, int64_t(nb) * len * int64_t(sizeof(C)), threadIdx.x, TPB);
  else
    for (int j = 0; j < nb; ++j) prefetch_range(src + (b2 + j) * idist, len * int64_t(sizeof(C)), threadIdx.x, TPB);
}

// Co-resident CTAs of a kernel on the current device (the prefetch distance).
template <typename F>
inline int64_t resident_ctas(F* fn, int tpb, int smem) {
  int dev = 0, sms = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, tpb, smem);
  cudaGetLastError();
  return int64_t(sms) * (occ > 0 ? occ : 1);
}

template <typename C>
struct GlobalLoad {
  static constexpr bool kShared = false;
  const C* in;
  bool valid;
  __device__ __forceinline__ C operator()(int e) const { return valid ? ld_stream(in + e) : C{0, 0}; }
};

template <typename C, bool SCALE>
struct GlobalStore {
  static constexpr bool kShared = false;
  C* out;
  bool valid;
  typename RealOf<C>::type scale;
  __device__ __forceinline__ void operator()(int e, C x) const {
    if constexpr (SCALE) x = cscale(x, scale);
    if (valid) st_stream(out + e, x);
  }
};

// This transform's padded row in shared memory as the first stage's input
// and the last stage's output (the CTA stages global I/O itself).
template <typename C, int N, int EPT>
struct RowShared {
  static constexpr bool kShared = true;
  C* sh;
  __device__ __forceinline__ C operator()(int e) const { return sh[Pow2Shape<N, EPT, sizeof(C)>::pad(e)]; }
  __device__ __forceinline__ void operator()(int e, C x) const { sh[Pow2Shape<N, EPT, sizeof(C)>::pad(e)] = x; }
};

// Batched C2C: transform b reads src[b*idist .. b*idist+N) and writes
// dst[b*odist ..).  src may equal dst (every CTA reads its whole transform
// before it writes any of it).  tw holds W_N^m, m < N.
//
// With ahead > 0 each CTA first asks for the input of CTA blockIdx + ahead
// to be prefetched into L2 (ahead = the number of co-resident CTAs, so the
// data arrives about one CTA lifetime before it is read): HBM keeps
// streaming while the SM's few resident CTAs are in their compute and
// store phases.  Prefetching only reads, so in-place calls use it too.
template <typename C, int N, int EPT, int DIR>
__global__ void __launch_bounds__(Pow2Shape<N, EPT, sizeof(C)>::TPB)
k_pow2(const C* src, C* dst, int64_t count, int64_t idist, int64_t odist, const C* __restrict__ tw,
       typename RealOf<C>::type scale, int64_t ahead) {
  using S = Pow2Shape<N, EPT, sizeof(C)>;
  prefetch_ahead<S::B, S::TPB>(src, count, idist, N, ahead);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw) + (threadIdx.x / S::T) * S::STRIDE;
  const int t = threadIdx.x % S::T;
  const int64_t b = int64_t(blockIdx.x) * S::B + threadIdx.x / S::T;
  const bool valid = b < count;
  // Few threads per transform (rows of under 128 bytes per thread group):
  // a direct load would touch short runs, so a contiguous batch is staged
  // through shared memory, the CTA's B transforms read and written as one
  // run with consecutive threads on consecutive elements.
  if constexpr (S::T * int(sizeof(C)) < 128 && S::B > 1 && S::SMEM > 0) {
    if (idist == N && odist == N) {
      const int64_t b0 = int64_t(blockIdx.x) * S::B;
      const int nb = int(count - b0 < S::B ? count - b0 : S::B);
      C* shc = reinterpret_cast<C*>(smem_raw);
      constexpr int LN = N == 1 ? 0 : (N == 2 ? 1 : (N == 4 ? 2 : (N == 8 ? 3 : (N == 16 ? 4 : (N == 32 ? 5 : (N == 64 ? 6 : (N == 128 ? 7 : 8)))))));
      static_assert((1 << LN) == N, "staged I/O covers N <= 256");
      const C* in = src + b0 * N;
      for (int e = threadIdx.x; e < nb * N; e += S::TPB)
        shc[(e >> LN) * S::STRIDE + S::pad(e & (N - 1))] = ld_stream(in + e);
      __syncthreads();
      RowShared<C, N, EPT> io{sh};
      pow2_fft<C, N, EPT, DIR>(sh, t, tw, io, io);
      __syncthreads();
      C* out = dst + b0 * N;
      for (int e = threadIdx.x; e < nb * N; e += S::TPB) {
        C y = shc[(e >> LN) * S::STRIDE + S::pad(e & (N - 1))];
        if constexpr (DIR > 0) y = cscale(y, scale);
        st_stream(out + e, y);
      }
      return;
    }
  }
  GlobalLoad<C> ld{src + (valid ? b * idist : 0), valid};
  GlobalStore<C, (DIR > 0)> st{dst + (valid ? b * odist : 0), valid, scale};
  pow2_fft<C, N, EPT, DIR>(sh, t, tw, ld, st);
}

}  // namespace gfft
