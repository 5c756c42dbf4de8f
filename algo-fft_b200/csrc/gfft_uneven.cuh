// Uneven-length batches (K8): thousands of transforms of different lengths,
// packed back to back, in a handful of launches.
//
// k_uneven: persistent CTAs pop items (one transform each) from a device
// work queue.  An item names a descriptor (one per distinct length): the
// runtime Stockham schedule and the offsets of its tables.  Direct items run
// the schedule on the transform; Bluestein items (length n, FFT length
// M = NextPow2(2n-1), plan_bluestein.go) run chirp-multiply, FFT_M, filter
// product, inverse FFT_M and chirp-multiply in the same CTA's shared memory.
// Items come sorted by decreasing cost, so the queue order is also a
// longest-first schedule.
#pragma once
#include "gfft_generic.cuh"

namespace gfft {

struct UnevenDesc {
  GenSched s;         // schedule of the FFT length s.n (n, or M for Bluestein)
  int64_t n;          // transform length
  int32_t bluestein;  // 1: Bluestein through an FFT of length s.n
  int32_t pad_;
  int64_t tw;         // W_{s.n} table (element offset into the tables)
  int64_t chirp;      // forward chirp exp(-i pi k^2/n), k < n
  int64_t filt;       // forward filter FFT_M(b), M entries
};

struct UnevenItem {
  int64_t off;   // element offset of the transform in src and dst
  int32_t desc;  // descriptor index
  int32_t pad_;
};

template <int DIR, typename C>
__device__ __forceinline__ C chirp_dir(C w) {
  if constexpr (DIR > 0) return cconj(w);
  else return w;
}

template <typename C, int DIR>
__global__ void __launch_bounds__(1024) k_uneven(const C* src, C* dst, const UnevenItem* __restrict__ items, int nitems,
                                                 const UnevenDesc* __restrict__ descs, const C* __restrict__ tab,
                                                 unsigned* counter) {
  using Re = typename RealOf<C>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* x = reinterpret_cast<C*>(smem_raw);
  __shared__ UnevenDesc d;
  __shared__ int s_w;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_w = int(atomicAdd(counter, 1u));
    __syncthreads();
    const int w = s_w;
    if (w >= nitems) break;
    const UnevenItem it = items[w];
    for (int i = tid; i < int(sizeof(UnevenDesc) / sizeof(int)); i += nthr)
      reinterpret_cast<int*>(&d)[i] = reinterpret_cast<const int*>(descs + it.desc)[i];
    __syncthreads();
    const int L = d.s.n;
    const int t = tid < d.s.T ? tid : kIdleThread;
    const C* W = tab + d.tw;
    const C* in = src + it.off;
    C* out = dst + it.off;
    if (!d.bluestein) {
      if (d.s.nst == 0) {  // length 1
        for (int e = tid; e < L; e += nthr) st_stream(out + e, ld_stream(in + e));
      } else {
        // first stage from HBM, last stage to HBM
        gen_fft_io<DIR>(x, x + d.s.half, in, out, Re(1.0 / double(L)), d.s, t, W);
      }
    } else {
      const int n = int(d.n);
      const C* ch = tab + d.chirp;
      const C* F = tab + d.filt;
      for (int e = tid; e < L; e += nthr)
        x[gpad(e)] = e < n ? cmul(ld_stream(in + e), chirp_dir<DIR>(__ldg(ch + e))) : C{0, 0};
      __syncthreads();
      C* y = gen_fft<-1>(x, x + d.s.half, d.s, t, W);
      C* other = y == x ? x + d.s.half : x;
      // the inverse filter is FFT_M(conj b) = conj(F[(M - k) mod M])
      for (int e = tid; e < L; e += nthr) {
        const C f = DIR < 0 ? __ldg(F + e) : cconj(__ldg(F + (e == 0 ? 0 : L - e)));
        y[gpad(e)] = cmul(y[gpad(e)], f);
      }
      __syncthreads();
      const C* res = gen_fft<+1>(y, other, d.s, t, W);
      const Re sc = Re(DIR > 0 ? 1.0 / (double(L) * double(n)) : 1.0 / double(L));
      for (int e = tid; e < n; e += nthr)
        st_stream(out + e, cscale(cmul(res[gpad(e)], chirp_dir<DIR>(__ldg(ch + e))), sc));
    }
  }
}

// ---- large items: rows gathered into per-length (or per-M) batches --------

struct BigItem {
  int64_t off;    // offset in src/dst
  int64_t n;      // transform length
  int64_t chirp;  // Bluestein: chirp offset in the tables
  int64_t filt;   // Bluestein: filter offset in the tables
};

// work[r][m] = m < n_r ? x_r[m] (* chirp for Bluestein) : 0
template <typename C, int DIR>
__global__ void k_big_gather(C* work, int64_t M, const C* src, const BigItem* items, int64_t rows, const C* tab,
                             int bluestein) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < rows * M; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / M, m = e - r * M;
    const BigItem it = items[r];
    C v{0, 0};
    if (m < it.n) {
      v = ld_stream(src + it.off + m);
      if (bluestein) v = cmul(v, chirp_dir<DIR>(tab[it.chirp + m]));
    }
    work[e] = v;
  }
}

template <typename C, int DIR>
__global__ void k_big_filter(C* work, int64_t M, const BigItem* items, int64_t rows, const C* tab) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < rows * M; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / M, m = e - r * M;
    const C* F = tab + items[r].filt;
    const C f = DIR < 0 ? F[m] : cconj(F[m == 0 ? 0 : M - m]);
    work[e] = cmul(work[e], f);
  }
}

// y_r[k] = work[r][k] (* chirp, and 1/n_r for the inverse, for Bluestein;
// the batched inverse FFT_M already applied 1/M), k < n_r
template <typename C, int DIR>
__global__ void k_big_scatter(C* dst, const C* work, int64_t M, const BigItem* items, int64_t rows, const C* tab,
                              int bluestein) {
  using Re = typename RealOf<C>::type;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < rows * M; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / M, k = e - r * M;
    const BigItem it = items[r];
    if (k >= it.n) continue;
    C v = work[e];
    if (bluestein) {
      v = cmul(v, chirp_dir<DIR>(tab[it.chirp + k]));
      if constexpr (DIR > 0) v = cscale(v, Re(1.0 / double(it.n)));
    }
    st_stream(dst + it.off + k, v);
  }
}

}  // namespace gfft
