// Real-input transforms (K5): N reals as N/2 complex, a half-length C2C and
// the recombination with U[k] = 0.5*(1 + i*W_N^k)
// (plan_real_generic.go:64-98,142-229; inverse repack internal/fft/
// real_repack.go:5-100).  For power-of-two N/2 that fits one CTA, the
// repacking is fused into the transform: the R2C kernel keeps the half-length
// spectrum in shared memory and recombines it on the way out; the C2R kernel
// builds the packed spectrum in its first stage's loads.
#pragma once
#include "gfft_pow2.cuh"

namespace gfft {

// X[k] for k in [0, h]: DC and Nyquist from Y[0] (plan_real_generic.go:174-191),
// else A - U[k] (A - conj(Y[h-k])) with A = Y[k] (:194-228).
template <typename C>
__device__ __forceinline__ C r2c_bin(C y0, C yk, C yhk, C u, int k, int h) {
  using Re = typename RealOf<C>::type;
  if (k == 0) return C{y0.x + y0.y, Re(0)};
  if (k == h) return C{y0.x - y0.y, Re(0)};
  const C b = cconj(yhk);
  const C cc = cmul(u, csub(yk, b));
  return csub(yk, cc);
}

// Packed z[k] of the inverse (internal/fft/real_repack.go:5-100):
// z[0] = (0.5(x0 + xh), 0.5(x0 - xh)); else
// z[k] = (X[k](1-u) - conj(X[h-k]) u) * conj(1 - 2u), u = U[k].  The
// reference writes pairs (k, h-k) from one k; the value it stores at h-k
// equals this formula evaluated at h-k, since U[h-k] = conj(U[k]).
template <typename C>
__device__ __forceinline__ C c2r_packed(C xk, C xhk, C x0, C xh, C u, int k) {
  using Re = typename RealOf<C>::type;
  if (k == 0) return C{Re(0.5) * (x0.x + xh.x), Re(0.5) * (x0.x - xh.x)};
  const C one{1, 0};
  const C omu = csub(one, u);
  const C det = csub(one, cadd(u, u));
  const C inv = cconj(det);  // det is on the unit circle
  return cmul(csub(cmul(xk, omu), cmul(cconj(xhk), u)), inv);
}

template <typename C, int N, int EPT>
struct PaddedStore {
  static constexpr bool kShared = true;
  C* sh;
  __device__ __forceinline__ void operator()(int e, C x) const { sh[Pow2Shape<N, EPT, sizeof(C)>::pad(e)] = x; }
};

// R2C: src holds the reals of transform b at src + b*idist (complex units,
// idist = real stride / 2); dst gets h+1 bins at dst + b*odist.
template <typename C, int H, int EPT>
__global__ void __launch_bounds__(Pow2Shape<H, EPT, sizeof(C)>::TPB)
k_r2c_pow2(const C* src, C* dst, int64_t count, int64_t idist, int64_t odist, const C* __restrict__ tw,
           const C* __restrict__ wt, typename RealOf<C>::type scale) {
  using S = Pow2Shape<H, EPT, sizeof(C)>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw) + (threadIdx.x / S::T) * S::STRIDE;
  const int t = threadIdx.x % S::T;
  const int64_t b = int64_t(blockIdx.x) * S::B + threadIdx.x / S::T;
  const bool valid = b < count;
  GlobalLoad<C> ld{src + (valid ? b * idist : 0), valid};
  PaddedStore<C, H, EPT> st{sh};
  pow2_fft<C, H, EPT, -1>(sh, t, tw, ld, st);
  xsync<S::T>();
  if (!valid) return;
  C* out = dst + b * odist;
  const C y0 = sh[0];
  if (t == 0) {
    st_stream(out, cscale(r2c_bin(y0, y0, y0, C{0, 0}, 0, H), scale));
    st_stream(out + H, cscale(r2c_bin(y0, y0, y0, C{0, 0}, H, H), scale));
  }
  // bins k and H - k share their two inputs: one pair of shared loads per
  // two outputs, stored as an ascending and a descending run
  for (int k = 1 + t; 2 * k <= H; k += S::T) {
    const C yk = sh[S::pad(k)], yhk = sh[S::pad(H - k)];
    st_stream(out + k, cscale(r2c_bin(y0, yk, yhk, __ldg(wt + k), k, H), scale));
    if (2 * k < H) st_stream(out + (H - k), cscale(r2c_bin(y0, yhk, yk, __ldg(wt + (H - k)), H - k, H), scale));
  }
}

template <typename C>
struct RepackLoad {
  static constexpr bool kShared = false;
  const C* X;
  const C* wt;
  int h;
  bool valid;
  C x0, xh;
  __device__ __forceinline__ C operator()(int e) const {
    if (!valid) return C{0, 0};
    return c2r_packed(e == 0 ? x0 : ld_stream(X + e), e == 0 ? x0 : ld_stream(X + (h - e)), x0, xh, __ldg(wt + e), e);
  }
};

// The packed input of the inverse from bins staged in shared memory
// (X[0..h) at the padded positions, X[h] in a register).
template <typename C, int H, int EPT>
struct RepackSharedLoad {
  static constexpr bool kShared = true;
  const C* sh;
  const C* wt;
  C x0, xh;
  __device__ __forceinline__ C operator()(int e) const {
    using S = Pow2Shape<H, EPT, sizeof(C)>;
    return c2r_packed(sh[S::pad(e)], sh[S::pad(e == 0 ? 0 : H - e)], x0, xh, __ldg(wt + e), e);
  }
};

// C2R: src holds h+1 bins of transform b at src + b*idist; dst gets the N
// reals at dst + b*odist (complex units).  scale = 1/h (the half-length
// inverse of the reference, plan_real_generic.go:333).  The bins are read
// once, coalesced, into shared memory; the packing of the first stage pairs
// bins k and h-k from there.
template <typename C, int H, int EPT>
__global__ void __launch_bounds__(Pow2Shape<H, EPT, sizeof(C)>::TPB)
k_c2r_pow2(const C* src, C* dst, int64_t count, int64_t idist, int64_t odist, const C* __restrict__ tw,
           const C* __restrict__ wt, typename RealOf<C>::type scale) {
  using S = Pow2Shape<H, EPT, sizeof(C)>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw) + (threadIdx.x / S::T) * S::STRIDE;
  const int t = threadIdx.x % S::T;
  const int64_t b = int64_t(blockIdx.x) * S::B + threadIdx.x / S::T;
  const bool valid = b < count;
  const C* X = src + (valid ? b * idist : 0);
#pragma unroll
  for (int i = 0; i < EPT; ++i) {
    const int k = t + i * S::T;
    sh[S::pad(k)] = valid ? ld_stream(X + k) : C{0, 0};
  }
  const C xh = valid ? X[H] : C{0, 0};
  xsync<S::T>();
  RepackSharedLoad<C, H, EPT> ld{sh, wt, sh[0], xh};
  GlobalStore<C, true> st{dst + (valid ? b * odist : 0), valid, scale};
  pow2_fft<C, H, EPT, +1>(sh, t, tw, ld, st);
}

// ------------------------------------------------------------ unfused path

// reals (row stride istride, in reals) -> packed complex rows of h
template <typename C>
__global__ void k_pack_real(C* z, const typename RealOf<C>::type* x, int64_t h, int64_t count, int64_t istride) {
  const int64_t total = count * h;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / h, k = e - b * h;
    const auto* p = x + b * istride + 2 * k;
    z[e] = C{p[0], p[1]};
  }
}

template <typename C>
__global__ void k_r2c_post(C* dst, const C* y, const C* wt, int64_t h, int64_t count, int64_t odist,
                           typename RealOf<C>::type scale) {
  const int64_t total = count * (h + 1);
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / (h + 1), k = e - b * (h + 1);
    const C* yb = y + b * h;
    const C yk = k < h ? yb[k] : C{0, 0};
    const C yhk = (k > 0 && k < h) ? yb[h - k] : C{0, 0};
    dst[b * odist + k] = cscale(r2c_bin(yb[0], yk, yhk, wt[k], int(k), int(h)), scale);
  }
}

template <typename C>
__global__ void k_c2r_pre(C* z, const C* X, const C* wt, int64_t h, int64_t count, int64_t idist) {
  const int64_t total = count * h;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / h, k = e - b * h;
    const C* xb = X + b * idist;
    z[e] = c2r_packed(xb[k], xb[k == 0 ? 0 : h - k], xb[0], xb[h], wt[k], int(k));
  }
}

template <typename C>
__global__ void k_unpack_real(typename RealOf<C>::type* x, const C* z, int64_t h, int64_t count, int64_t ostride) {
  const int64_t total = count * h;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / h, k = e - b * h;
    auto* p = x + b * ostride + 2 * k;
    const C v = z[e];
    p[0] = v.x;
    p[1] = v.y;
  }
}

// Flags a spectrum whose DC or Nyquist bin has |imag| > eps
// (plan_real_generic.go:301-316).
template <typename C>
__global__ void k_check_spectrum(const C* X, int64_t h, int64_t count, int64_t idist, double eps, unsigned* flag) {
  for (int64_t b = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; b < count; b += int64_t(gridDim.x) * blockDim.x) {
    const C* xb = X + b * idist;
    if (fabs(double(xb[0].y)) > eps || fabs(double(xb[h].y)) > eps) atomicOr(flag, 1u);
  }
}

}  // namespace gfft
