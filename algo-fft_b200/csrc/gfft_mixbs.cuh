// Bluestein's chain on the compiled mixed-radix column tiles, for FFT
// lengths M = M1 x M2 that are not powers of two.
//
// The reference pads to M = NextPow2(2n - 1) (plan.go:865), which costs
// 2..4 times n per FFT; any M >= 2n - 1 gives the same product up to
// rounding.  Here M is the smallest product of two compiled column lengths
// (18 multiples of 16 from 80 to 512) that is at least 2n - 1, used when it is below
// the power of two: about 0.76 of it on average over primes 8K..131K.  The
// element-wise steps ride in the passes, as in the power-of-two chain
// (kernels_bluestein_tp.cu), three launches per chunk of transforms:
//   BSK_IN   forward pass 1 (columns of M1), its loads the chirp-weighted,
//            zero-padded input a_m = x_m w_m (m < n), scratch out (rows n2
//            of M1, times W_M^{n2 k1});
//   BSK_MID  forward pass 2 on columns k1 of the scratch (length M2), the
//            spectrum times the filter, Z_k = A_k F_k (k = k1 + M1 k2), left
//            in shared memory; then the inverse FFT's pass 1 on the same
//            tile: the inverse splits M the other way (M2 rows of M1), so
//            its column k1 is exactly the tile's column, times
//            W_M^{-k1 j2}, stored as rows k1 of M2 into the work buffer;
//   BSK_OUT  inverse pass 2 (columns of M1), its stores y_k = w_k z_k / M
//            (and 1/n for the inverse transform) for k < n only, k = j2 +
//            M2 j1.
// About 4M + 2n element transfers per transform (6M + 2n with the filter
// product stored and the inverse pass 1 a launch of its own).  The chirp w
// and filter F of the forward direction serve the inverse as conj(w) and
// conj(F[(M - k) mod M]) (flag `inv`).
#pragma once
#include "gfft_mixcols.cuh"

namespace gfft {

enum { BSK_IN = 0, BSK_MID = 1, BSK_OUT = 2 };

// One transform of an uneven batch on this chain (offsets in elements).
struct MixBsItem {
  int64_t off;        // the transform in the user's input and output
  int64_t s;          // its M-element rows in the scratch and work buffers
  int64_t n, M;
  int64_t chirp, filt;  // forward chirp (n) and filter spectrum (M) in `tab`
  int64_t lo, hi;       // W_M split tables in `tab`
  int32_t shift;
  int32_t first[3];     // first CTA in its BSK_IN / BSK_MID / BSK_OUT launch
};

struct MixBsParams {
  const void* x;      // user input
  void* y;            // user output
  void* scratch;      // M elements per transform
  void* work;         // M elements per transform
  int64_t n, M, idist, odist;  // batch mode: every transform alike
  const void* w;      // batch mode: chirp of the direction asked for
  const void* f;      // batch mode: filter spectrum of that direction
  const void* tw;     // W_L, L the launch's column length
  BigTwiddle bt;      // W_M (BSK_IN, BSK_MID)
  int64_t tiles;      // batch mode: column tiles per transform; item mode: CTAs
  double scale;       // batch mode: output scale (1/n for the inverse)
  int inv;            // item mode: 1 for the inverse (conjugate tables, 1/n)
  const MixBsItem* items = nullptr;
  const int32_t* blk = nullptr;
  const void* tab = nullptr;
};

template <typename C>
__device__ __forceinline__ C bs_chirp(const C* w, int64_t m, int inv) {
  C v = __ldg(w + m);
  if (inv) v.y = -v.y;
  return v;
}

template <typename C>
struct MixBsIn {
  static constexpr bool kLoad = true, kStore = false;
  const C* x;
  const C* w;
  int64_t n, pitch, col0;
  int inv;
  __device__ __forceinline__ C load(int row, int c) const {
    const int64_t m = int64_t(row) * pitch + col0 + c;
    return m < n ? cmul(ld_stream(x + m), bs_chirp(w, m, inv)) : C{0, 0};
  }
};

// BSK_MID's forward stores: Z_k = A_k F_k into the tile's shared memory,
// row k2 of column c (k = k1 + M1 k2, k1 = col0 + c).
template <typename TL, typename C>
struct MixBsFiltSh {
  static constexpr bool kLoad = false, kStore = true, kShared = true;
  C* sh;
  const C* f;
  int64_t m1, col0, M;
  int inv;
  __device__ __forceinline__ void store(int row, int c, C v) const {
    const int64_t k = col0 + c + m1 * int64_t(row);
    // one load per element: the index first, then the conjugate
    C fk = __ldg(f + (inv ? (k == 0 ? 0 : M - k) : k));
    if (inv) fk.y = -fk.y;
    sh[TL::phys(row, c)] = cmul(v, fk);
  }
};

// BSK_MID's inverse loads: the same rows back out of shared memory.
template <typename TL, typename C>
struct MixBsLoadSh {
  static constexpr bool kLoad = true, kStore = false, kShared = true;
  const C* sh;
  __device__ __forceinline__ C load(int row, int c) const { return sh[TL::phys(row, c)]; }
};

template <typename C>
struct MixBsOut {
  static constexpr bool kLoad = false, kStore = true;
  C* y;
  const C* w;
  int64_t n, m2, col0;
  typename RealOf<C>::type scale;
  int inv;
  __device__ __forceinline__ void store(int row, int c, C v) const {
    const int64_t k = col0 + c + m2 * int64_t(row);
    if (k < n) st_stream(y + k, cscale(cmul(v, bs_chirp(w, k, inv)), scale));
  }
};

// One CTA per column tile of one transform (batch mode: blockIdx =
// transform * tiles + tile; item mode: items[blk[blockIdx]]).
template <typename C, typename SC, int NC, int KIND, int MINB = 1, int TT = 0>
__global__ void __launch_bounds__(MixTile<SC, NC, TT>::TPB, MINB) k_mix_bs(MixBsParams p) {
  using TL = MixTile<SC, NC, TT>;
  using Re = typename RealOf<C>::type;
  constexpr int L = SC::L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  int64_t col0, off_x, off_y, s, n, M;
  const C* w;
  const C* f;
  BigTwiddle bt = p.bt;
  Re oscale;
  if (p.items) {
    const MixBsItem m = p.items[p.blk[blockIdx.x]];
    col0 = int64_t(int(blockIdx.x) - m.first[KIND]) * NC;
    off_x = off_y = m.off;
    s = m.s;
    n = m.n;
    M = m.M;
    const C* tab = static_cast<const C*>(p.tab);
    w = tab + m.chirp;
    f = tab + m.filt;
    bt = BigTwiddle{tab + m.lo, tab + m.hi, m.shift};
    oscale = Re(p.inv ? 1.0 / double(m.n) : 1.0);
  } else {
    const int64_t b = blockIdx.x / p.tiles;
    col0 = (blockIdx.x % p.tiles) * NC;
    off_x = b * p.idist;
    off_y = b * p.odist;
    s = b * p.M;
    n = p.n;
    M = p.M;
    w = static_cast<const C*>(p.w);
    f = static_cast<const C*>(p.f);
    oscale = Re(p.scale);  // batch mode: the direction's own tables
  }
  const int64_t ncols = M / L;  // M2 for BSK_IN and BSK_OUT, M1 for BSK_MID
  const int c = threadIdx.x % NC, t = threadIdx.x / NC;
  const bool active = col0 + c < ncols;
  const C* tw = static_cast<const C*>(p.tw);
  C* scratch = static_cast<C*>(p.scratch);
  C v[TL::vmax()];
  if constexpr (KIND == BSK_IN) {
    const MixBsIn<C> io{static_cast<const C*>(p.x) + off_x, w, n, ncols, col0, p.inv};
    mix_stage<C, SC, TL, -1, 0, MIX_PASS1, MixBsIn<C>>(v, nullptr, nullptr, sh, t, c, active, tw, Re(1), bt,
                                                       col0 + c, ncols, 0, io);
    C* yt = scratch + s + col0 * L;
    const int nv = int(ncols - col0 < NC ? ncols - col0 : NC);
    for (int e = threadIdx.x; e < L * nv; e += TL::TPB) {
      const int cc = e / L, row = e - cc * L;
      __stcg(yt + e, sh[cc * TL::LP + row]);
    }
  } else if constexpr (KIND == BSK_MID) {
    const MixBsFiltSh<TL, C> fwd{sh, f, ncols, col0, M, p.inv};
    mix_stage<C, SC, TL, -1, 0, MIX_PASS2, MixBsFiltSh<TL, C>>(v, scratch + s + col0, nullptr, sh, t, c, active,
                                                               tw, Re(1), bt, 0, ncols, ncols, fwd);
    __syncthreads();
    const MixBsLoadSh<TL, C> back{sh};
    mix_stage<C, SC, TL, +1, 0, MIX_PASS1, MixBsLoadSh<TL, C>>(v, nullptr, nullptr, sh, t, c, active, tw, Re(1), bt,
                                                               col0 + c, 0, 0, back);
    C* yt = static_cast<C*>(p.work) + s + col0 * L;
    const int nv = int(ncols - col0 < NC ? ncols - col0 : NC);
    for (int e = threadIdx.x; e < L * nv; e += TL::TPB) {
      const int cc = e / L, row = e - cc * L;
      __stcg(yt + e, sh[cc * TL::LP + row]);
    }
  } else {
    const MixBsOut<C> io{static_cast<C*>(p.y) + off_y, w, n, ncols, col0, oscale, p.inv};
    mix_stage<C, SC, TL, +1, 0, MIX_PASS2, MixBsOut<C>>(v, static_cast<const C*>(p.work) + s + col0, nullptr, sh, t,
                                                        c, active, tw, Re(1.0 / double(M)), bt, 0, ncols, ncols, io);
  }
}

}  // namespace gfft
