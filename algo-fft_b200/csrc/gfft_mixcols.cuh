// Compile-time mixed-radix column tiles for 7-smooth column lengths.
//
// The runtime-radix column kernel (k_gen_cols) pays for its generality in
// instructions: a radix switch per stage, a runtime quotient and padded
// address per butterfly, and two extra shared-memory passes to load and
// store the tile.  For the column lengths the four-step splits of common
// 7-smooth sizes produce (147 x 343 = 50421, 250 x 400 = 100000,
// 1000 x 1000 = 10^6, ...) this header generates the same column FFTs with
// the radices fixed at compile time, in the register/shared-memory form of
// the power-of-two column tiles (col_stage): the first stage reads its
// butterflies straight from HBM (runs of NC contiguous elements), the last
// writes them straight back (pass 2) or, times the four-step twiddle,
// transposed into shared memory for stores of whole rows (pass 1), and only
// the exchanges between stages go through shared memory.
//
// A column of L = R_0 * R_1 * ... points is owned by T threads, L / max(R)
// by default (or L / min(R) for two-stage schedules whose larger radix is
// not a multiple of the smaller: every thread then holds at most max(R)
// values).  Stage s (radix R_s, prefix product P_s) is Stockham's
// self-sorting step:
// butterfly i < L / R_s reads rows i + r L/R_s, multiplies by W_L^{r k L/(P_s R_s)}
// (k = i mod P_s), runs DFT_{R_s} in registers and writes rows
// (i - k) R_s + k + r P_s.  A thread takes butterflies t, t + T, ...; the
// stages of the largest radix give every thread exactly one, smaller radices
// several (the last partial round masked).
//
// Replaces, for these lengths, the reference's mixed-radix recursion
// (internal/fft/mixedradix.go:45-188) inside the four-step of large
// 7-smooth lengths (internal/kernels/sixstep.go:29-91).
#pragma once
#include <type_traits>
#include "gfft_math.cuh"

namespace gfft {

// Stage radices R..., in the order the stages run.
template <int... R>
struct MixSched {
  static constexpr int NS = sizeof...(R);
  static constexpr int L = (1 * ... * R);
  __host__ __device__ static constexpr int radix(int s) {
    constexpr int a[] = {R...};
    return a[s];
  }
  __host__ __device__ static constexpr int prefix(int s) {
    int p = 1;
    for (int i = 0; i < s; ++i) p *= radix(i);
    return p;
  }
  __host__ __device__ static constexpr int rmax() {
    int m = 1;
    for (int i = 0; i < NS; ++i) m = radix(i) > m ? radix(i) : m;
    return m;
  }
};

// Tile of NC adjacent columns (NC a power of two) of length SC::L, TT
// threads per column (0: L / max radix).
// Shared memory: element (row, c) at row * PITCH + c, PITCH = NC + 1 (odd)
// for NC >= 16, else rows of NC with the column XOR-swizzled by the row.
// (Skipping a row every R0 rows for even first radices, as rows mode does,
// measured 2% slower here, up to 20% for some complex128 lengths.)
// Pass 1's transposed result: column c at c * LP, LP = L rounded up to odd,
// so the NC columns a warp writes at once fall in distinct banks.
template <typename SC, int NC, int TT = 0>
struct MixTile {
  static_assert((NC & (NC - 1)) == 0, "NC must be a power of two");
  static constexpr int L = SC::L;
  static constexpr int T = TT > 0 ? TT : L / SC::rmax();  // threads per column
  static constexpr int TPB = T * NC;
  static_assert(TPB <= 1024, "tile needs more than 1024 threads");
  static constexpr bool PITCHED = NC >= 16;
  static constexpr int PITCH = PITCHED ? NC + 1 : NC;
  static constexpr int LP = L | 1;
  static constexpr int ELEMS1 = L * PITCH > NC * LP ? L * PITCH : NC * LP;  // pass 1
  static constexpr int ELEMS2 = L * PITCH;                                  // pass 2
  __host__ __device__ static constexpr int q_at(int s) { return (L / SC::radix(s) + T - 1) / T; }
  __host__ __device__ static constexpr int vmax() {
    int m = 1;
    for (int s = 0; s < SC::NS; ++s) m = q_at(s) * SC::radix(s) > m ? q_at(s) * SC::radix(s) : m;
    return m;
  }
  __device__ static __forceinline__ int phys(int row, int c) {
    if constexpr (PITCHED) return row * PITCH + c;
    else return row * NC + (c ^ (row & (NC - 1)));
  }
};

enum { MIX_PASS1 = 1, MIX_PASS2 = 2 };

// Hooks of mix_stage: kLoad replaces the first stage's loads by
// io.load(row, c), kStore the last stage's pass-2 stores by
// io.store(row, c, value) (the value already scaled for the inverse).  A
// hook that declares kShared = true reads or writes the tile's shared
// memory, and the stage then adds the barriers that reuse needs.
struct MixNoIO {
  static constexpr bool kLoad = false, kStore = false;
};

template <typename IO, typename = void>
struct io_shared : std::false_type {};
template <typename IO>
struct io_shared<IO, std::void_t<decltype(IO::kShared)>> : std::bool_constant<IO::kShared> {};

// One stage of a column tile, then the next (compile-time recursion).
//   MIX_PASS1: the first stage streams rows `ip` elements apart; the last
//     multiplies output row k1 of column n2 by W_N^{n2 k1} and writes it to
//     sh[c * LP + k1] (the caller stores whole rows of L).
//   MIX_PASS2: the first stage reads rows `ip` apart through L2 (the
//     four-step intermediate, or a caller's column batch); the last writes
//     row k to out[k * op] scaled by `scale` for the inverse.
template <typename C, typename SC, typename TL, int DIR, int S, int PASS, typename IO = MixNoIO>
__device__ __forceinline__ void mix_stage(C* v, const C* in, C* out, C* sh, int t, int c, bool active,
                                          const C* __restrict__ tw, typename RealOf<C>::type scale,
                                          const BigTwiddle& bt, int64_t n2, int64_t ip, int64_t op,
                                          const IO& io = IO()) {
  constexpr int L = SC::L, T = TL::T;
  constexpr int RS = SC::radix(S);
  constexpr int P = SC::prefix(S);
  constexpr int NB = L / RS;          // butterflies of the stage
  constexpr int Q = (NB + T - 1) / T;  // per thread
  constexpr bool GUARD = NB % T != 0;
  constexpr bool FIRST = S == 0;
  constexpr bool LAST = S == SC::NS - 1;
  // the stage read shared memory, so it must sync before writing it
  constexpr bool READ_SH = !FIRST || (io_shared<IO>::value && IO::kLoad);
  constexpr bool STORE_SH = io_shared<IO>::value && IO::kStore;

  // Pass 1's four-step twiddles of the last stage, fetched before its loads
  // so their latency hides behind them: W_N^{n2 (i + r P)} = b * s^r with
  // b = W_N^{n2 i} (one lookup per butterfly) and s = W_N^{n2 P}.
  [[maybe_unused]] C tw_s{}, tw_b[Q];
  if constexpr (LAST && PASS == MIX_PASS1) {
    if (active) {
      tw_s = big_twiddle<C, DIR>(bt, n2 * P);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int i = t + q * T;
        tw_b[q] = big_twiddle<C, DIR>(bt, n2 * int64_t(GUARD && i >= NB ? 0 : i));
      }
    }
  }

  if (active) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = t + q * T;
      if (GUARD && i >= NB) break;
#pragma unroll
      for (int r = 0; r < RS; ++r) {
        const int row = i + r * NB;
        if constexpr (FIRST && IO::kLoad) {
          v[q * RS + r] = io.load(row, c);
        } else if constexpr (FIRST) {
          const C* p = in + int64_t(row) * ip + c;
          v[q * RS + r] = PASS == MIX_PASS1 ? ld_stream(p) : __ldcg(p);
        } else {
          v[q * RS + r] = sh[TL::phys(row, c)];
        }
      }
      if constexpr (P > 1) apply_twiddles<RS, DIR>(v + q * RS, __ldg(tw + (i % P) * (L / (P * RS))));
      dft<RS, DIR>(v + q * RS);
    }
  }

  if constexpr (LAST && PASS == MIX_PASS2) {
    if constexpr (STORE_SH && READ_SH) __syncthreads();
    if (active) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int i = t + q * T;
        if (GUARD && i >= NB) break;
#pragma unroll
        for (int r = 0; r < RS; ++r) {
          C o = v[q * RS + r];
          if constexpr (DIR > 0) o = cscale(o, scale);
          if constexpr (IO::kStore) io.store(i + r * P, c, o);
          else st_stream(out + int64_t(i + r * P) * op + c, o);
        }
      }
    }
  } else if constexpr (LAST) {
    if constexpr (READ_SH) __syncthreads();
    if (active) {
      // s^r = s^(r mod 8) (s^8)^(r / 8): eight low powers and RS / 8 high
      // ones from product trees, so a large last radix keeps few powers live
      constexpr int NL = RS < 8 ? RS : 8, NH = (RS + 7) / 8;
      C lo[NL], hi[NH];
      lo[0] = C{1, 0};
      if constexpr (NL > 1) lo[1] = tw_s;
#pragma unroll
      for (int r = 2; r < NL; ++r) lo[r] = cmul(lo[r / 2], lo[r - r / 2]);
      hi[0] = C{1, 0};
      if constexpr (NH > 1) hi[1] = cmul(lo[4], lo[4]);
#pragma unroll
      for (int h = 2; h < NH; ++h) hi[h] = cmul(hi[h / 2], hi[h - h / 2]);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int i = t + q * T;
        if (GUARD && i >= NB) break;
#pragma unroll
        for (int h = 0; h < NH; ++h) {
          const C bh = h == 0 ? tw_b[q] : cmul(tw_b[q], hi[h]);
#pragma unroll
          for (int a = 0; a < NL && h * 8 + a < RS; ++a) {
            const int r = h * 8 + a;
            const C w = a == 0 ? bh : cmul(bh, lo[a]);
            sh[c * TL::LP + i + r * P] = cmul(v[q * RS + r], w);
          }
        }
      }
    }
    __syncthreads();
  } else {
    if constexpr (READ_SH) __syncthreads();
    if (active) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int i = t + q * T;
        if (GUARD && i >= NB) break;
        const int k = i % P;
        const int j = (i - k) * RS + k;
#pragma unroll
        for (int r = 0; r < RS; ++r) sh[TL::phys(j + r * P, c)] = v[q * RS + r];
      }
    }
    __syncthreads();
    mix_stage<C, SC, TL, DIR, S + 1, PASS, IO>(v, in, out, sh, t, c, active, tw, scale, bt, n2, ip, op, io);
  }
}

// One transform of an uneven batch on the mixed-radix four-step: n = N1 x N2,
// both column lengths compiled.  Offsets are in elements.
struct MixItem {
  int64_t off;       // the transform in src and dst
  int64_t y;         // its N2 x N1 intermediate in the scratch
  int64_t n;
  int64_t lo, hi;    // W_n split tables in `tab`
  int32_t shift;     // of the split
  int32_t first[2];  // its first CTA in the pass-1 / pass-2 launch of its column length
  int32_t pad_;
};

struct MixColsParams {
  const void* src;
  void* dst;
  int64_t ncols;     // columns of each array (N2 in pass 1, N1 in pass 2)
  int64_t pitch;     // input row pitch (elements)
  int64_t opitch;    // pass 2: output row pitch
  int64_t in_dist;   // elements between arrays of the input
  int64_t out_dist;  // ... of the output
  int64_t tiles;     // column tiles per array (item mode: CTAs of the launch)
  const void* tw;    // W_L^m, m < L
  BigTwiddle bt;     // pass 1: W_N^m
  double scale;      // pass 2: 1/N for the inverse
  // Item mode (uneven batches): CTA i works on transform items[blk[i]];
  // src / dst are the packed batch and the scratch (pass 1) or the scratch
  // and the packed batch (pass 2), `tab` holds the items' W_n tables.
  const MixItem* items = nullptr;
  const int32_t* blk = nullptr;
  const void* tab = nullptr;
};

// One CTA per tile of NC columns of one array (blockIdx = array * tiles + tile);
// MINB resident CTAs per SM asked of the register allocation.
//   MIX_PASS1: array b of x (N1 rows of N2), columns n2 in [col0, col0 + NC):
//     column FFTs of length N1 = L, times W_N^{n2 k1}, stored as rows n2 of
//     the scratch (N2 rows of N1 = L).
//   MIX_PASS2: columns of L rows `pitch` apart, stored in place of their
//     natural order `opitch` apart.
// In item mode every CTA takes its transform, its columns (n / L of them,
// the row pitch) and, for pass 1, its W_n tables from its item.
template <typename C, typename SC, int NC, int DIR, int PASS, int MINB = 1, int TT = 0>
__global__ void __launch_bounds__(MixTile<SC, NC, TT>::TPB, MINB) k_mix_cols(MixColsParams p) {
  using TL = MixTile<SC, NC, TT>;
  using Re = typename RealOf<C>::type;
  constexpr int L = SC::L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  const C* src = static_cast<const C*>(p.src);
  C* dst = static_cast<C*>(p.dst);
  int64_t col0, ncols = p.ncols, pitch = p.pitch, opitch = p.opitch, ioff, ooff;
  BigTwiddle bt = p.bt;
  Re scale = Re(p.scale);
  if (p.items) {
    const MixItem m = p.items[p.blk[blockIdx.x]];
    ncols = m.n / L;
    pitch = opitch = ncols;
    col0 = int64_t(int(blockIdx.x) - m.first[PASS - 1]) * NC;
    ioff = PASS == MIX_PASS1 ? m.off : m.y;
    ooff = PASS == MIX_PASS1 ? m.y : m.off;
    const C* tab = static_cast<const C*>(p.tab);
    bt = BigTwiddle{tab + m.lo, tab + m.hi, m.shift};
    scale = Re(1.0 / double(m.n));
  } else {
    const int64_t b = blockIdx.x / p.tiles;
    col0 = (blockIdx.x % p.tiles) * NC;
    ioff = b * p.in_dist;
    ooff = b * p.out_dist;
  }
  const int c = threadIdx.x % NC, t = threadIdx.x / NC;
  const bool active = col0 + c < ncols;
  const C* in = src + ioff + col0;
  const C* tw = static_cast<const C*>(p.tw);
  C v[TL::vmax()];
  if constexpr (PASS == MIX_PASS1) {
    mix_stage<C, SC, TL, DIR, 0, MIX_PASS1>(v, in, nullptr, sh, t, c, active, tw, Re(1), bt, col0 + c, pitch, 0);
    C* y = dst + ooff + col0 * L;
    const int nv = int(ncols - col0 < NC ? ncols - col0 : NC);
    for (int e = threadIdx.x; e < L * nv; e += TL::TPB) {
      const int cc = e / L, row = e - cc * L;
      __stcg(y + e, sh[cc * TL::LP + row]);
    }
  } else {
    C* out = dst + ooff + col0;
    mix_stage<C, SC, TL, DIR, 0, MIX_PASS2>(v, in, out, sh, t, c, active, tw, scale, bt, 0, pitch, opitch);
  }
}

}  // namespace gfft

namespace gfft {

// Rows mode: NC whole contiguous transforms of length L per CTA, thread t of
// transform c at tid = c * T + t (consecutive threads walk one transform, so
// every load and store is coalesced); transform c's elements contiguous in
// shared memory, LP apart (odd).  The first stage writes its outputs R0 (its
// radix) apart across consecutive threads; an even R0 would put a half-warp
// in a few banks, so rows then get one element of padding every R0 rows.
template <typename SC, int NC, int TT = 0>
struct MixTileRows {
  static constexpr int L = SC::L;
  static constexpr int T = TT > 0 ? TT : L / SC::rmax();
  static constexpr int TPB = T * NC;
  static_assert(TPB <= 1024, "tile needs more than 1024 threads");
  static constexpr int R0 = SC::radix(0);
  static constexpr bool PAD = R0 % 2 == 0;
  static constexpr int LP = (PAD ? L + (L - 1) / R0 + 1 : L) | 1;
  static constexpr int ELEMS = NC * LP;
  __host__ __device__ static constexpr int q_at(int s) { return (L / SC::radix(s) + T - 1) / T; }
  __host__ __device__ static constexpr int vmax() {
    int m = 1;
    for (int s = 0; s < SC::NS; ++s) m = q_at(s) * SC::radix(s) > m ? q_at(s) * SC::radix(s) : m;
    return m;
  }
  __device__ static __forceinline__ int phys(int row, int c) {
    if constexpr (PAD) return c * LP + row + row / R0;
    else return c * LP + row;
  }
};

struct MixRowsParams {
  const void* src;
  void* dst;
  int64_t count, idist, odist;
  const void* tw;  // W_L^m, m < L
  double scale;    // 1/L for the inverse
};

template <typename C>
struct MixRowsIO {
  static constexpr bool kLoad = true, kStore = true;
  const C* x;
  C* y;
  int64_t idist, odist;
  __device__ __forceinline__ C load(int row, int c) const { return ld_stream(x + c * idist + row); }
  __device__ __forceinline__ void store(int row, int c, C v) const { st_stream(y + c * odist + row, v); }
};

// One CTA per NC consecutive transforms (the last CTA masks the missing ones).
template <typename C, typename SC, int NC, int DIR, int MINB = 1, int TT = 0>
__global__ void __launch_bounds__(MixTileRows<SC, NC, TT>::TPB, MINB) k_mix_rows(MixRowsParams p) {
  using TL = MixTileRows<SC, NC, TT>;
  using Re = typename RealOf<C>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  const int64_t b0 = int64_t(blockIdx.x) * NC;
  const int c = threadIdx.x / TL::T, t = threadIdx.x % TL::T;
  const bool active = b0 + c < p.count;
  const MixRowsIO<C> io{static_cast<const C*>(p.src) + b0 * p.idist, static_cast<C*>(p.dst) + b0 * p.odist, p.idist,
                        p.odist};
  C v[TL::vmax()];
  mix_stage<C, SC, TL, DIR, 0, MIX_PASS2, MixRowsIO<C>>(v, nullptr, nullptr, sh, t, c, active,
                                                        static_cast<const C*>(p.tw), Re(p.scale), BigTwiddle{}, 0,
                                                        0, 0, io);
}

}  // namespace gfft
