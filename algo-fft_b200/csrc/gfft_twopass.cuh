// Two-pass (four-step) transform for large N = N1 * N2 (K2), as one
// persistent kernel that keeps the intermediate in L2.
//
// Index maps: n = N2*n1 + n2 (input), k = k1 + N1*k2 (output).
//   pass 1: for each column n2, FFT_N1 over n1 of x[N2*n1 + n2], multiply by
//           W_N^{n2*k1}, store transposed: Y[n2][k1] (rows of N1, scratch).
//   pass 2: for each k1, FFT_N2 over n2 of Y[n2][k1] (a column of Y), store
//           X[k1 + N1*k2] (a column of the output viewed as N2 x N1).
// A tile is NC adjacent columns of one transform, so every global access is
// a run of NC contiguous elements (pass 1's store is a run of N1).
//
// Scheduling: the batch is cut into groups of G transforms; each group's
// intermediate lives in one of S scratch slots small enough to stay in the
// 126 MB L2, so HBM sees one read of the input and one write of the output.
// Persistent CTAs take tiles from a global counter in a fixed order
//   P1(0..S-2), then P2(k), P1(k+S-1) for k = 0, 1, ...
// A pass-2 tile of group g waits (bounded) until all pass-1 tiles of g are
// done; a pass-1 tile of group g >= S waits until pass 2 of g-S has released
// its slot.  Every wait targets tiles handed out earlier, which are held by
// running CTAs whose own waits target still earlier tiles, so the chain
// always ends: no deadlock, whatever the residency.  Waits are bounded
// anyway: on expiry the kernel records an error and returns.
//
// Replaces the reference's six-step / eight-step kernels
// (internal/kernels/sixstep.go:29-91, eightstep.go:27-154) and the packed
// Stockham for large power-of-two N (internal/transform/stockham_packed.go:86).
#pragma once
#include "gfft_pow2.cuh"
#include "gfft_sched.cuh"
#include "gfft_tma.cuh"

namespace gfft {

// Tile of NC columns of length L, EPT elements per thread.
// DENSE tiles keep rows of exactly NC elements, the layout a TMA tile copy
// writes.  With rows of 128 bytes or more every warp access of a stage
// (whole rows) is bank-conflict free; with 64-byte rows the first stage's
// scattered writes can take twice the minimum wavefronts.
template <int L, int EPT, int NC, int ES, bool DENSE = false>
struct ColShape {
  static_assert((NC & (NC - 1)) == 0, "NC must be a power of two");
  static_assert(!DENSE || NC * ES >= 64, "dense tiles need rows of at least 64 bytes");
  static constexpr int T = L / EPT;     // threads per column
  static constexpr int TPB = T * NC;    // threads per tile
  // Rows of NC+1 elements when NC >= 16 (odd pitch: row-wise and column-wise
  // accesses are both bank-conflict free); narrower tiles use an XOR swizzle
  // of the column index by the row, which keeps most of that property.
  static constexpr bool PITCHED = !DENSE && NC >= 16;
  static constexpr int PITCH = PITCHED ? NC + 1 : NC;
  static constexpr int SMEM = L * PITCH * ES;
  __device__ static __forceinline__ int phys(int row, int c) {
    if constexpr (DENSE) return row * NC + c;
    else if constexpr (PITCHED) return row * PITCH + c;
    else return row * NC + (c ^ (row & (NC - 1)));
  }
};

// LOAD_SMEM: the tile is already in shared memory (a TMA copy put it there).
// LOAD_FN: the first stage asks the caller's IO object, io.load(row, c).
enum { LOAD_STREAM = 0, LOAD_L2 = 1, LOAD_SMEM = 2, LOAD_FN = 3 };
// OUT_SMEM: the result, scaled, back into the tile's rows (for a TMA store);
// OUT_SMEM_TWIDDLE_T: times the big twiddle, transposed into rows of L + 1
// elements per column, for a coalesced store of whole columns.
// OUT_SMEM_TWIDDLE_SW: times the big twiddle, transposed into boxes of 128-byte
// rows in the copy engine's 128-byte swizzle (see swz128), for TMA stores of
// whole columns.
// OUT_FN: the last stage hands each (row, column, value) to io.store, the
// value already scaled for the inverse.
enum { OUT_COLUMNS = 0, OUT_SMEM_TWIDDLE = 1, OUT_SMEM = 2, OUT_SMEM_TWIDDLE_T = 3, OUT_SMEM_TWIDDLE_SW = 4, OUT_FN = 5 };

// Default IO of col_stage: no hooks.
struct NoIO {};

// Element (row, c) of a transposed tile held as L / RE boxes of NC rows (one
// per column c) of 128 bytes (RE elements of consecutive rows), in the
// layout of a TMA copy with 128-byte swizzle: the 16-byte chunk j of box row
// c sits at chunk j ^ (c mod 8).  Writes of a warp (whole rows of the
// untransposed tile) then spread over all banks.  The boxes start on
// 1024-byte boundaries.
template <typename C, int NC>
__device__ __forceinline__ int swz128(int row, int c) {
  constexpr int RE = 128 / int(sizeof(C)), EPC = 16 / int(sizeof(C));
  const int k = row % RE;
  return (row / RE) * (NC * RE) + c * RE + (((k / EPC) ^ (c & 7)) * EPC) + (k % EPC);
}

template <int LOADK, typename C>
__device__ __forceinline__ C gload(const C* p) {
  if constexpr (LOADK == LOAD_L2) return __ldcg(p);
  else return ld_stream(p);
}

// Barrier among the threads that run a tile's stages: the whole CTA
// (NSYNC = 0), or the NSYNC threads of named barrier 1 (kernels whose other
// warps copy tiles in and out and never take part in the stages).
template <int NSYNC>
__device__ __forceinline__ void tile_sync() {
  if constexpr (NSYNC == 0) __syncthreads();
  else asm volatile("bar.sync 1, %0;" ::"n"(NSYNC) : "memory");
}

// One Stockham stage of a column tile (see pow2_stage for the algebra).
// Element (row, c) of the tile lives at sh[phys(row, c)]; global row r of
// column c is at in[r*ISTRIDE + c].
// ISTRIDE / OSTRIDE = 0 take the row pitch from `pitch` at run time.
template <typename C, int L, int EPT, int NC, int DIR, int P, int LOADK, int MODE, int64_t ISTRIDE, int64_t OSTRIDE,
          bool DENSE = false, typename IO = NoIO, int NSYNC = 0, bool BTG = false>
__device__ __forceinline__ void col_stage(C* v, const C* in, C* out, C* sh,
                                          int t, int c, bool active, const C* __restrict__ tw,
                                          typename RealOf<C>::type scale, const BigTwiddle& bt, int64_t n2,
                                          int64_t pitch = 0, const IO& io = IO()) {
  const int64_t IS = ISTRIDE > 0 ? ISTRIDE : pitch;
  const int64_t OS = OSTRIDE > 0 ? OSTRIDE : pitch;
  using S = ColShape<L, EPT, NC, sizeof(C), DENSE>;
  using SC = Sched<L, EPT>;
  constexpr int T = S::T;
  constexpr int RS = SC::radix_at(P);
  constexpr int Q = EPT / RS;
  constexpr int STRIDE = L / RS;
  constexpr bool FIRST = (P == 1);
  constexpr bool LAST = (P * RS == L);
  // the stage read shared memory, so it must sync before writing it
  constexpr bool READ_SH = !FIRST || LOADK == LOAD_SMEM;
  constexpr bool BIGTW = LAST && (MODE == OUT_SMEM_TWIDDLE || MODE == OUT_SMEM_TWIDDLE_T || MODE == OUT_SMEM_TWIDDLE_SW);

  // The big twiddles of the last stage are fetched before the stage's own
  // reads and butterflies, so their latency hides behind that work.
  // W_N^{n2*(row0 + r*P)} = b * s^r with b = W_N^{n2*row0} (one lookup per
  // butterfly) and s = W_N^{n2*P} (one per thread); the powers of s come
  // from a product tree, so no per-element table lookup is scattered across
  // the warp.
  [[maybe_unused]] C tw_s{}, tw_b[Q];
  if constexpr (BIGTW) {
    if (active) {
      if constexpr (BTG) {  // tables in shared memory
        tw_s = big_twiddle_any<C, DIR>(bt, n2 * P);
#pragma unroll
        for (int q = 0; q < Q; ++q) tw_b[q] = big_twiddle_any<C, DIR>(bt, n2 * (t + q * T));
      } else {
        tw_s = big_twiddle<C, DIR>(bt, n2 * P);
#pragma unroll
        for (int q = 0; q < Q; ++q) tw_b[q] = big_twiddle<C, DIR>(bt, n2 * (t + q * T));
      }
    }
  }

  if (active) {
    if constexpr (FIRST && LOADK == LOAD_FN) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < RS; ++r) v[q * RS + r] = io.load(t + q * T + r * STRIDE, c);
    } else if constexpr (FIRST && LOADK != LOAD_SMEM) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < RS; ++r)
          v[q * RS + r] = gload<LOADK>(in + int64_t(t + q * T + r * STRIDE) * IS + c);
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < RS; ++r) v[q * RS + r] = sh[S::phys(t + q * T + r * STRIDE, c)];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if constexpr (P > 1) {
        const int k = (t + q * T) & (P - 1);
        // DENSE (TMA-staged) callers keep the W_L table in shared memory
        if constexpr (DENSE) apply_twiddles<RS, DIR>(v + q * RS, tw[k * (L / (P * RS))]);
        else apply_twiddles<RS, DIR>(v + q * RS, __ldg(tw + k * (L / (P * RS))));
      }
      dft<RS, DIR>(v + q * RS);
    }
  }

  if constexpr (LAST && (MODE == OUT_COLUMNS || MODE == OUT_FN)) {
    if (active) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < RS; ++r) {
          C o = v[q * RS + r];
          if constexpr (DIR > 0) o = cscale(o, scale);
          if constexpr (MODE == OUT_FN) io.store(t + q * T + r * P, c, o);
          else st_stream(out + int64_t(t + q * T + r * P) * OS + c, o);
        }
    }
  } else if constexpr (LAST && MODE == OUT_SMEM) {
    if constexpr (READ_SH) tile_sync<NSYNC>();
    if (active) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < RS; ++r) {
          C o = v[q * RS + r];
          if constexpr (DIR > 0) o = cscale(o, scale);
          sh[S::phys(t + q * T + r * P, c)] = o;
        }
    }
  } else if constexpr (LAST) {
    if constexpr (READ_SH) tile_sync<NSYNC>();
    if (active) {
      C pw[RS];
      pw[0] = C{1, 0};
      if constexpr (RS > 1) pw[1] = tw_s;
#pragma unroll
      for (int r = 2; r < RS; ++r) pw[r] = cmul(pw[r / 2], pw[r - r / 2]);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int row0 = t + q * T;
        const C b = tw_b[q];
#pragma unroll
        for (int r = 0; r < RS; ++r) {
          const C w = r == 0 ? b : cmul(b, pw[r]);
          if constexpr (MODE == OUT_SMEM_TWIDDLE_T) sh[c * (L + 1) + row0 + r * P] = cmul(v[q * RS + r], w);
          else if constexpr (MODE == OUT_SMEM_TWIDDLE_SW) sh[swz128<C, NC>(row0 + r * P, c)] = cmul(v[q * RS + r], w);
          else sh[S::phys(row0 + r * P, c)] = cmul(v[q * RS + r], w);
        }
      }
    }
    if constexpr (DENSE) fence_async_smem();  // the tile may leave by a TMA store
    tile_sync<NSYNC>();
  } else {
    if constexpr (READ_SH) tile_sync<NSYNC>();
    if (active) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int i = t + q * T;
        const int k = i & (P - 1);
        const int j = (i - k) * RS + k;
#pragma unroll
        for (int r = 0; r < RS; ++r) sh[S::phys(j + r * P, c)] = v[q * RS + r];
      }
    }
    tile_sync<NSYNC>();
    col_stage<C, L, EPT, NC, DIR, P * RS, LOADK, MODE, ISTRIDE, OSTRIDE, DENSE, IO, NSYNC, BTG>(v, in, out, sh, t, c, active, tw,
                                                                                    scale, bt, n2, pitch, io);
  }
}

struct TwoPassParams {
  const void* src;
  void* dst;
  void* scratch;       // S slots of G*N elements
  int64_t count, idist, odist;
  const void* tw1;     // W_N1^m, m < N1
  const void* tw2;     // W_N2^m, m < N2
  BigTwiddle bt;       // W_N^m
  unsigned* ctr;       // [0] next tile, [1 + g] pass-1 done, [1 + groups + g] pass-2 done
  unsigned* status;    // 0 ok, 1 a bounded wait expired (every CTA stops at its next tile)
  unsigned* report = nullptr;  // optional sticky word also set when a wait expires (the plan's)
  int groups, G, S;
  double scale;        // applied in pass 2 (1/N for the inverse)
  unsigned spin_limit;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Bounded wait of one thread for *p >= target.
__device__ __forceinline__ bool wait_at_least(const unsigned* p, unsigned target, unsigned limit) {
  unsigned it = 0;
  while (ld_acquire(p) < target) {
    if (++it > limit) return false;
    __nanosleep(128);
  }
  return true;
}

template <typename C, int N1, int EPT1, int NC1, int N2, int EPT2, int NC2, int DIR>
struct TwoPass {
  using S1 = ColShape<N1, EPT1, NC1, sizeof(C)>;
  using S2 = ColShape<N2, EPT2, NC2, sizeof(C)>;
  static constexpr int64_t N = int64_t(N1) * N2;
  static constexpr int TILES1 = N2 / NC1;  // pass-1 tiles per transform
  static constexpr int TILES2 = N1 / NC2;  // pass-2 tiles per transform
  static constexpr int TPB = S1::TPB > S2::TPB ? S1::TPB : S2::TPB;
  static constexpr int SMEM = S1::SMEM > S2::SMEM ? S1::SMEM : S2::SMEM;
  static constexpr int EPT = EPT1 > EPT2 ? EPT1 : EPT2;
  // resident CTAs per SM the register allocation must allow: as many as
  // the shared memory admits, but never so many that a thread gets fewer
  // registers than its elements need plus 32 (at least 64; below that the
  // stages spill)
  static constexpr int MB0 = (200 * 1024) / (SMEM > 0 ? SMEM : 1);
  static constexpr int REGS = EPT * int(sizeof(C)) / 4 + 32 > 64 ? EPT * int(sizeof(C)) / 4 + 32 : 64;
  static constexpr int MB_REG = 65536 / (TPB * REGS) < 1 ? 1 : 65536 / (TPB * REGS);
  static constexpr int MB1 = MB0 < MB_REG ? MB0 : MB_REG;
  static constexpr int MIN_BLOCKS = MB1 < 1 ? 1 : (MB1 > 4 ? 4 : MB1);
};

// Tile order decode (see the header comment).
__device__ __forceinline__ void decode_tile(int64_t w, int groups, int S, int64_t T1, int64_t T2, int& pass,
                                            int& g, int64_t& tile) {
  const int64_t init = groups < S - 1 ? groups : S - 1;
  if (w < init * T1) {
    pass = 1;
    g = int(w / T1);
    tile = w % T1;
    return;
  }
  w -= init * T1;
  const int64_t k1 = groups - (S - 1) > 0 ? groups - (S - 1) : 0;  // pairs that carry a pass-1 unit
  if (w < k1 * (T1 + T2)) {
    const int64_t k = w / (T1 + T2), rem = w % (T1 + T2);
    if (rem < T2) {
      pass = 2;
      g = int(k);
      tile = rem;
    } else {
      pass = 1;
      g = int(k + S - 1);
      tile = rem - T2;
    }
    return;
  }
  w -= k1 * (T1 + T2);
  pass = 2;
  g = int(k1 + w / T2);
  tile = w % T2;
}

template <typename C, int N1, int EPT1, int NC1, int N2, int EPT2, int NC2, int DIR>
__global__ void __launch_bounds__(TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>::TPB,
                                  TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>::MIN_BLOCKS)
k_twopass(TwoPassParams p) {
  using TP = TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>;
  using S1 = typename TP::S1;
  using S2 = typename TP::S2;
  using Re = typename RealOf<C>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  __shared__ int64_t s_w;
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  const int64_t T1 = int64_t(TP::TILES1) * p.G, T2 = int64_t(TP::TILES2) * p.G;
  const int64_t total = int64_t(p.groups) * (T1 + T2);
  const C* src = static_cast<const C*>(p.src);
  C* dst = static_cast<C*>(p.dst);
  C* scratch = static_cast<C*>(p.scratch);
  unsigned* done1 = p.ctr + 1;
  unsigned* done2 = p.ctr + 1 + p.groups;
  C v[TP::EPT];

  for (;;) {
    __syncthreads();
    if (tid == 0) {
      s_w = (ld_acquire(p.status) != 0) ? total : int64_t(atomicAdd(p.ctr, 1u));
    }
    __syncthreads();
    const int64_t w = s_w;
    if (w >= total) break;
    int pass, g;
    int64_t tile;
    decode_tile(w, p.groups, p.S, T1, T2, pass, g, tile);
    if (tid == 0) {
      bool ok = true;
      if (pass == 2) ok = wait_at_least(done1 + g, unsigned(T1), p.spin_limit);
      else if (g >= p.S) ok = wait_at_least(done2 + (g - p.S), unsigned(T2), p.spin_limit);
      if (!ok) {
        atomicExch(p.status, 1u);
        if (p.report) atomicOr(p.report, 1u);
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) break;
    const int slot = g % p.S;
    if (pass == 1) {
      const int64_t b = int64_t(g) * p.G + tile / TP::TILES1;  // transform index
      const int col0 = int(tile % TP::TILES1) * NC1;
      const bool valid = b < p.count;
      const bool active = valid && tid < S1::TPB;
      const int c = tid % NC1, t = tid / NC1;
      const C* in = src + (valid ? b * p.idist : 0) + col0;
      C* y = scratch + (int64_t(slot) * p.G + (b - int64_t(g) * p.G)) * TP::N;
      col_stage<C, N1, EPT1, NC1, DIR, 1, LOAD_STREAM, OUT_SMEM_TWIDDLE, N2, 0>(
          v, in, nullptr, sh, t, c, active, static_cast<const C*>(p.tw1), Re(1), p.bt, int64_t(col0 + c));
      if (valid) {
        // transposed store: Y[col0 + cc][row], rows of N1 contiguous
        for (int e = tid; e < N1 * NC1; e += TP::TPB) {
          const int cc = e / N1, row = e % N1;
          __stcg(y + int64_t(col0 + cc) * N1 + row, sh[S1::phys(row, cc)]);
        }
      }
    } else {
      const int64_t b = int64_t(g) * p.G + tile / TP::TILES2;
      const int col0 = int(tile % TP::TILES2) * NC2;
      const bool valid = b < p.count;
      const bool active = valid && tid < S2::TPB;
      const int c = tid % NC2, t = tid / NC2;
      const C* y = scratch + (int64_t(slot) * p.G + (b - int64_t(g) * p.G)) * TP::N + col0;
      C* out = dst + (valid ? b * p.odist : 0) + col0;
      col_stage<C, N2, EPT2, NC2, DIR, 1, LOAD_L2, OUT_COLUMNS, N1, N1>(v, y, out, sh, t, c, active,
                                                                        static_cast<const C*>(p.tw2), Re(p.scale),
                                                                        p.bt, 0);
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(pass == 1 ? done1 + g : done2 + g, 1u);
    }
  }
}

// Split form (the default schedule): one plain launch per pass over a chunk
// of transforms starting at b0, one tile per CTA, no cross-CTA waits.  Pass
// 1 writes the chunk's intermediate to scratch (the chunk's size); pass 2
// reads it back; the two launches are stream-ordered.  Measured on B200 it
// beats the persistent form above at every size, although its intermediate
// makes a round trip through HBM: the persistent form loses more to the
// three serialized L2 round trips per tile (work counter, dependency
// acquire, completion fence) than the L2-resident intermediate saves, and
// chunks small enough for L2 lose it again to launch gaps and tails.  The
// persistent form stays for callers that cannot allocate (a bounded static
// scratch).
template <typename C, int N1, int EPT1, int NC1, int N2, int EPT2, int NC2, int DIR, int PASS>
__global__ void __launch_bounds__(TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>::TPB,
                                  TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>::MIN_BLOCKS)
k_tp_split(TwoPassParams p, int64_t b0) {
  using TP = TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, DIR>;
  using S1 = typename TP::S1;
  using S2 = typename TP::S2;
  using Re = typename RealOf<C>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  const C* src = static_cast<const C*>(p.src);
  C* dst = static_cast<C*>(p.dst);
  C* scratch = static_cast<C*>(p.scratch);
  C v[TP::EPT];
  if constexpr (PASS == 1) {
    const int64_t bl = blockIdx.x / TP::TILES1;  // transform within the chunk
    const int col0 = int(blockIdx.x % TP::TILES1) * NC1;
    const bool active = tid < S1::TPB;
    const int c = tid % NC1, t = tid / NC1;
    const C* in = src + (b0 + bl) * p.idist + col0;
    C* y = scratch + bl * TP::N;
    col_stage<C, N1, EPT1, NC1, DIR, 1, LOAD_STREAM, OUT_SMEM_TWIDDLE, N2, 0>(
        v, in, nullptr, sh, t, c, active, static_cast<const C*>(p.tw1), Re(1), p.bt, int64_t(col0 + c));
    for (int e = tid; e < N1 * NC1; e += TP::TPB) {
      const int cc = e / N1, row = e % N1;
      __stcg(y + int64_t(col0 + cc) * N1 + row, sh[S1::phys(row, cc)]);
    }
  } else {
    const int64_t bl = blockIdx.x / TP::TILES2;
    const int col0 = int(blockIdx.x % TP::TILES2) * NC2;
    const bool active = tid < S2::TPB;
    const int c = tid % NC2, t = tid / NC2;
    const C* y = scratch + bl * TP::N + col0;
    C* out = dst + (b0 + bl) * p.odist + col0;
    col_stage<C, N2, EPT2, NC2, DIR, 1, LOAD_L2, OUT_COLUMNS, N1, N1>(v, y, out, sh, t, c, active,
                                                                      static_cast<const C*>(p.tw2), Re(p.scale),
                                                                      p.bt, 0);
  }
}

}  // namespace gfft
