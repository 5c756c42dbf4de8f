// TMA-staged column passes of the three-pass schedule (k_tp3t), with the
// same index maps and the same intermediate layout as k_tp3, so a pass of
// either form can follow a pass of the other.  The pass body is written for
// any column length (copies of up to 256 rows per box); a two-pass form
// built on it lost to the plain two-pass kernels at every length.
//
// Each pass is a persistent kernel: CTA b takes tiles b, b + grid, ...  A
// tile (L rows of NC adjacent columns) arrives in shared memory by TMA tile
// copies (boxes of at most 256 rows) into one of NST stage buffers; one
// thread keeps up to NST - 1 tiles in flight ahead of the tile being
// transformed, so the copy engine streams the next tiles while the threads
// run the Stockham stages in place on the current one (rows of NC
// elements, the layout the copy writes).  Three kinds of pass:
//   CT_TWID_T  (pass 1): column FFTs of x, times the
//              big twiddle W_N^{m k1}, written transposed into boxes of
//              128-byte rows in the copy engine's 128-byte swizzle
//              (bank-conflict free for the threads' writes) and stored by
//              L / RE TMA tile stores as whole columns, Y[m][k1];
//   CT_TWID_IN (three-pass pass 2): column FFTs of the intermediate times
//              W_M^{m2 k'1}, back in place by one TMA tile store;
//   CT_OUT     (last pass): column FFTs, scaled, to the output in natural
//              order by TMA tile stores.
// A stage buffer is refilled only after the store that read it has finished
// reading (bulk-group wait).  Waits on the copies are bounded: on expiry the
// kernel sets the plan's status word, waits (bounded) for its own copies in
// flight and returns.
#pragma once
#include "gfft_threepass.cuh"
#include "gfft_tma.cuh"

namespace gfft {

enum { CT_TWID_T = 1, CT_TWID_IN = 2, CT_OUT = 3 };

// Tile of a pass: NC = TE / L columns (at most 64), EPT = EMAX with at
// least 8 threads per column.
template <typename C, int L, int TE, int EMAX, int NST, int KIND>
struct ColT {
  static constexpr int ES = sizeof(C);
  static constexpr int NC0 = TE / L;
  static constexpr int NC = NC0 > 64 ? 64 : NC0;
  static constexpr int EPT = (L / EMAX >= 8) ? EMAX : (L / 8 >= 2 ? L / 8 : 2);
  using S = ColShape<L, EPT, NC, ES, true>;
  static constexpr int TPB = S::TPB;
  static constexpr int TILE_BYTES = L * NC * ES;
  static constexpr int BR = L < 256 ? L : 256;  // rows per copy box
  static constexpr int NBOX = L / BR;
  static constexpr int RE = 128 / ES;  // elements per 128-byte row of a swizzled box
  static_assert(KIND != CT_TWID_T || (L % RE == 0 && NC * 128 % 1024 == 0),
                "swizzled boxes: whole 128-byte rows, 1 KB per box");
  static_assert(KIND != CT_TWID_IN || L <= 256, "the in-place pass copies one box");
  // buffers on 1024-byte boundaries (the swizzle pattern repeats every 1 KB)
  static constexpr int BUF_BYTES = (TILE_BYTES + 1023) / 1024 * 1024;
  static constexpr int SMEM = NST * BUF_BYTES + 1024;  // + alignment slack
  static constexpr int MINB = (200 * 1024) / SMEM < 1 ? 1 : ((200 * 1024) / SMEM > 4 ? 4 : (200 * 1024) / SMEM);
  static constexpr int W = ES / 4;  // FP32 words per element (tensor-map x unit)
};

struct ColTArgs {
  int64_t tiles;    // tiles of this launch
  int64_t tpt;      // tiles per transform
  int groups;       // column groups per row block (CT_TWID_IN, CT_OUT)
  const void* tw;   // W_L table of the pass
  BigTwiddle bt;    // CT_TWID_T: W_N; CT_TWID_IN: W_M
  double scale;     // CT_OUT
  unsigned* status;
  unsigned spin_limit;
};

// Tensor maps (element units; x in FP32 words in the kernel):
//   CT_TWID_T:  tin 3D {row length, L, transforms}, box {NC, BR, 1};
//               tout 3D {L, row length, transforms} (rows of Y), box {RE, NC, 1}, 128-byte swizzle;
//   CT_TWID_IN: tin 4D {N1, M2, M1, transforms}, box {NC, 1, L, 1} (also the store);
//   CT_OUT:     tin 3D {N1, rows, transforms}, box {NC, BR, 1}, tile rows from rowc * L;
//               tout 4D {N1, row blocks, L, transforms}, box {NC, 1, BR, 1}.
template <typename C, int L, int TE, int EMAX, int NST, int DIR, int KIND>
__device__ __forceinline__ void colt_body(const CUtensorMap* tin, const CUtensorMap* tout, const ColTArgs& a) {
  using K = ColT<C, L, TE, EMAX, NST, KIND>;
  using Re = typename RealOf<C>::type;
  constexpr int NC = K::NC, EPT = K::EPT, W = K::W, BR = K::BR;
  constexpr int BUFE = K::BUF_BYTES / K::ES;
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[NST];
  __shared__ int s_fail;
  __shared__ C s_tw[L];  // W_L, read by every tile's stages
  C* bufs = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x;
  const int c = tid % NC, t = tid / NC;
  const int64_t nloc = a.tiles > blockIdx.x ? (a.tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

  // tile -> (transform, row block, first column)
  auto decode = [&](int64_t tile, int& bl, int& rowc, int& col0) {
    bl = int(tile / a.tpt);
    const int r = int(tile % a.tpt);
    if constexpr (KIND == CT_TWID_T) {
      rowc = 0;
      col0 = r * NC;
    } else {
      rowc = r / a.groups;
      col0 = (r % a.groups) * NC;
    }
  };
  auto issue = [&](int64_t j) {
    int bl, rowc, col0;
    decode(blockIdx.x + j * gridDim.x, bl, rowc, col0);
    const int s = int(j % NST);
    C* buf = bufs + s * BUFE;
    mbar_expect_tx(&bar[s], K::TILE_BYTES);
    if constexpr (KIND == CT_TWID_IN) {
      tma_load_4d(buf, tin, &bar[s], col0 * W, rowc, 0, bl);
    } else {
#pragma unroll
      for (int i = 0; i < K::NBOX; ++i)
        tma_load_3d(buf + i * BR * NC, tin, &bar[s], col0 * W, rowc * L + i * BR, bl);
    }
  };

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
    fence_async_smem();
    s_fail = 0;
  }
  for (int i = tid; i < L; i += K::TPB) s_tw[i] = static_cast<const C*>(a.tw)[i];
  __syncthreads();
  int64_t issued = 0;  // meaningful in thread 0
  if (tid == 0)
    for (; issued < NST - 1 && issued < nloc; ++issued) issue(issued);

  C v[EPT];
  int64_t j = 0;
  // Refill of the buffer tile j - 1 used, with tile j + NST - 1.  With three
  // or more stages it comes after tile j's butterflies, when the store that
  // read that buffer (committed one tile earlier) has long finished; with
  // two it must come first, or no copy would overlap the butterflies.
  constexpr bool LATE = NST >= 3;
  auto refill = [&]() {
    if (tid == 0 && issued < nloc) {
      bulk_wait_read();
      fence_async_smem();
      issue(issued);
      ++issued;
    }
  };
  for (; j < nloc; ++j) {
    const int s = int(j % NST);
    C* sh = bufs + s * BUFE;
    if constexpr (!LATE) refill();
    // one thread waits for the copy; the barrier passes its completion on
    // to the others (the copy's writes are ordered before the phase flip
    // that thread 0 observes, and the barrier orders the rest after it)
    if (tid == 0 && !mbar_wait(&bar[s], uint32_t((j / NST) & 1), a.spin_limit)) s_fail = 1;
    __syncthreads();
    if (s_fail) break;
    int bl, rowc, col0;
    decode(blockIdx.x + j * gridDim.x, bl, rowc, col0);
    // every branch ends its butterflies with a fence for the copy engine and
    // a barrier, so the tile is complete in shared memory before its store
    if constexpr (KIND == CT_TWID_T) {
      col_stage<C, L, EPT, NC, DIR, 1, LOAD_SMEM, OUT_SMEM_TWIDDLE_SW, 1, 1, true>(
          v, nullptr, nullptr, sh, t, c, true, s_tw, Re(1), a.bt, int64_t(col0 + c));
      if constexpr (LATE) refill();
      if (tid == 0) {  // Y[m][k1]: box i holds rows k1 = i*RE.. of columns m = col0..
        for (int i = 0; i < L / K::RE; ++i) tma_store_3d(tout, sh + i * NC * K::RE, i * K::RE * W, col0, bl);
        bulk_commit();
      }
    } else if constexpr (KIND == CT_TWID_IN) {
      col_stage<C, L, EPT, NC, DIR, 1, LOAD_SMEM, OUT_SMEM_TWIDDLE, 1, 1, true>(
          v, nullptr, nullptr, sh, t, c, true, s_tw, Re(1), a.bt, int64_t(rowc));
      if constexpr (LATE) refill();
      if (tid == 0) {
        tma_store_4d(tin, sh, col0 * W, rowc, 0, bl);  // in place
        bulk_commit();
      }
    } else {
      col_stage<C, L, EPT, NC, DIR, 1, LOAD_SMEM, OUT_SMEM, 1, 1, true>(
          v, nullptr, nullptr, sh, t, c, true, s_tw, Re(a.scale), a.bt, 0);
      fence_async_smem();
      __syncthreads();
      if constexpr (LATE) refill();
      if (tid == 0) {
#pragma unroll
        for (int i = 0; i < K::NBOX; ++i) tma_store_4d(tout, sh + i * BR * NC, col0 * W, rowc, i * BR, bl);
        bulk_commit();
      }
    }
    // the early refill of the next iteration reuses this buffer
    if constexpr (!LATE) __syncthreads();
  }
  if (tid == 0) {
    if (j < nloc) {
      // a wait expired: flag it, then let the copies still in flight land
      // (bounded) before the CTA's shared memory goes away
      atomicExch(a.status, 1u);
      for (int64_t k = j; k < issued; ++k)
        mbar_wait(&bar[int(k % NST)], uint32_t((k / NST) & 1), a.spin_limit);
    }
    bulk_wait_all();
  }
}

// Pass PASS (1..3) of the three-pass schedule N = N1 x M1 x M2.
template <int N1, int M1, int M2, int PASS>
struct Tp3Pass {
  static constexpr int L = PASS == 1 ? N1 : PASS == 2 ? M1 : M2;
  static constexpr int KIND = PASS == 1 ? CT_TWID_T : PASS == 2 ? CT_TWID_IN : CT_OUT;
};

template <typename C, int N1, int M1, int M2, int TE, int EMAX, int NST, int DIR, int PASS>
__global__ void __launch_bounds__(
    ColT<C, Tp3Pass<N1, M1, M2, PASS>::L, TE, EMAX, NST, Tp3Pass<N1, M1, M2, PASS>::KIND>::TPB,
    ColT<C, Tp3Pass<N1, M1, M2, PASS>::L, TE, EMAX, NST, Tp3Pass<N1, M1, M2, PASS>::KIND>::MINB)
k_tp3t(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout, ColTArgs a) {
  using P = Tp3Pass<N1, M1, M2, PASS>;
  colt_body<C, P::L, TE, EMAX, NST, DIR, P::KIND>(&tin, &tout, a);
}

}  // namespace gfft
