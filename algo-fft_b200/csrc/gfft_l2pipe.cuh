// L2-pipelined two-pass (four-step) transform, N = N1 x N2 (k_l2p).
//
// The same index maps as the two-pass schedule (gfft_twopass.cuh):
//   pass A: for each column n2, FFT_N1 over n1 of x[N2 n1 + n2], times
//           W_N^{n2 k1}, stored transposed as Y[n2][k1] (rows of N1);
//   pass B: for each k1, FFT_N2 over n2 of Y[n2][k1], stored as
//           X[k1 + N1 k2].
// What differs is where Y lives.  The batch is cut into groups of G
// transforms (a few MB each), and each group's Y goes into one of S scratch
// slots that stay in the 126 MB L2: HBM sees one read of x and one write of
// X, and Y makes its round trip through L2 only.  One persistent launch runs
// both passes over all groups, taking work items from a global counter in
// the order
//   A(0) .. A(S-2), then B(g), A(g+S-1) for g = 0, 1, ...
// so pass B of a group runs while pass A of the group S-1 later fills
// another slot.  A pass-B tile of group g waits until every pass-A tile of g
// is complete; a pass-A tile of group g >= S waits until pass B of group g-S
// has read its slot.  Both waits point at work items handed out earlier.
//
// Roles inside a CTA (warp specialised, so no CTA ever blocks on another
// CTA while it still holds unfinished work):
//   warp 0, lane 0 -- producer: takes the next work item, waits (bounded)
//     for its dependency, then copies the tile into a free stage buffer
//     with TMA tile loads (completion on full[s]);
//   warp 1, lane 0 -- storer: once the compute warps have a tile ready
//     (ready[s]), stores it with TMA tile stores, frees the buffer when the
//     stores have read it (empty[s]), and publishes pass-A completion after
//     the stores are complete;
//   warps 2.. -- compute: the Stockham stages of the tile in place in its
//     stage buffer (named barrier 1 among themselves).
// Work items are processed by each CTA in the order it took them, and every
// dependency points at a smaller item, so the smallest unfinished item can
// always proceed: no deadlock whatever the residency.  All waits are
// bounded anyway; on expiry the kernel sets the plan's status word and
// every role returns.
//
// Tiles: pass A takes NC1 adjacent columns n2 of one transform (N1 rows);
// pass B takes NC2 adjacent columns k1 of one slot (N2 rows).  Every copy is
// a local tile copy (no cluster multicast).
//
// Replaces the reference's six-step / eight-step kernels and the packed
// Stockham for large power-of-two N (internal/kernels/sixstep.go:29-91,
// eightstep.go:27-154, internal/transform/stockham_packed.go:86).
#pragma once
#include "gfft_cols_tma.cuh"
#include "gfft_twopass.cuh"

namespace gfft {

// One try_wait (the hardware suspends the thread for a short while).
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(sm_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of this parity that gives up early once
// *abort (a shared flag) is set.
__device__ __forceinline__ bool mbar_wait_abort(uint64_t* bar, uint32_t parity, unsigned limit,
                                                const volatile int* abort) {
  for (unsigned it = 0; it < limit; ++it) {
    if (mbar_test(bar, parity)) return true;
    if (*abort) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm_addr(bar)) : "memory");
}

// Orders this thread's earlier generic-proxy accesses of global memory with
// its later async-proxy (TMA) accesses, and the reverse.
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits until all but the N most recent bulk store groups are complete.
template <int N>
__device__ __forceinline__ void bulk_wait_n() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

// Bounded wait of one thread for *p >= target, stopping early once *abort
// (a shared flag) is set.
__device__ __forceinline__ bool wait_counter(const unsigned* p, unsigned target, unsigned limit,
                                             const volatile int* abort) {
  for (unsigned it = 0;; ++it) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    if (v >= target) return true;
    if (it > limit || *abort) return false;
    __nanosleep(64);
  }
}

struct L2pParams {
  const void* src;
  void* dst;
  void* scratch;      // S slots of G transforms
  unsigned* ctr;      // [0] next work item, [1 + g] pass-A tiles done, [1 + groups + g] pass-B tiles done
  unsigned* status;   // set to 1 when a bounded wait expires
  int64_t count, idist, odist;
  const void* tw1;    // W_N1^m, m < N1
  const void* tw2;    // W_N2^m, m < N2
  BigTwiddle bt;      // W_N^m
  double scale;       // pass B (1/N for the inverse)
  int G, S, groups;
  unsigned spin_limit;
};

template <typename C, int N1, int N2, int NC1, int NC2, int EPT1, int EPT2, int NST>
struct L2p {
  static constexpr int ES = int(sizeof(C));
  static constexpr int W = ES / 4;     // FP32 words per element (tensor-map x unit)
  static constexpr int RE = 128 / ES;  // elements per 128-byte row of a swizzled box
  using A = ColShape<N1, EPT1, NC1, ES, true>;
  using B = ColShape<N2, EPT2, NC2, ES, true>;
  static constexpr int TPBC = A::TPB > B::TPB ? A::TPB : B::TPB;  // compute threads
  static constexpr int TPB = TPBC + 64;                             // + producer and storer warps
  static constexpr int64_t N = int64_t(N1) * N2;
  static constexpr int TA = N2 / NC1;  // pass-A tiles per transform
  static constexpr int TB = N1 / NC2;  // pass-B tiles per transform
  static constexpr int BYTES_A = N1 * NC1 * ES, BYTES_B = N2 * NC2 * ES;
  static constexpr int BUF = ((BYTES_A > BYTES_B ? BYTES_A : BYTES_B) + 1023) / 1024 * 1024;
  static constexpr int BR1 = N1 < 256 ? N1 : 256, NBOX1 = N1 / BR1;
  static constexpr int BR2 = N2 < 256 ? N2 : 256, NBOX2 = N2 / BR2;
  static constexpr int SMEM = NST * BUF + 1024;  // + alignment slack (swizzled boxes on 1 KB)
  // the split table of W_N (m = a * LO + b: hi[a] * lo[b]), in shared memory
  static constexpr int LGN = []() { int l = 0; while ((int64_t(1) << l) < int64_t(N1) * N2) ++l; return l; }();
  static constexpr int SHIFT = (LGN + 1) / 2;
  static constexpr int LO = 1 << SHIFT, HI = int((int64_t(N1) * N2) >> SHIFT);
  static constexpr int TABLES = (N1 + N2 + LO + HI) * ES;  // static shared memory: W_N1, W_N2, split W_N
  // resident CTAs per SM the register allocation must allow (as many as
  // the shared memory admits, at most 2)
  static constexpr int MINB0 = (220 * 1024) / (SMEM + TABLES + 256);
  static constexpr int MINB = MINB0 < 1 ? 1 : (MINB0 > 2 ? 2 : MINB0);
  static_assert(TPBC % 32 == 0 && TPB <= 1024, "compute threads in whole warps, at most 1024 in all");
  static_assert(NC1 * 128 % 1024 == 0 && N1 % RE == 0, "pass A stores whole 1 KB swizzled boxes");
  static_assert(NC2 * ES % 16 == 0 && NC1 * ES % 16 == 0, "tile columns start on 16-byte boundaries");
  static_assert(SMEM + TABLES <= 227 * 1024, "shared memory per CTA");
};

template <typename C, int N1, int N2, int NC1, int NC2, int EPT1, int EPT2, int NST, int DIR>
__global__ void __launch_bounds__(L2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST>::TPB,
                                  L2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST>::MINB)
k_l2p(const __grid_constant__ CUtensorMap tx, const __grid_constant__ CUtensorMap tys,
      const __grid_constant__ CUtensorMap tyl, const __grid_constant__ CUtensorMap tz, L2pParams p) {
  using K = L2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST>;
  using Re = typename RealOf<C>::type;
  constexpr int BUFE = K::BUF / K::ES, W = K::W;
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[NST], ready[NST], empty[NST];
  __shared__ int64_t s_item[NST];  // work item of the tile in stage s; < 0: stop
  __shared__ volatile int s_abort;
  __shared__ C s_tw1[N1], s_tw2[N2], s_btlo[K::LO], s_bthi[K::HI];
  C* bufs = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int CWARPS = K::TPBC / 32;
  const int64_t TAg = int64_t(K::TA) * p.G, TBg = int64_t(K::TB) * p.G;
  const int64_t total = int64_t(p.groups) * (TAg + TBg);
  unsigned* doneA = p.ctr + 1;
  unsigned* doneB = p.ctr + 1 + p.groups;

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&ready[s], CWARPS);
      mbar_init(&empty[s], 1);
    }
    s_abort = 0;
    fence_mbar_init();
  }
  for (int i = tid; i < N1; i += K::TPB) s_tw1[i] = static_cast<const C*>(p.tw1)[i];
  for (int i = tid; i < N2; i += K::TPB) s_tw2[i] = static_cast<const C*>(p.tw2)[i];
  for (int i = tid; i < K::LO; i += K::TPB) s_btlo[i] = static_cast<const C*>(p.bt.lo)[i];
  for (int i = tid; i < K::HI; i += K::TPB) s_bthi[i] = static_cast<const C*>(p.bt.hi)[i];
  BigTwiddle sbt;
  sbt.lo = s_btlo;
  sbt.hi = s_bthi;
  sbt.shift = K::SHIFT;
  __syncthreads();

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane != 0) return;
    int64_t k = 0;
    for (;; ++k) {
      const int s = int(k % NST);
      if (k >= NST && !mbar_wait_abort(&empty[s], uint32_t(((k / NST) - 1) & 1), p.spin_limit, &s_abort)) {
        s_abort = 1;
        atomicExch(p.status, 1u);
        break;  // the compute warps see s_abort at their next full wait
      }
      const int64_t w = int64_t(atomicAdd(p.ctr, 1u));
      if (w >= total || s_abort) {
        s_item[s] = -1;
        mbar_arrive(&full[s]);
        break;
      }
      int pass, g;
      int64_t tile;
      decode_tile(w, p.groups, p.S, TAg, TBg, pass, g, tile);
      bool ok = true;
      if (pass == 2) ok = wait_counter(doneA + g, unsigned(TAg), p.spin_limit, &s_abort);
      else if (g >= p.S) ok = wait_counter(doneB + (g - p.S), unsigned(TBg), p.spin_limit, &s_abort);
      if (!ok) {
        s_abort = 1;
        atomicExch(p.status, 1u);
        s_item[s] = -2;
        mbar_arrive(&full[s]);
        break;
      }
      fence_async_global();  // the acquired slot contents before the copy engine reads them
      s_item[s] = w;
      C* buf = bufs + s * BUFE;
      if (pass == 1) {
        const int64_t bl = tile / K::TA;
        const int64_t b = int64_t(g) * p.G + bl;
        const int col0 = int(tile % K::TA) * NC1;
        if (b < p.count) {
          mbar_expect_tx(&full[s], K::BYTES_A);
#pragma unroll
          for (int i = 0; i < K::NBOX1; ++i) tma_load_3d(buf + i * K::BR1 * NC1, &tx, &full[s], col0 * W, i * K::BR1, int(b));
        } else {
          mbar_arrive(&full[s]);  // a transform past the batch's end: nothing to copy
        }
      } else {
        const int64_t bl = tile / K::TB;
        const int64_t b = int64_t(g) * p.G + bl;
        const int col0 = int(tile % K::TB) * NC2;
        const int z = int((g % p.S) * p.G + bl);
        if (b < p.count) {
          mbar_expect_tx(&full[s], K::BYTES_B);
#pragma unroll
          for (int i = 0; i < K::NBOX2; ++i) tma_load_3d(buf + i * K::BR2 * NC2, &tyl, &full[s], col0 * W, i * K::BR2, z);
        } else {
          mbar_arrive(&full[s]);
        }
      }
    }
    // let copies still in flight land before the CTA's shared memory goes
    // away (their phases complete; waits on completed phases return at once)
    for (int64_t j = k - 1; j >= 0 && j > k - NST; --j)
      mbar_wait(&full[int(j % NST)], uint32_t((j / NST) & 1), p.spin_limit);
    return;
  }

  if (warp == 1) {
    // ------------------------------------------------------------ storer
    if (lane != 0) return;
    int prev_g = -1;  // group of the previous pass-A tile whose completion is still unpublished
    auto publish = [&]() {
      fence_async_global();
      red_release_add(doneA + prev_g, 1u);
      prev_g = -1;
    };
    for (int64_t k = 0;; ++k) {
      const int s = int(k % NST);
      const uint32_t par = uint32_t((k / NST) & 1);
      // Publication of the previous tile waits for this one only while this
      // one is ready at once; otherwise it happens now (this CTA's own
      // producer may be waiting for exactly that group).
      if (prev_g >= 0 && !mbar_test(&ready[s], par)) {
        bulk_wait_n<0>();
        publish();
      }
      if (!mbar_wait_abort(&ready[s], par, 4 * p.spin_limit, &s_abort)) {
        s_abort = 1;
        atomicExch(p.status, 1u);
        break;
      }
      const int64_t w = s_item[s];
      if (w < 0 || s_abort) break;
      int pass, g;
      int64_t tile;
      decode_tile(w, p.groups, p.S, TAg, TBg, pass, g, tile);
      const C* sh = bufs + s * BUFE;
      if (pass == 1) {
        const int64_t bl = tile / K::TA;
        const int64_t b = int64_t(g) * p.G + bl;
        const int col0 = int(tile % K::TA) * NC1;
        const int z = int((g % p.S) * p.G + bl);
        fence_async_global();  // after the slot's release by pass B (observed through the producer)
        if (b < p.count)  // Y[n2][k1]: box i holds rows k1 = i*RE.. of columns n2 = col0..
          for (int i = 0; i < N1 / K::RE; ++i) tma_store_3d(&tys, sh + i * NC1 * K::RE, i * K::RE * W, col0, z);
      } else {
        const int64_t bl = tile / K::TB;
        const int64_t b = int64_t(g) * p.G + bl;
        const int col0 = int(tile % K::TB) * NC2;
        if (b < p.count)
#pragma unroll
          for (int i = 0; i < K::NBOX2; ++i) tma_store_3d(&tz, sh + i * K::BR2 * NC2, col0 * W, i * K::BR2, int(b));
      }
      bulk_commit();
      // the previous pass-A tile, once its stores are complete (this tile's
      // group may stay in flight)
      if (prev_g >= 0) {
        bulk_wait_n<1>();
        publish();
      }
      prev_g = pass == 1 ? g : -1;
      bulk_wait_read();  // the stores have read the buffer: free it
      mbar_arrive(&empty[s]);
    }
    bulk_wait_all();
    if (prev_g >= 0 && !s_abort) publish();
    return;
  }

  // -------------------------------------------------------------- compute
  const int ct = tid - 64;
  C v[EPT1 > EPT2 ? EPT1 : EPT2];
  for (int64_t k = 0;; ++k) {
    const int s = int(k % NST);
    const bool ok = mbar_wait_abort(&full[s], uint32_t((k / NST) & 1), 4 * p.spin_limit, &s_abort);
    // the decision to stop is taken together (named barrier with a vote)
    int stop;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, 1, %2, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(stop)
        : "r"(int(!ok || s_abort)), "n"(K::TPBC)
        : "memory");
    const int64_t w = stop ? -3 : s_item[s];
    if (w < 0) {
      if (stop && ct == 0) {
        s_abort = 1;  // before this warp's arrival: the storer then stores nothing
        atomicExch(p.status, 1u);
      }
      if (lane == 0) mbar_arrive(&ready[s]);  // the storer sees the stop too
      break;
    }
    int pass, g;
    int64_t tile;
    decode_tile(w, p.groups, p.S, TAg, TBg, pass, g, tile);
    C* sh = bufs + s * BUFE;
    // a pass-B tile has read its slot rows (they are in shared memory): one
    // more of the group's tiles no longer needs the slot
    if (pass == 2 && ct == 0) red_release_add(doneB + g, 1u);
    if (pass == 1) {
      const int64_t b = int64_t(g) * p.G + tile / K::TA;
      const int col0 = int(tile % K::TA) * NC1;
      if (b < p.count) {
        const int c = ct % NC1, t = ct / NC1;
        col_stage<C, N1, EPT1, NC1, DIR, 1, LOAD_SMEM, OUT_SMEM_TWIDDLE_SW, 1, 1, true, NoIO, K::TPBC, true>(
            v, nullptr, nullptr, sh, t, c, ct < K::A::TPB, s_tw1, Re(1), sbt, int64_t(col0 + c));
      }
    } else {
      const int64_t b = int64_t(g) * p.G + tile / K::TB;
      if (b < p.count) {
        const int c = ct % NC2, t = ct / NC2;
        col_stage<C, N2, EPT2, NC2, DIR, 1, LOAD_SMEM, OUT_SMEM, 1, 1, true, NoIO, K::TPBC>(
            v, nullptr, nullptr, sh, t, c, ct < K::B::TPB, s_tw2, Re(p.scale), p.bt, 0);
        fence_async_smem();
      }
    }
    // each warp hands the tile to the storer once its own writes are done
    // (every thread fenced its writes for the copy engine)
    __syncwarp();
    if (lane == 0) mbar_arrive(&ready[s]);
  }
}

}  // namespace gfft
