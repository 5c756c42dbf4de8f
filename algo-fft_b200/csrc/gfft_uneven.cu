// Uneven-length batch plans: many transforms of different lengths, packed
// back to back (transform i at the prefix sum of the lengths before it).
//
// The reference has no such entry point: a caller loops Plan.Forward over a
// plan per length, which is what gfft_uneven_exec_per_size does on the GPU
// (one launch chain per transform) as the baseline.  gfft_uneven_exec runs
// the whole batch as:
//   - every transform that fits one CTA (direct runtime Stockham, or
//     Bluestein whose FFT length fits) in persistent k_uneven launches, one
//     per CTA-size class, fed by a device work queue;
//   - larger power-of-two lengths: gathered into one batch per length, run
//     through that length's batched plan, scattered back;
//   - larger 7-smooth lengths whose four-step factors n = N1 x N2 both have
//     compiled mixed-radix column tiles: the two passes of every such
//     transform in one launch per distinct N1 (pass 1) and one per distinct
//     N2 (pass 2), each CTA finding its transform through an item table;
//   - larger lengths whose Bluestein FFT can be a product M = M1 x M2 of
//     compiled column lengths below NextPow2(2n-1): the chain of
//     gfft_mixbs.cuh as items, four phases (chirp-load pass, filter-store
//     pass, inverse pass 1, chirp-store pass), one launch per column length
//     and phase, in chunks that bound the scratch;
//   - every other larger length through Bluestein, grouped by FFT length M
//     (NextPow2(2n-1), plan.go:865): one gather (x chirp), one batched FFT_M,
//     one filter product, one batched inverse FFT_M, one scatter (x chirp).
// The launch sequence is captured once into a CUDA graph per (direction,
// dst, src) and replayed.  Plan tables (twiddles, chirps, filters) are built
// on the GPU at plan creation; filters of one M come from one batched FFT.
#include <algorithm>
#include <cmath>
#include <functional>
#include <map>
#include <mutex>
#include <new>
#include <vector>
#include "gfft_internal.h"
#include "gfft_mixbs.cuh"
#include "gfft_mixcols.cuh"
#include "gfft_uneven.cuh"

namespace gfft {
namespace {

struct Group {
  int64_t M = 0;           // FFT length of the group
  bool bluestein = false;
  PlanCore* plan = nullptr;
  std::vector<BigItem> items;
  BigItem* d_items = nullptr;
  void* work = nullptr;    // rows x M
};

struct Klass {
  std::vector<UnevenItem> items;
  UnevenItem* d_items = nullptr;
  int cta = 0;
  size_t smem = 0;
  int grid = 0;
};

unsigned grid1(int64_t total) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 32))); }

const size_t kSmemMax = 200 * 1024;

bool direct_ok(int64_t n, size_t es, GenSched* s) {
  if (n == 1) {
    *s = GenSched{};
    s->n = 1;
    s->nst = 0;
    s->T = 1;
    s->B = 1;
    s->stride = 1;
    return true;
  }
  return make_gen_sched(n, s) && size_t(s->stride) * es <= kSmemMax;
}

template <typename C>
cudaError_t set_uneven_attrs() {
  cudaError_t e = cudaFuncSetAttribute(&k_uneven<C, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemMax));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(&k_uneven<C, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemMax));
  return e;
}

}  // namespace
}  // namespace gfft

using namespace gfft;

struct gfft_plan_uneven {
  int prec = 0;
  int device = 0;
  int64_t count = 0, total = 0;
  std::vector<int64_t> len, off;
  void* tab = nullptr;
  std::vector<UnevenDesc> descs;
  UnevenDesc* d_descs = nullptr;
  Klass klass[2];
  std::vector<Group> groups;
  unsigned* counters = nullptr;
  std::map<int64_t, PlanCore*> single;  // per-length plans of the per-size path
  std::mutex mu;
  struct Graph {
    int dir;
    const void* src;
    void* dst;
    cudaGraphExec_t exec;
    uint64_t used;  // call tick of the last replay (least recently used goes first)
  };
  std::vector<Graph> graphs;
  uint64_t tick = 0;
  cudaStream_t cap = nullptr;
  // Side streams the batch's independent pieces run on, forked from the
  // caller's stream and joined back to it.
  static constexpr int kSide = 4;
  cudaStream_t side[kSide] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kSide] = {};
  // Large 7-smooth lengths on the mixed-radix four-step (item mode).
  struct MixLaunch {
    int64_t L;        // column length of the launch
    int pass;         // MIX_PASS1 / MIX_PASS2
    int64_t tw;       // W_L table offset
    int64_t blocks;   // CTAs
    int32_t* d_blk = nullptr;  // item of every CTA
  };
  std::vector<MixItem> mix_items;
  MixItem* d_mix_items = nullptr;
  std::vector<MixLaunch> mix_launches;  // pass-1 launches first
  int64_t mix_scratch = 0;              // elements of the intermediates
  // Bluestein on mixed FFT lengths (item mode): per chunk of transforms,
  // launches of the phases BSK_IN, BSK_MID and BSK_OUT, in that order.
  struct BsmLaunch {
    int kind;
    int64_t L, tw, blocks;
    int32_t* d_blk = nullptr;
  };
  struct BsmChunk {
    int64_t elems = 0;  // M summed over the chunk's transforms
    std::vector<BsmLaunch> launches;
  };
  std::vector<MixBsItem> bsm_items;
  MixBsItem* d_bsm_items = nullptr;
  std::vector<BsmChunk> bsm_chunks;
  int64_t bsm_buf = 0;  // elements of the largest chunk
  // Recorded after every call's work: the next call, on whatever stream,
  // waits for it, so calls on one plan never overlap on the device (they
  // share the work buffers and queue counters above).
  cudaEvent_t done = nullptr;
};

namespace {
constexpr size_t kMaxGraphs = 8;  // instantiated graphs kept per plan

bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// Orders this call after the plan's previous one (skipped while the caller
// captures `st` into its own graph: the capture orders its replays).
gfft_status after_previous_call(gfft_plan_uneven* p, cudaStream_t st) {
  if (capturing(st)) return GFFT_OK;
  GFFT_CUDA(cudaStreamWaitEvent(st, p->done, 0));
  return GFFT_OK;
}

gfft_status mark_call_done(gfft_plan_uneven* p, cudaStream_t st) {
  if (capturing(st)) return GFFT_OK;
  GFFT_CUDA(cudaEventRecord(p->done, st));
  return GFFT_OK;
}
}  // namespace

extern "C" GFFT_API void gfft_plan_uneven_close(gfft_plan_uneven* p);

namespace gfft {

static gfft_status uneven_build(gfft_plan_uneven* p) {
  const size_t es = elem_bytes(p->prec);
  const int64_t max_direct_bs = p->prec == kC64 ? 16384 : 8192;
  // distinct lengths and their handling
  std::map<int64_t, int> desc_of;                 // small lengths -> descriptor
  std::map<int64_t, std::vector<int64_t>> bs_by_m;  // Bluestein lengths per FFT length M
  std::map<int64_t, int64_t> tw_off;              // W_L table offsets
  std::map<int64_t, int64_t> chirp_off, filt_off;
  std::map<int64_t, int> big_pow2_group;          // large pow2 length -> group
  std::map<int64_t, int> big_bs_group;            // M -> group
  std::map<int64_t, int64_t> mix_n1;              // mixed-radix four-step length -> N1
  std::map<int64_t, int64_t> mix_lo, mix_hi;      // its W_n split tables
  std::map<int64_t, int> mix_shift;
  std::map<int64_t, int64_t> bsm_M, bsm_m1;       // mixed Bluestein length n -> M, M1
  std::map<int64_t, int64_t> bsm_lo, bsm_hi;      // W_M split tables per M
  std::map<int64_t, int> bsm_shift;
  int64_t cursor = 0;
  auto alloc = [&](int64_t n) {
    const int64_t at = cursor;
    cursor += (n + 1) & ~int64_t(1);  // keep every table 16-byte aligned
    return at;
  };
  std::vector<int64_t> distinct(p->len);
  std::sort(distinct.begin(), distinct.end());
  distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
  for (int64_t n : distinct) {
    GenSched s;
    if (direct_ok(n, es, &s)) {
      UnevenDesc d{};
      d.s = s;
      d.n = n;
      d.bluestein = 0;
      if (!tw_off.count(n)) tw_off[n] = alloc(n);
      d.tw = tw_off[n];
      desc_of[n] = int(p->descs.size());
      p->descs.push_back(d);
      continue;
    }
    if ((n & (n - 1)) == 0) {
      big_pow2_group[n] = int(p->groups.size());
      Group g;
      g.M = n;
      p->groups.push_back(g);
      continue;
    }
    const int64_t m1 = is_smooth7(n) ? mix_split(n) : 0;
    if (m1 >= 2) {
      mix_n1[n] = m1;
      for (int64_t L : {m1, n / m1})
        if (!tw_off.count(L)) tw_off[L] = alloc(L);
      int shift = 0;
      while ((int64_t(1) << (2 * shift)) < n) ++shift;
      mix_shift[n] = shift;
      mix_lo[n] = alloc(int64_t(1) << shift);
      mix_hi[n] = alloc((n + (int64_t(1) << shift) - 1) >> shift);
      continue;
    }
    int64_t M = 1;
    while (M < 2 * n - 1) M <<= 1;
    // beyond the one-CTA kernel: a smaller FFT length of two compiled
    // column lengths where the plans' rule prefers it (never a power of
    // two itself)
    int64_t bm1 = 0;
    const int64_t mx = M > max_direct_bs ? bs_mixed_choice(n, &bm1) : 0;
    if (bs_mixed_preferred(mx, M)) {
      bsm_M[n] = mx;
      bsm_m1[n] = bm1;
      bs_by_m[mx].push_back(n);
      chirp_off[n] = alloc(n);
      for (int64_t L : {bm1, mx / bm1})
        if (!tw_off.count(L)) tw_off[L] = alloc(L);
      if (!bsm_lo.count(mx)) {
        int shift = 0;
        while ((int64_t(1) << (2 * shift)) < mx) ++shift;
        bsm_shift[mx] = shift;
        bsm_lo[mx] = alloc(int64_t(1) << shift);
        bsm_hi[mx] = alloc((mx + (int64_t(1) << shift) - 1) >> shift);
      }
      continue;
    }
    bs_by_m[M].push_back(n);
    chirp_off[n] = alloc(n);
    GenSched sm;
    if (M <= max_direct_bs && direct_ok(M, es, &sm)) {
      UnevenDesc d{};
      d.s = sm;
      d.n = n;
      d.bluestein = 1;
      if (!tw_off.count(M)) tw_off[M] = alloc(M);
      d.tw = tw_off[M];
      d.chirp = chirp_off[n];
      desc_of[n] = int(p->descs.size());
      p->descs.push_back(d);
    } else if (!big_bs_group.count(M)) {
      big_bs_group[M] = int(p->groups.size());
      Group g;
      g.M = M;
      g.bluestein = true;
      p->groups.push_back(g);
    }
  }
  // filters: one contiguous block of rows per M, in bs_by_m order
  for (auto& kv : bs_by_m)
    for (int64_t n : kv.second) filt_off[n] = alloc(kv.first);
  for (auto& d : p->descs)
    if (d.bluestein) d.filt = filt_off[d.n];
  GFFT_CUDA(cudaMalloc(&p->tab, size_t(std::max<int64_t>(cursor, 1)) * es));
  char* tab = static_cast<char*>(p->tab);
  for (auto& kv : tw_off) {
    gfft_status s = fill_twiddles(p->prec, tab + kv.second * es, kv.first, kv.first, 1, 0);
    if (s != GFFT_OK) return s;
  }
  for (auto& kv : mix_n1) {
    const int64_t n = kv.first, nlo = int64_t(1) << mix_shift[n];
    gfft_status s = fill_twiddles(p->prec, tab + mix_lo[n] * es, n, nlo, 1, 0);
    if (s == GFFT_OK) s = fill_twiddles(p->prec, tab + mix_hi[n] * es, n, (n + nlo - 1) / nlo, nlo, 0);
    if (s != GFFT_OK) return s;
  }
  for (auto& kv : bsm_lo) {
    const int64_t M = kv.first, nlo = int64_t(1) << bsm_shift[M];
    gfft_status s = fill_twiddles(p->prec, tab + bsm_lo[M] * es, M, nlo, 1, 0);
    if (s == GFFT_OK) s = fill_twiddles(p->prec, tab + bsm_hi[M] * es, M, (M + nlo - 1) / nlo, nlo, 0);
    if (s != GFFT_OK) return s;
  }
  for (auto& kv : chirp_off) {
    const int64_t n = kv.first;
    if (p->prec == kC64)
      k_chirp<float2><<<grid1(n), 256>>>(reinterpret_cast<float2*>(tab + kv.second * es), n, -1);
    else
      k_chirp<double2><<<grid1(n), 256>>>(reinterpret_cast<double2*>(tab + kv.second * es), n, -1);
  }
  GFFT_CUDA(cudaGetLastError());
  for (auto& kv : bs_by_m) {
    const int64_t M = kv.first;
    for (int64_t n : kv.second) {
      if (p->prec == kC64)
        k_bs_filter_src<float2><<<grid1(M), 256>>>(reinterpret_cast<float2*>(tab + filt_off[n] * es),
                                                    reinterpret_cast<const float2*>(tab + chirp_off[n] * es), n, M);
      else
        k_bs_filter_src<double2><<<grid1(M), 256>>>(reinterpret_cast<double2*>(tab + filt_off[n] * es),
                                                     reinterpret_cast<const double2*>(tab + chirp_off[n] * es), n, M);
    }
    GFFT_CUDA(cudaGetLastError());
    PlanCore pc;
    gfft_status s = core_init(&pc, p->prec, M, p->device);
    if (s == GFFT_OK)
      s = core_exec(&pc, -1, tab + filt_off[kv.second.front()] * es, tab + filt_off[kv.second.front()] * es,
                    int64_t(kv.second.size()), M, M, 0);
    GFFT_CUDA(cudaStreamSynchronize(0));
    core_free(&pc);
    if (s != GFFT_OK) return s;
  }
  // items
  for (int64_t i = 0; i < p->count; ++i) {
    const int64_t n = p->len[i];
    auto it = desc_of.find(n);
    if (it != desc_of.end()) {
      const UnevenDesc& d = p->descs[it->second];
      Klass& k = p->klass[d.s.T <= 128 ? 0 : 1];
      k.items.push_back(UnevenItem{p->off[i], it->second, 0});
      continue;
    }
    if ((n & (n - 1)) == 0) {
      p->groups[big_pow2_group[n]].items.push_back(BigItem{p->off[i], n, 0, 0});
    } else if (bsm_M.count(n)) {
      MixBsItem m{};
      m.off = p->off[i];
      m.n = n;
      m.M = bsm_M[n];
      m.chirp = chirp_off[n];
      m.filt = filt_off[n];
      m.lo = bsm_lo[m.M];
      m.hi = bsm_hi[m.M];
      m.shift = bsm_shift[m.M];
      p->bsm_items.push_back(m);
    } else if (mix_n1.count(n)) {
      MixItem m{};
      m.off = p->off[i];
      m.y = p->mix_scratch;
      m.n = n;
      m.lo = mix_lo[n];
      m.hi = mix_hi[n];
      m.shift = mix_shift[n];
      p->mix_scratch += n;
      p->mix_items.push_back(m);
    } else {
      int64_t M = 1;
      while (M < 2 * n - 1) M <<= 1;
      p->groups[big_bs_group[M]].items.push_back(BigItem{p->off[i], n, chirp_off[n], filt_off[n]});
    }
  }
  // queue order: most expensive first (longest-first list schedule)
  auto cost = [&](const UnevenItem& u) {
    const UnevenDesc& d = p->descs[u.desc];
    return double(d.s.n) * std::log2(double(d.s.n) + 1.0) * (d.bluestein ? 2.0 : 1.0);
  };
  int dev = 0, sms = 0;
  GFFT_CUDA(cudaGetDevice(&dev));
  GFFT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GFFT_CUDA(p->prec == kC64 ? set_uneven_attrs<float2>() : set_uneven_attrs<double2>());
  for (Klass& k : p->klass) {
    if (k.items.empty()) continue;
    std::stable_sort(k.items.begin(), k.items.end(),
                     [&](const UnevenItem& a, const UnevenItem& b) { return cost(a) > cost(b); });
    int maxT = 32;
    size_t smem = 0;
    for (const auto& u : k.items) {
      maxT = std::max(maxT, p->descs[u.desc].s.T);
      smem = std::max(smem, size_t(p->descs[u.desc].s.stride) * es);
    }
    k.cta = std::min(1024, (maxT + 31) / 32 * 32);
    k.smem = smem;
    int occ = 0;
    const void* fn = p->prec == kC64 ? reinterpret_cast<const void*>(&k_uneven<float2, -1>)
                                     : reinterpret_cast<const void*>(&k_uneven<double2, -1>);
    GFFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, k.cta, k.smem));
    k.grid = int(std::min<int64_t>(int64_t(k.items.size()), int64_t(sms) * std::max(occ, 1)));
    GFFT_CUDA(cudaMalloc(&k.d_items, k.items.size() * sizeof(UnevenItem)));
    GFFT_CUDA(cudaMemcpy(k.d_items, k.items.data(), k.items.size() * sizeof(UnevenItem), cudaMemcpyHostToDevice));
  }
  if (!p->descs.empty()) {
    GFFT_CUDA(cudaMalloc(&p->d_descs, p->descs.size() * sizeof(UnevenDesc)));
    GFFT_CUDA(cudaMemcpy(p->d_descs, p->descs.data(), p->descs.size() * sizeof(UnevenDesc), cudaMemcpyHostToDevice));
  }
  for (Group& g : p->groups) {
    g.plan = new (std::nothrow) PlanCore;
    if (!g.plan) return GFFT_ERR_OUT_OF_MEMORY;
    gfft_status s = core_init(g.plan, p->prec, g.M, p->device);
    if (s != GFFT_OK) return s;
    GFFT_CUDA(cudaMalloc(&g.d_items, g.items.size() * sizeof(BigItem)));
    GFFT_CUDA(cudaMemcpy(g.d_items, g.items.data(), g.items.size() * sizeof(BigItem), cudaMemcpyHostToDevice));
    GFFT_CUDA(cudaMalloc(&g.work, g.items.size() * size_t(g.M) * es));
  }
  // mixed-radix four-step items: one launch per column length and pass,
  // each CTA one column tile of one item
  if (!p->mix_items.empty()) {
    for (int pass : {int(MIX_PASS1), int(MIX_PASS2)}) {
      std::map<int64_t, std::vector<int>> by_len;
      for (int i = 0; i < int(p->mix_items.size()); ++i) {
        const int64_t n = p->mix_items[i].n, n1 = mix_n1[n];
        by_len[pass == MIX_PASS1 ? n1 : n / n1].push_back(i);
      }
      for (auto& kv : by_len) {
        const int64_t L = kv.first;
        const int nc = mix_cols_width(p->prec, pass, L);
        if (nc <= 0) return GFFT_ERR_NOT_IMPLEMENTED;
        std::vector<int32_t> blk;
        for (int i : kv.second) {
          MixItem& m = p->mix_items[i];
          m.first[pass - 1] = int32_t(blk.size());
          const int64_t tiles = (m.n / L + nc - 1) / nc;
          blk.insert(blk.end(), size_t(tiles), int32_t(i));
        }
        gfft_plan_uneven::MixLaunch ml;
        ml.L = L;
        ml.pass = pass;
        ml.tw = tw_off[L];
        ml.blocks = int64_t(blk.size());
        GFFT_CUDA(cudaMalloc(&ml.d_blk, blk.size() * sizeof(int32_t)));
        p->mix_launches.push_back(ml);
        GFFT_CUDA(cudaMemcpy(ml.d_blk, blk.data(), blk.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
      }
    }
    GFFT_CUDA(cudaMalloc(&p->d_mix_items, p->mix_items.size() * sizeof(MixItem)));
    GFFT_CUDA(cudaMemcpy(p->d_mix_items, p->mix_items.data(), p->mix_items.size() * sizeof(MixItem),
                         cudaMemcpyHostToDevice));
  }
  // mixed Bluestein items: chunks of at most 2^27 FFT elements; per chunk one
  // launch per column length and phase, each CTA one column tile of one item
  if (!p->bsm_items.empty()) {
    const int64_t kChunk = int64_t(1) << 27;
    std::vector<std::pair<size_t, size_t>> spans;  // item ranges of the chunks
    for (size_t i = 0; i < p->bsm_items.size();) {
      size_t j = i;
      int64_t sum = 0;
      while (j < p->bsm_items.size() && (j == i || sum + p->bsm_items[j].M <= kChunk)) {
        p->bsm_items[j].s = sum;
        sum += p->bsm_items[j].M;
        ++j;
      }
      spans.push_back({i, j});
      gfft_plan_uneven::BsmChunk ch;
      ch.elems = sum;
      p->bsm_chunks.push_back(ch);
      p->bsm_buf = std::max(p->bsm_buf, sum);
      i = j;
    }
    for (size_t ci = 0; ci < spans.size(); ++ci) {
      for (int kind : {int(BSK_IN), int(BSK_MID), int(BSK_OUT)}) {
        const bool on_m1 = kind != BSK_MID;
        std::map<int64_t, std::vector<size_t>> by_len;
        for (size_t i = spans[ci].first; i < spans[ci].second; ++i) {
          const int64_t m1 = bsm_m1[p->bsm_items[i].n];
          by_len[on_m1 ? m1 : p->bsm_items[i].M / m1].push_back(i);
        }
        for (auto& kv : by_len) {
          const int64_t L = kv.first;
          const int nc = mix_bs_width(p->prec, L);
          if (nc <= 0) return GFFT_ERR_NOT_IMPLEMENTED;
          std::vector<int32_t> blk;
          for (size_t i : kv.second) {
            const int32_t first = int32_t(blk.size());
            p->bsm_items[i].first[kind] = first;
            const int64_t tiles = (p->bsm_items[i].M / L + nc - 1) / nc;
            blk.insert(blk.end(), size_t(tiles), int32_t(i));
          }
          gfft_plan_uneven::BsmLaunch bl;
          bl.kind = kind;
          bl.L = L;
          bl.tw = tw_off[L];
          bl.blocks = int64_t(blk.size());
          GFFT_CUDA(cudaMalloc(&bl.d_blk, blk.size() * sizeof(int32_t)));
          p->bsm_chunks[ci].launches.push_back(bl);
          GFFT_CUDA(cudaMemcpy(bl.d_blk, blk.data(), blk.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        }
      }
    }
    GFFT_CUDA(cudaMalloc(&p->d_bsm_items, p->bsm_items.size() * sizeof(MixBsItem)));
    GFFT_CUDA(cudaMemcpy(p->d_bsm_items, p->bsm_items.data(), p->bsm_items.size() * sizeof(MixBsItem),
                         cudaMemcpyHostToDevice));
  }
  GFFT_CUDA(cudaMalloc(&p->counters, 2 * sizeof(unsigned)));
  GFFT_CUDA(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking));
  for (int k = 0; k < gfft_plan_uneven::kSide; ++k) {
    GFFT_CUDA(cudaStreamCreateWithFlags(&p->side[k], cudaStreamNonBlocking));
    GFFT_CUDA(cudaEventCreateWithFlags(&p->ev_join[k], cudaEventDisableTiming));
  }
  GFFT_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
  GFFT_CUDA(cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming));
  return GFFT_OK;
}

// Pieces of an uneven batch that touch disjoint outputs and buffers; each is
// a launch sequence on one stream.
template <typename C, int DIR>
static gfft_status run_klass(gfft_plan_uneven* p, int k, C* dst, const C* src, cudaStream_t s) {
  const Klass& K = p->klass[k];
  k_uneven<C, DIR><<<K.grid, K.cta, K.smem, s>>>(src, dst, K.d_items, int(K.items.size()), p->d_descs,
                                                 static_cast<const C*>(p->tab), p->counters + k);
  GFFT_CUDA(cudaGetLastError());
  return GFFT_OK;
}

template <typename C, int DIR>
static gfft_status run_mixc(gfft_plan_uneven* p, C* dst, const C* src, cudaStream_t s) {
  void* scratch = nullptr;
  GFFT_CUDA(ws_alloc(&scratch, size_t(p->mix_scratch) * sizeof(C), s));
  cudaError_t e = cudaSuccess;
  for (const auto& ml : p->mix_launches) {
    MixColsParams mp{};
    mp.src = ml.pass == MIX_PASS1 ? static_cast<const void*>(src) : scratch;
    mp.dst = ml.pass == MIX_PASS1 ? scratch : static_cast<void*>(dst);
    mp.tw = static_cast<const C*>(p->tab) + ml.tw;
    mp.items = p->d_mix_items;
    mp.blk = ml.d_blk;
    mp.tab = p->tab;
    e = exec_mix_cols(p->prec, DIR, ml.pass, ml.L, mp, ml.blocks, s);
    if (e != cudaSuccess) break;
  }
  cudaFreeAsync(scratch, s);
  if (e != cudaSuccess) return cuda_status(e, "k_mix_cols");
  return GFFT_OK;
}

template <typename C, int DIR>
static gfft_status run_bsm(gfft_plan_uneven* p, C* dst, const C* src, cudaStream_t s) {
  void* buf = nullptr;
  GFFT_CUDA(ws_alloc(&buf, 2 * size_t(p->bsm_buf) * sizeof(C), s));
  void* scratch = buf;
  void* work = static_cast<C*>(buf) + p->bsm_buf;
  cudaError_t e = cudaSuccess;
  for (const auto& ch : p->bsm_chunks) {
    for (const auto& bl : ch.launches) {
      MixBsParams bp{};
      bp.x = src;
      bp.y = dst;
      bp.scratch = scratch;
      bp.work = work;
      bp.tw = static_cast<const C*>(p->tab) + bl.tw;
      bp.inv = DIR > 0;
      bp.items = p->d_bsm_items;
      bp.blk = bl.d_blk;
      bp.tab = p->tab;
      e = exec_mix_bs(p->prec, bl.kind, bl.L, bp, bl.blocks, s);
      if (e != cudaSuccess) break;
    }
    if (e != cudaSuccess) break;
  }
  cudaFreeAsync(buf, s);
  if (e != cudaSuccess) return cuda_status(e, "k_mix_bs");
  return GFFT_OK;
}

template <typename C, int DIR>
static gfft_status run_group(gfft_plan_uneven* p, Group& g, C* dst, const C* src, cudaStream_t s) {
  const int64_t rows = int64_t(g.items.size());
  C* work = static_cast<C*>(g.work);
  const C* tab = static_cast<const C*>(p->tab);
  const bool tp = (g.plan->algo == Algo::TwoPass || g.plan->algo == Algo::L2Pipe) &&
                  bluestein_tp_supported(p->prec, g.M, g.plan->tp[0]->n1);
  if (tp) {
    // on the two-pass FFT: rows read and written in place in the packed
    // batch, no gather or scatter pass (Bluestein: the chain fused in)
    void* scratch = nullptr;
    GFFT_CUDA(ws_alloc(&scratch, bluestein_tp_chunk_bytes(p->prec, g.M, rows), s));
    BigTwiddle bt;
    bt.lo = g.plan->bt_lo;
    bt.hi = g.plan->bt_hi;
    bt.shift = g.plan->bt_shift;
    const cudaError_t e =
        g.bluestein ? exec_bluestein_tp_items(p->prec, g.M, DIR, src, dst, g.d_items, rows, p->tab, g.plan->tw1,
                                              g.plan->tw2, bt, scratch, work, s)
                    : exec_twopass_items(p->prec, g.M, DIR, src, dst, g.d_items, rows, g.plan->tw1, g.plan->tw2, bt,
                                         scratch, s);
    cudaFreeAsync(scratch, s);
    GFFT_CUDA(e);
    return GFFT_OK;
  }
  k_big_gather<C, DIR><<<grid1(rows * g.M), 256, 0, s>>>(work, g.M, src, g.d_items, rows, tab, g.bluestein);
  GFFT_CUDA(cudaGetLastError());
  if (!g.bluestein) {
    const gfft_status r = core_exec(g.plan, DIR, work, work, rows, g.M, g.M, s);
    if (r != GFFT_OK) return r;
  } else {
    gfft_status r = core_exec(g.plan, -1, work, work, rows, g.M, g.M, s);
    if (r != GFFT_OK) return r;
    k_big_filter<C, DIR><<<grid1(rows * g.M), 256, 0, s>>>(work, g.M, g.d_items, rows, tab);
    GFFT_CUDA(cudaGetLastError());
    r = core_exec(g.plan, +1, work, work, rows, g.M, g.M, s);  // includes 1/M
    if (r != GFFT_OK) return r;
  }
  k_big_scatter<C, DIR><<<grid1(rows * g.M), 256, 0, s>>>(dst, work, g.M, g.d_items, rows, tab, g.bluestein);
  GFFT_CUDA(cudaGetLastError());
  return GFFT_OK;
}

using Piece = std::pair<double, std::function<gfft_status(cudaStream_t)>>;

// Runs the pieces on the plan's side streams, forked from `st` and joined
// back to it (parallel branches when `st` is being captured): longest
// first, each onto the stream with the least work so far.  Every side
// stream rejoins `st` even when a piece fails, so a capture stays whole.
static gfft_status run_pieces(gfft_plan_uneven* p, cudaStream_t st, std::vector<Piece>& pieces) {
  if (pieces.size() < 2) {
    for (auto& pc : pieces) {
      const gfft_status r = pc.second(st);
      if (r != GFFT_OK) return r;
    }
    return GFFT_OK;
  }
  std::stable_sort(pieces.begin(), pieces.end(), [](const Piece& a, const Piece& b) { return a.first > b.first; });
  const int ns = int(std::min<size_t>(pieces.size(), gfft_plan_uneven::kSide));
  GFFT_CUDA(cudaEventRecord(p->ev_fork, st));
  for (int k = 0; k < ns; ++k) GFFT_CUDA(cudaStreamWaitEvent(p->side[k], p->ev_fork, 0));
  std::vector<double> load(ns, 0.0);
  gfft_status first = GFFT_OK;
  for (auto& pc : pieces) {
    const int k = int(std::min_element(load.begin(), load.end()) - load.begin());
    load[k] += pc.first;
    if (first == GFFT_OK) first = pc.second(p->side[k]);
  }
  for (int k = 0; k < ns; ++k) {
    const cudaError_t e1 = cudaEventRecord(p->ev_join[k], p->side[k]);
    const cudaError_t e2 = cudaStreamWaitEvent(st, p->ev_join[k], 0);
    if (first == GFFT_OK && (e1 != cudaSuccess || e2 != cudaSuccess))
      first = cuda_status(e1 != cudaSuccess ? e1 : e2, "uneven join");
  }
  return first;
}

template <typename C, int DIR>
static gfft_status uneven_run(gfft_plan_uneven* p, C* dst, const C* src, cudaStream_t st) {
  GFFT_CUDA(cudaMemsetAsync(p->counters, 0, 2 * sizeof(unsigned), st));
  // rough costs (elements moved) for spreading the pieces over the streams
  std::vector<Piece> pieces;
  for (int k = 0; k < 2; ++k) {
    const Klass& K = p->klass[k];
    if (K.items.empty()) continue;
    double cost = 0;
    for (const UnevenItem& u : K.items) cost += double(p->descs[u.desc].s.n) * (p->descs[u.desc].bluestein ? 4 : 2);
    pieces.push_back({cost, [=](cudaStream_t s) { return run_klass<C, DIR>(p, k, dst, src, s); }});
  }
  if (!p->mix_items.empty())
    pieces.push_back({4.0 * double(p->mix_scratch), [=](cudaStream_t s) { return run_mixc<C, DIR>(p, dst, src, s); }});
  if (!p->bsm_items.empty()) {
    double cost = 0;
    for (const auto& ch : p->bsm_chunks) cost += 5.0 * double(ch.elems);
    pieces.push_back({cost, [=](cudaStream_t s) { return run_bsm<C, DIR>(p, dst, src, s); }});
  }
  for (Group& g : p->groups) {
    if (g.items.empty()) continue;
    Group* gp = &g;
    pieces.push_back({double(g.items.size()) * double(g.M) * (g.bluestein ? 6 : 4),
                      [=](cudaStream_t s) { return run_group<C, DIR>(p, *gp, dst, src, s); }});
  }
  return run_pieces(p, st, pieces);
}

static gfft_status uneven_dispatch(gfft_plan_uneven* p, int dir, void* dst, const void* src, cudaStream_t st) {
  if (p->prec == kC64)
    return dir < 0 ? uneven_run<float2, -1>(p, static_cast<float2*>(dst), static_cast<const float2*>(src), st)
                   : uneven_run<float2, +1>(p, static_cast<float2*>(dst), static_cast<const float2*>(src), st);
  return dir < 0 ? uneven_run<double2, -1>(p, static_cast<double2*>(dst), static_cast<const double2*>(src), st)
                 : uneven_run<double2, +1>(p, static_cast<double2*>(dst), static_cast<const double2*>(src), st);
}

}  // namespace gfft

extern "C" {

gfft_status gfft_plan_uneven_new(gfft_plan_uneven** out, int32_t precision, int64_t count, const int64_t* lengths,
                                 const gfft_plan_options* opts) {
  clear_error();
  if (!out) return GFFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (count < 1 || !lengths) return GFFT_ERR_INVALID_LENGTH;
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  for (int64_t i = 0; i < count; ++i)
    if (lengths[i] < 1 || lengths[i] > (int64_t(1) << 24)) {
      set_error("transform " + std::to_string(i) + " has an unsupported length");
      return GFFT_ERR_INVALID_LENGTH;
    }
  gfft_plan_options o{};
  if (opts) o = *opts;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GFFT_ERR_NO_DEVICE;
  if (o.device < 0 || o.device >= ndev) return GFFT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(o.device));
  auto* p = new (std::nothrow) gfft_plan_uneven;
  if (!p) return GFFT_ERR_OUT_OF_MEMORY;
  p->prec = precision;
  p->device = o.device;
  p->count = count;
  p->len.assign(lengths, lengths + count);
  p->off.resize(count);
  for (int64_t i = 0; i < count; ++i) {
    p->off[i] = p->total;
    p->total += lengths[i];
  }
  gfft_status s = uneven_build(p);
  if (s != GFFT_OK) {
    gfft_plan_uneven_close(p);
    return s;
  }
  *out = p;
  return GFFT_OK;
}

void gfft_plan_uneven_close(gfft_plan_uneven* p) {
  if (!p) return;
  for (auto& g : p->graphs) cudaGraphExecDestroy(g.exec);
  for (Klass& k : p->klass)
    if (k.d_items) cudaFree(k.d_items);
  for (Group& g : p->groups) {
    if (g.plan) {
      core_free(g.plan);
      delete g.plan;
    }
    if (g.d_items) cudaFree(g.d_items);
    if (g.work) cudaFree(g.work);
  }
  for (auto& kv : p->single) {
    core_free(kv.second);
    delete kv.second;
  }
  for (auto& ml : p->mix_launches)
    if (ml.d_blk) cudaFree(ml.d_blk);
  if (p->d_mix_items) cudaFree(p->d_mix_items);
  for (auto& ch : p->bsm_chunks)
    for (auto& bl : ch.launches)
      if (bl.d_blk) cudaFree(bl.d_blk);
  if (p->d_bsm_items) cudaFree(p->d_bsm_items);
  if (p->d_descs) cudaFree(p->d_descs);
  if (p->tab) cudaFree(p->tab);
  if (p->counters) cudaFree(p->counters);
  if (p->cap) cudaStreamDestroy(p->cap);
  for (int k = 0; k < gfft_plan_uneven::kSide; ++k) {
    if (p->side[k]) cudaStreamDestroy(p->side[k]);
    if (p->ev_join[k]) cudaEventDestroy(p->ev_join[k]);
  }
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->done) cudaEventDestroy(p->done);
  delete p;
}

int64_t gfft_plan_uneven_total(const gfft_plan_uneven* p) { return p ? p->total : 0; }

gfft_status gfft_uneven_exec(gfft_plan_uneven* p, int32_t direction, void* dst, const void* src, int32_t use_graph,
                             void* stream) {
  clear_error();
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (direction != -1 && direction != 1) return GFFT_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> g(p->mu);  // the plan's work buffers are shared
  DeviceGuard dg;
  GFFT_CUDA(dg.set(p->device));
  gfft_status s0 = after_previous_call(p, st);
  if (s0 != GFFT_OK) return s0;
  if (!use_graph) {
    s0 = uneven_dispatch(p, direction, dst, src, st);
    return s0 != GFFT_OK ? s0 : mark_call_done(p, st);
  }
  cudaGraphExec_t exec = nullptr;
  ++p->tick;
  for (auto& gr : p->graphs)
    if (gr.dir == direction && gr.src == src && gr.dst == dst) {
      exec = gr.exec;
      gr.used = p->tick;
    }
  if (!exec && p->graphs.size() >= kMaxGraphs) {
    // drop the least recently used graph; every replay of it has finished
    // once the plan's previous call has (calls are ordered on the device)
    auto lru = std::min_element(p->graphs.begin(), p->graphs.end(),
                                [](const auto& a, const auto& b) { return a.used < b.used; });
    GFFT_CUDA(cudaEventSynchronize(p->done));
    cudaGraphExecDestroy(lru->exec);
    p->graphs.erase(lru);
  }
  if (!exec) {
    cudaGraph_t graph = nullptr;
    GFFT_CUDA(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
    gfft_status s = uneven_dispatch(p, direction, dst, src, p->cap);
    cudaError_t e = cudaStreamEndCapture(p->cap, &graph);
    if (s != GFFT_OK) {
      if (graph) cudaGraphDestroy(graph);
      return s;
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
    p->graphs.push_back({direction, src, dst, exec, p->tick});
  }
  GFFT_CUDA(cudaGraphLaunch(exec, st));
  return mark_call_done(p, st);
}

gfft_status gfft_uneven_exec_per_size(gfft_plan_uneven* p, int32_t direction, void* dst, const void* src,
                                      void* stream) {
  clear_error();
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (direction != -1 && direction != 1) return GFFT_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> g(p->mu);
  DeviceGuard dg;
  GFFT_CUDA(dg.set(p->device));
  gfft_status s0 = after_previous_call(p, st);
  if (s0 != GFFT_OK) return s0;
  const size_t es = elem_bytes(p->prec);
  for (int64_t i = 0; i < p->count; ++i) {
    const int64_t n = p->len[i];
    auto it = p->single.find(n);
    if (it == p->single.end()) {
      auto* c = new (std::nothrow) PlanCore;
      if (!c) return GFFT_ERR_OUT_OF_MEMORY;
      gfft_status s = core_init(c, p->prec, n, p->device);
      if (s != GFFT_OK) {
        core_free(c);
        delete c;
        return s;
      }
      it = p->single.emplace(n, c).first;
    }
    gfft_status s = core_exec(it->second, direction, static_cast<char*>(dst) + size_t(p->off[i]) * es,
                              static_cast<const char*>(src) + size_t(p->off[i]) * es, 1, n, n, st);
    if (s != GFFT_OK) return s;
  }
  return mark_call_done(p, st);
}

}  // extern "C"
