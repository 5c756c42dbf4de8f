// Kernel registry, device twiddle generation and the 1-D schedule choice.
#include <algorithm>
#include <atomic>
#include <map>
#include <cstdlib>
#include <cstdio>
#include <mutex>
#include <vector>
#include "gfft_internal.h"
#include "gfft_math.cuh"
#include "gfft_l2pipe.cuh"
#include "gfft_threepass.cuh"
#include "gfft_twopass.cuh"

namespace gfft {

// ---------------------------------------------------------------- registry

static std::vector<Pow2Kernel>& pow2_table() {
  static std::vector<Pow2Kernel> t;
  return t;
}

static std::vector<TwoPassKernel>& twopass_table() {
  static std::vector<TwoPassKernel> t;
  return t;
}

static std::vector<ThreePassKernel>& threepass_table() {
  static std::vector<ThreePassKernel> t;
  return t;
}

void register_pow2(const Pow2Kernel& k) { pow2_table().push_back(k); }
void register_threepass(const ThreePassKernel& k) { threepass_table().push_back(k); }

const ThreePassKernel* find_threepass(int prec, int64_t n, int dir, int tma, int te, int emax, int nst) {
  for (const auto& k : threepass_table())
    if (k.prec == prec && int64_t(k.n1) * k.m1 * k.m2 == n && k.dir == dir && k.tma == tma &&
        (tma == 0 || (k.te == te && k.emax == emax && k.nst == nst)))
      return &k;
  return nullptr;
}

std::vector<const ThreePassKernel*> threepass_variants(int prec, int64_t n, int dir) {
  std::vector<const ThreePassKernel*> v;
  for (const auto& k : threepass_table())
    if (k.prec == prec && int64_t(k.n1) * k.m1 * k.m2 == n && k.dir == dir) v.push_back(&k);
  return v;
}
void register_twopass(const TwoPassKernel& k) { twopass_table().push_back(k); }

static std::vector<L2PipeKernel>& l2pipe_table() {
  static std::vector<L2PipeKernel> t;
  return t;
}

void register_l2pipe(const L2PipeKernel& k) { l2pipe_table().push_back(k); }

const L2PipeKernel* find_l2pipe(int prec, int64_t n, int dir, int n1, int nc1, int nc2, int nst) {
  for (const auto& k : l2pipe_table())
    if (k.prec == prec && int64_t(k.n1) * k.n2 == n && k.dir == dir && (n1 == 0 || k.n1 == n1) &&
        (nc1 == 0 || k.nc1 == nc1) && (nc2 == 0 || k.nc2 == nc2) && (nst == 0 || k.nst == nst))
      return &k;
  return nullptr;
}

std::vector<const L2PipeKernel*> l2pipe_variants(int prec, int64_t n, int dir) {
  std::vector<const L2PipeKernel*> v;
  for (const auto& k : l2pipe_table())
    if (k.prec == prec && int64_t(k.n1) * k.n2 == n && k.dir == dir) v.push_back(&k);
  return v;
}

const TwoPassKernel* find_twopass(int prec, int64_t n, int dir, int te, int emax) {
  for (const auto& k : twopass_table())
    if (k.prec == prec && int64_t(k.n1) * k.n2 == n && k.dir == dir && (te == 0 || k.te == te) &&
        (emax == 0 || k.emax == emax))
      return &k;
  return nullptr;
}

std::vector<const TwoPassKernel*> twopass_variants(int prec, int64_t n, int dir) {
  std::vector<const TwoPassKernel*> v;
  for (const auto& k : twopass_table())
    if (k.prec == prec && int64_t(k.n1) * k.n2 == n && k.dir == dir) v.push_back(&k);
  return v;
}

const Pow2Kernel* find_pow2(int prec, int n, int ept, int dir) {
  for (const auto& k : pow2_table())
    if (k.prec == prec && k.n == n && k.ept == ept && k.dir == dir) return &k;
  return nullptr;
}

std::vector<const Pow2Kernel*> pow2_variants(int prec, int n, int dir) {
  std::vector<const Pow2Kernel*> v;
  for (const auto& k : pow2_table())
    if (k.prec == prec && k.n == n && k.dir == dir) v.push_back(&k);
  std::sort(v.begin(), v.end(), [](auto a, auto b) { return a->ept < b->ept; });
  return v;
}

cudaError_t prepare_kernels() {
  static std::mutex mu;
  static std::vector<int> done;  // devices already prepared
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  if (std::find(done.begin(), done.end(), dev) != done.end()) return cudaSuccess;
  for (const auto& k : pow2_table()) {
    if (k.smem > 48 * 1024) {
      e = cudaFuncSetAttribute(k.func, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
      if (e != cudaSuccess) return e;
    }
  }
  for (const auto& k : twopass_table()) {
    if (k.smem > 48 * 1024) {
      for (const void* f : {k.func, k.split_func[0], k.split_func[1]}) {
        e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
        if (e != cudaSuccess) return e;
      }
    }
  }
  for (const auto& k : threepass_table())
    if (k.smem > 48 * 1024)
      for (const void* f : k.func) {
        e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
        if (e != cudaSuccess) return e;
      }
  done.push_back(dev);
  return cudaSuccess;
}

// ---------------------------------------------------------------- twiddles

// W_n^m in FP64: the angle is folded into (-1/2, 1/2] turns with integer
// arithmetic first, so sincospi sees an argument of at most 1 in magnitude
// and the result is accurate to a few ulp of double before rounding to the
// element type.
template <typename C>
__global__ void k_twiddles(C* tw, int64_t n, int64_t count, int64_t step) {
  using Re = typename RealOf<C>::type;
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < count; j += int64_t(gridDim.x) * blockDim.x) {
    int64_t mm = (j * step) % n;  // callers keep j*step < 2^62
    if (2 * mm > n) mm -= n;  // exp(-2πi m/n) == exp(-2πi (m-n)/n)
    double s, c;
    sincospi(-2.0 * double(mm) / double(n), &s, &c);
    tw[j] = C{Re(c), Re(s)};
  }
}

gfft_status fill_twiddles(int prec, void* dst, int64_t n, int64_t count, int64_t step, cudaStream_t st) {
  int blocks = int(std::min<int64_t>((count + 255) / 256, 4096));
  if (blocks < 1) return GFFT_OK;
  if (prec == kC64)
    k_twiddles<float2><<<blocks, 256, 0, st>>>(static_cast<float2*>(dst), n, count, step);
  else
    k_twiddles<double2><<<blocks, 256, 0, st>>>(static_cast<double2*>(dst), n, count, step);
  GFFT_CUDA(cudaGetLastError());
  return GFFT_OK;
}

gfft_status make_twiddles(int prec, int64_t n, void** out, cudaStream_t st) {
  *out = nullptr;
  void* p = nullptr;
  GFFT_CUDA(cudaMalloc(&p, size_t(n) * elem_bytes(prec)));
  gfft_status s = fill_twiddles(prec, p, n, n, 1, st);
  if (s != GFFT_OK) {
    cudaFree(p);
    return s;
  }
  *out = p;
  return GFFT_OK;
}

// ---------------------------------------------------------------- workspace

// Per-call workspace (two-pass scratch, Bluestein and N-D temporaries, host
// staging) comes from one stream-ordered pool per device that keeps freed
// memory (release threshold = max): the device's default pool returns its
// memory at every synchronize, so each call would map its workspace anew.
cudaError_t ws_alloc(void** p, size_t bytes, cudaStream_t st) {
  static std::mutex mu;
  static std::vector<std::pair<int, cudaMemPool_t>> pools;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> g(mu);
    for (auto& kv : pools)
      if (kv.first == dev) pool = kv.second;
    if (!pool) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&pool, &props);
      if (e != cudaSuccess) return e;
      uint64_t keep = ~uint64_t(0);
      e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
      pools.emplace_back(dev, pool);
    }
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

// ---------------------------------------------------------------- copy kernel

template <typename C>
__global__ void k_copy_batch(C* dst, const C* src, int64_t n, int64_t count, int64_t idist, int64_t odist) {
  const int64_t total = n * count;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    int64_t b = e / n, i = e - b * n;
    dst[b * odist + i] = src[b * idist + i];
  }
}

// ---------------------------------------------------------------- schedules

static int ilog2(int64_t n) {
  int l = 0;
  while ((int64_t(1) << l) < n) ++l;
  return l;
}

// Default elements-per-thread of the single-pass kernel (the autotuner may
// override it through wisdom): enough threads per transform for coalesced
// 128-byte rows, radix-32 stages where the register budget allows.
static int default_ept(int prec, int64_t n) {
  if (n <= 4) return int(n);
  if (n == 8) return 4;
  if (n <= 64) return n == 16 ? 4 : 8;
  if (n <= 256) return 16;
  if (prec == kC64 && n == 1024) return 32;
  if (prec == kC64 && n == 16384) return 16;
  return 16;
}

static std::string twopass_token(const TwoPassKernel* k);
static std::string threepass_token(const ThreePassKernel* k);

// Two-pass plan: tables W_N1, W_N2 and the split table of W_N in one
// allocation; slot geometry sized so the live intermediate stays in L2.
static gfft_status init_twopass(PlanCore* c, const TwoPassKernel* f, const TwoPassKernel* inv) {
  const int64_t n = c->n, n1 = f->n1, n2 = f->n2;
  const size_t es = elem_bytes(c->prec);
  int shift = (ilog2(n) + 1) / 2;
  const int64_t nlo = int64_t(1) << shift, nhi = n >> shift;
  GFFT_CUDA(cudaMalloc(&c->tw, size_t(n1 + n2 + nlo + nhi) * es));
  char* base = static_cast<char*>(c->tw);
  gfft_status s = fill_twiddles(c->prec, base, n1, n1, 1, 0);
  if (s == GFFT_OK) s = fill_twiddles(c->prec, base + n1 * es, n2, n2, 1, 0);
  if (s == GFFT_OK) s = fill_twiddles(c->prec, base + (n1 + n2) * es, n, nlo, 1, 0);
  if (s == GFFT_OK) s = fill_twiddles(c->prec, base + (n1 + n2 + nlo) * es, n, nhi, nlo, 0);
  if (s != GFFT_OK) return s;
  GFFT_CUDA(cudaStreamSynchronize(0));
  c->tp[0] = f;
  c->tp[1] = inv;
  c->tw1 = base;
  c->tw2 = base + n1 * es;
  c->bt_lo = base + (n1 + n2) * es;
  c->bt_hi = base + (n1 + n2 + nlo) * es;
  c->bt_shift = shift;
  const int64_t slot_target = int64_t(8) << 20, live_target = int64_t(48) << 20;
  const int64_t tbytes = n * int64_t(es);
  c->group = int(std::max<int64_t>(1, slot_target / tbytes));
  c->slots = int(std::max<int64_t>(2, std::min<int64_t>(8, live_target / (c->group * tbytes))));
  int dev = 0, sms = 0, occ = 0;
  GFFT_CUDA(cudaGetDevice(&dev));
  GFFT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GFFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f->func, f->tpb, f->smem));
  c->resident = std::max(1, sms * std::max(occ, 1));
  GFFT_CUDA(cudaMalloc(&c->status, sizeof(unsigned)));
  GFFT_CUDA(cudaMemset(c->status, 0, sizeof(unsigned)));
  c->algo = Algo::TwoPass;
  c->name = twopass_token(f);
  return GFFT_OK;
}

static std::string l2pipe_token(const L2PipeKernel* k, int gmb) {
  return "gpu-sm100-l2p-" + std::to_string(k->n1) + "x" + std::to_string(k->n2) + "-c" + std::to_string(k->nc1) +
         "x" + std::to_string(k->nc2) + "-e" + std::to_string(k->ept1) + "x" + std::to_string(k->ept2) + "-s" +
         std::to_string(k->nst) + "-g" + std::to_string(gmb);
}

// L2-pipelined plan: the two-pass tables of the same split (and its split
// kernels, for buffers the copy engine cannot address), groups of about
// gmb MB in three scratch slots.
static gfft_status init_l2pipe(PlanCore* c, const L2PipeKernel* f, const L2PipeKernel* inv, int gmb) {
  const TwoPassKernel* tf = nullptr;
  const TwoPassKernel* ti = nullptr;
  for (const TwoPassKernel* k : twopass_variants(c->prec, c->n, -1))
    if (k->n1 == f->n1 && !tf) tf = k;
  for (const TwoPassKernel* k : twopass_variants(c->prec, c->n, +1))
    if (k->n1 == f->n1 && tf && k->te == tf->te && k->emax == tf->emax) ti = k;
  if (!tf || !ti) {
    set_error("no two-pass kernel of the split " + std::to_string(f->n1) + " x " + std::to_string(f->n2));
    return GFFT_ERR_NOT_IMPLEMENTED;
  }
  gfft_status s = init_twopass(c, tf, ti);
  if (s != GFFT_OK) return s;
  c->l2[0] = f;
  c->l2[1] = inv;
  c->l2_gmb = gmb;
  c->l2_slots = 3;
  c->algo = Algo::L2Pipe;
  c->name = l2pipe_token(f, gmb);
  return GFFT_OK;
}

// Three-pass plan: W_N1 | W_M1 | W_M2 | split W_N | split W_M in one
// allocation.
static gfft_status init_threepass(PlanCore* c, const ThreePassKernel* f, const ThreePassKernel* inv) {
  const int64_t n = c->n, n1 = f->n1, m1 = f->m1, m2 = f->m2, m = m1 * m2;
  const size_t es = elem_bytes(c->prec);
  const int shn = (ilog2(n) + 1) / 2, shm = (ilog2(m) + 1) / 2;
  const int64_t nlo = int64_t(1) << shn, nhi = n >> shn, mlo = int64_t(1) << shm, mhi = m >> shm;
  const int64_t total = n1 + m1 + m2 + nlo + nhi + mlo + mhi;
  GFFT_CUDA(cudaMalloc(&c->tw, size_t(total) * es));
  char* base = static_cast<char*>(c->tw);
  int64_t off = 0;
  auto put = [&](int64_t len, int64_t cnt, int64_t step, const void** where) -> gfft_status {
    gfft_status s = fill_twiddles(c->prec, base + off * es, len, cnt, step, 0);
    if (where) *where = base + off * es;
    off += cnt;
    return s;
  };
  gfft_status s = put(n1, n1, 1, &c->tw1);
  if (s == GFFT_OK) s = put(m1, m1, 1, &c->tw2);
  if (s == GFFT_OK) s = put(m2, m2, 1, &c->tw3);
  if (s == GFFT_OK) s = put(n, nlo, 1, &c->bt_lo);
  if (s == GFFT_OK) s = put(n, nhi, nlo, &c->bt_hi);
  if (s == GFFT_OK) s = put(m, mlo, 1, &c->btm_lo);
  if (s == GFFT_OK) s = put(m, mhi, mlo, &c->btm_hi);
  if (s != GFFT_OK) return s;
  GFFT_CUDA(cudaStreamSynchronize(0));
  c->bt_shift = shn;
  c->btm_shift = shm;
  GFFT_CUDA(cudaMalloc(&c->status, sizeof(unsigned)));
  GFFT_CUDA(cudaMemset(c->status, 0, sizeof(unsigned)));
  c->t3[0] = f;
  c->t3[1] = inv;
  c->algo = Algo::ThreePass;
  c->name = threepass_token(f);
  return GFFT_OK;
}

static std::string pow2_token(int n, int ept) {
  return "gpu-sm100-p2-n" + std::to_string(n) + "-e" + std::to_string(ept);
}

static std::string threepass_token(const ThreePassKernel* k) {
  std::string t = std::string(k->tma ? "gpu-sm100-tp3t-" : "gpu-sm100-tp3-") + std::to_string(k->n1) + "x" +
                  std::to_string(k->m1) + "x" + std::to_string(k->m2);
  if (k->tma) t += "-t" + std::to_string(k->te) + "-e" + std::to_string(k->emax) + "-s" + std::to_string(k->nst);
  return t;
}

static std::string twopass_token(const TwoPassKernel* k) {
  return "gpu-sm100-tp-" + std::to_string(k->n1) + "x" + std::to_string(k->n2) + "-t" + std::to_string(k->te) +
         "-e" + std::to_string(k->emax);
}

std::vector<std::string> variant_tokens(int prec, int64_t n) {
  std::vector<std::string> v;
  if (n > 1 && (n & (n - 1)) == 0) {
    if (n <= (prec == kC64 ? 16384 : 8192))
      for (const Pow2Kernel* k : pow2_variants(prec, int(n), -1)) v.push_back(pow2_token(k->n, k->ept));
    for (const TwoPassKernel* k : twopass_variants(prec, n, -1)) v.push_back(twopass_token(k));
    for (const L2PipeKernel* k : l2pipe_variants(prec, n, -1))
      for (int gmb : {8, 16}) v.push_back(l2pipe_token(k, gmb));
    for (const ThreePassKernel* k : threepass_variants(prec, n, -1)) v.push_back(threepass_token(k));
  } else if (n > 1 && is_smooth7(n)) {
    // runtime-radix schedules (single CTA when it fits, two passes when n
    // has a 7-smooth divisor >= 2 below sqrt n) against Bluestein
    // (planner.go:50-55 picks by smoothness alone)
    for (const std::string& t : mixed_tokens(prec, n)) v.push_back(t);
    v.push_back("gpu-sm100-bluestein-n" + std::to_string(n));
  } else if (n > 1) {
    // Bluestein: a smaller mixed FFT length (a product of compiled column
    // lengths) against NextPow2(2n - 1)
    int64_t m1 = 0;
    if (bs_mixed_choice(n, &m1) > 0) {
      v.push_back("gpu-sm100-bluestein-n" + std::to_string(n) + "-mx");
      v.push_back("gpu-sm100-bluestein-n" + std::to_string(n) + "-p2");
    }
  }
  return v;
}

static gfft_status init_pow2(PlanCore* c, int ept) {
  const Pow2Kernel* f = find_pow2(c->prec, int(c->n), ept, -1);
  const Pow2Kernel* i = find_pow2(c->prec, int(c->n), ept, +1);
  if (!f || !i) {
    set_error("no compiled power-of-two kernel for this size");
    return GFFT_ERR_NOT_IMPLEMENTED;
  }
  c->algo = Algo::Pow2Smem;
  c->k[0] = f;
  c->k[1] = i;
  gfft_status s = make_twiddles(c->prec, c->n, &c->tw, 0);
  if (s != GFFT_OK) return s;
  GFFT_CUDA(cudaStreamSynchronize(0));
  c->name = pow2_token(int(c->n), ept);
  return GFFT_OK;
}

gfft_status core_init_variant(PlanCore* c, int prec, int64_t n, int device, const std::string& tok) {
  c->prec = prec;
  c->n = n;
  c->device = device;
  GFFT_CUDA(prepare_kernels());
  int a = 0, b = 0, te = 0, e = 0;
  if (std::sscanf(tok.c_str(), "gpu-sm100-p2-n%d-e%d", &a, &e) == 2 && a == n) return init_pow2(c, e);
  if (std::sscanf(tok.c_str(), "gpu-sm100-tp-%dx%d-t%d-e%d", &a, &b, &te, &e) == 4 && int64_t(a) * b == n) {
    const TwoPassKernel* f = find_twopass(prec, n, -1, te, e);
    const TwoPassKernel* i = find_twopass(prec, n, +1, te, e);
    if (f && i) return init_twopass(c, f, i);
  }
  if (std::sscanf(tok.c_str(), "gpu-sm100-tp3-%dx%dx%d", &a, &b, &te) == 3 && int64_t(a) * b * te == n) {
    const ThreePassKernel* f = find_threepass(prec, n, -1);
    const ThreePassKernel* i = find_threepass(prec, n, +1);
    if (f && i && f->n1 == a && f->m1 == b && f->m2 == te) return init_threepass(c, f, i);
  }
  int m2 = 0, ns = 0;
  {
    int c1 = 0, c2 = 0, e1 = 0, e2 = 0, gmb = 0;
    if (std::sscanf(tok.c_str(), "gpu-sm100-l2p-%dx%d-c%dx%d-e%dx%d-s%d-g%d", &a, &b, &c1, &c2, &e1, &e2, &ns, &gmb) ==
            8 &&
        int64_t(a) * b == n && gmb >= 1 && gmb <= 64) {
      const L2PipeKernel* f = find_l2pipe(prec, n, -1, a, c1, c2, ns);
      const L2PipeKernel* i = find_l2pipe(prec, n, +1, a, c1, c2, ns);
      if (f && i && f->ept1 == e1 && f->ept2 == e2) return init_l2pipe(c, f, i, gmb);
    }
  }
  if (std::sscanf(tok.c_str(), "gpu-sm100-tp3t-%dx%dx%d-t%d-e%d-s%d", &a, &b, &m2, &te, &e, &ns) == 6 &&
      int64_t(a) * b * m2 == n) {
    const ThreePassKernel* f = find_threepass(prec, n, -1, 1, te, e, ns);
    const ThreePassKernel* i = find_threepass(prec, n, +1, 1, te, e, ns);
    if (f && i && f->n1 == a && f->m1 == b && f->m2 == m2) return init_threepass(c, f, i);
  }
  long long ln = 0, l1 = 0, l2 = 0;
  if (std::sscanf(tok.c_str(), "gpu-sm100-mixed-n%lld", &ln) == 1 && ln == n && is_smooth7(n)) return init_generic(c);
  if (std::sscanf(tok.c_str(), "gpu-sm100-mixr-n%lld", &ln) == 1 && ln == n && is_smooth7(n)) return init_generic(c, true);
  if (std::sscanf(tok.c_str(), "gpu-sm100-mixed2-%lldx%lld", &l1, &l2) == 2 && l1 * l2 == n && is_smooth7(n)) {
    gfft_status s = init_gen_twopass(c);
    if (s == GFFT_OK && c->gn1 == l1) return s;
    core_free(c);
  }
  if (std::sscanf(tok.c_str(), "gpu-sm100-mixc-%lldx%lld", &l1, &l2) == 2 && l1 * l2 == n && is_smooth7(n)) {
    gfft_status s = init_gen_twopass(c, true);
    if (s == GFFT_OK && c->gn1 == l1) return s;
    core_free(c);
  }
  if (std::sscanf(tok.c_str(), "gpu-sm100-bluestein-n%lld", &ln) == 1 && ln == n && n >= 2) {
    const std::string head = "gpu-sm100-bluestein-n" + std::to_string(n);
    const bool mx = tok.compare(0, head.size() + 3, head + "-mx") == 0;
    const bool p2 = tok.compare(0, head.size() + 3, head + "-p2") == 0;
    return init_bluestein(c, mx ? kBsMixed : p2 ? kBsPow2 : kBsAuto);
  }
  if (std::sscanf(tok.c_str(), "gpu-sm100-tc16-n%lld", &ln) == 1 && ln == n) return init_tc(c);
  set_error("unknown or uncompiled variant '" + tok + "' for length " + std::to_string(n));
  return GFFT_ERR_INVALID_ARGUMENT;
}

// SetKernelStrategy / RecordBenchmarkDecision (plan.go:110-125,
// internal/planner/selection.go:22-60): a process-wide strategy that
// overrides automatic selection for plans created with KernelAuto, and
// per-length strategy classes used while selection is automatic.
namespace {
std::atomic<int> g_strategy{GFFT_KERNEL_AUTO};
std::mutex g_decision_mu;
std::map<int64_t, int> g_decisions;
}  // namespace

void set_kernel_strategy(int s) { g_strategy.store(s); }
int get_kernel_strategy() { return g_strategy.load(); }
void record_decision(int64_t n, int s) {
  std::lock_guard<std::mutex> g(g_decision_mu);
  g_decisions[n] = s;
}

static int recorded_decision(int64_t n) {
  std::lock_guard<std::mutex> g(g_decision_mu);
  auto it = g_decisions.find(n);
  return it == g_decisions.end() ? GFFT_KERNEL_AUTO : it->second;
}

gfft_status core_init(PlanCore* c, int prec, int64_t n, int device, int strategy, const PlanHint* hint) {
  // the process-wide strategy and recorded decisions steer the plans users
  // create, not the sub-plans built inside other schedules
  const bool user = hint && hint->user;
  if (user && strategy == GFFT_KERNEL_AUTO) strategy = g_strategy.load();
  c->prec = prec;
  c->n = n;
  c->device = device;
  if (n == 1) {
    c->algo = Algo::Trivial;
    c->name = "gpu-sm100-copy-n1";
    return GFFT_OK;
  }
  GFFT_CUDA(prepare_kernels());
  const bool pow2 = (n & (n - 1)) == 0;
  const int64_t max_single = prec == kC64 ? 16384 : 8192;
  if (strategy == GFFT_KERNEL_AUTO) {
    std::string tok;
    if (wisdom_lookup(n, prec, &tok) && core_init_variant(c, prec, n, device, tok) == GFFT_OK) return GFFT_OK;
    core_free(c);
    // PlannerMeasure/Patient/Exhaustive (plan_options.go:15-33): time the
    // compiled variants once and remember the winner in the wisdom store
    // (internal/fft/measure.go:89-141); later plans reuse it.
    if (hint && hint->planner >= GFFT_PLANNER_MEASURE && hint->planner <= GFFT_PLANNER_EXHAUSTIVE &&
        variant_tokens(prec, n).size() > 1) {
      const int iters = hint->planner == GFFT_PLANNER_MEASURE ? 10 : hint->planner == GFFT_PLANNER_PATIENT ? 50 : 100;
      std::string best, report;
      gfft_status ts = autotune(prec, n, hint->batch > 0 ? hint->batch : 0, iters, &best, &report);
      if (ts != GFFT_OK) return ts;
      if (!best.empty() && core_init_variant(c, prec, n, device, best) == GFFT_OK) return GFFT_OK;
      core_free(c);
    }
    if (hint && hint->planner == GFFT_PLANNER_LEARNED && learned_choose(prec, n, *hint, &tok) &&
        core_init_variant(c, prec, n, device, tok) == GFFT_OK)
      return GFFT_OK;
    core_free(c);
    c->prec = prec;
    c->n = n;
    c->device = device;
    clear_error();
    if (user) strategy = recorded_decision(n);  // a recorded class, else the size-class rules
  }
  // A forced strategy (SetKernelStrategy / PlanOptions.Strategy,
  // internal/planner/selection.go:71-78) picks the schedule class: the
  // step kernels map to the two-pass schedule, DIT/Stockham to the
  // single-pass one; a class that cannot serve n falls back to auto.
  const bool want_twopass = strategy == GFFT_KERNEL_SIXSTEP || strategy == GFFT_KERNEL_EIGHTSTEP;
  const bool want_single = strategy == GFFT_KERNEL_DIT || strategy == GFFT_KERNEL_STOCKHAM;
  const bool want_bluestein = strategy == GFFT_KERNEL_BLUESTEIN;
  if (pow2 && n <= max_single && !want_twopass && !want_bluestein) return init_pow2(c, default_ept(prec, n));
  if (pow2 && !want_single && strategy != GFFT_KERNEL_BLUESTEIN) {
    const TwoPassKernel* f = find_twopass(prec, n, -1, prec == kC64 ? 8192 : 4096, prec == kC64 ? 16 : 8);
    const TwoPassKernel* i = find_twopass(prec, n, +1, prec == kC64 ? 8192 : 4096, prec == kC64 ? 16 : 8);
    if (f && i) return init_twopass(c, f, i);
  }
  if (pow2 && n <= max_single && strategy != GFFT_KERNEL_BLUESTEIN) return init_pow2(c, default_ept(prec, n));
  if (pow2 && strategy != GFFT_KERNEL_BLUESTEIN) {
    const TwoPassKernel* f = find_twopass(prec, n, -1);
    const TwoPassKernel* i = find_twopass(prec, n, +1);
    if (f && i) return init_twopass(c, f, i);
  }
  // 7-smooth lengths run the runtime-radix Stockham (one CTA per transform
  // when it fits, else two passes); everything else, or a forced
  // KernelBluestein, goes through Bluestein (planner.go:50-55).
  if (strategy != GFFT_KERNEL_BLUESTEIN && is_smooth7(n)) {
    gfft_status s = init_generic(c, true);
    if (s == GFFT_OK) return s;
    core_free(c);
    s = init_generic(c);
    if (s == GFFT_OK) return s;
    core_free(c);
    s = init_gen_twopass(c, true);
    if (s == GFFT_OK) return s;
    core_free(c);
    s = init_gen_twopass(c);
    if (s == GFFT_OK) return s;
    core_free(c);
  }
  if (n >= 2 && n <= (int64_t(1) << 26)) return init_bluestein(c);
  set_error("length " + std::to_string(n) + " has no GPU schedule");
  return GFFT_ERR_INVALID_LENGTH;
}

unsigned core_device_status(const PlanCore* c) {
  if (!c->status) return 0;
  unsigned v = 0;
  if (cudaMemcpy(&v, c->status, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
  return v;
}

void core_free(PlanCore* c) {
  for (void** p : {&c->tw, reinterpret_cast<void**>(&c->status)}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (c->sub) {
    core_free(c->sub);
    delete c->sub;
    c->sub = nullptr;
  }
  c->mixc = false;
  c->mixr = false;
  c->bsm = false;
  c->algo = Algo::Trivial;
}

// Two-pass execution in the split schedule (k_tp_split): per chunk of up to
// 1 GiB of intermediate, one pass-1 launch and one pass-2 launch.  The
// scratch comes from the library's workspace pool.
static gfft_status exec_twopass(const PlanCore* c, int dir, void* dst, const void* src, int64_t count,
                                int64_t idist, int64_t odist, cudaStream_t st) {
  const TwoPassKernel* k = c->tp[dir < 0 ? 0 : 1];
  const int64_t tbytes = c->n * int64_t(elem_bytes(c->prec));
  const int64_t nb = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(1) << 30) / tbytes));
  void* ws = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&ws), size_t(nb) * size_t(tbytes), st));
  TwoPassParams p{};
  p.src = src;
  p.dst = dst;
  p.scratch = ws;
  p.count = count;
  p.idist = idist;
  p.odist = odist;
  p.tw1 = c->tw1;
  p.tw2 = c->tw2;
  p.bt.lo = c->bt_lo;
  p.bt.hi = c->bt_hi;
  p.bt.shift = c->bt_shift;
  p.scale = dir < 0 ? 1.0 : 1.0 / double(c->n);
  p.status = c->status;
  p.spin_limit = 1u << 22;
  cudaError_t e = cudaSuccess;
  for (int64_t b0 = 0; b0 < count && e == cudaSuccess; b0 += nb) {
    const int64_t m = std::min(nb, count - b0);
    e = k->split(p, 1, b0, m, st);
    if (e == cudaSuccess) e = k->split(p, 2, b0, m, st);
  }
  cudaFreeAsync(ws, st);
  if (e != cudaSuccess) return cuda_status(e, "k_tp_split");
  return GFFT_OK;
}

// Three-pass execution: per chunk of up to 1 GiB of intermediate, one
// launch per pass (pass 2 works in place on the intermediate).
static gfft_status exec_threepass(const PlanCore* c, int dir, void* dst, const void* src, int64_t count,
                                  int64_t idist, int64_t odist, cudaStream_t st) {
  const ThreePassKernel* k = c->t3[dir < 0 ? 0 : 1];
  const int64_t tbytes = c->n * int64_t(elem_bytes(c->prec));
  const int64_t nb = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(1) << 30) / tbytes));
  void* ws = nullptr;
  GFFT_CUDA(ws_alloc(&ws, size_t(nb) * size_t(tbytes), st));
  ThreePassParams p{};
  p.src = src;
  p.dst = dst;
  p.scratch = ws;
  p.idist = idist;
  p.odist = odist;
  p.tw1 = c->tw1;
  p.tw2 = c->tw2;
  p.tw3 = c->tw3;
  p.bt.lo = c->bt_lo;
  p.bt.hi = c->bt_hi;
  p.bt.shift = c->bt_shift;
  p.btm.lo = c->btm_lo;
  p.btm.hi = c->btm_hi;
  p.btm.shift = c->btm_shift;
  p.scale = dir < 0 ? 1.0 : 1.0 / double(c->n);
  p.status = c->status;
  p.spin_limit = 1u << 22;
  cudaError_t e = cudaSuccess;
  for (int64_t b0 = 0; b0 < count && e == cudaSuccess; b0 += nb) {
    const int64_t m = std::min(nb, count - b0);
    for (int pass = 1; pass <= 3 && e == cudaSuccess; ++pass) e = k->launch(p, pass, b0, m, st);
  }
  cudaFreeAsync(ws, st);
  if (e != cudaSuccess) return cuda_status(e, "k_tp3");
  return GFFT_OK;
}

// L2-pipelined execution: one persistent launch over the whole batch, the
// intermediate in S slots of G transforms (about l2_gmb MB each) that stay
// in L2, the work counter and per-group completion counters cleared first.
static gfft_status exec_l2pipe(const PlanCore* c, int dir, void* dst, const void* src, int64_t count,
                               int64_t idist, int64_t odist, cudaStream_t st) {
  const L2PipeKernel* k = c->l2[dir < 0 ? 0 : 1];
  const int64_t tbytes = c->n * int64_t(elem_bytes(c->prec));
  const int64_t G = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(c->l2_gmb) << 20) / tbytes));
  const int64_t groups = (count + G - 1) / G;
  const int S = c->l2_slots;
  const int64_t tiles = groups * G * (k->n2 / k->nc1 + k->n1 / k->nc2);
  if (tiles >= (int64_t(1) << 31)) return exec_twopass(c, dir, dst, src, count, idist, odist, st);
  const size_t ctr_bytes = (size_t(1 + 2 * groups) * sizeof(unsigned) + 1023) & ~size_t(1023);
  void* ws = nullptr;
  GFFT_CUDA(ws_alloc(&ws, ctr_bytes + size_t(S) * size_t(G) * size_t(tbytes), st));
  cudaError_t e = cudaMemsetAsync(ws, 0, ctr_bytes, st);
  L2pParams p{};
  p.src = src;
  p.dst = dst;
  p.scratch = static_cast<char*>(ws) + ctr_bytes;
  p.ctr = static_cast<unsigned*>(ws);
  p.status = c->status;
  p.count = count;
  p.idist = idist;
  p.odist = odist;
  p.tw1 = c->tw1;
  p.tw2 = c->tw2;
  p.bt.lo = c->bt_lo;
  p.bt.hi = c->bt_hi;
  p.bt.shift = c->bt_shift;
  p.scale = dir < 0 ? 1.0 : 1.0 / double(c->n);
  p.G = int(G);
  p.S = S;
  p.groups = int(groups);
  p.spin_limit = 1u << 22;
  if (e == cudaSuccess) e = k->launch(p, st);
  cudaFreeAsync(ws, st);
  if (e == cudaErrorNotSupported) {  // buffers the copy engine cannot address
    cudaGetLastError();
    return exec_twopass(c, dir, dst, src, count, idist, odist, st);
  }
  if (e != cudaSuccess) return cuda_status(e, "k_l2p");
  return GFFT_OK;
}

gfft_status core_exec(const PlanCore* c, int dir, void* dst, const void* src, int64_t count, int64_t idist,
                      int64_t odist, cudaStream_t st) {
  if (count <= 0) return GFFT_OK;
  switch (c->algo) {
    case Algo::Trivial: {
      if (dst == src && idist == odist) return GFFT_OK;
      int blocks = int(std::min<int64_t>((count + 255) / 256, 65535));
      if (c->prec == kC64)
        k_copy_batch<float2><<<blocks, 256, 0, st>>>(static_cast<float2*>(dst), static_cast<const float2*>(src), 1,
                                                      count, idist, odist);
      else
        k_copy_batch<double2><<<blocks, 256, 0, st>>>(static_cast<double2*>(dst), static_cast<const double2*>(src),
                                                       1, count, idist, odist);
      GFFT_CUDA(cudaGetLastError());
      return GFFT_OK;
    }
    case Algo::TwoPass:
      return exec_twopass(c, dir, dst, src, count, idist, odist, st);
    case Algo::L2Pipe:
      return exec_l2pipe(c, dir, dst, src, count, idist, odist, st);
    case Algo::ThreePass:
      return exec_threepass(c, dir, dst, src, count, idist, odist, st);
    case Algo::Generic:
    case Algo::GenTwoPass:
    case Algo::Bluestein:
      return exec_runtime_plan(c, dir, dst, src, count, idist, odist, st);
    case Algo::TensorCore:
      return exec_tc(c, dir, dst, src, count, idist, odist, st);
    case Algo::Pow2Smem: {
      const Pow2Kernel* k = c->k[dir < 0 ? 0 : 1];
      const double scale = dir < 0 ? 1.0 : 1.0 / double(c->n);
      GFFT_CUDA(k->launch(src, dst, count, idist, odist, c->tw, scale, st));
      return GFFT_OK;
    }
  }
  return GFFT_ERR_NOT_IMPLEMENTED;
}

}  // namespace gfft
