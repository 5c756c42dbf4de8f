// N-dimensional plans (K6): Plan2D / Plan3D / PlanND (plan_2d.go, plan_3d.go,
// plan_nd.go) and PlanReal2D / PlanReal3D (plan_real_2d.go, plan_real_3d.go),
// plus batched strided transforms.
//
// Row-column decomposition, last axis first (plan_3d.go:319-403 order).  The
// last axis is contiguous and runs the 1-D batched plan.  Every other axis
// is a batch of columns: element j of column c at j*inner + c.  When the
// axis length is 7-smooth and a column tile fits shared memory, one launch
// of the runtime column kernel transforms the columns in place with
// NC-element coalesced rows; otherwise the axis is transposed to rows in
// scratch, transformed by the 1-D plan, and transposed back.  Real plans run
// the real-input plan on the last axis (compact n/2+1 spectrum) and complex
// column passes on the rest.
#include <algorithm>
#include <new>
#include <vector>
#include "gfft_internal.h"

namespace gfft {

// dst[b][c][r] = src[b][r][c] for r < rows, c < cols (32x32 tiles).
template <typename C>
__global__ void k_transpose(C* dst, const C* src, int64_t rows, int64_t cols, int64_t count, int64_t sdist,
                            int64_t ddist) {
  __shared__ C tile[32][33];
  const int64_t tr = (rows + 31) / 32, tc = (cols + 31) / 32;
  for (int64_t blk = blockIdx.x; blk < count * tr * tc; blk += gridDim.x) {
    const int64_t b = blk / (tr * tc), rem = blk % (tr * tc);
    const int64_t r0 = (rem / tc) * 32, c0 = (rem % tc) * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
      const int64_t r = r0 + i, c = c0 + threadIdx.x;
      if (r < rows && c < cols) tile[i][threadIdx.x] = src[b * sdist + r * cols + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
      const int64_t c = c0 + i, r = r0 + threadIdx.x;
      if (r < rows && c < cols) dst[b * ddist + c * rows + r] = tile[threadIdx.x][i];
    }
    __syncthreads();
  }
}

static gfft_status transpose(int prec, void* dst, const void* src, int64_t rows, int64_t cols, int64_t count,
                             int64_t sdist, int64_t ddist, cudaStream_t st) {
  const int64_t tiles = count * ((rows + 31) / 32) * ((cols + 31) / 32);
  const unsigned grid = unsigned(std::max<int64_t>(1, std::min<int64_t>(tiles, 148 * 16)));
  dim3 block(32, 8);
  if (prec == kC64)
    k_transpose<float2><<<grid, block, 0, st>>>(static_cast<float2*>(dst), static_cast<const float2*>(src), rows, cols,
                                                count, sdist, ddist);
  else
    k_transpose<double2><<<grid, block, 0, st>>>(static_cast<double2*>(dst), static_cast<const double2*>(src), rows,
                                                 cols, count, sdist, ddist);
  GFFT_CUDA(cudaGetLastError());
  return GFFT_OK;
}

// One transform axis of an N-D array: length n, columns `inner` apart,
// `outer` independent blocks of n*inner elements.
struct Axis {
  int64_t n = 1, inner = 1, outer = 1;
  PlanCore core;       // 1-D plan of length n (rows)
  bool cols = false;   // column kernel usable
  GenSched cs{};
  void* w = nullptr;   // W_n for the column kernel
};

static gfft_status axis_init(Axis* a, int prec, int64_t n, int64_t inner, int64_t outer, int device, int planner,
                             int64_t batch) {
  a->n = n;
  a->inner = inner;
  a->outer = outer;
  PlanHint hint;
  hint.planner = planner;
  hint.batch = std::max<int64_t>(1, batch) * inner * outer;  // transforms of this axis per call
  hint.stride = inner;
  hint.user = true;
  gfft_status s = core_init(&a->core, prec, n, device, GFFT_KERNEL_AUTO, &hint);
  if (s != GFFT_OK) return s;
  if (inner > 1 && n > 1 && column_sched(n, prec, &a->cs)) {
    s = make_twiddles(prec, n, &a->w, 0);
    if (s != GFFT_OK) return s;
    GFFT_CUDA(cudaStreamSynchronize(0));
    a->cols = true;
  }
  return GFFT_OK;
}

static void axis_free(Axis* a) {
  core_free(&a->core);
  if (a->w) cudaFree(a->w);
  a->w = nullptr;
}

// Transforms axis `a` of `reps` arrays `dist` apart (out may equal in).
static gfft_status axis_exec(const Axis& a, int prec, int dir, void* out, const void* in, int64_t reps,
                             int64_t dist, cudaStream_t st) {
  if (a.n == 1) {
    if (out != in) {
      GFFT_CUDA(cudaMemcpy2DAsync(out, size_t(dist) * elem_bytes(prec), in, size_t(dist) * elem_bytes(prec),
                                  size_t(a.outer * a.inner) * elem_bytes(prec), size_t(reps), cudaMemcpyDeviceToDevice,
                                  st));
    }
    return GFFT_OK;
  }
  const int64_t block = a.n * a.inner;  // elements per outer block
  if (a.inner == 1) {
    if (dist == a.outer * block) return core_exec(&a.core, dir, out, in, reps * a.outer, a.n, a.n, st);
    for (int64_t r = 0; r < reps; ++r) {
      const size_t off = size_t(r) * size_t(dist) * elem_bytes(prec);
      gfft_status s = core_exec(&a.core, dir, static_cast<char*>(out) + off, static_cast<const char*>(in) + off,
                                a.outer, a.n, a.n, st);
      if (s != GFFT_OK) return s;
    }
    return GFFT_OK;
  }
  if (a.cols) {
    if (dist == a.outer * block)
      return exec_columns(a.cs, prec, dir, out, in, reps * a.outer, block, a.inner, a.inner, a.w, st);
    for (int64_t r = 0; r < reps; ++r) {
      const size_t off = size_t(r) * size_t(dist) * elem_bytes(prec);
      gfft_status s = exec_columns(a.cs, prec, dir, static_cast<char*>(out) + off,
                                   static_cast<const char*>(in) + off, a.outer, block, a.inner, a.inner, a.w, st);
      if (s != GFFT_OK) return s;
    }
    return GFFT_OK;
  }
  // transpose [n][inner] -> [inner][n], rows, transpose back
  const size_t es = elem_bytes(prec);
  void* tmp = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&tmp), size_t(a.outer) * size_t(block) * es, st));
  gfft_status s = GFFT_OK;
  for (int64_t r = 0; r < reps && s == GFFT_OK; ++r) {
    const size_t off = size_t(r) * size_t(dist) * es;
    s = transpose(prec, tmp, static_cast<const char*>(in) + off, a.n, a.inner, a.outer, block, block, st);
    if (s == GFFT_OK) s = core_exec(&a.core, dir, tmp, tmp, a.outer * a.inner, a.n, a.n, st);
    if (s == GFFT_OK)
      s = transpose(prec, static_cast<char*>(out) + off, tmp, a.inner, a.n, a.outer, block, block, st);
  }
  cudaFreeAsync(tmp, st);
  return s;
}

// Full spectrum from the compact one (Hermitian symmetry): for the last
// index k >= h+1, X[i0.., k] = conj(X[-i0 mod n0, .., n-k]) (plan_real_2d.go:231-276).
template <typename C>
__global__ void k_expand_full(C* full, const C* compact, const int64_t* dims, int nd, int64_t total, int64_t reps,
                              int64_t fdist, int64_t cdist) {
  const int64_t n = dims[nd - 1], h1 = n / 2 + 1;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total * reps; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / total;
    int64_t rem = e % total;
    const int64_t k = rem % n;
    int64_t outer = rem / n;  // flattened leading index
    C v;
    if (k < h1) {
      v = compact[r * cdist + outer * h1 + k];
    } else {
      // negate every leading index
      int64_t neg = 0, mul = 1, o = outer;
      for (int d = nd - 2; d >= 0; --d) {
        const int64_t i = o % dims[d];
        o /= dims[d];
        neg += ((dims[d] - i) % dims[d]) * mul;
        mul *= dims[d];
      }
      v = cconj(compact[r * cdist + neg * h1 + (n - k)]);
    }
    full[r * fdist + rem] = v;
  }
}

// Compact half of a full spectrum (the part InverseFull feeds the inverse).
template <typename C>
__global__ void k_take_compact(C* compact, const C* full, int64_t n, int64_t rows, int64_t reps, int64_t fdist,
                               int64_t cdist) {
  const int64_t h1 = n / 2 + 1, total = rows * h1;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total * reps; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / total, rem = e % total, row = rem / h1, k = rem % h1;
    compact[r * cdist + rem] = full[r * fdist + row * n + k];
  }
}

}  // namespace gfft

using namespace gfft;

struct gfft_plan_nd {
  int prec = 0;
  bool real = false;
  int nd = 0;
  int64_t dims[8] = {};
  int64_t len = 1;   // elements of the input (reals for real plans)
  int64_t clen = 1;  // complex elements of the (compact) spectrum
  gfft_plan_options opts{};
  std::vector<Axis*> axes;  // complex axes, last first
  gfft_plan_real* rplan = nullptr;
  int64_t* ddims = nullptr;  // device copy of dims (full-spectrum expansion)
};

extern "C" GFFT_API void gfft_plan_nd_close(gfft_plan_nd* p);

extern "C" gfft_status gfft_plan_nd_new(gfft_plan_nd** out, int32_t precision, int32_t ndims, const int64_t* dims,
                                        int32_t real_input, const gfft_plan_options* opts) {
  clear_error();
  if (!out) return GFFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (ndims < 1 || ndims > 8 || !dims) return GFFT_ERR_INVALID_LENGTH;  // plan_nd.go:51-53
  for (int i = 0; i < ndims; ++i)
    if (dims[i] < 1) return GFFT_ERR_INVALID_LENGTH;                     // plan_nd.go:61-66
  if (real_input && (dims[ndims - 1] < 2 || dims[ndims - 1] % 2)) return GFFT_ERR_INVALID_LENGTH;
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  gfft_plan_options o{};
  if (opts) o = *opts;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GFFT_ERR_NO_DEVICE;
  if (o.device < 0 || o.device >= ndev) return GFFT_ERR_INVALID_ARGUMENT;
  DeviceGuard dg;
  GFFT_CUDA(dg.set(o.device));
  auto* p = new (std::nothrow) gfft_plan_nd;
  if (!p) return GFFT_ERR_OUT_OF_MEMORY;
  p->prec = precision;
  p->real = real_input != 0;
  p->nd = ndims;
  p->opts = o;
  for (int i = 0; i < ndims; ++i) {
    p->dims[i] = dims[i];
    p->len *= dims[i];
  }
  // complex view: real plans keep n/2+1 bins on the last axis
  int64_t cd[8];
  for (int i = 0; i < ndims; ++i) cd[i] = dims[i];
  if (p->real) cd[ndims - 1] = dims[ndims - 1] / 2 + 1;
  p->clen = 1;
  for (int i = 0; i < ndims; ++i) p->clen *= cd[i];
  gfft_status s = GFFT_OK;
  if (p->real) {
    gfft_plan_options ro{};
    ro.device = o.device;
    ro.planner = o.planner;  // (ro.batch would change the real plan's buffer layout)
    s = gfft_plan_real_new(&p->rplan, precision, dims[ndims - 1], &ro);
  }
  int64_t inner = 1;
  for (int i = ndims - 1; i >= 0 && s == GFFT_OK; --i) {
    const int64_t n = cd[i];
    const int64_t outer = p->clen / (n * inner);
    if (!(p->real && i == ndims - 1)) {
      Axis* a = new (std::nothrow) Axis;
      if (!a) {
        s = GFFT_ERR_OUT_OF_MEMORY;
        break;
      }
      p->axes.push_back(a);
      s = axis_init(a, precision, n, inner, outer, o.device, o.planner, o.batch);
    }
    inner *= n;
  }
  if (s == GFFT_OK && p->real) {
    cudaError_t e = cudaMalloc(&p->ddims, sizeof(int64_t) * 8);
    if (e == cudaSuccess) e = cudaMemcpy(p->ddims, p->dims, sizeof(int64_t) * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) s = cuda_status(e, "nd dims");
  }
  if (s != GFFT_OK) {
    gfft_plan_nd_close(p);
    return s;
  }
  *out = p;
  return GFFT_OK;
}

extern "C" void gfft_plan_nd_close(gfft_plan_nd* p) {
  if (!p) return;
  for (Axis* a : p->axes) {
    axis_free(a);
    delete a;
  }
  if (p->rplan) gfft_plan_real_close(p->rplan);
  if (p->ddims) cudaFree(p->ddims);
  delete p;
}

extern "C" int64_t gfft_plan_nd_len(const gfft_plan_nd* p) { return p ? p->len : 0; }
extern "C" int64_t gfft_plan_nd_spectrum_len(const gfft_plan_nd* p) { return p ? p->clen : 0; }

namespace gfft {

// plan_batch.go:3-19 resolveBatchStride (complex) / :21-42 (real): returns
// reps and the element distances between consecutive arrays.
static gfft_status nd_layout(const gfft_plan_nd* p, int64_t in_len, int64_t out_len, bool forward, int64_t* reps,
                             int64_t* din, int64_t* dout) {
  const int64_t a = forward ? p->len : p->clen;   // input elements per array
  const int64_t b = forward ? p->clen : p->len;   // output elements per array
  const int64_t ra = p->real ? a : p->len, rb = p->real ? b : p->len;
  if (p->opts.batch <= 1 && p->opts.stride <= 0) {
    if (in_len != ra || out_len != rb) return GFFT_ERR_LENGTH_MISMATCH;
    *reps = 1;
    *din = ra;
    *dout = rb;
    return GFFT_OK;
  }
  const int64_t n = p->opts.batch < 1 ? 1 : p->opts.batch;
  const int64_t si = p->opts.stride <= 0 ? ra : p->opts.stride;
  const int64_t so = p->opts.stride <= 0 ? rb : p->opts.stride;
  if (si < ra || so < rb) return GFFT_ERR_INVALID_STRIDE;
  if ((n - 1) * si + ra > in_len || (n - 1) * so + rb > out_len) return GFFT_ERR_LENGTH_MISMATCH;
  *reps = n;
  *din = si;
  *dout = so;
  return GFFT_OK;
}

static unsigned grid1(int64_t total) { return unsigned(std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 32))); }

// complex axes, last first; the first pass may read from `in`
static gfft_status nd_complex_axes(const gfft_plan_nd* p, int dir, void* out, const void* in, int64_t reps,
                                   int64_t dist, cudaStream_t st) {
  const void* cur = in;
  for (Axis* a : p->axes) {
    gfft_status s = axis_exec(*a, p->prec, dir, out, cur, reps, dist, st);
    if (s != GFFT_OK) return s;
    cur = out;
  }
  return GFFT_OK;
}

static gfft_status nd_forward(gfft_plan_nd* p, bool full, void* dst, const void* src, int64_t reps, int64_t din,
                              int64_t dout, cudaStream_t st) {
  if (!p->real) return nd_complex_axes(p, -1, dst, src, reps, din, st);
  const size_t es = elem_bytes(p->prec);
  const int64_t n = p->dims[p->nd - 1], h1 = n / 2 + 1, rows = p->len / n;
  void* comp = dst;
  int64_t cdist = dout;
  void* tmp = nullptr;
  if (full) {
    GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&tmp), size_t(reps) * size_t(p->clen) * es, st));
    comp = tmp;
    cdist = p->clen;
  }
  gfft_status s = GFFT_OK;
  for (int64_t r = 0; r < reps && s == GFFT_OK; ++r) {
    s = real_forward(p->rplan, 0, static_cast<char*>(comp) + size_t(r) * size_t(cdist) * es,
                     static_cast<const char*>(src) + size_t(r) * size_t(din) * es / 2, rows, n, h1, st);
  }
  if (s == GFFT_OK) s = nd_complex_axes(p, -1, comp, comp, reps, cdist, st);
  if (s == GFFT_OK && full) {
    if (p->prec == kC64)
      k_expand_full<float2><<<grid1(p->len * reps), 256, 0, st>>>(static_cast<float2*>(dst), static_cast<const float2*>(comp),
                                                                   p->ddims, p->nd, p->len, reps, dout, cdist);
    else
      k_expand_full<double2><<<grid1(p->len * reps), 256, 0, st>>>(static_cast<double2*>(dst), static_cast<const double2*>(comp),
                                                                    p->ddims, p->nd, p->len, reps, dout, cdist);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = cuda_status(e, "k_expand_full");
  }
  if (tmp) cudaFreeAsync(tmp, st);
  return s;
}

static gfft_status nd_inverse(gfft_plan_nd* p, bool full, void* dst, const void* src, int64_t reps, int64_t din,
                              int64_t dout, cudaStream_t st) {
  if (!p->real) return nd_complex_axes(p, +1, dst, src, reps, din, st);
  // the spectrum is not modified: column passes run on a copy
  const size_t es = elem_bytes(p->prec);
  const int64_t n = p->dims[p->nd - 1], h1 = n / 2 + 1, rows = p->len / n;
  void* tmp = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&tmp), size_t(reps) * size_t(p->clen) * es, st));
  cudaError_t e = cudaSuccess;
  if (full) {
    if (p->prec == kC64)
      k_take_compact<float2><<<grid1(p->clen * reps), 256, 0, st>>>(static_cast<float2*>(tmp), static_cast<const float2*>(src),
                                                                     n, rows, reps, din, p->clen);
    else
      k_take_compact<double2><<<grid1(p->clen * reps), 256, 0, st>>>(static_cast<double2*>(tmp), static_cast<const double2*>(src),
                                                                      n, rows, reps, din, p->clen);
    e = cudaGetLastError();
  } else {
    e = cudaMemcpy2DAsync(tmp, size_t(p->clen) * es, src, size_t(din) * es, size_t(p->clen) * es, size_t(reps),
                          cudaMemcpyDeviceToDevice, st);
  }
  gfft_status s = e == cudaSuccess ? GFFT_OK : cuda_status(e, "nd inverse staging");
  if (s == GFFT_OK) s = nd_complex_axes(p, +1, tmp, tmp, reps, p->clen, st);
  for (int64_t r = 0; r < reps && s == GFFT_OK; ++r) {
    s = real_inverse(p->rplan, static_cast<char*>(dst) + size_t(r) * size_t(dout) * es / 2,
                     static_cast<char*>(tmp) + size_t(r) * size_t(p->clen) * es, rows, n, h1, st);
  }
  cudaFreeAsync(tmp, st);
  return s;
}

static gfft_status nd_call(gfft_plan_nd* p, bool inverse, bool full, void* dst, int64_t dst_len, const void* src,
                           int64_t src_len, cudaStream_t st) {
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (full && !p->real) return GFFT_ERR_INVALID_ARGUMENT;
  int64_t reps, din, dout;
  gfft_status s;
  if (full) {
    // ForwardFull / InverseFull take full-size spectra (plan_real_2d.go:231,370)
    if (p->opts.batch > 1 || p->opts.stride > 0) return GFFT_ERR_NOT_IMPLEMENTED;
    if (src_len != p->len || dst_len != p->len) return GFFT_ERR_LENGTH_MISMATCH;
    reps = 1;
    din = dout = p->len;
    s = GFFT_OK;
  } else {
    s = nd_layout(p, src_len, dst_len, !inverse, &reps, &din, &dout);
  }
  if (s != GFFT_OK) return s;
  return inverse ? nd_inverse(p, full, dst, src, reps, din, dout, st) : nd_forward(p, full, dst, src, reps, din, dout, st);
}

// Host-slice wrapper (copies the whole slices in and out).
static gfft_status nd_host(gfft_plan_nd* p, bool inverse, bool full, void* dst, int64_t dst_len, const void* src,
                           int64_t src_len) {
  if (!p) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  const size_t es = elem_bytes(p->prec);
  const bool src_real = p->real && !inverse, dst_real = p->real && inverse;
  const size_t sb = size_t(src_len) * (src_real ? es / 2 : es), db = size_t(dst_len) * (dst_real ? es / 2 : es);
  cudaStream_t st = nullptr;
  GFFT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  void *ds = nullptr, *dd = nullptr;
  gfft_status s = GFFT_OK;
  cudaError_t e = ws_alloc(reinterpret_cast<void**>(&ds), sb ? sb : 1, st);
  if (e == cudaSuccess) e = ws_alloc(reinterpret_cast<void**>(&dd), db ? db : 1, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ds, src, sb, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dd, dst, db, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    s = nd_call(p, inverse, full, dd, dst_len, ds, src_len, st);
    if (s == GFFT_OK) e = cudaMemcpyAsync(dst, dd, db, cudaMemcpyDeviceToHost, st);
  }
  if (ds) cudaFreeAsync(ds, st);
  if (dd) cudaFreeAsync(dd, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) return cuda_status(e, "nd host path");
  if (e2 != cudaSuccess) return cuda_status(e2, "cudaStreamSynchronize");
  return s;
}

}  // namespace gfft

extern "C" {

gfft_status gfft_nd_forward(gfft_plan_nd* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                            void* stream) {
  clear_error();
  return nd_call(p, false, false, dst, dst_len, src, src_len, static_cast<cudaStream_t>(stream));
}
gfft_status gfft_nd_inverse(gfft_plan_nd* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                            void* stream) {
  clear_error();
  return nd_call(p, true, false, dst, dst_len, src, src_len, static_cast<cudaStream_t>(stream));
}
gfft_status gfft_nd_forward_full(gfft_plan_nd* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                 void* stream) {
  clear_error();
  return nd_call(p, false, true, dst, dst_len, src, src_len, static_cast<cudaStream_t>(stream));
}
gfft_status gfft_nd_inverse_full(gfft_plan_nd* p, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                 void* stream) {
  clear_error();
  return nd_call(p, true, true, dst, dst_len, src, src_len, static_cast<cudaStream_t>(stream));
}
gfft_status gfft_nd_forward_host(gfft_plan_nd* p, void* dst, int64_t dst_len, const void* src, int64_t src_len) {
  clear_error();
  return nd_host(p, false, false, dst, dst_len, src, src_len);
}
gfft_status gfft_nd_inverse_host(gfft_plan_nd* p, void* dst, int64_t dst_len, const void* src, int64_t src_len) {
  clear_error();
  return nd_host(p, true, false, dst, dst_len, src, src_len);
}

// Batched strided transforms of a 1-D plan: element j of transform b at
// b*dist + j*stride, same layout for dst and src.
gfft_status gfft_exec_strided_batch(gfft_plan* plan, int32_t direction, void* dst, int64_t dst_len, const void* src,
                                    int64_t src_len, int64_t count, int64_t stride, int64_t dist, void* stream) {
  clear_error();
  if (!plan) return GFFT_ERR_INVALID_ARGUMENT;
  if (!dst || !src) return GFFT_ERR_NIL_SLICE;
  if (direction != -1 && direction != 1) return GFFT_ERR_INVALID_ARGUMENT;
  if (count < 1) return GFFT_ERR_INVALID_LENGTH;
  if (stride < 1 || dist < 1) return GFFT_ERR_INVALID_STRIDE;
  const int64_t n = plan->core.n;
  if ((n - 1) > (INT64_MAX - 1 - (count - 1) * dist) / stride) return GFFT_ERR_INVALID_STRIDE;
  const int64_t required = (count - 1) * dist + (n - 1) * stride + 1;
  if (dst_len < required || src_len < required) return GFFT_ERR_LENGTH_MISMATCH;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DeviceGuard dg;
  GFFT_CUDA(dg.set(plan->core.device));
  const int prec = plan->core.prec;
  if (stride == 1) return core_exec(&plan->core, direction, dst, src, count, dist, dist, st);
  if (dist == 1 && count <= stride) {
    // columns: count adjacent transforms with rows `stride` apart
    GenSched cs;
    if (column_sched(n, prec, &cs)) {
      void* w = nullptr;
      GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&w), size_t(n) * elem_bytes(prec), st));
      gfft_status s = fill_twiddles(prec, w, n, n, 1, st);
      if (s == GFFT_OK) s = exec_columns(cs, prec, direction, dst, src, 1, 0, count, stride, w, st);
      cudaFreeAsync(w, st);
      return s;
    }
  }
  // general layout: gather into rows, transform, scatter back
  const size_t es = elem_bytes(prec);
  void* tmp = nullptr;
  GFFT_CUDA(ws_alloc(reinterpret_cast<void**>(&tmp), size_t(count) * size_t(n) * es, st));
  cudaError_t e = cudaSuccess;
  for (int64_t b = 0; b < count && e == cudaSuccess; ++b)
    e = cudaMemcpy2DAsync(static_cast<char*>(tmp) + size_t(b) * size_t(n) * es, es,
                          static_cast<const char*>(src) + size_t(b) * size_t(dist) * es, size_t(stride) * es, es,
                          size_t(n), cudaMemcpyDeviceToDevice, st);
  gfft_status s = e == cudaSuccess ? core_exec(&plan->core, direction, tmp, tmp, count, n, n, st) : cuda_status(e, "gather");
  for (int64_t b = 0; b < count && s == GFFT_OK && e == cudaSuccess; ++b)
    e = cudaMemcpy2DAsync(static_cast<char*>(dst) + size_t(b) * size_t(dist) * es, size_t(stride) * es,
                          static_cast<char*>(tmp) + size_t(b) * size_t(n) * es, es, es, size_t(n),
                          cudaMemcpyDeviceToDevice, st);
  cudaFreeAsync(tmp, st);
  if (e != cudaSuccess) return cuda_status(e, "scatter");
  return s;
}

}  // extern "C"
