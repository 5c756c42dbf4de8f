/*
 * gfft.h — C ABI of the B200 (sm_100a) FFT engine behind algo-fft's
 * batched-transform path.
 *
 * Every entry point takes plain pointers and sizes and returns a status code,
 * so a cgo binding can call it directly.  Each entry point names the
 * reference API it replaces as file:line inside CWBudde/algo-fft.
 *
 * Devices: a plan lives on the device of its options; every call on it runs
 * with that device current and gives the calling thread its previous current
 * device back before returning.  A stream passed in must belong to the
 * plan's device (or be NULL).
 *
 * Conventions
 *  - Complex data is interleaved (re, im): complex64 = 2 x float32,
 *    complex128 = 2 x float64, exactly Go's []complex64 / []complex128 layout.
 *  - Lengths (`*_len`) are counted in elements of the slice type, as Go's
 *    len() would report them.
 *  - Functions without the `_host` suffix take DEVICE pointers (the
 *    gpu.Buffer path, gpu/backend.go:29-37) and are ordered on `stream`
 *    (a cudaStream_t; NULL = the legacy default stream).  They return as soon
 *    as the work is queued.
 *  - Functions with the `_host` suffix take HOST pointers (the Go-slice
 *    path): they copy in, compute and copy out before returning, and retain
 *    no pointer after they return (cgo pointer rules).
 *  - Forward transforms are unscaled; inverse transforms scale by 1/n
 *    (plan.go:320-330, 372-385).
 *  - A plan is immutable after creation and may be used from several threads
 *    at once (plan.go:13-17); host-call staging buffers are per call.
 */
#ifndef GFFT_H
#define GFFT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GFFT_API __attribute__((visibility("default")))
#else
#define GFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1..6 map one-to-one onto the reference's sentinel errors
 * (errors.go:6-30); the Go binding converts them back to those values so
 * errors.Is keeps working.  100+ are device-side conditions the CPU library
 * never had. */
typedef enum gfft_status {
  GFFT_OK = 0,
  GFFT_ERR_INVALID_LENGTH = 1,   /* ErrInvalidLength   errors.go:11 */
  GFFT_ERR_NIL_SLICE = 2,        /* ErrNilSlice        errors.go:14 */
  GFFT_ERR_LENGTH_MISMATCH = 3,  /* ErrLengthMismatch  errors.go:18 */
  GFFT_ERR_INVALID_STRIDE = 4,   /* ErrInvalidStride   errors.go:22 */
  GFFT_ERR_INVALID_SPECTRUM = 5, /* ErrInvalidSpectrum errors.go:26 */
  GFFT_ERR_NOT_IMPLEMENTED = 6,  /* ErrNotImplemented  errors.go:30 */
  GFFT_ERR_CUDA = 100,           /* a CUDA runtime call failed */
  GFFT_ERR_OUT_OF_MEMORY = 101,  /* device or pinned-host allocation failed */
  GFFT_ERR_TIMEOUT = 102,        /* a bounded device wait gave up */
  GFFT_ERR_NO_DEVICE = 103,      /* no CUDA device (gpu.ErrBackendUnavailable) */
  GFFT_ERR_INVALID_ARGUMENT = 104,
  GFFT_ERR_WISDOM = 105          /* malformed wisdom text */
} gfft_status;

/* gpu/types.go:11-14 PrecisionKind. */
typedef enum gfft_precision { GFFT_COMPLEX64 = 0, GFFT_COMPLEX128 = 1 } gfft_precision;

/* plan_options.go:15-33 PlannerMode. */
enum { GFFT_PLANNER_ESTIMATE = 0, GFFT_PLANNER_MEASURE = 1, GFFT_PLANNER_PATIENT = 2, GFFT_PLANNER_EXHAUSTIVE = 3,
       /* no counterpart in the reference: the learned cost model picks the
        * variant when the wisdom store has none (gfft_planner_* below) */
       GFFT_PLANNER_LEARNED = 4 };

/* internal/fftypes/strategy.go:4-13 KernelStrategy. */
enum {
  GFFT_KERNEL_AUTO = 0, GFFT_KERNEL_DIT = 1, GFFT_KERNEL_STOCKHAM = 2, GFFT_KERNEL_SIXSTEP = 3,
  GFFT_KERNEL_EIGHTSTEP = 4, GFFT_KERNEL_BLUESTEIN = 5, GFFT_KERNEL_RECURSIVE = 6
};

/* plan_options.go:46-76 PlanOptions (Radices and Workspace are accepted by
 * the reference but unused; Wisdom is the process-wide store below) plus
 * gpu/types.go:32-42 DeviceIndex. */
typedef struct gfft_plan_options {
  int32_t planner;  /* GFFT_PLANNER_* */
  int32_t strategy; /* GFFT_KERNEL_* */
  int64_t batch;    /* PlanOptions.Batch (0 = 1) */
  int64_t stride;   /* PlanOptions.Stride (0 = contiguous) */
  int32_t in_place; /* PlanOptions.InPlace */
  int32_t device;   /* gpu.PlanOptions.DeviceIndex */
} gfft_plan_options;

/* Opaque 1-D complex plan: Plan[T] (plan.go:18). */
typedef struct gfft_plan gfft_plan;

/* ---- plan lifecycle ---------------------------------------------------- */

/* NewPlanT[T](n) / NewPlanWithOptions (plan.go:596-603; NewPlan32/NewPlan64
 * plan.go:1013-1027).  opts may be NULL.  n < 1 -> GFFT_ERR_INVALID_LENGTH. */
GFFT_API gfft_status gfft_plan_new(gfft_plan** out, int32_t precision, int64_t n, const gfft_plan_options* opts);

/* Plan.Close (plan.go:1223).  NULL is ignored. */
GFFT_API void gfft_plan_close(gfft_plan* plan);
/* Clone (plan.go:1300): an independent plan with the same schedule (its
 * tables rebuilt on the device; GPU plans keep no per-call scratch, so the
 * copy exists for callers that want separately closable handles).  Closing
 * either leaves the other intact. */
GFFT_API gfft_status gfft_plan_clone(gfft_plan** out, const gfft_plan* src);
/* SetKernelStrategy / GetKernelStrategy (plan.go:110-120): a process-wide
 * GFFT_KERNEL_* applied to plans created with GFFT_KERNEL_AUTO;
 * GFFT_KERNEL_AUTO restores automatic selection. */
GFFT_API void gfft_set_kernel_strategy(int32_t strategy);
GFFT_API int32_t gfft_get_kernel_strategy(void);
/* RecordBenchmarkDecision (plan.go:122-125, internal/planner/
 * selection.go:42-60): the strategy class automatic selection uses for
 * length n when the wisdom store, measurement and the learned model have
 * not decided; only DIT, Stockham, SixStep and EightStep are recorded. */
GFFT_API void gfft_record_benchmark_decision(int64_t n, int32_t strategy);
/* NewPlanPooled / NewPlanPooledWithOptions (plan.go:1040-1118): like
 * gfft_plan_new, but gfft_plan_close returns the plan to a process-wide pool
 * keyed by (device, precision, n, planner, strategy) and the next pooled
 * request of that shape reuses it instead of rebuilding its tables.  Batch
 * layouts (opts->batch > 1 or opts->stride > 0) are not pooled.
 * gfft_plan_pool_clear frees every pooled plan. */
GFFT_API gfft_status gfft_plan_new_pooled(gfft_plan** out, int32_t precision, int64_t n,
                                          const gfft_plan_options* opts);
GFFT_API void gfft_plan_pool_clear(void);

/* Plan.Len (plan.go:148). */
GFFT_API int64_t gfft_plan_len(const gfft_plan* plan);

/* Plan.Algorithm (plan.go:159): the bound GPU schedule as a
 * NUL-terminated string, e.g. "gpu:sm100:pow2:n1024:ept32". */
GFFT_API gfft_status gfft_plan_algorithm(const gfft_plan* plan, char* buf, size_t cap);

/* Creates a plan bound to one compiled kernel variant named by a wisdom
 * token (as listed by gfft_plan_variants), bypassing the planner: the
 * forced-strategy path of SetKernelStrategy (internal/planner/selection.go:22-29)
 * at kernel granularity. */
GFFT_API gfft_status gfft_plan_new_variant(gfft_plan** out, int32_t precision, int64_t n, const char* token);

/* Newline-separated tokens of every compiled variant for (precision, n).
 * With buf == NULL only *needed (bytes incl. NUL) is set. */
GFFT_API gfft_status gfft_plan_variants(int32_t precision, int64_t n, char* buf, size_t cap, size_t* needed);

/* Returns GFFT_ERR_TIMEOUT if a bounded device wait in this plan's kernels
 * has expired (the kernels then stop early and set a device flag instead of
 * hanging); synchronous. */
GFFT_API gfft_status gfft_plan_check(gfft_plan* plan);

/* ---- planner: autotuner and wisdom (wisdom.go:13-82, measure.go:89-228) ---- */

/* MeasureAndSelect (internal/fft/measure.go:89-141) on the GPU: times every
 * compiled variant of length n on `count` transforms (0 = about 2^25
 * elements) with CUDA events, `iters` timed runs each (median), records the
 * fastest in the wisdom store and writes a JSON report into report/cap
 * (may be NULL; *needed gets the size). */
GFFT_API gfft_status gfft_autotune(int32_t precision, int64_t n, int64_t count, int32_t iters, char* report,
                                   size_t cap, size_t* needed);

/* ImportWisdomFromString / ImportWisdom / ExportWisdom / ClearWisdom /
 * WisdomLen (wisdom.go:13-82).  Lines are size:precision:features:algorithm:ts;
 * a malformed line fails the whole import with GFFT_ERR_WISDOM and changes
 * nothing.  Unlike the reference (plan.go:832), imported entries steer
 * every later plan creation. */
GFFT_API gfft_status gfft_wisdom_import_string(const char* text);
GFFT_API gfft_status gfft_wisdom_export_string(char* buf, size_t cap, size_t* needed);
GFFT_API gfft_status gfft_wisdom_import_file(const char* path);
GFFT_API gfft_status gfft_wisdom_export_file(const char* path);
GFFT_API void gfft_wisdom_clear(void);
GFFT_API int64_t gfft_wisdom_len(void);

/* ---- device-resident execution (gpu.PlanImpl, gpu/backend.go:44-51) ---- */

/* Plan.Forward / Inverse (plan.go:332,382): one transform; dst may equal src. */
GFFT_API gfft_status gfft_forward(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len, void* stream);
GFFT_API gfft_status gfft_inverse(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len, void* stream);

/* Plan.ForwardBatch / InverseBatch (plan.go:504-571): count transforms on
 * [i*n, (i+1)*n).  Validation order: nil -> count < 1 -> lengths. */
GFFT_API gfft_status gfft_forward_batch(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                               int64_t count, void* stream);
GFFT_API gfft_status gfft_inverse_batch(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                               int64_t count, void* stream);

/* Plan.ForwardStrided / InverseStrided (plan_strided.go:16,25): one
 * transform over src[i*stride], written to dst[i*stride]. */
GFFT_API gfft_status gfft_forward_strided(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                 int64_t stride, void* stream);
GFFT_API gfft_status gfft_inverse_strided(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                 int64_t stride, void* stream);

/* Batched transform (direction -1 forward, +1 inverse; contiguous
 * [i*n, (i+1)*n) layout, validated like ForwardBatch) that allocates
 * nothing.  No counterpart in the reference: it exists for callers that must
 * not allocate while they run a transform (a real-time or callback context,
 * a process whose GPU allocator belongs to another runtime, a service that
 * reserves its memory up front).  It runs the plan's two-pass large-N
 * kernel with its scratch in a fixed 64 MiB array inside the library (held
 * on every GPU that loads the library until the process exits) instead of
 * the stream-ordered pool, so a length-n transform needs 2*n*element_size
 * bytes of it at most 63.5 MiB (n <= 2^21 complex64, 2^20 complex128);
 * larger lengths, or plans on another schedule, are rejected with an error.
 * The first call on a device looks the array up (make it before any stream
 * capture).  All calls share the array: calls that overlap on the GPU race.
 * The kernel's waits are bounded: if one expires, that call stops early and
 * leaves dst incomplete, and the plan's status word is set, which
 * gfft_plan_check then reports as GFFT_ERR_TIMEOUT (the next call starts
 * afresh).  A caller that must know a call completed checks the plan after
 * synchronizing its stream. */
GFFT_API gfft_status gfft_exec_batch_noalloc(gfft_plan* plan, int32_t direction, void* dst, int64_t dst_len,
                                             const void* src, int64_t src_len, int64_t count, void* stream);

/* ---- host-slice execution (the Go-slice methods) ------------------------ */

GFFT_API gfft_status gfft_forward_host(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len);
GFFT_API gfft_status gfft_inverse_host(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len);
GFFT_API gfft_status gfft_forward_batch_host(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                    int64_t count);
GFFT_API gfft_status gfft_inverse_batch_host(gfft_plan* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                    int64_t count);

/* ---- real-input plans (PlanReal, plan_real_generic.go) -------------------- */

/* Opaque PlanRealT[F, C] (plan_real_generic.go:22-36). */
typedef struct gfft_plan_real gfft_plan_real;

/* NewPlanReal32/64 / NewPlanRealTWithOptions (plan_real_constructors.go:8-43,
 * plan_real_generic.go:48-99): n reals, n even (else GFFT_ERR_INVALID_LENGTH).
 * precision GFFT_COMPLEX64 means float32 in / complex64 out.  opts->batch and
 * opts->stride give the batch layout of plan_batch.go:21-42 (the stride, in
 * elements, applies to the reals and to the bins alike). */
GFFT_API gfft_status gfft_plan_real_new(gfft_plan_real** out, int32_t precision, int64_t n,
                                        const gfft_plan_options* opts);
GFFT_API void gfft_plan_real_close(gfft_plan_real* plan);
/* Len / SpectrumLen (plan_real_generic.go:101-109): n and n/2+1. */
GFFT_API int64_t gfft_plan_real_len(const gfft_plan_real* plan);
GFFT_API int64_t gfft_plan_real_spectrum_len(const gfft_plan_real* plan);

/* Forward (R2C, plan_real_generic.go:111), ForwardNormalized (scaling 1,
 * x 1/n, :231) and ForwardUnitary (scaling 2, x 1/sqrt(n), :243); scaling 0 is
 * the plain Forward.  dst: n/2+1 complex bins, src: n reals (per transform). */
GFFT_API gfft_status gfft_real_forward(gfft_plan_real* plan, int32_t scaling, void* dst, int64_t dst_len,
                                       const void* src, int64_t src_len, void* stream);
/* Inverse (C2R, plan_real_generic.go:256): returns GFFT_ERR_INVALID_SPECTRUM
 * if a DC or Nyquist bin has |imag| > 1e-4 (float32) / 1e-12 (float64)
 * (:301-316); checking it synchronizes the stream. */
GFFT_API gfft_status gfft_real_inverse(gfft_plan_real* plan, void* dst, int64_t dst_len, const void* src,
                                       int64_t src_len, void* stream);
GFFT_API gfft_status gfft_real_forward_host(gfft_plan_real* plan, int32_t scaling, void* dst, int64_t dst_len,
                                            const void* src, int64_t src_len);
GFFT_API gfft_status gfft_real_inverse_host(gfft_plan_real* plan, void* dst, int64_t dst_len, const void* src,
                                            int64_t src_len);

/* ---- N-dimensional plans ------------------------------------------------- */

/* Opaque Plan2D / Plan3D / PlanND (plan_2d.go, plan_3d.go, plan_nd.go) and,
 * with real_input = 1, PlanReal2D / PlanReal3D (plan_real_2d.go,
 * plan_real_3d.go; any rank here). */
typedef struct gfft_plan_nd gfft_plan_nd;

/* NewPlan2D/3D/ND[WithOptions] (plan_2d.go:28, plan_3d.go:42-49,
 * plan_nd.go:43-50), NewPlanReal2D/3D (plan_real_2d.go:43-48,
 * plan_real_3d.go:42): row-major dims[0] x ... x dims[ndims-1], 1 <= ndims
 * <= 8, every dim >= 1 (real: last dim even) else GFFT_ERR_INVALID_LENGTH.
 * opts->batch / opts->stride: the batch layout of plan_batch.go:3-42. */
GFFT_API gfft_status gfft_plan_nd_new(gfft_plan_nd** out, int32_t precision, int32_t ndims, const int64_t* dims,
                                      int32_t real_input, const gfft_plan_options* opts);
GFFT_API void gfft_plan_nd_close(gfft_plan_nd* plan);
/* Len (plan_nd.go:151): product of dims.  SpectrumLen (plan_real_2d.go:121):
 * the compact spectrum, product of dims with the last one n/2+1 (= Len for
 * complex plans). */
GFFT_API int64_t gfft_plan_nd_len(const gfft_plan_nd* plan);
GFFT_API int64_t gfft_plan_nd_spectrum_len(const gfft_plan_nd* plan);
/* Forward / Inverse (plan_nd.go:188, plan_real_2d.go:139,278): complex plans
 * map Len -> Len elements (dst may equal src); real plans map Len reals to
 * SpectrumLen bins and back (the inverse leaves src untouched and checks the
 * last axis' DC/Nyquist bins like PlanReal.Inverse). */
GFFT_API gfft_status gfft_nd_forward(gfft_plan_nd* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                     void* stream);
GFFT_API gfft_status gfft_nd_inverse(gfft_plan_nd* plan, void* dst, int64_t dst_len, const void* src, int64_t src_len,
                                     void* stream);
/* ForwardFull / InverseFull of real plans (plan_real_2d.go:231,370): the
 * full Len-bin spectrum, redundant half from Hermitian symmetry. */
GFFT_API gfft_status gfft_nd_forward_full(gfft_plan_nd* plan, void* dst, int64_t dst_len, const void* src,
                                          int64_t src_len, void* stream);
GFFT_API gfft_status gfft_nd_inverse_full(gfft_plan_nd* plan, void* dst, int64_t dst_len, const void* src,
                                          int64_t src_len, void* stream);
GFFT_API gfft_status gfft_nd_forward_host(gfft_plan_nd* plan, void* dst, int64_t dst_len, const void* src,
                                          int64_t src_len);
GFFT_API gfft_status gfft_nd_inverse_host(gfft_plan_nd* plan, void* dst, int64_t dst_len, const void* src,
                                          int64_t src_len);

/* Batched strided transforms with a 1-D plan: element j of transform b at
 * b*dist + j*stride in both dst and src (the column batches behind the N-D
 * plans; plan_strided.go:35-99 for one transform).  Columns (dist = 1,
 * count <= stride) run one coalesced column kernel. */
GFFT_API gfft_status gfft_exec_strided_batch(gfft_plan* plan, int32_t direction, void* dst, int64_t dst_len,
                                             const void* src, int64_t src_len, int64_t count, int64_t stride,
                                             int64_t dist, void* stream);

/* ---- convolution and correlation (convolve.go, convolve_real.go, correlate.go) */

/* Convolve / Convolve128 (convolve.go:9,65): dst = a (*) b, complex, length
 * exactly a_len + b_len - 1 (else GFFT_ERR_LENGTH_MISMATCH); empty inputs ->
 * GFFT_ERR_INVALID_LENGTH.  Device pointers, ordered on stream. */
GFFT_API gfft_status gfft_convolve(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                                   const void* b, int64_t b_len, void* stream);
/* CrossCorrelate / Correlate128 (correlate.go:13,48): Convolve with the
 * conjugate reverse of b; AutoCorrelate is (a, a). */
GFFT_API gfft_status gfft_correlate(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                                    const void* b, int64_t b_len, void* stream);
/* ConvolveReal (convolve_real.go:9): real inputs (float32 for
 * GFFT_COMPLEX64, float64 for GFFT_COMPLEX128), FFT length
 * NextPow2(a_len + b_len - 1). */
GFFT_API gfft_status gfft_convolve_real(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                                        const void* b, int64_t b_len, void* stream);
GFFT_API gfft_status gfft_convolve_host(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                                        const void* b, int64_t b_len);
GFFT_API gfft_status gfft_correlate_host(int32_t precision, void* dst, int64_t dst_len, const void* a, int64_t a_len,
                                         const void* b, int64_t b_len);
GFFT_API gfft_status gfft_convolve_real_host(int32_t precision, void* dst, int64_t dst_len, const void* a,
                                             int64_t a_len, const void* b, int64_t b_len);
/* ConvolveReal of `count` signals (a_len reals, a_dist apart) with one kernel
 * b, results of a_len + b_len - 1 reals dst_dist apart: the reference's
 * per-signal ConvolveReal loop as one batched computation. */
GFFT_API gfft_status gfft_convolve_real_batch(int32_t precision, void* dst, int64_t dst_dist, const void* a,
                                              int64_t a_len, int64_t a_dist, int64_t count, const void* b,
                                              int64_t b_len, void* stream);

/* ---- uneven-length batches ------------------------------------------------ */

/* No single reference entry point: a Go caller loops Plan.Forward over one
 * plan per length.  A plan for `count` transforms of the given lengths
 * (1 .. 2^24 each), packed back to back: transform i starts at the sum of
 * the lengths before it.  Plan creation builds every twiddle, chirp and
 * Bluestein filter on the GPU. */
typedef struct gfft_plan_uneven gfft_plan_uneven;
GFFT_API gfft_status gfft_plan_uneven_new(gfft_plan_uneven** out, int32_t precision, int64_t count,
                                          const int64_t* lengths, const gfft_plan_options* opts);
GFFT_API void gfft_plan_uneven_close(gfft_plan_uneven* plan);
/* Total elements of the packed batch (sum of the lengths). */
GFFT_API int64_t gfft_plan_uneven_total(const gfft_plan_uneven* plan);
/* The whole batch in a few launches (persistent work-queue kernel for
 * every transform that fits one CTA, grouped batches for the rest),
 * replayed from a CUDA graph captured on first use per (direction, dst,
 * src) when use_graph is set (the plan keeps the 8 most recently used
 * graphs).  dst may equal src.  Safe to call from several threads and
 * streams at once: the calls of one plan share its work buffers, so each is
 * ordered on the device after the plan's previous call (an event recorded
 * by every call, waited on by the next; the calls do not overlap on the
 * GPU).  Inside a caller's own stream capture that ordering is left to the
 * captured graph. */
GFFT_API gfft_status gfft_uneven_exec(gfft_plan_uneven* plan, int32_t direction, void* dst, const void* src,
                                      int32_t use_graph, void* stream);
/* The plain per-size path: one plan per distinct length and one transform
 * call per transform, as a loop over Plan.Forward would do. */
GFFT_API gfft_status gfft_uneven_exec_per_size(gfft_plan_uneven* plan, int32_t direction, void* dst,
                                               const void* src, void* stream);

/* ---- learned planner (no counterpart in the reference) -------------------- */

/* The cost model: an FP32 MLP, in_dim -> hidden -> hidden -> 1 with ReLU,
 * nparams floats laid out W1[hidden][in_dim] b1 W2[hidden][hidden] b2 w3 b3
 * (row-major).  in_dim = 16, hidden = 64. */
GFFT_API void gfft_mlp_sizes(int32_t* in_dim, int32_t* hidden, int64_t* nparams);
/* out[i] = model(x[i*in_dim ..]) for n samples; device pointers. */
GFFT_API gfft_status gfft_mlp_forward(const float* params, const float* x, int64_t n, float* out, void* stream);
/* Gradient of the mean squared error (1/n) sum (model(x_i) - y_i)^2 over
 * samples 0..n-1 (1 <= n <= 64) with respect to every parameter, and the
 * loss; device pointers. */
GFFT_API gfft_status gfft_mlp_grad(const float* params, const float* x, const float* y, int64_t n, float* grad,
                                   float* loss, void* stream);
/* `steps` Adam steps (beta1 0.9, beta2 0.999, eps 1e-8, step counter
 * starting after step0) on mini-batches of `batch` (<= 64) samples drawn
 * deterministically from (seed, step) out of the n samples; params and the
 * Adam moments adam_m, adam_v (nparams each, zero at the start) are updated
 * in place; *loss (device) = mean mini-batch loss of these steps. */
GFFT_API gfft_status gfft_mlp_train(float* params, float* adam_m, float* adam_v, const float* x, const float* y,
                                    int64_t n, int32_t steps, int32_t batch, float lr, uint64_t seed, int64_t step0,
                                    float* loss, void* stream);
/* Raw features (in_dim floats, host) of the variant `token` for a shape:
 * complex length n (the complex child length for real = 1), batch
 * transforms per call (<= 0: unknown, taken as 128 MB of data), element
 * stride.  Host-only. */
GFFT_API gfft_status gfft_planner_features(int32_t precision, int64_t n, int64_t batch, int64_t stride, int32_t real,
                                           const char* token, float* out);
/* Installs the model used by GFFT_PLANNER_LEARNED (host arrays: nparams
 * parameters; norm = feature means[in_dim], deviations[in_dim], target mean,
 * target deviation), or unloads it (params NULL).  Without a call, the file
 * wisdom/planner_b200.bin next to the library is loaded on first use. */
GFFT_API gfft_status gfft_planner_set_model(const float* params, const float* norm);
GFFT_API gfft_status gfft_planner_load_model(const char* path);
GFFT_API int32_t gfft_planner_has_model(void);
/* The model's pick among gfft_plan_variants(n) for a shape (one inference
 * launch on the current device). */
GFFT_API gfft_status gfft_planner_choose(int32_t precision, int64_t n, int64_t batch, int64_t stride, int32_t real,
                                         char* token, size_t cap);

/* ---- errors -------------------------------------------------------------- */

/* Text of a status code (the reference's error strings for 1..6). */
GFFT_API const char* gfft_status_string(int32_t status);
/* Detail of the last failure on the calling thread ("" if none). */
GFFT_API const char* gfft_last_error(void);

/* ---- devices, streams and buffers (gpu.Context / Buffer / Stream) ------- */

/* Backend.Devices (gpu/backend.go:10): number of CUDA devices (0 if none). */
GFFT_API gfft_status gfft_device_count(int32_t* count);
/* Context.NewBuffer (gpu/backend.go:18): device allocation of `bytes`. */
GFFT_API gfft_status gfft_buffer_alloc(void** ptr, int64_t bytes);
/* Buffer.Close (gpu/backend.go:36). */
GFFT_API gfft_status gfft_buffer_free(void* ptr);
/* Buffer.Upload / Download (gpu/backend.go:32-35): synchronous copies. */
GFFT_API gfft_status gfft_buffer_upload(void* dst_device, const void* src_host, int64_t bytes);
GFFT_API gfft_status gfft_buffer_download(void* dst_host, const void* src_device, int64_t bytes);
/* Context.NewStream / Stream.Synchronize / Stream.Close (gpu/backend.go:19,40-41). */
GFFT_API gfft_status gfft_stream_create(void** stream);
GFFT_API gfft_status gfft_stream_synchronize(void* stream);
GFFT_API gfft_status gfft_stream_destroy(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GFFT_H */
