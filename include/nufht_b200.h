/*
 * nufht_b200.h -- C ABI of the B200 batched nonuniform fast Hankel transform.
 *
 *   g[i, t] = sum_j c[j, t] * J_nu(k_i * r_j),   i < n targets, j < m sources, t < batch.
 *
 * Part 1 re-declares, with identical names, struct layouts, argument meaning and
 * return codes, the public interface of the reference library Ansal06/NUFHT
 * (src/fast_hankel_nufht.h).  A program compiled against the reference header links
 * against libnufht_b200.so unchanged; every transform then runs on the GPU.
 * Pointers passed to Part 1 may be host or device pointers (detected per call).
 *
 * Part 2 is this library's own extension: a device-resident plan, explicit CUDA
 * streams, device pointers and precision selection.
 *
 * Deliberate deviations from the reference (each one also has a test):
 *   - inputs rs and ws must be finite, non-negative and non-decreasing; the reference
 *     assumes this without checking (src/fast_hankel_nufht.c:454-466).  Violations
 *     return NUFHT_E_UNSORTED_RS / NUFHT_E_UNSORTED_WS from nufht_plan_init.
 *   - for odd integer nu < 0 the sign (-1)^nu is applied exactly once for every batch
 *     size (the reference applies it twice when batch == 1,
 *     src/fast_hankel_nufht.c:916-920 and :1090-1095);
 *   - the all-direct path (m*n < min_dim_prod) evaluates J_|nu| like every other path
 *     (the reference hands the signed nu to GSL there, src/fast_hankel_nufht.c:1049).
 */
#ifndef NUFHT_B200_H
#define NUFHT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================= Part 1: reference-compatible ABI ======================= */

/* Replaces NufhtOptions, src/fast_hankel_nufht.h:21-28 (same layout). */
typedef struct {
    double tol;          /* default 1e-8 */
    int    max_levels;   /* <= 0: floor(log2(min(m,n)^2 / min_dim_prod)) */
    int    min_dim_prod; /* default 10000 */
    double z_split;      /* NaN: from the tables */
    int    K_asy;        /* <= 0: from the tolerance formula */
    int    K_loc;        /* <= 0: from the tables */
} NufhtOptions;

/* Replaces nufht_default_options, src/fast_hankel_nufht.h:31. */
NufhtOptions nufht_default_options(void);

/* Replaces Box / BoxVector / Boxes, src/fast_hankel_nufht.h:35-55 (same layouts).
 * i indexes targets (ws), j indexes sources (rs); bounds are inclusive. */
typedef struct { int i0, i1; int j0, j1; } Box;
typedef struct { Box *data; size_t length; size_t capacity; } BoxVector;
typedef struct { BoxVector loc; BoxVector asy; BoxVector dir; } Boxes;

/* Replaces boxes_free, src/fast_hankel_nufht.h:59. */
void boxes_free(Boxes *boxes);

/* Replaces NufhtPlan, src/fast_hankel_nufht.h:64-83 (same layout).  The GPU state of
 * a plan (device copies of rs/ws, work lists, FFT plans, workspace) is kept by the
 * library, keyed by the plan's address, and released by nufht_plan_free. */
typedef struct {
    double nu;
    double tol;
    double z_split;
    int    K_asy;
    int    K_loc;
    double asy_coef[64];
    int m;
    int n;
    const double *rs;
    const double *ws;
    int max_levels;
    int min_dim_prod;
    Boxes boxes;
    int tables_loaded;
} NufhtPlan;

/* Replaces NufhtScratch, src/fast_hankel_nufht.h:86-101 (same layout).  The buffers are
 * allocated with the reference's sizes for ABI compatibility; GPU execution keeps its
 * own device workspace inside the plan state. */
typedef struct {
    double *in_buffer;
    double *out_buffer;
    double *real_buffer_1;
    double *real_buffer_2;
    double *cheb_buffer;
    double *bessel_buffer_1;
    double *bessel_buffer_2;
    int m_alloc;
    int n_alloc;
    int Kloc_alloc;
    int extra_alloc;
} NufhtScratch;

/* Replaces nufht_plan_init, src/fast_hankel_nufht.h:106-111 / .c:759-786.
 * Returns 0, or -1..-6 (parameter errors as the reference), -200 (NULL / empty),
 * NUFHT_E_UNSORTED_RS, NUFHT_E_UNSORTED_WS. */
int nufht_plan_init(NufhtPlan *plan, double nu, const double *rs, int m, const double *ws,
                    int n, const NufhtOptions *opt);

/* Replaces nufht_plan_free, src/fast_hankel_nufht.h:114. */
void nufht_plan_free(NufhtPlan *plan);

/* Replaces nufht_scratch_init / nufht_scratch_free, src/fast_hankel_nufht.h:117-119.
 * Returns 0, -300 (NULL), -301 (allocation failure). */
int nufht_scratch_init(NufhtScratch *scratch, const NufhtPlan *plan);
void nufht_scratch_free(NufhtScratch *scratch);

/* Replaces generate_boxes, src/fast_hankel_nufht.h:128-134 / .c:578-744 (same boxes,
 * found by binary search instead of a linear scan). */
Boxes generate_boxes(const double *rs, int m, const double *ws, int n, double z_split,
                     int max_levels, int min_dim_prod, int K_loc_threshold);

/* Replaces split_box, src/fast_hankel_nufht.h:138-144 / .c:523-574. */
void split_box(const double *rs, int m, const double *ws, int n, const Box *box, double z,
               int *ispl_out, int *jspl_out);

/* Replaces nufht_batch, src/fast_hankel_nufht.h:155-160 / .c:989-1107.
 * cs: m x batch column-major, leading dimension ld_cs >= m; gs: n x batch, ld_gs >= n,
 * overwritten.  Host or device pointers.  scratch may be NULL.
 * Returns 0, -400 (bad args), -401 (leading dims), or NUFHT_E_CUDA / NUFHT_E_NO_DEVICE. */
int nufht_batch(const NufhtPlan *plan, const double *cs, int ld_cs, double *gs, int ld_gs,
                int batch, NufhtScratch *scratch);

/* Replaces nufht_inplace and nufht, src/fast_hankel_nufht.h:163-177 / .c:1111-1159.
 * On failure they print to stderr and leave gs zeroed, as the reference does. */
void nufht_inplace(double *gs, double nu, const double *rs, int m, const double *cs,
                   const double *ws, int n, const NufhtOptions *opt);
double *nufht(double nu, const double *rs, int m, const double *cs, const double *ws, int n,
              const NufhtOptions *opt);

/* Replaces generate_tables, src/fast_hankel_nufht.h:181 / src/bounds.c:306-324: fills the
 * library's planning tables from their defining formulas. */
void generate_tables(void);

/* Replace the evaluators of src/fast_hankel_nufht.h:185-238 (src/expansions.c).  Each
 * adds one box's contribution to gs on the GPU.  Host or device pointers.  The
 * scratch-buffer arguments are accepted for ABI compatibility and not used. */
void add_dir(double *gs, double nu, const double *rs, const double *cs, const double *ws,
             int m, int n);
void add_dir_batch(double *gs, double nu, const double *rs, const double *cs,
                   const double *ws, int m, int n, int batch, int ld_cs, int ld_gs);
void add_asy(double *gs, double nu, const double *rs, const double *cs, const double *ws,
             int m, int n, int K, double tol, const double *asy_coef, double *real_buffer_1,
             double *real_buffer_2, double *in_buffer, double *out_buffer);
void add_asy_batch(double *gs, double nu, const double *rs, const double *cs,
                   const double *ws, int m, int n, int K, double tol, const double *asy_coef,
                   int batch, int ld_cs, int ld_gs, double *in_buffer, double *out_buffer);
void add_loc(double *gs, double nu, const double *rs, const double *cs, const double *ws,
             int m, int n, int K, double *cheb_buffer, double *bessel_buffer_1,
             double *bessel_buffer_2);
void add_loc_batch(double *gs, double nu, const double *rs, const double *cs,
                   const double *ws, int m, int n, int K, int batch, int ld_cs, int ld_gs,
                   double *cheb_buffer_batch, double *bessel_buffer_1, double *bessel_buffer_2);

/* ======================= Part 2: B200 extension ======================= */

/* Error codes added by this library (the reference's codes are kept as they are). */
#define NUFHT_E_UNSORTED_RS  (-410) /* rs not finite, non-negative and non-decreasing */
#define NUFHT_E_UNSORTED_WS  (-411) /* ws not finite, non-negative and non-decreasing */
#define NUFHT_E_CUDA         (-420) /* a CUDA runtime or cuFFT call failed */
#define NUFHT_E_NO_DEVICE    (-422) /* no CUDA device */
#define NUFHT_E_TOO_LARGE    (-423) /* sizes exceed what this entry point accepts */
#define NUFHT_E_BAD_FLAGS    (-424) /* unknown flag bits */

/* Plan flags. */
#define NUFHT_B200_FP64            0x0   /* all arithmetic in FP64 (default) */
#define NUFHT_B200_MIXED           0x1   /* asymptotic boxes in FP32 where the modelled worst-case
                                            FP32 error is at most tol / 4 (plan info: mixed = 1),
                                            FP64 otherwise */
#define NUFHT_B200_MIXED_AVERAGED  0x2   /* asymptotic boxes in FP32 for tol >= 1e-9 whatever the
                                            worst case: within tol for coefficient columns spread
                                            over many sources (their FP32 rounding averages out;
                                            measured against FP64 direct sums), up to the
                                            plan_stats bound out[14] * ||c||_1 for a column
                                            concentrated on one source */
#define NUFHT_B200_EXTENDED_TABLES 0x10  /* fill the asymptotic table at K_asy = 10, which the
                                            reference leaves empty (affects |nu| >= 35) */

typedef struct NufhtDevicePlan NufhtDevicePlan;

/* Summary of a device plan. */
typedef struct {
    double nu, tol, z_split;
    int K_asy, K_loc;
    long n_loc, n_asy, n_dir;      /* box counts */
    long fft_points;               /* sum over asymptotic boxes of the FFT length */
    int spread_width;              /* exponential-of-semicircle kernel width */
    int path;                      /* 0 boxes, 1 all-direct, 2 half-integer order */
    size_t workspace_bytes;        /* device workspace for the last batch size executed */
    int mixed;                     /* 1 when the asymptotic boxes run in FP32 */
} NufhtB200Info;

/* Build a device plan.  rs (m) and ws (n) may be host or device pointers; they are
 * copied, so the caller may free them afterwards.  device: CUDA ordinal.
 * Returns 0 or a negative code (same codes as nufht_plan_init, plus Part 2 codes). */
int nufht_b200_plan_create(NufhtDevicePlan **out, double nu, const double *rs, int m,
                           const double *ws, int n, const NufhtOptions *opt, int flags,
                           int device);

/* g = H c on `stream` (a cudaStream_t; NULL = legacy default stream).  cs and gs are
 * DEVICE pointers; column-major with leading dimensions ld_cs >= m, ld_gs >= n.  The call
 * is asynchronous with respect to the host. */
int nufht_b200_execute(NufhtDevicePlan *plan, const double *cs, int ld_cs, double *gs,
                       int ld_gs, int batch, void *stream);

int nufht_b200_plan_info(const NufhtDevicePlan *plan, NufhtB200Info *info);
void nufht_b200_plan_destroy(NufhtDevicePlan *plan);

/* Copy the plan's boxes (4 ints each, loc then asy then dir) into out (cap boxes).
 * Returns the total number of boxes. */
long nufht_b200_plan_boxes(const NufhtDevicePlan *plan, int *out, long cap);

/* Replaces generate_boxes (src/fast_hankel_nufht.c:578-744) computed on the GPU: the same
 * boxes in the same order, from sorted grids in host or device memory (validated on the
 * device first: NUFHT_E_UNSORTED_RS / _WS).  The lists in `out` are host memory, released
 * with boxes_free.  nufht_b200_plan_create partitions this way unless the environment sets
 * NUFHT_B200_HOST_PLANNER=1.  Returns 0 or a negative code. */
int nufht_b200_generate_boxes_device(const double *rs, int m, const double *ws, int n,
                                     double z_split, int max_levels, int min_dim_prod,
                                     int K_loc_threshold, Boxes *out);

/* Human-readable text for any code returned by this library. */
const char *nufht_b200_strerror(int code);

/* Number of kernel launches made by this library in the calling process so far. */
long long nufht_b200_launch_count(void);

/* Device-side Bessel function values J_nu(x[i]) for nu integer (|nu| <= 200) or
 * half-integer (|nu| <= 19/2); x and out are device pointers.  Exposed for testing the
 * device special-function code. */
int nufht_b200_besselj(double nu, const double *x, double *out, long count, void *stream);

/* Device timing of the phases of every transform executed while enabled: CUDA events on
 * the launching stream.  nufht_b200_phase_times() waits for them, adds the milliseconds
 * per phase into ms[0..nphase) -- 0 zeroing of g, 1 local projection, 2 local evaluation,
 * 3 asymptotic spreading, 4 FFT, 5 asymptotic interpolation, 6 direct boxes -- releases
 * them and returns how many phase records it read. */
void nufht_b200_set_phase_timing(int on);
int nufht_b200_phase_times(double *ms, int nphase);

/* Algorithmic work of a plan, per batch column where it scales with the batch:
 * out[0..14] = asymptotic sources, asymptotic targets, FFT cells, spreading taps,
 * interpolation taps, direct pairs, local sources, local targets, FFT cells read by
 * interpolation, FFT flops per vector, expansion terms (2 (K_asy + 1)), K_loc + 1,
 * asymptotic boxes oversampled below 2, 1 if the asymptotic boxes run in FP32 (mixed
 * precision) else 0, and the modelled worst-case error of FP32 asymptotic boxes per unit
 * ||c||_1 (mixed precision is used only where it is at most tol / 4); out[15..17] the
 * planning time in ms (grid validation and box partition, work lists, device tables and
 * uploads), out[18] 1 when the partition ran on the device, and out[19..20] the bytes of the
 * plan-time source records (read by spreading) and target records (read by interpolation). */
int nufht_b200_plan_stats(const NufhtDevicePlan *plan, double *out, int n);

/* Measured FP64 fused-multiply-add throughput of the current device (TFLOP/s). */
int nufht_b200_fp64_peak(double *tflops);
/* Measured FP32 throughput of the packed two-lane multiply-add (fma.rn.f32x2) that the
 * single-precision asymptotic kernels use (TFLOP/s). */
int nufht_b200_fp32_peak(double *tflops);

/* No counterpart in the reference.  Allocation-free variant of add_loc_batch for callers
 * that cannot call cudaMalloc at call time (a fixed memory budget or pool, allocation
 * forbidden after start-up): adds the local (Wimp) expansion of the single box
 * [0,n) x [0,m) to gs, with its scratch (work lists, partial projections, coefficients) in
 * a 4 MiB device array inside the library that every GPU loading the library holds until
 * exit.  gs, rs, cs, ws are DEVICE pointers of the current device (or managed memory) and
 * `stream` belongs to it; nu is an integer order (a negative odd order adds the negated
 * expansion, J_{-n} = (-1)^n J_n); asynchronous on `stream`.  Returns 0, -400/-401
 * (arguments, including buffers or a stream of another device), -2 (order), NUFHT_E_TOO_LARGE when the
 * scratch would exceed 4 MiB (about ceil(m/2048) (K+1) batch 8 bytes plus work lists),
 * NUFHT_E_CUDA.  The first call on a device looks up the array's address and should come
 * before any stream capture; calls that overlap on the GPU share the array and race. */
int nufht_b200_add_loc_batch_noalloc(double *gs, double nu, const double *rs, const double *cs,
                                     const double *ws, int m, int n, int K, int batch, int ld_cs,
                                     int ld_gs, void *stream);

/* No counterpart in the reference (one problem per call there).  Many independent
 * transforms -- each a device plan with its own order, grids, tolerance and batch width --
 * executed by ONE CUDA-graph launch.  Items that share a plan run one after another; other
 * items run concurrently on up to `branches` parallel branches of the graph, dealt by
 * estimated work.  branches = 0 tunes the count at creation (1, 2, 4, ... 32) by timing the
 * graph on the items' own buffers.  cs / gs are DEVICE pointers, fixed for the life of the
 * batch (the graph records them); g is overwritten.  Creation runs every item once and
 * sizes all workspaces, so a launch allocates nothing.  The plans must not be executed
 * elsewhere while a launch of the batch is in flight. */
/* Replaces the copies around nufht_batch in src/_pynufht.c:156,222-237 (the forced
 * Fortran-order copy of cs and the transpose copy of g).  nufht_batch with a choice of
 * layout for cs and gs: layout 0 = column-major as nufht_batch (column t at p + t * ld,
 * ld >= m or n), 1 = row-major (row j at p + j * ld, ld >= batch: a C-order (m, batch)
 * NumPy array).  Host or device pointers; synchronous.  Row-major batches are transposed
 * on the GPU after / before one contiguous copy, so no host-side copy is made; with both
 * layouts 0 this is nufht_batch.  Returns 0, -400 (null pointer, batch <= 0, layout not
 * 0 or 1), -401 (leading dimension too small), or a plan / CUDA error code. */
int nufht_b200_batch_layout(const NufhtPlan *plan, const double *cs, int c_rowmajor, int ld_cs,
                            double *gs, int g_rowmajor, int ld_gs, int batch);

typedef struct NufhtB200Batch NufhtB200Batch;
typedef struct {
    NufhtDevicePlan *plan;
    const double *cs;  /* m x batch, leading dimension ld_cs >= m */
    int ld_cs;
    double *gs;        /* n x batch, leading dimension ld_gs >= n */
    int ld_gs;
    int batch;
} NufhtB200BatchItem;

int nufht_b200_batch_create(NufhtB200Batch **out, const NufhtB200BatchItem *items, int count,
                            int branches);
/* A batch keeps every plan it uses alive (destroying a plan's handle while a batch uses it
 * is safe) and pins it: while pinned, running the plan on its own at a larger width gives
 * it new workspace buffers and leaves the ones the graph recorded allocated until the last
 * batch using the plan is destroyed.  Items may share a plan at different widths.
 * Creation synchronizes the device (it first runs every item once on its own stream). */
/* One graph launch on `stream` (a cudaStream_t; asynchronous). */
int nufht_b200_batch_launch(NufhtB200Batch *batch, void *stream);
/* Branch count in use, the tuned graph time (ms, 0 when branches was given) and the
 * number of kernel nodes of the graph. */
int nufht_b200_batch_info(const NufhtB200Batch *batch, int *branches, float *tuned_ms,
                          long *kernel_nodes);
void nufht_b200_batch_destroy(NufhtB200Batch *batch);
/* Introspection (tests): the plan's current asymptotic-grid workspace, how many older
 * workspace buffers it keeps allocated for batches that recorded them, and how many
 * batches pin it. */
int nufht_b200_plan_buffers(const NufhtDevicePlan *plan, const void **grid, int *retired,
                            int *pins);

/* Where the planning tables were read from (a cache file path), or "generated". */
const char *nufht_b200_table_source(void);

/* Generate the planning tables from their formulas and write them to `path` in the
 * reference's cache format.  Returns 0 on success. */
int nufht_b200_write_tables(const char *path);

#ifdef __cplusplus
}
#endif
#endif /* NUFHT_B200_H */
