/* libttgpu: B200-native TT rounding and AMEn inner loop behind a C ABI.
 *
 * Plain pointers and sizes only.  Column-major FP64 arrays throughout, in the
 * layouts of TT-Toolbox (paths relative to the TT-Toolbox source tree):
 *   TT tensor core k : [r_k, n_k, r_{k+1}]        (@tt_tensor/core2cell.m:9-11)
 *   TT matrix core k : [r_k, n_k, m_k, r_{k+1}]   (@tt_matrix/core2cell.m:9-11)
 *   flat core vector : cores concatenated, offsets ps (@tt_tensor/tt_tensor.m:33-41)
 *
 * Conventions
 *   - Every function returns TTG_OK (0) or an error code; ttg_last_error()
 *     gives a message for the calling thread.  Nothing aborts the process.
 *   - Handles (ttg_context, ttg_tt) are owned by the library; host buffers are
 *     borrowed for the duration of the call; *_download copies out.
 *   - One context = one device and one CUDA stream.  Calls are synchronous at
 *     the ABI.  A context must not be used by two threads at once.
 *   - Kernel-level entries (ttg_local_matvec, ttg_next_phi, ttg_local_solve)
 *     take DEVICE pointers of the context's device.
 */
#ifndef TTGPU_H
#define TTGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TTG_OK = 0,
  TTG_ERR_INVALID = 1,     /* bad argument / inconsistent shapes            */
  TTG_ERR_CUDA = 2,        /* CUDA runtime error                            */
  TTG_ERR_SOLVER = 3,      /* cuSOLVER error or LAPACK info != 0            */
  TTG_ERR_NOCONV = 4,      /* iteration cap reached without convergence     */
  TTG_ERR_ALLOC = 5,       /* device allocation failed                      */
  TTG_ERR_TIMEOUT = 6,     /* a bounded device-side wait gave up            */
  TTG_ERR_UNSUPPORTED = 7  /* option value not implemented                  */
};

/* Arithmetic of the contractions.  TTG_FP64: everything in FP64 (parity mode).
 * TTG_MIXED: local matvecs / Phi contractions on BF16 tensor cores with FP32
 * accumulation inside the Krylov solver, FP64 residuals and refinement,
 * FP64 QR/SVD. */
enum { TTG_FP64 = 0, TTG_MIXED = 1 };

typedef struct ttg_context_s* ttg_context;
typedef struct ttg_tt_s* ttg_tt;

/* ---- library / context --------------------------------------------------- */
const char* ttg_last_error(void);
int ttg_version(void);
int ttg_context_create(int device, ttg_context* out);
int ttg_context_destroy(ttg_context ctx);
int ttg_context_sync(ttg_context ctx);

/* Context options.  TTG_OPT_JACOBI_MAX_SWEEPS (default 40, 1..1000): sweep
 * limit of the one-sided Jacobi SVDs.  An SVD that reaches it without
 * converging makes ttg_dense_svd and ttg_amen_solve fail with
 * TTG_ERR_NOCONV (MATLAB's svd errors there, which aborts amen_solve2), and
 * makes ttg_round take the fallback SVD of the core, as round.m:64-74 falls
 * back to svds.  TTG_OPT_GROUP_SMS (default 0): the SM count each solve of a
 * grouped batch sizes its own grids with (cooperative Krylov grids, split-K
 * slices, grid-stride loops); 0 = twice the device's SMs divided among the
 * solves in flight, re-evaluated at every flush; the device's SM count gives
 * every solve the launch configurations of a solve run alone. */
enum { TTG_OPT_JACOBI_MAX_SWEEPS = 1, TTG_OPT_GROUP_SMS = 2 };
int ttg_context_set_option(ttg_context ctx, int32_t key, int64_t value);

/* Self-test of the bounded device waits.  No counterpart in the reference.
 * Every kernel of this library that waits on the device (the grid barriers
 * of the Householder GMRES (which = 0), of the cooperative Jacobi SVD (2)
 * and of the mixed-precision Arnoldi kernels (3), the mbarrier waits of the
 * tcgen05 pipeline (1)) gives up after a bounded number of polls, raises a
 * device error flag and returns, so that a lost participant ends in an
 * error status instead of a hang.  This entry runs the chosen wait helper
 * on a condition that nothing satisfies, with a small poll limit, and
 * returns TTG_ERR_TIMEOUT when the wait gave up as designed; the context
 * stays usable. */
int ttg_selftest_wait(ttg_context ctx, int32_t which);

/* Device memory helpers for callers without an allocator of their own. */
int ttg_malloc(ttg_context ctx, size_t bytes, void** out);
int ttg_free(ttg_context ctx, void* p);
int ttg_memcpy_h2d(ttg_context ctx, void* dst_dev, const void* src_host, size_t bytes);
int ttg_memcpy_d2h(ttg_context ctx, void* dst_host, const void* src_dev, size_t bytes);
/* Fill device memory with a byte value (e.g. to evict the L2 cache between
 * timed runs). */
int ttg_memset(ttg_context ctx, void* dst_dev, int value, size_t bytes);
/* Number of kernels this library launched on the context so far. */
int ttg_launch_count(ttg_context ctx, int64_t* out);

/* ---- device-resident TT tensors / matrices -------------------------------
 * Replaces the MATLAB objects built by @tt_tensor/tt_tensor.m:33-41 and
 * @tt_matrix/tt_matrix.m:33-40.  m == NULL makes a TT tensor, otherwise a TT
 * matrix with row sizes n and column sizes m.  r has d+1 entries.  The flat
 * core is copied from host memory. */
int ttg_tt_upload(ttg_context ctx, int64_t d, const int64_t* n, const int64_t* m,
                  const int64_t* r, const double* core_host, ttg_tt* out);
/* Any output pointer may be NULL.  n, m: d entries; r: d+1 entries. */
int ttg_tt_shape(ttg_tt t, int64_t* d, int64_t* n, int64_t* m, int64_t* r,
                 int64_t* numel);
int ttg_tt_download(ttg_tt t, double* core_host);
int ttg_tt_free(ttg_tt t);

/* ---- TT rounding ----------------------------------------------------------
 * Replaces tt = round(tt, eps[, rmax])  (@tt_tensor/round.m:1, algorithm
 * round.m:20-108 with my_chop2, core/my_chop2.m:18-35): left-to-right QR
 * sweep, right-to-left truncated SVD sweep with threshold
 * eps/sqrt(d-1)*||s||, then norm balancing.  rmax: NULL (no cap), one value
 * (nrmax == 1) or d+1 values.  *out is a new handle. */
typedef struct {
  double ms_total;     /* device time of the whole rounding            */
  double ms_qr_sweep;  /* left-to-right QR sweep                       */
  double ms_svd_sweep; /* right-to-left SVD sweep                      */
  int64_t max_rank;    /* max rank of the result                       */
  int64_t svd_fallbacks; /* cores whose Jacobi SVD reached the sweep limit
                            and took the fallback SVD (round.m:64-74)    */
} ttg_round_stats;

int ttg_round(ttg_tt in, double eps, const int64_t* rmax, int64_t nrmax,
              int32_t precision, ttg_tt* out, ttg_round_stats* stats);

/* ---- AMEn solve -----------------------------------------------------------
 * Replaces [x,testdata,z] = amen_solve2(A, y, tol, 'name', value, ...)
 * (solve/amen_solve2.m:1, options :75-107,161-203) on the default path:
 * kicktype 'als', trunc_norm 'residual', local GMRES per fmex/solve3d_2.c
 * (Householder Arnoldi, fmex/solve3d.c:339-518).  Also the whole-solve seam of
 * fmex/fort_amen_solve_mex.F90:20-21.
 * x0 / z0 may be NULL: then a right-orthogonal random TT of rank 2 / kickrank
 * is drawn on the device (the reference's tt_rand(n,d,2,-1),
 * amen_solve2.m:222-224,250-252; the random stream differs from MATLAB's). */
/* One local step of an AMEn sweep (core `core` of sweep `sweep`), recorded
 * when ttg_amen_opts.trace is set.  It holds the discrete decisions of the
 * step and the two local residuals that enter them, so that a caller can
 * compare a solve decision by decision with another implementation of
 * solve/amen_solve2.m. */
typedef struct {
  int64_t sweep;    /* 1-based sweep number                                   */
  int64_t core;     /* 0-based core index                                     */
  int64_t rank;     /* rank kept by the residual-based truncation, after the
                       caps (amen_solve2.m:539-594), before the kick; -1 at
                       the last core, which is not truncated                  */
  int64_t iters;    /* Krylov steps of the local solve (over all restarts);
                       -1: dense branch (:468-492) or zero right-hand side    */
  double res_prev;  /* ||B x_prev - rhs|| / ||rhs||                   (:495)  */
  double res_new;   /* ||B x_new - rhs|| / ||rhs||                    (:504)  */
} ttg_amen_step;

typedef struct {
  int64_t nswp;          /* 50   */
  int64_t rmax;          /* 1000 */
  int64_t max_full_size; /* 50   */
  int64_t local_restart; /* 40   */
  int64_t local_iters;   /* 2    */
  int64_t kickrank;      /* 4    */
  double resid_damp;     /* 2    */
  double tol_exit;       /* <= 0: tol                       */
  int32_t trunc_norm;    /* 1 = 'residual' (only value supported) */
  int32_t local_prec;    /* 0 '', 1 'cjacobi', 2 'ljacobi', 3 'rjacobi' (FP64 only);
                            amen_solve2.m:205-207                           */
  int32_t precision;     /* TTG_FP64 or TTG_MIXED           */
  int32_t verb;          /* 0 silent, 1 per-sweep line on stderr */
  uint64_t seed;         /* seed for device-drawn x0/z0     */
  int32_t timing;        /* 1: time every local matvec with CUDA events */
  int32_t reserved;
  ttg_amen_step* trace;  /* NULL, or room for trace_cap steps (host memory) */
  int64_t trace_cap;     /* steps beyond the capacity are counted, not stored */
} ttg_amen_opts;

#define TTG_MAX_SWEEPS_RECORDED 64
typedef struct {
  int64_t sweeps;
  int64_t matvecs;        /* local matvecs in the working precision      */
  int64_t matvecs_fp64;   /* FP64 local matvecs (residual checks)        */
  int64_t local_solves;
  int64_t gmres_iters;
  int64_t max_rank;
  double max_res[TTG_MAX_SWEEPS_RECORDED]; /* per sweep, amen_solve2.m:521 */
  double max_dx[TTG_MAX_SWEEPS_RECORDED];
  double ms_total;
  double ms_matvec;       /* device time inside local matvecs (if timed)  */
  double matvec_gflop;    /* algorithmic FLOPs of all local matvecs / 1e9 */
  int64_t launches;       /* kernels launched by the solve                */
  int64_t matvecs_lp;     /* BF16 tensor-core local matvecs (mixed)       */
  double gflop_lp;        /* their algorithmic FLOPs / 1e9                */
  double ms_lp;           /* their device time (opts.timing = 1)          */
  double gflop_fp64;      /* FP64 local-matvec FLOPs / 1e9                */
  double ms_fp64;         /* their device time (opts.timing = 1)          */
  int64_t trace_len;      /* local steps run (entries written to opts.trace,
                             up to its capacity)                          */
  double gbyte_lp;        /* algorithmic DRAM bytes of the BF16 matvecs / 1e9
                             (operand, operators and result once each)    */
} ttg_amen_stats;

void ttg_amen_opts_default(ttg_amen_opts* opts);
int ttg_amen_solve(ttg_tt A, ttg_tt y, double tol, const ttg_amen_opts* opts,
                   ttg_tt x0, ttg_tt z0, ttg_tt* x_out, ttg_amen_stats* stats);

/* ---- ALS(t+z) solve ---------------------------------------------------------
 * Replaces [x,testdata] = alstpz_solve(A, y, tol, 'name', value, ...)
 * (solve/alstpz_solve.m:1) on its default path, kicktype 'svd': each of
 * nswp sweeps rounds x to tol (:140), rounds the exact residual y - A x to
 * rank kickrank (:189-195), appends it to x with weight zero (:199-201) and
 * runs one ALS sweep of local solves (als_solve, :217-428: QR
 * orthogonalisation, dense local solve below max_full_size, else the MEX
 * local solver).  Every sweep runs (the reference has no stopping test).
 * The options are ttg_amen_opts: nswp, max_full_size, local_restart,
 * local_iters, kickrank, resid_damp, local_prec, precision, verb, seed are
 * read; opts = NULL takes ttg_alstpz_opts_default (nswp 10, max_full_size
 * 50, kickrank 4, :56-67).  x0 may be NULL: a right-orthogonal random TT of
 * rank 2 is drawn on the device (tt_rand, :116-118).  stats (nullable):
 * sweeps, per-sweep max_res / max_dx of the ALS sweeps (:371-373), local
 * solves, Krylov steps, max rank, launches; ms_total is host-clock time. */
void ttg_alstpz_opts_default(ttg_amen_opts* opts);
int ttg_alstpz_solve(ttg_tt A, ttg_tt y, double tol, const ttg_amen_opts* opts, ttg_tt x0,
                     ttg_tt* x_out, ttg_amen_stats* stats);

/* ---- kernel-level entries (device pointers) --------------------------------
 * Local matvec y = (Phi1 x A x Phi2) x, the reference's bfun3
 * (solve/amen_solve2.m:924-951; twin fmex/solve3d.c:141-195).
 * Phi1 [rx1, rx1, ra1], A [ra1, n, n, ra2], Phi2 [rx2, ra2, rx2],
 * x, y [rx1, n, rx2].  x and y must not overlap. */
int ttg_local_matvec(ttg_context ctx, int64_t rx1, int64_t n, int64_t rx2,
                     int64_t ra1, int64_t ra2, const double* Phi1,
                     const double* A, const double* Phi2, const double* x,
                     double* y, int32_t precision);

/* Interface update, the reference's compute_next_Phi
 * (solve/amen_solve2.m:834-920).  dir 0 = 'lr': Phi_prev [rx1, ry1, ra1] ->
 * Phi_out [rx2, ry2, ra2];  dir 1 = 'rl': Phi_prev [ry2, ra2, rx2] ->
 * Phi_out [ry1, ra1, rx1].  x [rx1, n, rx2], y [ry1, n, ry2],
 * A [ra1, n, n, ra2] or NULL (then ra1 = ra2 = 1, the X'Y variant).
 * If nrm_out != NULL the result is divided by its Frobenius norm, which is
 * returned in *nrm_out (host), as with nargout > 1 (:907-914). */
int ttg_next_phi(ttg_context ctx, int32_t dir, int64_t rx1, int64_t n,
                 int64_t rx2, int64_t ry1, int64_t ry2, int64_t ra1,
                 int64_t ra2, const double* Phi_prev, const double* x,
                 const double* A, const double* y, double* Phi_out,
                 double* nrm_out);

/* Local solve with the signature of the MEX gateway
 * sol = solve3d_2(Phi1, A, Phi2, rhs, tol, trunc_norm, sol_prev, prec,
 *                 nrestart, niters, verb)       (fmex/solve3d_2.c:121-122)
 * Residual branch (trunc_norm = 1) only; prec 0 (none), 1 ('cjacobi'),
 * 2 ('ljacobi') or 3 ('rjacobi'): the block-Jacobi right preconditioners
 * of solve/solve3d_2ml.m:21-70, FP64 only (the ljacobi / rjacobi inverse
 * blocks are limited to 2^28 doubles in total).  tol is relative to
 * ||rhs|| as in the MEX (fmex/solve3d_2.c:263-267).  nrestart is clamped to
 * rx1*n*rx2 (:184).  *iters_out (nullable) receives the Krylov iterations. */
int ttg_local_solve(ttg_context ctx, int64_t rx1, int64_t n, int64_t rx2,
                    int64_t ra1, int64_t ra2, const double* Phi1,
                    const double* A, const double* Phi2, const double* rhs,
                    double tol, int32_t trunc_norm, const double* sol_prev,
                    int32_t prec, int64_t nrestart, int64_t niters,
                    double* sol_out, int32_t precision, int64_t* iters_out);

/* Local matvec that allocates nothing.  No counterpart in the reference: it
 * is ttg_local_matvec (FP64) for callers that may not allocate device memory
 * -- hosts whose memory budget is owned by another pool, time-critical loops
 * that must not hit cudaMalloc's implicit synchronisation or out-of-memory
 * failure, plugin hosts whose memory manager forbids untracked allocations.
 * The caller passes device inputs and outputs only; the two contraction
 * intermediates use a fixed scratch array built into the library, 64 MiB per
 * GPU (8 Mi doubles), held by every GPU that loads the library until exit.
 * Sizes whose intermediates (rx1*n*ra2*rx2 + rx1*ra1*n*rx2 doubles) exceed
 * it are rejected with TTG_ERR_INVALID.  stream: a cudaStream_t (NULL = the
 * legacy default stream) of the current device; the call returns after the
 * stream has finished.  The first call on a device looks up the array's
 * device address and caches it for the life of the process, so make that
 * first call before any stream capture; after a cudaDeviceReset the cached
 * address is stale, so do not call it again in that process.  All calls on
 * a device share the array: calls whose GPU
 * work overlaps (other streams, other host threads) race on it and must be
 * serialised by the caller. */
int ttg_local_matvec_noalloc(void* stream, int64_t rx1, int64_t n, int64_t rx2,
                             int64_t ra1, int64_t ra2, const double* Phi1,
                             const double* A, const double* Phi2, const double* x,
                             double* y);

/* ---- device FP64 factorizations used by the sweeps (device pointers) -------
 * Thin QR A = Q R (Q m x k, R k x n, k = min(m,n); Householder with LAPACK's
 * sign convention, as MATLAB's qr(A,0) at round.m:41 / amen_solve2.m:342) and
 * economy SVD A = U diag(S) VT (U m x k, S k descending, VT k x n; as
 * svd(A,'econ') at round.m:65 / amen_solve2.m:533).  Column-major, leading
 * dimension = row count.  A is not modified. */
int ttg_dense_qr(ttg_context ctx, int64_t m, int64_t n, const double* A, double* Q, double* R);
int ttg_dense_svd(ttg_context ctx, int64_t m, int64_t n, const double* A, double* U, double* S,
                  double* VT);

/* AMEn approximate matrix-by-vector product y ~ A x
 * ([y, z] = amen_mv(A, x, tol, ...), core/amen_mv.m:1-419, default path:
 * renorm 'direct', fkick false, kickrank2 0).  A: TT matrix with square
 * cores matching x.  y0 / z0 (nullable: right-orthogonal random TTs of
 * ranks 2 / kickrank drawn from opts->seed) as the options 'y0', 'z0'.
 * y_out receives the approximation; z_out (nullable) the error TT;
 * sweeps_out (nullable) the sweeps run. */
typedef struct {
  int64_t nswp;      /* 20 (amen_mv.m:55)            */
  int64_t kickrank;  /* 4  (:56); 0 disables z        */
  int32_t init_qr;   /* 1  (:61)                      */
  int32_t verb;      /* 0                             */
  uint64_t seed;     /* random y0 / z0 when NULL      */
  int64_t reserved[4];
} ttg_amen_mv_opts;

int ttg_amen_mv_opts_default(ttg_amen_mv_opts* opts);
int ttg_amen_mv(ttg_tt A, ttg_tt x, double tol, const ttg_amen_mv_opts* opts, ttg_tt y0,
                ttg_tt z0, ttg_tt* y_out, ttg_tt* z_out, int64_t* sweeps_out);

/* AMEn approximation of linear combinations of TT tensors
 * ([y, z] = amen_sum(X, v, tol, 'name', value, ...), core/amen_sum.m:1-483,
 * default path for TT inputs: renorm 'direct', fkick false, kickrank2 0,
 * multrank false).  X: `count` TT tensors of one context with equal mode
 * sizes and boundary ranks 1; coef: count x M host array (column-major):
 * y(:, m) ~ sum_j X[j] coef(j, m), m = 1..M, returned as one TT whose last
 * rank is M (one tensor for M = 1).  y0 / z0 (nullable) as the options
 * 'y0' / 'z0'; when NULL, right-orthogonal random TTs of ranks 2 /
 * kickrank are drawn from opts->seed (the reference draws its own,
 * amen_sum.m:152-187, from MATLAB's generator).  z_out (nullable) receives
 * the error TT, sweeps_out (nullable) the sweeps run. */
typedef struct {
  int64_t nswp;      /* 20 (amen_sum.m:56)             */
  int64_t kickrank;  /* 4  (:57); 0 disables z          */
  int32_t init_qr;   /* 1  (:63)                        */
  int32_t verb;      /* 0                               */
  uint64_t seed;     /* random y0 / z0 when NULL        */
  int64_t rmax;      /* <= 0: no cap (:67, Inf)         */
  int64_t reserved[3];
} ttg_amen_sum_opts;

int ttg_amen_sum_opts_default(ttg_amen_sum_opts* opts);
int ttg_amen_sum(int64_t count, const ttg_tt* X, const double* coef, int64_t M, double tol,
                 const ttg_amen_sum_opts* opts, ttg_tt y0, ttg_tt z0, ttg_tt* y_out,
                 ttg_tt* z_out, int64_t* sweeps_out);

/* TT algebra on device-resident handles (the caller side of the path: the
 * true residual ||A x - y|| / ||y||, round's inputs).  Results are new
 * handles of the operands' context; tensors need boundary ranks 1 for dot.
 *   ttg_tt_matvec : exact A x, ranks multiply   (@tt_matrix/mtimes.m:38-65)
 *   ttg_tt_axpby  : a x + b y, ranks add         (@tt_tensor/plus.m:40-86)
 *   ttg_tt_norm   : QR-based Frobenius norm      (@tt_tensor/norm.m:16-42)
 *   ttg_tt_dot    : <x, y>                       (@tt_tensor/dot.m:92-111) */
int ttg_tt_matvec(ttg_tt A, ttg_tt x, ttg_tt* out);
int ttg_tt_axpby(double a, ttg_tt x, double b, ttg_tt y, ttg_tt* out);
int ttg_tt_norm(ttg_tt x, double* nrm);
int ttg_tt_dot(ttg_tt x, ttg_tt y, double* val);

/* SDV TT files (the toolbox's binary format: fmex/tt_read.c:13-100,
 * fmex/tt_write.c:21-80; read by tt_tensor(filename),
 * @tt_tensor/tt_tensor.m:150).  Reading gives a TT tensor handle of ctx
 * (float files are widened to double; complex files fail with
 * TTG_ERR_UNSUPPORTED).  Writing stores a tensor, or a TT matrix as the tensor
 * of its cores with mode sizes n_k m_k; precision 0 = double, 1 = float. */
int ttg_tt_read_sdv(ttg_context ctx, const char* path, ttg_tt* out);
int ttg_tt_write_sdv(ttg_tt tt, const char* path, int32_t precision);

/* Batched amen_solve2: `count` independent systems A[i] x = y[i] solved
 * concurrently on the context's device.  No single reference counterpart:
 * each system is amen_solve2(A{i}, y{i}, tol(i), opts{i}) (solve/amen_solve2.m:1);
 * the batch replaces a MATLAB loop over systems.  `workers` host threads
 * (0 = 8; at most count and 64), each with its own CUDA stream, allocator
 * and solver handle, take systems in index order, so the systems' kernels
 * overlap on the GPU.  All handles belong to ctx; x0 / z0 (nullable arrays,
 * NULL entries allowed) as in ttg_amen_solve; tol[i] per system; opts
 * (nullable = defaults) is an array of `count` option sets; stats
 * (nullable) an array of `count`.  x_out[i] receives a new handle of ctx, or
 * NULL when system i failed; status (nullable) receives each system's code.
 * Every system runs even when some fail; the call then returns the code of
 * the lowest-numbered failing system with its message. */
int ttg_amen_solve_batch(ttg_context ctx, int64_t count, const ttg_tt* A, const ttg_tt* y,
                         const double* tol, const ttg_amen_opts* opts, const ttg_tt* x0,
                         const ttg_tt* z0, int32_t workers, ttg_tt* x_out,
                         ttg_amen_stats* stats, int32_t* status);

/* Counters of a grouped batch (ttg_amen_solve_grouped). */
typedef struct {
  int64_t flushes;          /* times every solve in flight waited for the device */
  int64_t launches;         /* launches and stream operations issued */
  int64_t records;          /* launches and stream operations the solves recorded */
  int64_t grouped_records;  /* recorded launches issued inside grouped launches */
  double ms_plan;           /* host time merging records and writing argument packs */
  double ms_issue_wait;     /* host time issuing and waiting for the device */
  double ms_total;          /* wall time of the call */
  int64_t lanes_max;        /* most streams one flush issued on */
  double ms_record;         /* wall time the solves spent recording between flushes */
  int64_t allocs;           /* device blocks the solves took from the shared allocator */
  int64_t device_mallocs;   /* of which new cudaMalloc blocks */
  double ms_alloc;          /* thread time in the shared allocator (lock waits included) */
  double ms_issue;          /* host time issuing (part of ms_issue_wait) */
  /* BF16 tensor-core GEMM launches (the local matvec stages), counted and,
   * with TTG_GROUP_TIME=1 in the environment, timed by CUDA events around
   * each launch on its stream (the events cost the launches their
   * programmatic overlap: use it in a separate, instrumented run). */
  int64_t tc_launches;      /* issued launches of the BF16 GEMM kernel */
  int64_t tc_records;       /* recorded GEMMs inside those launches */
  double tc_gflop;          /* algorithmic GFLOP of those GEMMs (2 M N K) */
  double tc_ms;             /* summed event time of those launches (0 untimed) */
} ttg_group_stats;

/* Grouped batch: the same solves as ttg_amen_solve_batch (same arguments,
 * results and per-system status), advanced together on the context's
 * stream.  Every system in flight runs on a host thread of its own whose
 * stream work is recorded; whenever all of them wait for the device, the
 * recorded launches of all systems are merged kernel by kernel into grouped
 * launches (one launch runs a kernel's CTAs for many systems, each system
 * with its own grid and arguments) and issued with one copy of their
 * arguments.  Each system's kernels run in its own order with its own
 * arguments, so every system gets the result of its own sequential solve.
 * `width` systems are in flight at once (<= 0: all of them, at most 1024);
 * group_stats (nullable) receives the counters above. */
int ttg_amen_solve_grouped(ttg_context ctx, int64_t count, const ttg_tt* A, const ttg_tt* y,
                           const double* tol, const ttg_amen_opts* opts, const ttg_tt* x0,
                           const ttg_tt* z0, int32_t width, ttg_tt* x_out,
                           ttg_amen_stats* stats, int32_t* status,
                           ttg_group_stats* group_stats);

/* ---- Gradients with respect to every core (FP64) ----------------------
 * No counterpart in the reference: TT-Toolbox has no derivative code.  The
 * forward maps are the reference's own, cited per entry.  x is a TT tensor
 * with boundary ranks 1; grad is a DEVICE buffer of numel(x) doubles
 * (ttg_malloc), written in x's flat core layout (grad of core k at the
 * offset of core k); value (nullable, host) receives f(x).  Operands must
 * belong to the same context. */

/* f(x) = <x, A x>: @tt_matrix/mtimes.m:38-65 then @tt_tensor/dot.m:92-111.
 * A: TT matrix with A.n = A.m = x.n. */
int ttg_grad_xAx(ttg_tt x, ttg_tt A, double* grad, double* value);

/* f(x) = <x, b>: @tt_tensor/dot.m:92-111.  b: TT tensor with b.n = x.n. */
int ttg_grad_xb(ttg_tt x, ttg_tt b, double* grad, double* value);

/* f(x) = sum_s (X[idx_s] - y_s)^2 with X[idx_s] the entry of the element
 * path @tt_tensor/subsref.m:93-123.  idx: DEVICE int32 array, column-major
 * nsamples x d (column k holds the mode-k indices, as MATLAB's ind(:,k)),
 * 0-based; an index outside [0, n_k) fails with TTG_ERR_INVALID.
 * y: DEVICE array of nsamples doubles.  Mode sizes up to 8192. */
int ttg_grad_sampled(ttg_tt x, int64_t nsamples, const int32_t* idx, const double* y,
                     double* grad, double* value);

#ifdef __cplusplus
}
#endif
#endif /* TTGPU_H */
