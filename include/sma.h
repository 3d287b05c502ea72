/*
 * sma.h -- C ABI of libsma, the B200 (sm_100a) implementation of the two solve-free
 * interior eigensolvers of MathiasTensor/sparse_matrix_algorithms:
 *
 *   chebyshev_poly_real_symm_sparse(A, emin, emax; ...)    chebyshev_subspace_iteration.jl:667
 *   chebyshev_poly_real_symm_sparse(matvec!, n, emin, emax; ...)   chebyshev_subspace_iteration.jl:771
 *   polfed(A::MatrixFreeRealSymOp, nev, degree; ...)        polfed.jl:1128
 *   polfed(matvec!, n, nev, degree; matblock!=nothing, ...) polfed.jl:1183
 *
 * Every entry point takes plain pointers and sizes.  Unless stated otherwise pointers
 * are HOST pointers.  Dense blocks handed to the device entry points (suffix _dev) are
 * ROW-MAJOR: element (i, j) of an n x b block with leading dimension ld sits at
 * X[i*ld + j] (ld >= b).  Blocks exchanged with host callers are column-major, as a
 * Julia Matrix{Float64} is.
 *
 * Status codes mirror the reference's error behaviour: SMA_ERR_ARG is Julia's
 * ArgumentError, SMA_ERR_BOUNDS the `error(...)` of polfed.jl:1130, SMA_ERR_WINDOW the
 * unknown-window error of polfed.jl:413.  sma_last_error() returns the message of the
 * calling thread's last failure.
 *
 * Threading: a context owns one CUDA stream and its library handles; use a context
 * from one host thread at a time.  Different contexts are independent.
 */
#ifndef SMA_H
#define SMA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMA_ABI_VERSION 1

enum sma_status {
  SMA_OK = 0,
  SMA_ERR_ARG = 1,          /* ArgumentError (chebyshev_subspace_iteration.jl:669-674) */
  SMA_ERR_NONSYMMETRIC = 2, /* issymmetric(Ain) failed (chebyshev_subspace_iteration.jl:669) */
  SMA_ERR_INTERVAL = 3,     /* mapped interval not inside [-1,1] (chebyshev_subspace_iteration.jl:689) */
  SMA_ERR_CUDA = 4,         /* CUDA / cuBLAS / cuSOLVER failure */
  SMA_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
  SMA_ERR_NOCONV = 6,
  SMA_ERR_NOMEM = 7,
  SMA_ERR_BOUNDS = 8,       /* "Matrix-free POLFED requires spectral bounds" (polfed.jl:1130) */
  SMA_ERR_WINDOW = 9,       /* "Unknown window type" (polfed.jl:413) */
  SMA_ERR_CALLBACK = 10,    /* a user operator callback returned non-zero */
  SMA_ERR_INTERNAL = 11
};

enum sma_window { SMA_WINDOW_STEP = 0, SMA_WINDOW_DELTA = 1, SMA_WINDOW_SMOOTH = 2 };

/* Arithmetic of the block Clenshaw filter.  FP64 is the reference's arithmetic.  MIXED
 * (solvers only) filters in FP32 while that still reduces the residuals, then in FP64 for
 * the final iterations; orthogonalization, Rayleigh-Ritz and residuals are always FP64. */
enum sma_precision { SMA_PREC_FP64 = 0, SMA_PREC_FP32 = 1, SMA_PREC_MIXED = 2 };

typedef struct sma_ctx sma_ctx;
typedef struct sma_op sma_op;
typedef struct sma_result sma_result;

/* Device block operator supplied by the caller (the GPU form of the reference's
 * matblock!, chebyshev_subspace_iteration.jl:186-197 / polfed.jl:209-219): write
 * Y = A X for the row-major n x b blocks X_dev, Y_dev (leading dimension ld, FP64),
 * enqueuing all work on `stream` (a cudaStream_t).  Return 0 on success. */
typedef int (*sma_matblock_fn)(void *user, const double *X_dev, double *Y_dev, int64_t n,
                               int64_t b, int64_t ld, void *stream);

/* Keyword arguments of chebyshev_poly_real_symm_sparse (chebyshev_subspace_iteration.jl:667). */
typedef struct sma_cheb_opts {
  double smin, smax;      /* spectral bounds, used when has_bounds != 0 */
  int64_t has_bounds;     /* 0: Gershgorin bounds (smin=nothing / smax=nothing) */
  double sigma;           /* centre of the :delta window */
  int64_t m0;             /* subspace size (default 200) */
  int64_t degree;         /* filter degree (default 80) */
  int64_t maxiter;        /* default 8 */
  double tol;             /* default 1e-10 */
  double res_gate;        /* default 1e-6 */
  int64_t jackson;        /* default 1 */
  int64_t debug;          /* print the per-iteration line */
  int64_t two_hit;        /* default 1 */
  int64_t seed;           /* start block seed (default 1) */
  int64_t window_type;    /* enum sma_window, default SMA_WINDOW_STEP */
  int64_t matrix_free;    /* 0: sparse overload semantics (always maxiter iterations,
                             chebyshev_subspace_iteration.jl:731-749); 1: matrix-free overload
                             semantics (two_hit early exit, chebyshev_subspace_iteration.jl:827-836) */
  int64_t precision;      /* enum sma_precision of the filter, default SMA_PREC_FP64 */
  int64_t lock;           /* 1: lock converged pairs (an extension: the reference's TODO at
                             chebyshev_subspace_iteration.jl:117 and its unused append_locked!,
                             :282-290).  Pairs inside [emin, emax] with residual < tol leave
                             the filtered block; later blocks are orthogonalized against them.
                             Default 0 (the reference's behaviour). */
  int64_t reserved[7];
} sma_cheb_opts;

/* Keyword arguments of polfed (polfed.jl:1128). */
typedef struct sma_polfed_opts {
  int64_t s;              /* block size (default 8) */
  double smin, smax;      /* spectral bounds (required) */
  int64_t has_bounds;     /* 0 -> SMA_ERR_BOUNDS, as polfed.jl:1130 */
  double sigma;           /* default 0 */
  double emin, emax;      /* default -Inf, +Inf */
  double tol;             /* default 1e-10 */
  int64_t threaded;       /* accepted, unused (as in the reference) */
  int64_t overextract;    /* default 2 */
  int64_t refine;         /* default 1 */
  int64_t window_type;    /* default SMA_WINDOW_STEP */
  int64_t jackson;        /* default 1 */
  int64_t mmax;           /* 0: ceil(2.8*nev/s) (polfed.jl:1132) */
  double rtol;            /* default 1e-12 */
  int64_t reorth_passes;  /* default 1 */
  int64_t extra_keep;     /* default 8 */
  int64_t seed;           /* default 1 */
  int64_t show_progress;  /* print the _progress_line summary (polfed.jl:991-1000) */
  int64_t chunk;          /* default 64 (extraction chunking; results do not depend on it) */
  int64_t precision;      /* enum sma_precision of the filter, default SMA_PREC_FP64 */
  int64_t reserved[8];
} sma_polfed_opts;

/* Per-solve counters and phase timings (device time, CUDA events). */
typedef struct sma_stats {
  int64_t iterations;     /* Chebyshev iterations or POLFED blocks */
  int64_t basis_dim;      /* POLFED basis dimension M; Chebyshev m0 */
  int64_t spmm_steps;     /* block sparse products issued by the filter */
  int64_t spmm_columns;   /* sum over those products of the block width */
  double filter_ms;       /* block Clenshaw filter (the POLFED basis / Chebyshev iterations;
                             the MIXED polish is counted in polish_ms) */
  double orth_ms;         /* orthogonalization / reorthogonalization */
  double rr_ms;           /* Rayleigh-Ritz, residuals, extraction */
  double total_ms;        /* whole solve, wall clock from call to return */
  double filter_bytes;    /* algorithmic bytes of those filter products */
  int64_t qr_fallbacks;   /* blocks that left CholQR2 for shifted CholQR3 / Householder */
  int64_t warnings;       /* bit 0: interval outside the spectral bounds */
  int64_t kernel_launches; /* this library's own CUDA kernels launched by the solve
                              (cuBLAS / cuSOLVER launches not included) */
  int64_t fp32_filter_calls; /* filter applications run in FP32 (FP32 / MIXED precision) */
  int64_t locked;         /* pairs locked during the solve (Chebyshev with lock = 1) */
  int64_t polish_iterations; /* FP64 polishing iterations after an FP32 POLFED basis */
  int64_t graph_replays;  /* CUDA graph launches of the batched slicing filter */
  double polish_ms;       /* MIXED POLFED polish: filters, orthonormalization, Rayleigh-Ritz */
  double polish_bytes;    /* algorithmic bytes of the polish's filter products */
  int64_t reserved[1];
} sma_stats;

/* Options of batched spectrum slicing (sma_slice_solve); every window runs Chebyshev
 * subspace iteration with the matrix-free overload's termination rule
 * (chebyshev_subspace_iteration.jl:827-836). */
typedef struct sma_slice_opts {
  double smin, smax;       /* spectral bounds, used when has_bounds != 0 (else Gershgorin) */
  int64_t has_bounds;
  int64_t maxiter;         /* iterations per window, at most */
  double tol;              /* absolute residual below which a window has converged */
  double res_gate;         /* residual gate of the convergence count */
  int64_t jackson;
  int64_t two_hit;         /* 1: a window stops after two consecutive converged iterations */
  int64_t seed;            /* window w starts from the random block of seed + w */
  int64_t window_type;     /* sma_window; delta windows centre on (emin + emax) / 2 */
  int64_t precision;       /* sma_precision; MIXED switches each window separately */
  int64_t graph;           /* 1: record the batched filter into a CUDA graph and replay it */
  int64_t debug;           /* 1: one progress line per window and iteration on stdout */
  int64_t reserved[8];
} sma_slice_opts;

/* ---------------------------------------------------------------- library, context */
int sma_abi_version(void);
const char *sma_last_error(void);
/* Kernels of this library launched by this process so far (all contexts; graph replays
 * count every kernel they contain; cuBLAS / cuSOLVER launches are not included). */
int64_t sma_kernel_launch_count(void);
int sma_ctx_create(int device, sma_ctx **out);
int sma_ctx_destroy(sma_ctx *ctx);
int sma_ctx_synchronize(sma_ctx *ctx);
/* The context's cudaStream_t. */
void *sma_ctx_stream(sma_ctx *ctx);

/* ---------------------------------------------------------------- operators */
/* Upload a sparse symmetric matrix given as CSC arrays (Julia's SparseMatrixCSC
 * colptr/rowval/nzval, chebyshev_subspace_iteration.jl:667; for a symmetric matrix
 * these are also its CSR arrays).  index_base 1 for Julia, 0 for C.  Row indices must
 * be sorted within each column.  check_symmetric != 0 verifies A == A^T exactly on the
 * device (the issymmetric check of chebyshev_subspace_iteration.jl:669). */
int sma_op_create_csc(sma_ctx *ctx, int64_t n, int64_t nnz, const int64_t *colptr,
                      const int64_t *rowval, const double *nzval, int64_t index_base,
                      int64_t check_symmetric, sma_op **out);
/* Symmetric half storage (no counterpart in the reference; the "next" item of its CSC
 * path): the same CSC arguments as sma_op_create_csc, but only the upper triangle
 * (diagonal included) is kept on the device, about half the entries and indices.  Products
 * are a row pass plus an atomic scatter of the transposed half, so they agree with full
 * storage to rounding, not bit for bit; the filter runs as product + axpy.  The lower
 * triangle is ignored: the operator applied is U + U^T - D for the stored upper triangle
 * U (diagonal D), whatever the lower triangle held; check_symmetric != 0 verifies
 * a_ij == a_ji on the host first and rejects a non-symmetric input.  Gershgorin bounds are
 * those of the operator applied.  Not accepted by sma_slice_solve. */
int sma_op_create_csc_upper(sma_ctx *ctx, int64_t n, int64_t nnz, const int64_t *colptr,
                            const int64_t *rowval, const double *nzval, int64_t index_base,
                            int64_t check_symmetric, sma_op **out);
/* Matrix-free 1D Laplacian tridiag(-1,2,-1) as a device stencil (the reference's
 * lap1d_matblock!, polfed.jl:1209-1219). */
int sma_op_create_lap1d(sma_ctx *ctx, int64_t n, sma_op **out);
/* Matrix-free 3D Anderson model on an L^3 periodic lattice (L >= 3) as a device stencil:
 * eps[i] (i = x + L*(y + L*z), L^3 host doubles) on the diagonal, hopping t to the six
 * neighbours.  Products are bit-identical to the stored CSR matrix's.  An extension that
 * gives the reference's matrix-free signatures (MatrixFreeRealSymOp, polfed.jl:165) a GPU
 * operator for this model with no index arrays. */
int sma_op_create_anderson(sma_ctx *ctx, int64_t L, const double *eps, double t, sma_op **out);
/* Matrix-free random-field XXZ chain (even L in 4..30, periodic) in the Sz = 0 sector as a
 * device stencil: H = J sum (SxSx + SySy + Delta SzSz) + sum h_i Sz_i, S = sigma/2, basis
 * ordered by the states' integer values (bit i = site i up); h holds L host doubles. */
int sma_op_create_xxz(sma_ctx *ctx, int64_t L, double J, double Delta, const double *h,
                      sma_op **out);
/* Matrix-free operator from a caller-supplied device block callback
 * (MatrixFreeRealSymOp(n, matvec!, matblock!), polfed.jl:165). */
int sma_op_create_matblock(sma_ctx *ctx, int64_t n, sma_matblock_fn fn, void *user,
                           sma_op **out);
int sma_op_destroy(sma_op *op);
int sma_op_info(const sma_op *op, int64_t *n, int64_t *nnz);
/* Gershgorin bounds (chebyshev_subspace_iteration.jl:351-367); explicit matrices only. */
int sma_gershgorin_bounds(sma_op *op, double *smin, double *smax);
/* Tighter spectral bounds than Gershgorin's (an extension; the reference has only
 * gershgorin_bounds): `steps` Lanczos steps in FP64 with full reorthogonalization from a
 * seeded random vector; the extreme Ritz values widened by their residual norms (at least
 * 1e-3 of the Ritz range), clipped to the Gershgorin interval when the operator has one
 * (explicit matrices, model stencils).  An estimate.  Any operator kind. */
int sma_lanczos_bounds(sma_op *op, int64_t steps, int64_t seed, double *smin, double *smax);

/* Stochastic Chebyshev moments of the spectral density, the kernel polynomial method (an
 * extension; the reference has no density-of-states estimate):
 *   mu[k] = (1/(n R)) sum_r z_r^T T_k(A_hat) z_r,  k < M,  A_hat = (A - c I)/d,
 * with c, d the centre and half-width of [smin, smax] and R Rademacher vectors z_r drawn
 * from the seeded SplitMix64 stream (mu[0] = 1 exactly).  FP64, ceil(M/2) block products
 * of width R.  per_vec (may be NULL) receives the M x R per-vector moments, row-major.
 * Any operator kind.  Synchronous. */
int sma_kpm_moments(sma_op *op, int64_t M, int64_t R, int64_t seed, double smin, double smax,
                    double *mu, double *per_vec);
/* Number of eigenvalues in [emin, emax] predicted by the moments of an n x n operator:
 * n times the integral of the Jackson-damped (jackson != 0) Chebyshev density series. */
int sma_kpm_count(const double *mu, int64_t M, int64_t n, double smin, double smax,
                  double emin, double emax, int64_t jackson, double *count);

/* ---------------------------------------------------------------- filter coefficients */
/* jackson_kernel(K): g[0..K] (chebyshev_subspace_iteration.jl:376-387). */
int sma_jackson_kernel(int64_t K, double *g);
/* cheb_delta_coeffs (chebyshev_subspace_iteration.jl:400-414). */
int sma_cheb_delta_coeffs(double sigma_hat, int64_t K, int64_t jackson, double *c);
/* cheb_window_coeffs (chebyshev_subspace_iteration.jl:430-447). */
int sma_cheb_window_coeffs(double a, double b, int64_t K, int64_t jackson, double *c);
/* cheb_smooth_window_coeffs (chebyshev_subspace_iteration.jl:465-489). */
int sma_cheb_smooth_window_coeffs(double a, double b, int64_t K, int64_t jackson,
                                  int64_t nsamp, double delta, double *c);
/* _build_coeffs (polfed.jl:404-414): c has degree+1 entries. */
int sma_build_coeffs(int64_t degree, double smin, double smax, double sigma, double emin,
                     double emax, int64_t window_type, int64_t jackson, double *c);

/* ---------------------------------------------------------------- the hot path */
/* Y = p(A_hat) Q by the block Clenshaw recurrence (apply_poly_block!,
 * chebyshev_subspace_iteration.jl:554-591 and 598-635, polfed.jl:464-545) on device
 * blocks.  coeffs: K+1 host doubles.  precision selects the element type of Q_dev and
 * Y_dev (double for SMA_PREC_FP64, float for SMA_PREC_FP32).  Synchronous. */
int sma_apply_poly_block_dev(sma_op *op, const double *coeffs, int64_t K, double smin,
                             double smax, const void *Q_dev, int64_t ldq, void *Y_dev,
                             int64_t ldy, int64_t b, int64_t precision);
/* Same filter on host column-major n x b FP64 blocks (copies in and out). */
int sma_apply_poly_block(sma_op *op, const double *coeffs, int64_t K, double smin,
                         double smax, const double *Q, double *Y, int64_t b,
                         int64_t precision);
/* The block filter with one polynomial per column (an extension; the reference filters a
 * block with one polynomial): column j of Y_dev is sum_m coeffs[m*b + j] T_m(A_hat) applied
 * to column j of Q_dev, by the same Clenshaw recurrence, for row-major n x b device blocks
 * with leading dimension b.  coeffs: (K+1) x b host doubles, row-major.  precision as in
 * sma_apply_poly_block_dev.  On a CSR matrix each column is bit-identical to
 * sma_apply_poly_block_dev with that column's coefficients.  Device operators only.
 * MIXED-precision POLFED uses it to apply, per Ritz vector, the divided difference of its
 * filter in FP32.  Synchronous. */
int sma_apply_poly_block_percol_dev(sma_op *op, const double *coeffs, int64_t K, double smin,
                                    double smax, const void *Q_dev, void *Y_dev, int64_t b,
                                    int64_t precision);
/* Divided difference of p = sum_{m=0..K} coeffs[m] T_m at t (K >= 1): e[0..K-1] with
 * (p(s) - p(t)) / (s - t) = sum_m e[m] T_m(s), and *pt = p(t) (an extension used by the
 * MIXED POLFED polish). */
int sma_divided_difference(const double *coeffs, int64_t K, double t, double *e, double *pt);
/* The tall-skinny FP64 products of the block orthogonalization and Rayleigh-Ritz steps
 * (the reference's Q' W and W - Q C of orth_against!/reorth_full!, polfed.jl:605-631, and
 * X = Q Xq of chebyshev_subspace_iteration.jl:735-740), on this library's FP64 tensor-core
 * (DMMA) kernels, exposed for callers and tests:
 *   gram:   C (m x k, column-major, ldc) = alpha X^T Y + beta C, X n x m and Y n x k
 *           row-major device blocks; deterministic (split-n partials summed in order);
 *   update: Y (n x p, row-major) = alpha X B + beta Y, X n x m row-major, B = C (m x p,
 *           column-major, ldc) or, with transC != 0, B = C^T (C p x m column-major).
 * Device pointers; synchronous. */
int sma_dense_gram_dev(sma_ctx *ctx, int64_t n, int64_t m, int64_t k, const double *X_dev,
                       int64_t ldx, const double *Y_dev, int64_t ldy, double *C_dev, int64_t ldc,
                       double alpha, double beta);
int sma_dense_update_dev(sma_ctx *ctx, int64_t n, int64_t m, int64_t p, const double *X_dev,
                         int64_t ldx, const double *C_dev, int64_t ldc, int64_t transC,
                         double *Y_dev, int64_t ldy, double alpha, double beta);
/* Y = A X on device row-major FP64 blocks (apply_A_block!). Synchronous. */
int sma_spmm_dev(sma_op *op, const double *X_dev, int64_t ldx, double *Y_dev, int64_t ldy,
                 int64_t b);
/* The FP64 filter of sma_apply_poly_block_dev without any device allocation, for callers
 * that cannot allocate device memory: processes whose GPU memory another allocator has
 * reserved up front, or latency-critical loops that must not pay for cudaMalloc/cudaFree.
 * No counterpart in the reference (its filter allocates Julia arrays).  Its three n x b
 * recurrence blocks live in one static device array of 48 MiB (held on every device that
 * loads it until exit), so n*b must be <= 2,097,152 (else SMA_ERR_ARG).  Device operators
 * only: CSR or a model stencil (1D Laplacian, Anderson, XXZ); half storage and caller
 * callbacks are rejected.  All calls on a device share the array: calls that overlap on
 * the GPU race, so serialize them.  The first call on a device looks the array up; make
 * it before any stream capture.  Synchronous. */
int sma_apply_poly_block_noalloc(sma_op *op, const double *coeffs, int64_t K, double smin,
                                 double smax, const double *Q_dev, int64_t ldq, double *Y_dev,
                                 int64_t ldy, int64_t b);

/* ---------------------------------------------------------------- solvers */
void sma_cheb_opts_default(sma_cheb_opts *o);
void sma_polfed_opts_default(sma_polfed_opts *o);
/* chebyshev_poly_real_symm_sparse; result sorted by eigenvalue, absolute residuals
 * (chebyshev_subspace_iteration.jl:750-756). */
int sma_cheb_solve(sma_op *op, double emin, double emax, const sma_cheb_opts *opts,
                   sma_result **out);
/* polfed; result order follows polfed.jl:1148-1157 (by eigenvalue when the nev-th
 * smallest residual is below tol, else by residual). */
int sma_polfed_solve(sma_op *op, int64_t nev, int64_t degree, const sma_polfed_opts *opts,
                     sma_result **out);

/* Batched POLFED (no counterpart in the reference, which runs polfed on one window per call,
 * polfed.jl:1128): nwin windows [emin[w], emax[w]] over the same explicit sparse matrix, each
 * a POLFED solve with its own nev[w], filter degree[w] and basis size mmax[w] blocks, its
 * filter centred on the window (sigma = (emin[w] + emax[w]) / 2) and start block seed
 * opts->seed + w.  The other options (s, smin, smax, tol, window_type, jackson, precision,
 * overextract, refine, rtol, reorth_passes, extra_keep, show_progress) apply to every
 * window; opts->emin/emax/sigma/mmax are ignored.  Every block step filters all active
 * windows' blocks in ONE segmented Clenshaw recurrence (windows sorted by degree, each
 * column with its own window's coefficients, recorded into a CUDA graph and replayed), so
 * each window's filtered block is bit-identical to its single-window filter and the matrix
 * is read once per step for all windows; a window leaves the batch when its basis is
 * complete.  MIXED: the basis filter in FP32, each window's pairs polished to FP64 accuracy.
 * The result holds window 0's pairs (in polfed's return order), then window 1's, ...;
 * sma_result_windows gives the window of every pair, sma_result_window_info each window's
 * blocks and whether the return rule's by-eigenvalue branch applied (the nev-th residual
 * below tol). */
int sma_polfed_batch_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                           const int64_t *nev, const int64_t *degree, const int64_t *mmax,
                           const sma_polfed_opts *opts, sma_result **out);

/* Batched spectrum slicing (no counterpart in the reference, which solves one window per
 * call): nwin windows [emin[w], emax[w]] over the same operator, each with its own filter
 * degree[w] and subspace width m0[w] (rounded up to a multiple of 8), solved together.
 * Every filter application runs ONE batched Clenshaw recurrence over the concatenation
 * of the windows' blocks: windows sorted by degree, each with its own coefficients, a
 * window's columns joining the recurrence at its own degree, so each window's filtered
 * block is bit-identical to a single-window filter.  Converged windows leave the batch.
 * Explicit sparse matrices only.  The result holds the pairs of window 0, then window 1,
 * ..., each by eigenvalue; sma_result_windows gives the window of every pair. */
void sma_slice_opts_default(sma_slice_opts *o);
int sma_slice_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                    const int64_t *degree, const int64_t *m0, const sma_slice_opts *opts,
                    sma_result **out);

/* ---------------------------------------------------------------- learned window planner */
/* A three-layer perceptron (in -> hid -> hid -> out, relu) with BF16 weights, FP32
 * biases and FP32 arithmetic, trained on the GPU by the library's own forward, backward
 * and Adam kernels (an extension: the reference picks degree and subspace size by hand).
 * It maps a window's KPM moments and mapped bounds to corrections of the plain rule's
 * filter degree, subspace width and eigenvalue count.  Parameters are packed as
 * W1 (hid x in, row-major), b1, W2 (hid x hid), b2, W3 (out x hid), b3: FP32 masters,
 * count = hid*in + hid + hid*hid + hid + out*hid + out.  Rows of X are samples. */
typedef struct sma_mlp sma_mlp;
int sma_mlp_create(sma_ctx *ctx, int64_t in, int64_t hid, int64_t out, int64_t seed,
                   sma_mlp **net);
int sma_mlp_destroy(sma_mlp *net);
int sma_mlp_num_params(const sma_mlp *net, int64_t *count);
int sma_mlp_get_params(const sma_mlp *net, float *params);
/* Loads FP32 masters (their BF16 copies are made on the device) and resets Adam. */
int sma_mlp_set_params(sma_mlp *net, const float *params);
/* Y (B x out) = network(X (B x in)), host arrays. */
int sma_mlp_forward(sma_mlp *net, const float *X, int64_t B, float *Y);
/* Loss (1/B) sum w (Y - T)^2 (w may be NULL: ones) and its gradient with respect to the
 * packed parameters (grad may be NULL), for host arrays X (B x in), T and w (B x out). */
int sma_mlp_grad(sma_mlp *net, const float *X, const float *T, const float *w, int64_t B,
                 float *loss, float *grad);
/* steps of minibatch Adam (lr, minibatch rows, L2 weight decay) over N host rows, all on
 * the device; loss_hist (may be NULL) receives the minibatch loss before each step. */
int sma_mlp_train(sma_mlp *net, const float *X, const float *T, const float *w, int64_t N,
                  int64_t steps, double lr, int64_t minibatch, int64_t seed,
                  double weight_decay, float *loss_hist);

/* Self-test of the bounded device wait (no counterpart in the reference): launches the
 * persistent filter's grid barrier with one CTA fewer than it awaits, so the wait must
 * give up after ~10 ms and report through its error flag.  Returns SMA_OK when the test
 * observed SMA_ERR_TIMEOUT (stored in *observed) and the context is usable afterwards. */
int sma_selftest_barrier_timeout(sma_ctx *ctx, int64_t *observed);

/* ---------------------------------------------------------------- results */
/* k = number of returned pairs, n = vector length. */
int sma_result_count(const sma_result *r, int64_t *k, int64_t *n);
/* Copy eigenvalues (k), eigenvectors (n x k, column-major) and residuals (k); any of
 * the three pointers may be NULL. */
int sma_result_copy(const sma_result *r, double *lam, double *X, double *res);
int sma_result_stats(const sma_result *r, sma_stats *stats);
/* Window index of each returned pair (k int64 values; 0 for single-window solvers). */
int sma_result_windows(const sma_result *r, int64_t *win);
/* Per window of a slicing result (nwin entries each, either pointer may be NULL): the
 * iterations it ran and whether it met its convergence rule (1) or ran out (0).  A
 * single-window solver's result reports one window. */
int sma_result_window_info(const sma_result *r, int64_t nwin, int64_t *iterations,
                           int64_t *converged);
int sma_result_free(sma_result *r);

#ifdef __cplusplus
}
#endif
#endif /* SMA_H */
