// Internal declarations shared by the libsma translation units.
#pragma once

#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <atomic>
#include <functional>
#include <cstdint>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sma.h"

namespace sma {

// ------------------------------------------------------------------ errors
// Internal code throws sma::Error; the extern "C" layer turns it into a status code
// and the thread-local message returned by sma_last_error().
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &msg);

#define SMA_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw ::sma::Error(e_ == cudaErrorMemoryAllocation ? SMA_ERR_NOMEM : SMA_ERR_CUDA, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

#define SMA_CUBLAS(call)                                                                 \
  do {                                                                                   \
    cublasStatus_t s_ = (call);                                                          \
    if (s_ != CUBLAS_STATUS_SUCCESS)                                                     \
      throw ::sma::Error(SMA_ERR_CUDA, std::string(#call) + ": cublas status " +        \
                                           std::to_string((int)s_));                    \
  } while (0)

#define SMA_CUSOLVER(call)                                                               \
  do {                                                                                   \
    cusolverStatus_t s_ = (call);                                                        \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                                   \
      throw ::sma::Error(SMA_ERR_CUDA, std::string(#call) + ": cusolver status " +      \
                                           std::to_string((int)s_));                    \
  } while (0)

// Every launch of this library's own kernels goes through SMA_CHECK_LAUNCH, which
// also counts it (sma_stats.kernel_launches).
extern std::atomic<int64_t> g_kernel_launches;
#define SMA_CHECK_LAUNCH()                                                     \
  do {                                                                         \
    ::sma::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);          \
    SMA_CUDA(cudaGetLastError());                                              \
  } while (0)

inline void require(bool ok, int code, const std::string &msg) {
  if (!ok) throw Error(code, msg);
}

// Online autotuner state of the CSR Clenshaw step for one (element type, vector width,
// variant, block width, leading dimension) key of an operator (csr_clenshaw.cuh).
struct CsrTune {
  std::vector<int> cands;           // encoded candidate configurations
  std::vector<int> trial;           // configuration of each timed launch so far
  std::vector<cudaEvent_t> events;  // start/stop event pair per timed launch
  int round = 0;                    // 0: every candidate twice; 1: the four best again
  int chosen = -1;                  // encoded winner once decided
  CsrTune() = default;
  CsrTune(const CsrTune &) = delete;
  CsrTune &operator=(const CsrTune &) = delete;
  void release() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    events.clear();
    trial.clear();
  }
  ~CsrTune() { release(); }
};

}  // namespace sma

// ------------------------------------------------------------------ context
struct sma_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  int num_sms = 148;
  bool autotune = true;  // SMA_AUTOTUNE=0 in the environment turns the kernel autotuner off
  // SMA_FILTER_GRAPHS=0 turns off the CUDA-graph replay of repeated filters (filter.cu)
  bool filter_graphs = true;
  // SMA_PERSISTENT=1: CSR filters run as one persistent cooperative launch (persistent.cu)
  bool persistent = false;
  // SMA_CUBLAS_DENSE=1: the tall-skinny products go through cuBLAS DGEMM instead of this
  // library's DMMA kernels (dgemm.cu) -- for comparisons
  bool cublas_dense = false;
  // SMA_PDL=0 turns off programmatic dependent launch of the fused CSR steps (the next
  // step's CTAs start on SMs the previous step's last wave leaves idle)
  bool pdl = true;
};

// OP_CSR_HALF: the upper triangle of a symmetric matrix only (half.cu)
enum op_kind { OP_CSR = 0, OP_LAP1D = 1, OP_MATBLOCK = 2, OP_ANDERSON = 3, OP_XXZ = 4, OP_CSR_HALF = 5 };

// Data of the matrix-free model stencils (kernels.cu): the 3D Anderson model on an L^3
// periodic lattice and the XXZ chain in its Sz = 0 sector.
struct sma_stencil {
  int L = 0;                   // lattice / chain length
  double hop = 0.0;            // Anderson hopping t, or the XXZ flip amplitude J/2
  double *diag = nullptr;      // n on-site energies / diagonal entries (device)
  unsigned *states = nullptr;  // XXZ: basis state (bit string) of each row (device)
  int *binom = nullptr;        // XXZ: C(p, k) for p < 32, k <= 16, row-major 32 x 17 (device)
};

struct sma_op {
  sma_ctx *ctx = nullptr;
  int kind = OP_CSR;
  int64_t n = 0, nnz = 0;
  // CSR (== CSC of the symmetric matrix), 0-based, int32 indices
  int *rowptr = nullptr;
  int *colind = nullptr;
  double *val64 = nullptr;
  float *val32 = nullptr;  // created on first FP32 use
  // Gershgorin bounds, computed on upload
  double gersh_min = 0, gersh_max = 0;
  bool has_gersh = false;
  int sym_state = 0;  // 0 unknown, 1 A == A^T, 2 not symmetric
  // caller callback
  sma_matblock_fn fn = nullptr;
  void *user = nullptr;
  // autotuned CSR kernel configurations
  std::map<uint64_t, sma::CsrTune> tuned;
  // BULK family of the CSR step (csr_clenshaw.cuh): the most CSR entries any CTA of RC rows
  // holds, per RC (from a host copy of the row pointers), and the device flag its bounded
  // wait sets when it gives up
  std::map<int, int> bulk_pairs;
  std::vector<int> host_rowptr;
  int *bulk_err = nullptr;
  // matrix-free model stencils
  sma_stencil stencil;
};

namespace sma {

// ------------------------------------------------------------------ device buffers
// Stream-ordered device allocation owned by one solve.
template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t count = 0;
  cudaStream_t stream = nullptr;
  DevBuf() = default;
  DevBuf(size_t n, cudaStream_t s) { alloc(n, s); }
  void alloc(size_t n, cudaStream_t s) {
    release();
    stream = s;
    count = n;
    if (n) SMA_CUDA(cudaMallocAsync((void **)&p, n * sizeof(T), s));
  }
  void release() {
    if (p) cudaFreeAsync(p, stream);
    p = nullptr;
    count = 0;
  }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), count(o.count), stream(o.stream) { o.p = nullptr; o.count = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; count = o.count; stream = o.stream; o.p = nullptr; o.count = 0; }
    return *this;
  }
  T *get() const { return p; }
};

// A row-major block view: element (i, j) at ptr[i*ld + j].
template <typename T>
struct Block {
  T *ptr;
  int64_t ld;
};

// ------------------------------------------------------------------ kernels (kernels.cu)
// out = ck*Q + alpha*(A*B1) + beta*B1 - B2 over b columns (one Clenshaw step).
// Q may be null (ck ignored), B2 may be null, has_self=false drops the beta*B1 term.
template <typename T>
void launch_clenshaw_step(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                          const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                          double alpha, double beta, bool has_self);
// The CSR form of launch_clenshaw_step (csr_clenshaw_f64.cu / csr_clenshaw_f32.cu).
template <typename T>
void csr_clenshaw_step(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                       const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                       double alpha, double beta, bool has_self);
// Throws SMA_ERR_TIMEOUT (and clears the flag) when a BULK-family launch of the CSR step on
// this operator gave up its bounded wait; synchronizes the stream when the family was used.
void check_bulk_error(const sma_op *op, cudaStream_t st);
// The CSR step without the autotuner (cached or default configuration, no events).
template <typename T>
void csr_clenshaw_step_untuned(const sma_op *op, cudaStream_t st, int64_t b, const T *Q,
                               int64_t ldq, const T *B1, const T *B2, int64_t ldb, T *out,
                               int64_t ldo, double ck, double alpha, double beta, bool has_self);
// The segmented CSR step (batched slicing, the POLFED polish): column c uses the
// coefficient cseg[colseg[c]] (csr_clenshaw.cuh).
template <typename T>
void csr_clenshaw_step_seg(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                           const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo,
                           const T *cseg, const int *colseg, double alpha, double beta,
                           bool tuned);
// out = ck * Q
template <typename T>
void launch_scale_block(cudaStream_t st, int64_t n, int64_t b, const T *Q, int64_t ldq, T *out,
                        int64_t ldo, double ck);
// out = ck*Q + alpha*AX + beta*B1 - B2 (the matrix-free axpy of
// chebyshev_subspace_iteration.jl:616-620); B2 may be null.
template <typename T>
void launch_clenshaw_axpy(cudaStream_t st, int64_t n, int64_t b, const T *Q, int64_t ldq,
                          const T *AX, int64_t ldax, const T *B1, const T *B2, int64_t ldb,
                          T *out, int64_t ldo, double ck, double alpha, double beta);

void launch_randn(cudaStream_t st, int64_t n, int64_t m, uint64_t seed, double *out, int64_t ld);
// Column reductions over row-major n x k blocks (deterministic two-stage sums).
//   mode 0: out[j] = sum_i X[i,j]*Y[i,j]
//   mode 1: out[j] = sqrt(sum_i (Y[i,j] - lam[j]*X[i,j])^2)
void column_reduce(cudaStream_t st, int mode, int64_t n, int64_t k, const double *X, int64_t ldx,
                   const double *Y, int64_t ldy, const double *lam, double *out,
                   DevBuf<double> &scratch);
// dst (row-major n x b, ldd) <- src (row-major, lds); optional type conversion
template <typename TS, typename TD>
void launch_copy_block(cudaStream_t st, int64_t n, int64_t b, const TS *src, int64_t lds, TD *dst,
                       int64_t ldd);
// dst column-major n x k (ld n) <- src row-major n x k (ld lds)
void launch_rowmajor_to_colmajor(cudaStream_t st, int64_t n, int64_t k, const double *src,
                                 int64_t lds, double *dst);
void launch_colmajor_to_rowmajor(cudaStream_t st, int64_t n, int64_t k, const double *src,
                                 double *dst, int64_t ldd);
// H = 0.5*(G + G^T) for a k x k column-major G (ld ldg) into H (ld ldh)
void launch_symmetrize(cudaStream_t st, int64_t k, const double *G, int64_t ldg, double *H,
                       int64_t ldh);
// T[o:o+r, o:o+r] = Aj ; T[o+r:o+r+r2, o:o+r] = Bj ; T[o:o+r, o+r:o+r+r2] = Bj^T
void launch_place_blocks(cudaStream_t st, double *T, int64_t ldt, int64_t o, int64_t r,
                         const double *Aj, int64_t lda, const double *Bj, int64_t ldbj,
                         int64_t r2);
// dst[:, j] = src[:, idx[j]] for column-major M x k (device idx)
void launch_gather_columns_cm(cudaStream_t st, int64_t M, int64_t k, const double *src,
                              int64_t lds, const int64_t *idx, double *dst, int64_t ldd);
// dst[i, j] = src[i, idx[j]] for row-major blocks (device idx)
void launch_gather_columns_rm(cudaStream_t st, int64_t n, int64_t k, const double *src,
                              int64_t lds, const int64_t *idx, double *dst, int64_t ldd);
// Gershgorin partial bounds of a CSR matrix
void gershgorin_device(const sma_op *op, double *smin, double *smax);
// Device arrays of a model stencil operator (stencils.cu)
void free_stencil_arrays(sma_op *op);
// Exact symmetry and sortedness check; returns 0 ok, 1 unsorted, 2 non-symmetric
int check_csr_device(const sma_op *op);
// In-place shift of the diagonal of a k x k column-major matrix
void launch_add_diagonal(cudaStream_t st, int64_t k, double *G, int64_t ld, double shift);
// Zero the strict lower triangle of a k x k column-major matrix
void launch_zero_lower(cudaStream_t st, int64_t k, double *G, int64_t ld);
// I (k x k, column-major, ld)
void launch_identity(cudaStream_t st, int64_t k, double *G, int64_t ld);

// ------------------------------------------------------------------ KPM (kpm.cu)
void kpm_moments(const sma_op *op, int64_t M, int64_t R, uint64_t seed, double smin,
                 double smax, double *mu, double *per_vec);
double kpm_count(const double *mu, int64_t M, int64_t n, double smin, double smax, double emin,
                 double emax, bool jackson);

// ------------------------------------------------------------------ host coefficient builders
std::vector<double> jackson_kernel(int64_t K);
std::vector<double> cheb_delta_coeffs(double sh, int64_t K, bool jackson);
std::vector<double> cheb_window_coeffs(double a, double b, int64_t K, bool jackson);
std::vector<double> cheb_smooth_window_coeffs(double a, double b, int64_t K, bool jackson,
                                              int64_t nsamp, double delta);
std::vector<double> build_coeffs(int64_t degree, double smin, double smax, double sigma,
                                 double emin, double emax, int64_t window_type, bool jackson);

// ------------------------------------------------------------------ filter (filter.cu)
// Work space of the block Clenshaw recurrence: three n x b blocks (+ AX for matrix-free),
// and the CUDA graph of a repeated filter: from the second call with the same operator,
// width, coefficients and bounds, the whole recurrence (on staging blocks q -> y at fixed
// addresses) is replayed from a graph instead of launched step by step.
template <typename T>
struct ClenshawWork {
  DevBuf<T> b1, b2, tmp, ax, q, y, coef;
  DevBuf<unsigned> barrier;  // persistent filter: arrival count, generation, error flag
  int64_t n = 0, bcap = 0;
  // graph cache
  const sma_op *g_op = nullptr;
  int64_t g_b = -1;
  double g_smin = 0, g_smax = 0;
  std::vector<double> g_coeffs;
  int64_t g_calls = 0, g_launches = 0, replays = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void ensure(const sma_op *op, int64_t n_, int64_t b, cudaStream_t st);
  void drop_graph();
  ClenshawWork() = default;
  ClenshawWork(const ClenshawWork &) = delete;
  ClenshawWork &operator=(const ClenshawWork &) = delete;
  ~ClenshawWork() { drop_graph(); }
};

// Y = p(A_hat) Q.  Returns the sparse block products issued and their algorithmic bytes.
struct FilterCount {
  int64_t steps = 0;
  double bytes = 0.0;
};
template <typename T>
FilterCount apply_poly_block(const sma_op *op, cudaStream_t st, const std::vector<double> &coeffs,
                         double smin, double smax, const T *Q, int64_t ldq, T *Y, int64_t ldy,
                         int64_t b, ClenshawWork<T> &work);

// The whole filter as one persistent cooperative launch (CSR operators, K >= 1); same
// results as apply_poly_block's step-by-step recurrence (persistent.cu).
template <typename T>
FilterCount persistent_filter(const sma_op *op, cudaStream_t st, const std::vector<double> &coeffs,
                              double smin, double smax, const T *Q, int64_t ldq, T *Y, int64_t ldy,
                              int64_t b, T *buf0, T *buf1, T *buf2, T *coeff_dev,
                              unsigned *barrier_words);

// persistent.cu: the bounded grid barrier with a missing CTA; SMA_ERR_TIMEOUT expected
int barrier_selftest(sma_ctx *ctx);

// Y = A X for a half-storage operator (row pass + atomic scatter of the transposed half)
template <typename T>
void half_product(const sma_op *op, cudaStream_t st, const T *X, int64_t ldx, T *Y, int64_t ldy,
                  int64_t b);

// AX = A X for FP64 blocks (any operator kind)
void op_apply(const sma_op *op, cudaStream_t st, const double *X, int64_t ldx, double *Y,
              int64_t ldy, int64_t b);

// Algorithmic bytes of one fused Clenshaw step over b columns
double clenshaw_step_bytes(const sma_op *op, int64_t b, int elem_bytes);

// ------------------------------------------------------------------ dense (dense.cu)
// FP64 tensor-core products of this library (dgemm.cu).
// Y (n x p, row-major) = alpha X B + beta Y, X n x m row-major, B = C (m x p column-major,
// ldc) or B = C^T (transC; C p x m column-major).  In place over X allowed when p <= 64 and
// beta = 0.
void dgemm_update(cudaStream_t st, int num_sms, int64_t n, int64_t m, int64_t p, const double *X,
                  int64_t ldx, const double *C, int64_t ldc, bool transC, double *Y, int64_t ldy,
                  double alpha, double beta);
// C (m x k, column-major, ldc) = alpha X^T Y + beta C; deterministic split-n reduction
// through `work` (grown as needed).  upper (m == k): only the 64 x 64 tiles on and above
// the diagonal are computed and written -- the upper triangle of a symmetric product.
void dgemm_gram(cudaStream_t st, int num_sms, int64_t n, int64_t m, int64_t k, const double *X,
                int64_t ldx, const double *Y, int64_t ldy, double *C, int64_t ldc, double alpha,
                double beta, DevBuf<double> &work, bool upper = false);

struct Dense {
  sma_ctx *ctx;
  DevBuf<double> work;  // split-n partial products of gram()
  explicit Dense(sma_ctx *c) : ctx(c) {}
  // C (col-major, m x k, ldc) = alpha * X^T Y + beta*C, X row-major n x m (ldx), Y n x k
  void gram(int64_t n, int64_t m, int64_t k, const double *X, int64_t ldx, const double *Y,
            int64_t ldy, double *C, int64_t ldc, double alpha = 1.0, double beta = 0.0,
            bool upper = false);
  // Y (row-major n x p, ldy) = alpha * X C + beta*Y, X row-major n x m, C col-major m x p
  void mul_small(int64_t n, int64_t m, int64_t p, const double *X, int64_t ldx, const double *C,
                 int64_t ldc, double *Y, int64_t ldy, double alpha, double beta, bool transC = false);
  // Symmetric eigen-decomposition of a k x k column-major matrix in place (vectors
  // overwrite A, eigenvalues ascending in w_dev). uplo_upper selects the triangle read.
  void syevd(int64_t k, double *A, int64_t lda, double *w_dev, bool uplo_upper);
  // Generalized symmetric-definite eigenproblem A E = B E diag(w) (k x k column-major, the
  // upper triangles read): E overwrites A (B-orthonormal), B its Cholesky factor,
  // eigenvalues ascending in w_dev.  Returns false when B is not positive definite.
  bool sygvd(int64_t k, double *A, int64_t lda, double *B, int64_t ldb, double *w_dev);
};

// Orthonormalize the columns of a row-major n x k block in place and return the
// upper-triangular factor R (k x k, column-major, host) with X_in = Q R.
// truncate: apply the reference's rank rule (keep the first count(|R_ii| > rtol*max|R_ii|)
// columns).  Returns the kept rank.  *fallbacks is incremented when CholQR2 is not used.
int64_t orthonormalize(sma_ctx *ctx, int64_t n, int64_t k, double *X, int64_t ldx,
                       bool truncate, double rtol, std::vector<double> *R_out,
                       int64_t *fallbacks);

// ------------------------------------------------------------------ polish (polish.cu)
// Y = q(A_hat) Q with a polynomial per column: coef[m * b + j] is coefficient m of column
// j (m = 0..K), blocks n x b row-major with ld = b, colseg the identity map on the device.
template <typename T>
FilterCount percol_filter(const sma_op *op, cudaStream_t st, const T *coef, int64_t K,
                          double smin, double smax, const T *Q, T *Y, int64_t b,
                          const int *colseg, T *B1, T *B2, T *TMP, T *AX);
// e[0..K-1]: Chebyshev coefficients of (p(s) - p(t)) / (s - t) for p = sum c_m T_m; *pt = p(t).
void divided_difference(const std::vector<double> &c, double t, double *e, double *pt);
struct PolishOut {
  std::vector<double> lam, res;  // Ritz values and residual norms of X's columns
  int64_t passes = 0;
  int64_t columns = 0;  // columns filtered, summed over the passes
  int64_t degree = 0;   // polish degree of the last pass
};
// coeffs_of(K): the polish polynomial of degree K (Chebyshev coefficients, K + 1 values).
using PolishCoeffs = std::function<std::vector<double>(int64_t)>;
// done(lam, res) ends the passes early; trace(pass, lam, res) sees every pass (pass 0: the
// columns before any filtering); needs(lam, res): whether a column is filtered (converged
// in-window columns and guards pass through to the Rayleigh-Ritz unchanged).
using PolishDone = std::function<bool(const std::vector<double> &, const std::vector<double> &)>;
using PolishTrace =
    std::function<void(int64_t, const std::vector<double> &, const std::vector<double> &)>;
using PolishNeeds = std::function<bool(double, double)>;
// Polish settings, from the environment: SMA_POLISH_FILTER=step (an undamped step window
// over the guards' span) or same (the basis filter, default); SMA_POLISH_GUARDS (guards as a
// fraction of the in-window candidates, default 3, or 1 with filtered guards);
// SMA_POLISH_FILTER_GUARDS=1 (the first
// pass filters the guards too, and a Rayleigh-Ritz of all columns precedes it; default 0:
// guards enter the Rayleigh-Ritz unfiltered); SMA_POLISH_DEGREE (degree scale of the
// polish polynomial, default 1); SMA_POLISH_PASSES (default 5); SMA_POLISH_VERBOSE=1.
struct PolishConfig {
  bool step_filter = false;
  double guard_fraction = 3.0;
  bool filter_guards = false;
  double degree_scale = 1.0;
  int64_t max_passes = 5;
  bool verbose = false;
  bool refine = false;  // SMA_POLISH_REFINE=1: keep the refinement before the polish
};
PolishConfig polish_config();
// Up to max_passes filtered subspace iterations on the k columns of X (n x k, ld k, FP64,
// in place) with p = sum coeffs[m] T_m(A_hat), each applying p as
// p(theta) x + q_theta(A_hat) r / d with q in FP32 to the columns needs() selects (with
// filter_all, every column in the first pass), then FP64 orthonormalization and
// Rayleigh-Ritz with A on all k columns; X ends as the last Ritz vectors.
// lam0/res0: each column's Rayleigh quotient and residual norm on entry (its columns unit
// vectors); when empty (or with filter_all), a Rayleigh-Ritz of the k columns comes first.
// Without filter_all, each Rayleigh-Ritz lifts the Ritz vectors with values in [emin, emax]
// first and the others only when done() is false; after a pass that ends the polish, the
// columns past the in-window ones are not lifted (their lam is the Ritz value, res inf).
// The degree starts at K0; after a pass (other than the first) that cut the worst unconverged
// residual by less than 3x the next pass doubles it, up to Kmax.
PolishOut polish_mixed(const sma_op *op, const PolishCoeffs &coeffs_of, int64_t K0, int64_t Kmax,
                       double smin, double smax, double *X, int64_t k, const PolishDone &done,
                       const PolishNeeds &needs, int64_t max_passes, FilterCount &fc,
                       int64_t *qr_fallbacks, const std::vector<double> &lam0,
                       const std::vector<double> &res0, double emin, double emax,
                       bool filter_all, bool verbose, const PolishTrace &trace = PolishTrace());

// ------------------------------------------------------------------ result
}  // namespace sma

struct sma_result {
  int64_t n = 0, k = 0;
  std::vector<double> lam, res;
  double *X_dev = nullptr;  // row-major n x k (ld k), owned
  int64_t ldx = 0;
  std::vector<int64_t> win;  // window of each pair (batched slicing); empty means all 0
  std::vector<int64_t> win_iters, win_done;  // per window: iterations run, converged flag
  sma_ctx *ctx = nullptr;
  sma_stats stats{};
};

// ------------------------------------------------------------------ learned window planner (mlp.cu)
// A three-layer perceptron with BF16 weights (FP32 masters) and its training state.
struct sma_mlp {
  sma_ctx *ctx = nullptr;
  int64_t in = 0, hid = 0, out = 0;
  int64_t nparam = 0;
  // offsets into the packed parameter vector: W1 (hid x in), b1, W2 (hid x hid), b2,
  // W3 (out x hid), b3
  int64_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0;
  sma::DevBuf<float> master, grad, m, v;
  sma::DevBuf<__nv_bfloat16> wbf;
  int64_t adam_t = 0;
  // activations for the current batch
  int64_t bcap = 0;
  sma::DevBuf<float> h1, h2, y, d2, d1, dy, partial, loss;
  void ensure(int64_t B) {
    if (B <= bcap) return;
    cudaStream_t st = ctx->stream;
    bcap = B;
    h1.alloc(B * hid, st);
    h2.alloc(B * hid, st);
    y.alloc(B * out, st);
    d2.alloc(B * hid, st);
    d1.alloc(B * hid, st);
    dy.alloc(B * out, st);
    partial.alloc(B, st);
    loss.alloc(1, st);
  }
};

namespace sma {
void mlp_init(sma_mlp *net, int64_t in, int64_t hid, int64_t out, uint64_t seed);
void mlp_set_params(sma_mlp *net, const float *p);
void mlp_get_params(const sma_mlp *net, float *p);
void mlp_forward(sma_mlp *net, const float *X_host, int64_t B, float *Y_host);
float mlp_grad(sma_mlp *net, const float *X_host, const float *T_host, const float *w_host,
               int64_t B, float *grad_host);
void mlp_train(sma_mlp *net, const float *X_host, const float *T_host, const float *w_host,
               int64_t N, int64_t steps, double lr, int64_t mb, uint64_t seed, double weight_decay,
               float *loss_hist);
}  // namespace sma
