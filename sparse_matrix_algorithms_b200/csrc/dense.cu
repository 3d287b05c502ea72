// Dense block operations: Gram products, small-matrix updates, symmetric
// eigensolves, and orthonormalization.
//
// Blocks are row-major n x k; cuBLAS sees such a block as the column-major k x n
// matrix X^T, so X^T Y is GEMM(N, T) and X C is GEMM(T, N).
//
// Orthonormalization replaces the reference's Householder QR (`qr!`/`geqrf!`+`orgqr!`,
// chebyshev_subspace_iteration.jl:223-231, polfed.jl:561-594 and 644-685) by CholQR2:
// two passes of  G = X^T X,  R = chol(G),  X <- X R^{-1}.  Its cost is two GEMM-shaped
// Gram products and two triangular solves, all HBM-bound tall-skinny sweeps.  CholQR
// needs cond(X) well below 1/sqrt(eps); when the first Cholesky fails or its pivots
// spread by more than 1e6, the shifted CholQR3 of Fukaya, Kannan, Nakatsukasa,
// Yamamoto and Yanagisawa ("Shifted Cholesky QR for computing the QR factorization of
// ill-conditioned matrices", SIAM J. Sci. Comput. 42 (2020)) takes over, and when that
// fails too (numerically rank-deficient X) the block goes through Householder QR
// (cuSOLVER geqrf/orgqr) exactly as the reference does.  Every rung multiplies X by the
// inverse of an upper-triangular factor, so the leading j columns keep spanning the
// leading j input columns and the accumulated R is the QR factor of the input.  The
// reference's rank rule -- keep the first count(|R_ii| > rtol*max|R_ii|) columns -- is
// applied to diag(R), the product of the rungs' diagonals.
#include <algorithm>
#include <cmath>

#include "sma_internal.h"

namespace sma {

void Dense::gram(int64_t n, int64_t m, int64_t k, const double *X, int64_t ldx, const double *Y,
                 int64_t ldy, double *C, int64_t ldc, double alpha, double beta, bool upper) {
  if (m == 0 || k == 0) return;
  if (!ctx->cublas_dense) {
    dgemm_gram(ctx->stream, ctx->num_sms, n, m, k, X, ldx, Y, ldy, C, ldc, alpha, beta, work,
               upper && m == k);
    return;
  }
  SMA_CUBLAS(cublasDgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)m, (int)k, (int)n, &alpha, X,
                         (int)ldx, Y, (int)ldy, &beta, C, (int)ldc));
}

void Dense::mul_small(int64_t n, int64_t m, int64_t p, const double *X, int64_t ldx,
                      const double *C, int64_t ldc, double *Y, int64_t ldy, double alpha,
                      double beta, bool transC) {
  if (p == 0 || n == 0) return;
  if (!ctx->cublas_dense) {
    dgemm_update(ctx->stream, ctx->num_sms, n, m, p, X, ldx, C, ldc, transC, Y, ldy, alpha, beta);
    return;
  }
  if (m == 0) {  // Y = beta*Y
    const double zero = 0.0;
    if (beta != 1.0)
      SMA_CUBLAS(cublasDgeam(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)p, (int)n, &beta, Y,
                             (int)ldy, &zero, Y, (int)ldy, Y, (int)ldy));
    return;
  }
  SMA_CUBLAS(cublasDgemm(ctx->cublas, transC ? CUBLAS_OP_N : CUBLAS_OP_T, CUBLAS_OP_N, (int)p,
                         (int)n, (int)m, &alpha, C, (int)ldc, X, (int)ldx, &beta, Y, (int)ldy));
}

void Dense::syevd(int64_t k, double *A, int64_t lda, double *w_dev, bool uplo_upper) {
  if (k == 0) return;
  const cublasFillMode_t uplo = uplo_upper ? CUBLAS_FILL_MODE_UPPER : CUBLAS_FILL_MODE_LOWER;
  int lwork = 0;
  SMA_CUSOLVER(cusolverDnDsyevd_bufferSize(ctx->cusolver, CUSOLVER_EIG_MODE_VECTOR, uplo, (int)k,
                                           A, (int)lda, w_dev, &lwork));
  DevBuf<double> work(std::max(lwork, 1), ctx->stream);
  DevBuf<int> info(1, ctx->stream);
  SMA_CUSOLVER(cusolverDnDsyevd(ctx->cusolver, CUSOLVER_EIG_MODE_VECTOR, uplo, (int)k, A,
                                (int)lda, w_dev, work.p, lwork, info.p));
  int h = 0;
  SMA_CUDA(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  require(h == 0, SMA_ERR_INTERNAL, "cusolverDnDsyevd failed, info=" + std::to_string(h));
}

bool Dense::sygvd(int64_t k, double *A, int64_t lda, double *B, int64_t ldb, double *w_dev) {
  if (k == 0) return true;
  int lwork = 0;
  SMA_CUSOLVER(cusolverDnDsygvd_bufferSize(ctx->cusolver, CUSOLVER_EIG_TYPE_1,
                                           CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER,
                                           (int)k, A, (int)lda, B, (int)ldb, w_dev, &lwork));
  DevBuf<double> work(std::max(lwork, 1), ctx->stream);
  DevBuf<int> info(1, ctx->stream);
  SMA_CUSOLVER(cusolverDnDsygvd(ctx->cusolver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                CUBLAS_FILL_MODE_UPPER, (int)k, A, (int)lda, B, (int)ldb, w_dev,
                                work.p, lwork, info.p));
  int h = 0;
  SMA_CUDA(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  require(h >= 0, SMA_ERR_INTERNAL, "cusolverDnDsygvd: bad argument " + std::to_string(-h));
  return h == 0;  // h > k: B is not positive definite; 0 < h <= k: no convergence
}

namespace {

// Upper Cholesky of the k x k column-major G in place. Returns cuSOLVER's info.
int potrf_upper(sma_ctx *ctx, int64_t k, double *G, int64_t ldg) {
  int lwork = 0;
  SMA_CUSOLVER(cusolverDnDpotrf_bufferSize(ctx->cusolver, CUBLAS_FILL_MODE_UPPER, (int)k, G,
                                           (int)ldg, &lwork));
  DevBuf<double> work(std::max(lwork, 1), ctx->stream);
  DevBuf<int> info(1, ctx->stream);
  SMA_CUSOLVER(cusolverDnDpotrf(ctx->cusolver, CUBLAS_FILL_MODE_UPPER, (int)k, G, (int)ldg, work.p,
                                lwork, info.p));
  int h = 0;
  SMA_CUDA(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  return h;
}

// X <- X R^{-1} for row-major X (n x k) and upper-triangular R (k x k column-major).
// This library's path: R^{-1} (k x k, a triangular solve against the identity -- tiny) and
// then one tensor-core product X R^{-1}, in place when k <= 64, else through a copy.  With
// SMA_CUBLAS_DENSE=1: cuBLAS DTRSM on X^T (column-major k x n), X^T <- R^{-T} X^T.
void trsm_right_upper(sma_ctx *ctx, int64_t n, int64_t k, const double *R, int64_t ldr, double *X,
                      int64_t ldx) {
  const double one = 1.0;
  if (ctx->cublas_dense) {
    SMA_CUBLAS(cublasDtrsm(ctx->cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T,
                           CUBLAS_DIAG_NON_UNIT, (int)k, (int)n, &one, R, (int)ldr, X, (int)ldx));
    return;
  }
  cudaStream_t st = ctx->stream;
  DevBuf<double> Rinv(k * k, st);
  launch_identity(st, k, Rinv.p, k);
  SMA_CUBLAS(cublasDtrsm(ctx->cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                         CUBLAS_DIAG_NON_UNIT, (int)k, (int)k, &one, R, (int)ldr, Rinv.p, (int)k));
  if (k <= 64) {
    dgemm_update(st, ctx->num_sms, n, k, k, X, ldx, Rinv.p, k, false, X, ldx, 1.0, 0.0);
  } else {
    DevBuf<double> tmp(n * k, st);
    dgemm_update(st, ctx->num_sms, n, k, k, X, ldx, Rinv.p, k, false, tmp.p, k, 1.0, 0.0);
    launch_copy_block<double, double>(st, n, k, tmp.p, k, X, ldx);
  }
}

std::vector<double> to_host(sma_ctx *ctx, const double *d, size_t count) {
  std::vector<double> h(count);
  if (count) {
    SMA_CUDA(cudaMemcpyAsync(h.data(), d, count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return h;
}

// Diagonal of a k x k column-major device matrix.
std::vector<double> diag_to_host(sma_ctx *ctx, const double *G, int64_t k) {
  std::vector<double> d(k);
  SMA_CUDA(cudaMemcpy2DAsync(d.data(), sizeof(double), G, (k + 1) * sizeof(double), sizeof(double),
                             k, cudaMemcpyDeviceToHost, ctx->stream));
  SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  return d;
}

int64_t rank_rule(const std::vector<double> &diag, double rtol) {
  double r0 = 0.0;
  for (double d : diag) r0 = std::max(r0, std::fabs(d));
  if (r0 == 0.0) return 0;
  int64_t r = 0;
  for (double d : diag) r += std::fabs(d) > rtol * r0 ? 1 : 0;
  return r;
}

// Accumulated upper-triangular factor: R_acc <- R_new * R_acc (device, k x k).
struct Factor {
  sma_ctx *ctx;
  int64_t k;
  bool want_matrix;
  DevBuf<double> R, tmp;
  std::vector<double> diag;
  bool empty = true;
  Factor(sma_ctx *c, int64_t k_, bool want) : ctx(c), k(k_), want_matrix(want), diag(k_, 1.0) {}
  void push(const double *Rnew, const std::vector<double> &dnew) {
    for (int64_t i = 0; i < k; ++i) diag[i] *= dnew[i];
    if (!want_matrix) return;
    cudaStream_t st = ctx->stream;
    if (empty) {
      R.alloc(k * k, st);
      SMA_CUDA(cudaMemcpyAsync(R.p, Rnew, k * k * sizeof(double), cudaMemcpyDeviceToDevice, st));
      launch_zero_lower(st, k, R.p, k);  // potrf leaves the strict lower part untouched
    } else {
      if (tmp.count < (size_t)(k * k)) tmp.alloc(k * k, st);
      const double one = 1.0;
      // tmp = triu(Rnew) * R  (cublas reads only the upper triangle of Rnew)
      SMA_CUBLAS(cublasDtrmm(ctx->cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                             CUBLAS_DIAG_NON_UNIT, (int)k, (int)k, &one, Rnew, (int)k, R.p, (int)k,
                             tmp.p, (int)k));
      std::swap(R.p, tmp.p);
    }
    empty = false;
  }
};

// One Cholesky-QR pass: G = X^T X (+ shift I), R = chol(G), X <- X R^{-1}.  Returns
// false with X untouched when the factorization fails or (max_spread > 0) when its
// pivots spread by more than max_spread.
bool cholqr_pass(sma_ctx *ctx, int64_t n, int64_t k, double *X, int64_t ldx, double shift,
                 double max_spread, Factor &F, DevBuf<double> &G) {
  Dense dn(ctx);
  if (G.count < (size_t)(k * k)) G.alloc(k * k, ctx->stream);
  dn.gram(n, k, k, X, ldx, X, ldx, G.p, k);
  if (shift > 0.0) launch_add_diagonal(ctx->stream, k, G.p, k, shift);
  if (potrf_upper(ctx, k, G.p, k) != 0) return false;
  std::vector<double> d = diag_to_host(ctx, G.p, k);
  double dmax = 0.0, dmin = INFINITY;
  for (double v : d) {
    if (!(std::isfinite(v) && v > 0.0)) return false;
    dmax = std::max(dmax, v);
    dmin = std::min(dmin, v);
  }
  if (max_spread > 0.0 && dmax / dmin > max_spread) return false;
  trsm_right_upper(ctx, n, k, G.p, k, X, ldx);
  F.push(G.p, d);
  return true;
}

// Householder QR of the row-major block (geqrf + orgqr on its column-major copy).
void householder(sma_ctx *ctx, int64_t n, int64_t k, double *X, int64_t ldx, Factor &F) {
  cudaStream_t st = ctx->stream;
  DevBuf<double> A(n * k, st), tau(k, st), Rk(k * k, st);
  launch_rowmajor_to_colmajor(st, n, k, X, ldx, A.p);
  int lw1 = 0, lw2 = 0;
  SMA_CUSOLVER(cusolverDnDgeqrf_bufferSize(ctx->cusolver, (int)n, (int)k, A.p, (int)n, &lw1));
  SMA_CUSOLVER(cusolverDnDorgqr_bufferSize(ctx->cusolver, (int)n, (int)k, (int)k, A.p, (int)n,
                                           tau.p, &lw2));
  const int lw = std::max(1, std::max(lw1, lw2));
  DevBuf<double> work(lw, st);
  DevBuf<int> info(1, st);
  SMA_CUSOLVER(cusolverDnDgeqrf(ctx->cusolver, (int)n, (int)k, A.p, (int)n, tau.p, work.p, lw, info.p));
  SMA_CUDA(cudaMemcpy2DAsync(Rk.p, k * sizeof(double), A.p, n * sizeof(double), k * sizeof(double),
                             k, cudaMemcpyDeviceToDevice, st));
  std::vector<double> d = diag_to_host(ctx, Rk.p, k);
  SMA_CUSOLVER(cusolverDnDorgqr(ctx->cusolver, (int)n, (int)k, (int)k, A.p, (int)n, tau.p, work.p,
                                lw, info.p));
  launch_colmajor_to_rowmajor(st, n, k, A.p, X, ldx);
  int h = 0;
  SMA_CUDA(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  require(h == 0, SMA_ERR_INTERNAL, "Householder QR failed, info=" + std::to_string(h));
  F.push(Rk.p, d);
}

}  // namespace

int64_t orthonormalize(sma_ctx *ctx, int64_t n, int64_t k, double *X, int64_t ldx, bool truncate,
                       double rtol, std::vector<double> *R_out, int64_t *fallbacks) {
  if (k == 0) {
    if (R_out) R_out->clear();
    return 0;
  }
  require(k <= n, SMA_ERR_ARG, "block wider than the operator dimension");
  cudaStream_t st = ctx->stream;
  DevBuf<double> G;
  Factor F(ctx, k, R_out != nullptr);
  // CholQR2; every pass that fails leaves X untouched, and X always equals
  // X_in * R_acc^{-1}, so the next rung continues from the current X.
  bool ok = cholqr_pass(ctx, n, k, X, ldx, 0.0, 1e6, F, G) &&
            cholqr_pass(ctx, n, k, X, ldx, 0.0, 0.0, F, G);
  if (!ok) {
    if (fallbacks) ++*fallbacks;
    // shifted CholQR3: shift = 11 (n k + k (k+1)) u ||X||_2^2, ||X||_2^2 <= trace(X^T X)
    DevBuf<double> nrm(k, st);
    column_reduce(st, 0, n, k, X, ldx, X, ldx, nullptr, nrm.p, G);
    std::vector<double> nh = to_host(ctx, nrm.p, k);
    double fro2 = 0.0;
    for (double v : nh) fro2 += v;
    const double u = 1.1102230246251565e-16;
    const double shift = 11.0 * ((double)n * k + (double)k * (k + 1)) * u * fro2;
    ok = fro2 > 0.0 && std::isfinite(fro2) && cholqr_pass(ctx, n, k, X, ldx, shift, 0.0, F, G) &&
         cholqr_pass(ctx, n, k, X, ldx, 0.0, 0.0, F, G) &&
         cholqr_pass(ctx, n, k, X, ldx, 0.0, 0.0, F, G);
  }
  if (!ok) householder(ctx, n, k, X, ldx, F);
  const int64_t r = truncate ? rank_rule(F.diag, rtol) : k;
  if (R_out) *R_out = to_host(ctx, F.R.p, k * k);
  return r;
}

}  // namespace sma
