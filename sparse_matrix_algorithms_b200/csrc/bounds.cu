// Spectral bounds by Lanczos on the GPU (sma_lanczos_bounds).
//
// The reference estimates [smin, smax] with Gershgorin discs (gershgorin_bounds,
// chebyshev_subspace_iteration.jl:351-367), which can be loose: for the XXZ chain the
// discs give [-22.6, 20.0] around a spectrum in [-17.8, 16.6].  A loose interval wastes
// filter degree in proportion to its excess width.  Here k Lanczos steps (FP64, full
// reorthogonalization) give Ritz values theta_1 <= ... <= theta_k whose extremes converge
// quickly to the spectrum's ends.  Each end is widened by the residual norm of its Ritz
// pair, beta_k |u_k(last)|, but at least by 1e-3 of the Ritz range (residual-based bound
// estimates as discussed by Y. Zhou and R.-C. Li, "Bound estimation for Chebyshev filtered
// subspace iteration", Linear Algebra Appl. 435 (2011)), and clipped to the Gershgorin
// interval, which is always valid, when the operator has one.  This is an estimate: an
// unconverged end could lie further out, which the solvers' tests guard against.  The
// Ritz pairs come from the small tridiagonal matrix (cuSOLVER syevd).
#include <algorithm>
#include <cmath>
#include <vector>

#include "sma_internal.h"

namespace sma {

void lanczos_bounds(sma_op *op, int64_t steps, uint64_t seed, double *smin, double *smax) {
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  const int64_t n = op->n;
  const int64_t k = std::min<int64_t>(steps, n);
  require(k >= 2, SMA_ERR_ARG, "Lanczos bounds need at least 2 steps and n >= 2");
  // V: k+1 column vectors of length n, each contiguous (a row-major n x 1 block, ld 1)
  DevBuf<double> V((k + 1) * n, st), w(n, st), c(k + 1, st);
  launch_randn(st, n, 1, seed, V.p, 1);
  const double one = 1.0, zero = 0.0, mone = -1.0;
  double nv = 0.0;
  SMA_CUBLAS(cublasDnrm2(ctx->cublas, (int)n, V.p, 1, &nv));
  SMA_CUDA(cudaStreamSynchronize(st));
  require(nv > 0.0, SMA_ERR_INTERNAL, "zero start vector");
  const double inv = 1.0 / nv;
  SMA_CUBLAS(cublasDscal(ctx->cublas, (int)n, &inv, V.p, 1));
  std::vector<double> alpha, beta;
  double beta_last = 0.0;
  for (int64_t j = 0; j < k; ++j) {
    double *vj = V.p + j * n;
    op_apply(op, st, vj, 1, w.p, 1, 1);  // w = A v_j
    // full reorthogonalization against v_0..v_j (twice), which also forms alpha_j
    double a = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
      SMA_CUBLAS(cublasDgemv(ctx->cublas, CUBLAS_OP_T, (int)n, (int)(j + 1), &one, V.p, (int)n,
                             w.p, 1, &zero, c.p, 1));
      SMA_CUBLAS(cublasDgemv(ctx->cublas, CUBLAS_OP_N, (int)n, (int)(j + 1), &mone, V.p, (int)n,
                             c.p, 1, &one, w.p, 1));
      double cj = 0.0;
      SMA_CUDA(cudaMemcpyAsync(&cj, c.p + j, sizeof(double), cudaMemcpyDeviceToHost, st));
      SMA_CUDA(cudaStreamSynchronize(st));
      a += cj;
    }
    double b = 0.0;
    SMA_CUBLAS(cublasDnrm2(ctx->cublas, (int)n, w.p, 1, &b));
    SMA_CUDA(cudaStreamSynchronize(st));
    alpha.push_back(a);
    beta_last = b;
    if (j + 1 == k || b <= 1e-14 * std::fabs(a)) break;  // invariant subspace found
    beta.push_back(b);
    const double ib = 1.0 / b;
    SMA_CUDA(cudaMemcpyAsync(V.p + (j + 1) * n, w.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    SMA_CUBLAS(cublasDscal(ctx->cublas, (int)n, &ib, V.p + (j + 1) * n, 1));
  }
  // Ritz values: eigenvalues of the m x m tridiagonal T = tridiag(beta, alpha, beta)
  const int64_t m = (int64_t)alpha.size();
  std::vector<double> T(m * m, 0.0);
  for (int64_t i = 0; i < m; ++i) {
    T[i + i * m] = alpha[i];
    if (i + 1 < m) T[(i + 1) + i * m] = T[i + (i + 1) * m] = beta[i];
  }
  DevBuf<double> Td(m * m, st), theta_d(m, st);
  SMA_CUDA(cudaMemcpyAsync(Td.p, T.data(), m * m * sizeof(double), cudaMemcpyHostToDevice, st));
  Dense(ctx).syevd(m, Td.p, m, theta_d.p, true);
  std::vector<double> theta(m), U(m * m);
  SMA_CUDA(cudaMemcpyAsync(theta.data(), theta_d.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaMemcpyAsync(U.data(), Td.p, m * m * sizeof(double), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  // residual norms of the extreme Ritz pairs: beta_k |last component of their eigenvector|
  const double r_lo = beta_last * std::fabs(U[(m - 1) + 0 * m]);
  const double r_hi = beta_last * std::fabs(U[(m - 1) + (m - 1) * m]);
  const double margin = 1e-3 * (theta.back() - theta.front());
  double lo = theta.front() - std::max(r_lo, margin), hi = theta.back() + std::max(r_hi, margin);
  if (op->has_gersh) {  // explicit matrices and the model stencils carry a valid interval
    lo = std::max(lo, op->gersh_min);
    hi = std::min(hi, op->gersh_max);
  }
  *smin = lo;
  *smax = hi;
}

}  // namespace sma

extern "C" int sma_lanczos_bounds(sma_op *op, int64_t steps, int64_t seed, double *smin,
                                  double *smax) {
  try {
    sma::require(op != nullptr && op->ctx != nullptr, SMA_ERR_ARG, "null operator");
    sma::require(smin != nullptr && smax != nullptr, SMA_ERR_ARG, "null output");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != op->ctx->device) SMA_CUDA(cudaSetDevice(op->ctx->device));
    sma::lanczos_bounds(op, steps, (uint64_t)seed, smin, smax);
    if (prev >= 0 && prev != op->ctx->device) cudaSetDevice(prev);
    return SMA_OK;
  } catch (const sma::Error &e) {
    sma::set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    sma::set_last_error(e.what());
    return SMA_ERR_INTERNAL;
  }
}
