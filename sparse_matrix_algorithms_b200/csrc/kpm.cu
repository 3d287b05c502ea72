// Stochastic Chebyshev moments of the spectral density (the kernel polynomial method) and
// the eigenvalue count they predict for a window.  An extension: the reference has no
// density-of-states estimate; here it places windows by eigenvalue count, sizes filters,
// and is the input of the learned degree / subspace-size predictor.
//
//   mu_k = (1 / (n R)) sum_{r=1..R} z_r^T T_k(A_hat) z_r,     A_hat = (A - c I) / d
//
// with R Rademacher (+-1) vectors z_r, so mu_0 = 1 exactly.  The block recurrence
// T_{k+1} = 2 A_hat T_k - T_{k-1} is the fused Clenshaw step of the filter with
// Q = T_{k-1} and coefficient -1; the doubling identities
//   mu_{2k} = 2 <T_k, T_k> - mu_0,   mu_{2k+1} = 2 <T_{k+1}, T_k> - mu_1
// give two moments per sparse product, so M moments take ceil(M/2) products.
#include <cmath>

#include "sma_internal.h"

namespace sma {

namespace {

__device__ __forceinline__ uint64_t kpm_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Element (i, j) of an n x R Rademacher block: flat index k = i + j*n, value +1 when the
// top bit of SplitMix64 output k+1 of the stream seed ^ 0x2545F4914F6CDD1D is clear,
// else -1.
__global__ void rademacher_kernel(int64_t n, int64_t R, uint64_t seed, double *__restrict__ out,
                                  int64_t ld) {
  const uint64_t s = seed ^ 0x2545F4914F6CDD1DULL;
  const uint64_t golden = 0x9E3779B97F4A7C15ULL;
  const int64_t total = n * R;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / R, j = t % R;
    const uint64_t k = (uint64_t)i + (uint64_t)j * (uint64_t)n;
    out[i * ld + j] = (kpm_mix64(s + (k + 1) * golden) >> 63) ? -1.0 : 1.0;
  }
}

}  // namespace

// Moments mu[0..M-1] (and, when per_vec is given, the M x R per-vector moments row-major,
// each normalized by n).
void kpm_moments(const sma_op *op, int64_t M, int64_t R, uint64_t seed, double smin,
                 double smax, double *mu, double *per_vec) {
  cudaStream_t st = op->ctx->stream;
  const int64_t n = op->n;
  require(M >= 1 && R >= 1, SMA_ERR_ARG, "need at least one moment and one vector");
  require(smax > smin, SMA_ERR_ARG, "need smin < smax");
  const double c = 0.5 * (smin + smax), invd = 2.0 / (smax - smin);
  DevBuf<double> t0(n * R, st), t1(n * R, st), t2(n * R, st), dots(2 * (M / 2 + 1) * R, st),
      scratch;
  {
    const int64_t total = n * R;
    const unsigned grid = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 16);
    rademacher_kernel<<<std::max(grid, 1u), 256, 0, st>>>(n, R, seed, t0.p, R);
    SMA_CHECK_LAUNCH();
  }
  // out = ck Q + alpha A B1 + beta B1: the fused step for device operators, the caller's
  // block product followed by the axpy kernel for callback operators
  DevBuf<double> ax;
  const bool product_then_axpy = op->kind == OP_MATBLOCK || op->kind == OP_CSR_HALF;
  if (product_then_axpy) ax.alloc(n * R, st);
  auto step = [&](const double *Q, const double *B1, double *out, double ck, double alpha,
                  double beta) {
    if (product_then_axpy) {
      op_apply(op, st, B1, R, ax.p, R, R);
      launch_clenshaw_axpy<double>(st, n, R, Q, R, ax.p, R, B1, nullptr, R, out, R, ck, alpha, beta);
    } else {
      launch_clenshaw_step<double>(op, st, R, Q, R, B1, nullptr, R, out, R, ck, alpha, beta, true);
    }
  };
  // dots[2k] = <T_k, T_k>, dots[2k+1] = <T_{k+1}, T_k> (R values each)
  double *Tprev = t0.p, *Tcur = t1.p, *Tnext = t2.p;
  column_reduce(st, 0, n, R, t0.p, R, t0.p, R, nullptr, dots.p, scratch);  // <T0, T0>
  if (M > 1) {
    // T1 = A_hat T0 = invd A T0 - c invd T0 (Q term with coefficient 0)
    step(t0.p, t0.p, Tcur, 0.0, invd, -c * invd);
    column_reduce(st, 0, n, R, Tcur, R, t0.p, R, nullptr, dots.p + R, scratch);  // <T1, T0>
  }
  const int64_t kmax = (M - 1) / 2;  // need <T_k,T_k> for 2k <= M-1, <T_{k+1},T_k> for 2k+1 <= M-1
  for (int64_t k = 1; k <= kmax; ++k) {
    column_reduce(st, 0, n, R, Tcur, R, Tcur, R, nullptr, dots.p + 2 * k * R, scratch);
    if (2 * k + 1 <= M - 1) {
      // T_{k+1} = 2 invd A T_k - 2 c invd T_k - T_{k-1}
      step(Tprev, Tcur, Tnext, -1.0, 2.0 * invd, -2.0 * c * invd);
      column_reduce(st, 0, n, R, Tnext, R, Tcur, R, nullptr, dots.p + (2 * k + 1) * R, scratch);
      double *t = Tprev;
      Tprev = Tcur;
      Tcur = Tnext;
      Tnext = t;
    }
  }
  std::vector<double> h((size_t)M * R);
  SMA_CUDA(cudaMemcpyAsync(h.data(), dots.p, (size_t)M * R * sizeof(double),
                           cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  std::vector<double> pv((size_t)M * R);
  for (int64_t j = 0; j < R; ++j) {
    const double m0 = h[j], m1 = M > 1 ? h[R + j] : 0.0;
    pv[j] = m0;
    if (M > 1) pv[R + j] = m1;
    for (int64_t q = 2; q < M; ++q) {
      const double dq = h[q * R + j];
      pv[q * R + j] = 2.0 * dq - ((q % 2 == 0) ? m0 : m1);
    }
  }
  for (int64_t q = 0; q < M; ++q) {
    double s = 0.0;
    for (int64_t j = 0; j < R; ++j) {
      pv[q * R + j] /= (double)n;
      s += pv[q * R + j];
    }
    mu[q] = s / (double)R;
  }
  if (per_vec) std::copy(pv.begin(), pv.end(), per_vec);
}

// Eigenvalue count in [emin, emax] predicted by the moments: n times the integral of the
// (Jackson-damped) Chebyshev series of the density,
//   int_a^b T_k(x) / (pi sqrt(1 - x^2)) dx = (sin(k acos a) - sin(k acos b)) / (k pi).
double kpm_count(const double *mu, int64_t M, int64_t n, double smin, double smax, double emin,
                 double emax, bool jackson) {
  require(M >= 1, SMA_ERR_ARG, "need at least one moment");
  require(smax > smin && emax >= emin, SMA_ERR_ARG, "bad interval");
  const double c = 0.5 * (smin + smax), d = 0.5 * (smax - smin);
  const double a = std::min(1.0, std::max(-1.0, (emin - c) / d));
  const double b = std::min(1.0, std::max(-1.0, (emax - c) / d));
  const double ta = std::acos(a), tb = std::acos(b);
  const std::vector<double> g = jackson ? jackson_kernel(M - 1) : std::vector<double>(M, 1.0);
  double s = g[0] * mu[0] * (ta - tb);
  for (int64_t k = 1; k < M; ++k)
    s += 2.0 * g[k] * mu[k] * (std::sin(k * ta) - std::sin(k * tb)) / (double)k;
  return (double)n * s / M_PI;
}

}  // namespace sma
