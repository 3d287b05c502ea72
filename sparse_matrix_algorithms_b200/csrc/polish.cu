// FP64 polish of Ritz vectors at FP32 cost (POLFED in MIXED precision).
//
// An FP32-filtered POLFED basis yields Ritz vectors whose residuals stop near 1e-6 of the
// spectral scale: the FP32 rounding of every filtered block enters the Krylov basis.  The
// polish refines them by subspace iteration with the same filter polynomial p, but
// never applies p in FP32 to the vectors themselves.  For a unit vector x with Rayleigh
// quotient theta and residual r = (A - theta) x, the divided difference
//
//     q_t(s) = (p(s) - p(t)) / (s - t),   t = (theta - c) / d   (A_hat = (A - c) / d)
//
// is a polynomial of degree K - 1 and
//
//     p(A_hat) x = p(t) x + q_t(A_hat) r / d.
//
// The first term is exact in FP64; the second applies q_t in FP32 to r / ||r||, so its
// rounding error is ~1e-7 of ||r|| / d instead of ~1e-7 of ||x||: the filtered block comes
// out with FP64-level accuracy while the recurrence streams FP32 blocks.  Each column has
// its own t, so every column runs its own polynomial: one segmented Clenshaw recurrence
// with one coefficient segment per column.  The coefficients of q_t are the Clenshaw
// intermediates of p at t: with b_m = c_m + 2 t b_{m+1} - b_{m+2} (b_{K+1} = b_{K+2} = 0),
// q_t = b_1 T_0 + sum_{m>=2} 2 b_m T_{m-1} and p(t) = c_0 + t b_1 - b_2 (synthetic division
// by (s - t) in the Chebyshev basis).
//
// One pass: residuals, the FP32 per-column recurrence, Y = p(t) X + Z diag(||r|| / d) in
// FP64, orthonormalization (CholQR2) and Rayleigh-Ritz with A, all in FP64.  The reference's
// only post-processing is Rayleigh-Ritz (refine_original_rr, polfed.jl:837-880); this
// filtered pass is what an FP32 basis needs on top of it to reach its tolerance.
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <string>

#include "solver_common.h"
#include "vec.cuh"

namespace sma {
namespace {

// Residual block of the filtered columns: R[i, a] = (AX[i, j] - theta[j] X[i, j]) inv_s[j]
// for j = act[a], a < ka; zero for ka <= a < kapad (padding to full vector width).
__global__ void residual_f32_kernel(int64_t n, int64_t ka, int64_t kapad, const int *__restrict__ act,
                                    const double *__restrict__ X, int64_t ldx,
                                    const double *__restrict__ AX, int64_t ldax,
                                    const double *__restrict__ theta,
                                    const double *__restrict__ inv_s, float *__restrict__ R) {
  const int64_t total = n * kapad;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / kapad, a = t % kapad;
    float v = 0.f;
    if (a < ka) {
      const int j = act[a];
      v = (float)((AX[i * ldax + j] - theta[j] * X[i * ldx + j]) * inv_s[j]);
    }
    R[i * kapad + a] = v;
  }
}

// Y[i, j] = pt[j] X[i, j] + sd[j] Z[i, slot[j]] for filtered columns (slot[j] >= 0), and
// Y[i, j] = X[i, j] for the others (FP64 result from the FP32 correction block).
__global__ void combine_kernel(int64_t n, int64_t k, const double *__restrict__ X, int64_t ldx,
                               const float *__restrict__ Z, int64_t ldz, const int *__restrict__ slot,
                               const double *__restrict__ pt, const double *__restrict__ sd,
                               double *__restrict__ Y, int64_t ldy) {
  const int64_t total = n * k;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / k, j = t % k;
    const int a = slot[j];
    const double x = X[i * ldx + j];
    Y[i * ldy + j] = a >= 0 ? pt[j] * x + sd[j] * (double)Z[i * ldz + a] : x;
  }
}

// out = crow[j] Q + alpha AX + beta B1 - B2 (per-column coefficient; operators without a
// fused step: the model stencils and half storage).
template <typename T>
__global__ void percol_axpy_kernel(int64_t n, int64_t b, const T *__restrict__ Q,
                                   const T *__restrict__ AX, const T *__restrict__ B1,
                                   const T *__restrict__ B2, T *__restrict__ out, int64_t ld,
                                   const T *__restrict__ crow, T alpha, T beta) {
  const int64_t total = n * b;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / b, j = t % b;
    const int64_t e = i * ld + j;
    out[e] = clenshaw_combine<true, true, true>(AX[e], Q[e], B1[e], B2[e], crow[j], alpha, beta);
  }
}

int grid_of(int64_t total) {
  const int64_t g = (total + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

}  // namespace

// Y = q(A_hat) Q where column j of the n x b blocks (ld = b) runs its own polynomial with
// coefficients coef[m * b + j], m = 0..K (row-major (K+1) x b table, FP32 or FP64 like
// the blocks).  colseg is the identity map 0..b-1 on the device; B1, B2, TMP (and AX for
// operators without a fused step) are n x b work blocks.  The recurrence starts from zero
// blocks, so its first product multiplies zeros (one extra step out of K+1).
template <typename T>
FilterCount percol_filter(const sma_op *op, cudaStream_t st, const T *coef, int64_t K,
                          double smin, double smax, const T *Q, T *Y, int64_t b,
                          const int *colseg, T *B1, T *B2, T *TMP, T *AX) {
  FilterCount fc;
  const int64_t n = op->n;
  require(op->kind != OP_MATBLOCK, SMA_ERR_ARG, "the per-column filter needs a device operator");
  const double c = 0.5 * (smin + smax), invd = 2.0 / (smax - smin);
  const double alpha = 2.0 * invd, beta = -2.0 * c * invd;
  const size_t bytes = (size_t)(n * b) * sizeof(T);
  SMA_CUDA(cudaMemsetAsync(B1, 0, bytes, st));
  SMA_CUDA(cudaMemsetAsync(B2, 0, bytes, st));
  const bool fused = op->kind == OP_CSR;
  auto step = [&](const T *crow, T *out, double al, double be) {
    if (fused) {
      csr_clenshaw_step_seg<T>(op, st, b, Q, b, B1, B2, b, out, b, crow, colseg, al, be, true);
    } else {
      if (op->kind == OP_CSR_HALF)
        half_product<T>(op, st, B1, b, AX, b, b);
      else
        launch_clenshaw_step<T>(op, st, b, nullptr, 0, B1, nullptr, b, AX, b, 0.0, 1.0, 0.0, false);
      percol_axpy_kernel<T><<<grid_of(n * b), 256, 0, st>>>(n, b, Q, AX, B1, B2, out, b, crow,
                                                           (T)al, (T)be);
      SMA_CHECK_LAUNCH();
    }
  };
  const double mat_bytes = clenshaw_step_bytes(op, 0, sizeof(T));
  const double blk = (double)n * (double)b * sizeof(T);
  for (int64_t k = K; k >= 1; --k) {
    step(coef + k * b, TMP, alpha, beta);
    T *t = B2;  // B1, B2, TMP = TMP, B1, B2
    B2 = B1;
    B1 = TMP;
    TMP = t;
  }
  step(coef, Y, invd, -(c * invd));
  check_bulk_error(op, st);
  fc.steps = K + 1;
  fc.bytes = (double)(K + 1) * (mat_bytes + 4 * blk);
  return fc;
}

template FilterCount percol_filter<float>(const sma_op *, cudaStream_t, const float *, int64_t,
                                          double, double, const float *, float *, int64_t,
                                          const int *, float *, float *, float *, float *);
template FilterCount percol_filter<double>(const sma_op *, cudaStream_t, const double *, int64_t,
                                           double, double, const double *, double *, int64_t,
                                           const int *, double *, double *, double *, double *);

// Coefficients e_0..e_{K-1} of q_t (p's divided difference at t) and p(t), from the
// Clenshaw intermediates of p at t.
void divided_difference(const std::vector<double> &c, double t, double *e, double *pt) {
  const int64_t K = (int64_t)c.size() - 1;
  double b1 = 0.0, b2 = 0.0;  // b_{m+1}, b_{m+2}
  for (int64_t m = K; m >= 1; --m) {
    const double bm = c[m] + 2.0 * t * b1 - b2;
    if (m >= 2) e[m - 1] = 2.0 * bm;
    else e[0] = bm;
    b2 = b1;
    b1 = bm;
  }
  *pt = c[0] + t * b1 - b2;
}

using detail::dev_to_host;

PolishConfig polish_config() {
  PolishConfig c;
  if (const char *f = std::getenv("SMA_POLISH_FILTER")) c.step_filter = std::string(f) == "step";
  if (const char *f = std::getenv("SMA_POLISH_FILTER_GUARDS")) c.filter_guards = std::string(f) == "1";
  // unfiltered guards: three times the in-window count, so that one pass converges C3-sized
  // windows; filtered guards: as many as the in-window candidates
  c.guard_fraction = c.filter_guards ? 1.0 : 3.0;
  if (const char *g = std::getenv("SMA_POLISH_GUARDS")) c.guard_fraction = std::max(0.0, std::atof(g));
  if (const char *d = std::getenv("SMA_POLISH_DEGREE")) c.degree_scale = std::max(0.05, std::atof(d));
  if (const char *p = std::getenv("SMA_POLISH_PASSES")) c.max_passes = std::max(0, std::atoi(p));
  if (const char *v = std::getenv("SMA_POLISH_VERBOSE")) c.verbose = std::string(v) == "1";
  if (const char *r = std::getenv("SMA_POLISH_REFINE")) c.refine = std::string(r) == "1";
  return c;
}

PolishOut polish_mixed(const sma_op *op, const PolishCoeffs &coeffs_of, int64_t K0, int64_t Kmax,
                       double smin, double smax, double *X, int64_t k, const PolishDone &done,
                       const PolishNeeds &needs, int64_t max_passes, FilterCount &fc,
                       int64_t *qr_fallbacks, const std::vector<double> &lam0,
                       const std::vector<double> &res0, double emin, double emax,
                       bool filter_all, bool verbose, const PolishTrace &trace) {
  PolishOut out;
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  const int64_t n = op->n;
  require(K0 >= 1 && Kmax >= K0, SMA_ERR_ARG, "the polish needs a filter of degree >= 1");
  int64_t K = K0;
  std::vector<double> coeffs = coeffs_of(K);
  const double c = 0.5 * (smin + smax), d = 0.5 * (smax - smin);
  const int64_t kpad = (k + 7) / 8 * 8;  // FP32 rows of 32-byte multiples: full vector width
  Dense dn(ctx);
  DevBuf<double> AX(n * k, st), Y(n * k, st), H(k * k, st), mu(k, st), lam_d(k, st), res_d(k, st),
      scratch, theta_d(k, st), inv_s_d(k, st), pt_d(k, st), sd_d(k, st);
  // the FP32 recurrence blocks hold the filtered columns only (the guards are never
  // filtered unless filter_all), sized by the first pass and grown if a later pass needs more
  DevBuf<float> R32, Z32, B1, B2, TMP, AX32, coef32;
  int64_t fcap = 0;
  auto ensure_fp32 = [&](int64_t kap) {
    if (kap <= fcap) return;
    fcap = kap;
    R32.alloc(n * kap, st);
    Z32.alloc(n * kap, st);
    B1.alloc(n * kap, st);
    B2.alloc(n * kap, st);
    TMP.alloc(n * kap, st);
    coef32.alloc(Kmax * kap, st);
    if (op->kind != OP_CSR) AX32.alloc(n * kap, st);
  };
  DevBuf<int> colseg(kpad, st), act_d(kpad, st), slot_d(k, st);
  {
    std::vector<int> idn(kpad);
    for (int64_t j = 0; j < kpad; ++j) idn[j] = (int)j;
    SMA_CUDA(cudaMemcpyAsync(colseg.p, idn.data(), kpad * sizeof(int), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaStreamSynchronize(st));
  }
  // Rayleigh-Ritz with A on span(V) (V n x k, orthonormalized in place): X = V E,
  // out.lam/out.res its Ritz values (ascending) and residual norms.
  auto rayleigh_ritz = [&](double *V) {
    orthonormalize(ctx, n, k, V, k, false, 0.0, nullptr, qr_fallbacks);
    op_apply(op, st, V, k, AX.p, k, k);
    dn.gram(n, k, k, V, k, AX.p, k, H.p, k);
    dn.syevd(k, H.p, k, mu.p, true);
    dn.mul_small(n, k, k, V, k, H.p, k, X, k, 1.0, 0.0);
    op_apply(op, st, X, k, AX.p, k, k);
    column_reduce(st, 0, n, k, X, k, AX.p, k, nullptr, lam_d.p, scratch);
    column_reduce(st, 1, n, k, X, k, AX.p, k, lam_d.p, res_d.p, scratch);
    out.lam = dev_to_host(st, lam_d.p, k);
    out.res = dev_to_host(st, res_d.p, k);
  };
  // The same Rayleigh-Ritz without orthonormalizing V first: S = V^T V, H = V^T A V and
  // the generalized eigenproblem H E = S E diag(mu), X = V E (S-orthonormal E, so X has
  // orthonormal columns): three n k^2 products instead of the six of CholQR2 followed by
  // Rayleigh-Ritz.  The columns of V (filtered candidates and Ritz vectors of the basis)
  // are nearly orthogonal, so S is well conditioned; when it is not positive definite the
  // orthonormalizing path runs instead.
  // Both products are symmetric, so only their upper triangles are formed.  The Ritz
  // vectors with values in [emin, emax] are lifted first (columns 0..kin-1 of X); the
  // others only when done() says the polish goes on.
  DevBuf<double> S, E;
  DevBuf<int64_t> perm_d;
  auto rayleigh_ritz_gen = [&](double *V) {
    if (!S.p) {
      S.alloc(k * k, st);
      E.alloc(k * k, st);
      perm_d.alloc(k, st);
    }
    op_apply(op, st, V, k, AX.p, k, k);
    dn.gram(n, k, k, V, k, V, k, S.p, k, 1.0, 0.0, true);
    dn.gram(n, k, k, V, k, AX.p, k, H.p, k, 1.0, 0.0, true);
    if (!dn.sygvd(k, H.p, k, S.p, k, mu.p)) {
      if (qr_fallbacks) ++*qr_fallbacks;
      rayleigh_ritz(V);
      return;
    }
    const std::vector<double> muh = dev_to_host(st, mu.p, k);
    std::vector<int64_t> perm;
    for (int64_t j = 0; j < k; ++j)
      if (emin <= muh[j] && muh[j] <= emax) perm.push_back(j);
    const int64_t kin = (int64_t)perm.size();
    for (int64_t j = 0; j < k; ++j)
      if (!(emin <= muh[j] && muh[j] <= emax)) perm.push_back(j);
    SMA_CUDA(cudaMemcpyAsync(perm_d.p, perm.data(), k * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    launch_gather_columns_cm(st, k, k, H.p, k, perm_d.p, E.p, k);
    SMA_CUDA(cudaStreamSynchronize(st));  // perm must outlive its copy
    out.lam.assign(k, 0.0);
    out.res.assign(k, INFINITY);
    for (int64_t j = kin; j < k; ++j) out.lam[j] = muh[perm[j]];
    auto lift = [&](int64_t c0, int64_t c1) {  // Ritz vectors c0..c1-1 (perm order) into X
      const int64_t c = c1 - c0;
      if (c <= 0) return;
      dn.mul_small(n, k, c, V, k, E.p + c0 * k, k, X + c0, k, 1.0, 0.0);
      op_apply(op, st, X + c0, k, AX.p + c0, k, c);
      column_reduce(st, 0, n, c, X + c0, k, AX.p + c0, k, nullptr, lam_d.p, scratch);
      column_reduce(st, 1, n, c, X + c0, k, AX.p + c0, k, lam_d.p, res_d.p, scratch);
      const std::vector<double> l = dev_to_host(st, lam_d.p, c), r = dev_to_host(st, res_d.p, c);
      std::copy(l.begin(), l.end(), out.lam.begin() + c0);
      std::copy(r.begin(), r.end(), out.res.begin() + c0);
    };
    lift(0, kin);
    if (!done(out.lam, out.res)) lift(kin, k);
  };
  // phase times for the verbose trace (the stream is synchronized only then)
  auto now_ms = [&]() {
    if (!verbose) return 0.0;
    SMA_CUDA(cudaStreamSynchronize(st));
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
  };
  double t_mark = now_ms();
  if (filter_all || lam0.size() != (size_t)k || res0.size() != (size_t)k) {
    // consistent start: Rayleigh-Ritz on the columns themselves
    SMA_CUDA(cudaMemcpyAsync(Y.p, X, n * k * sizeof(double), cudaMemcpyDeviceToDevice, st));
    rayleigh_ritz(Y.p);
  } else {
    out.lam = lam0;
    out.res = res0;
    op_apply(op, st, X, k, AX.p, k, k);  // the residual block of the first pass reads A X
  }
  if (verbose) {
    const double t = now_ms();
    fprintf(stderr, "polish start: k=%lld %.1f ms\n", (long long)k, t - t_mark);
    t_mark = t;
  }
  if (trace) trace(0, out.lam, out.res);
  std::vector<double> inv_s(k), pt(k), sd(k), e;
  std::vector<float> cf;
  std::vector<int> act, slot(k);
  // the largest residual among the columns still to converge
  auto worst = [&]() {
    double w = 0.0;
    for (int64_t j = 0; j < k; ++j)
      if (needs(out.lam[j], out.res[j])) w = std::max(w, out.res[j]);
    return w;
  };
  double prev = worst();
  for (int64_t pass = 0; pass < max_passes && !done(out.lam, out.res); ++pass) {
    e.resize(K);
    // the columns to filter: all of them in the first pass, then those the caller still needs
    act.clear();
    for (int64_t j = 0; j < k; ++j) {
      const bool f = (pass == 0 && filter_all) || needs(out.lam[j], out.res[j]);
      slot[j] = f ? (int)act.size() : -1;
      if (f) act.push_back((int)j);
    }
    const int64_t ka = (int64_t)act.size(), kapad = (ka + 7) / 8 * 8;
    if (ka == 0) break;
    ensure_fp32(kapad);
    cf.assign(K * kapad, 0.f);
    for (int64_t a = 0; a < ka; ++a) {
      const int64_t j = act[a];
      const double s = out.res[j];
      inv_s[j] = s > 0.0 ? 1.0 / s : 0.0;
      sd[j] = s / d;
      divided_difference(coeffs, (out.lam[j] - c) / d, e.data(), &pt[j]);
      for (int64_t m = 0; m < K; ++m) cf[m * kapad + a] = (float)e[m];
    }
    SMA_CUDA(cudaMemcpyAsync(theta_d.p, out.lam.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(inv_s_d.p, inv_s.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(pt_d.p, pt.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(sd_d.p, sd.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(act_d.p, act.data(), ka * sizeof(int), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(slot_d.p, slot.data(), k * sizeof(int), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(coef32.p, cf.data(), cf.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    residual_f32_kernel<<<grid_of(n * kapad), 256, 0, st>>>(n, ka, kapad, act_d.p, X, k, AX.p, k,
                                                           theta_d.p, inv_s_d.p, R32.p);
    SMA_CHECK_LAUNCH();
    const FilterCount f = percol_filter<float>(op, st, coef32.p, K - 1, smin, smax, R32.p, Z32.p,
                                               kapad, colseg.p, B1.p, B2.p, TMP.p, AX32.p);
    fc.steps += f.steps;
    fc.bytes += f.bytes;
    combine_kernel<<<grid_of(n * k), 256, 0, st>>>(n, k, X, k, Z32.p, kapad, slot_d.p, pt_d.p,
                                                   sd_d.p, Y.p, k);
    SMA_CHECK_LAUNCH();
    const double t_filt = now_ms();
    if (filter_all) rayleigh_ritz(Y.p);
    else rayleigh_ritz_gen(Y.p);
    SMA_CUDA(cudaStreamSynchronize(st));  // the host tables above are rewritten next pass
    if (verbose) {
      const double t = now_ms();
      fprintf(stderr, "polish pass %lld: filtered %lld columns at degree %lld in %.1f ms, "
              "Rayleigh-Ritz of %lld in %.1f ms\n", (long long)pass + 1, (long long)ka,
              (long long)K, t_filt - t_mark, (long long)k, t - t_filt);
      t_mark = t;
    }
    out.passes += 1;
    out.columns += ka;
    out.degree = K;
    if (trace) trace(out.passes, out.lam, out.res);
    // a pass that cut the worst unconverged residual by less than 3x met the filter's ratio
    // just outside the window, not the FP32 floor: sharpen the polynomial for the next pass
    const double now = worst();
    if (pass > 0 && now > prev / 3.0 && K < Kmax) {
      K = std::min(2 * K, Kmax);
      coeffs = coeffs_of(K);
    }
    prev = now;
  }
  return out;
}

}  // namespace sma
