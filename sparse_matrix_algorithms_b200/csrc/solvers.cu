// Solver driver: chebyshev_poly_real_symm_sparse on one GPU (POLFED: polfed.cu).
//
// All n-sized data stays on the device for the whole solve; the host sees only
// eigenvalues, residuals, block factors and rank decisions (a few KB per step).
// Control flow, selection rules and return ordering follow the reference line by line;
// the numerical kernels are this library's (kernels.cu, filter.cu, dense.cu).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>

#include "solver_common.h"

namespace sma {

using namespace detail;

namespace {

// Chebyshev subspace iteration with locking (sma_cheb_opts.lock = 1, matrix-free overload
// semantics for termination): the in-window Ritz pairs whose residual is below tol are
// moved to a locked set, the remaining Ritz vectors form the next (narrower) block, and
// every filtered block is projected against the locked vectors (two classical Gram-Schmidt
// passes) before its orthonormalization -- the reference's append_locked!
// (chebyshev_subspace_iteration.jl:282-290) put to use.
sma_result *cheb_solve_locked(sma_op *op, double emin, double emax, const sma_cheb_opts &o,
                              int64_t m0, double smin, double smax, Filter &flt, sma_stats &stats,
                              std::chrono::steady_clock::time_point t0, int64_t launches0) {
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  const int64_t n = op->n;
  Dense dn(ctx);
  PhaseClock clk(st);
  DevBuf<double> Q(n * m0, st), Y(n * m0, st), X(n * m0, st), Xlock(n * m0, st),
      Aq(m0 * m0, st), C(m0 * m0, st), lam_d(m0, st), res_d(m0, st), scratch;
  launch_randn(st, n, m0, (uint64_t)o.seed, Q.p, m0);
  std::vector<double> lam, res, lam_lock, res_lock;
  int64_t m = m0, nlock = 0, it = 0;
  bool prev_ok = false;
  MixedSwitch mixed;
  for (it = 1; it <= o.maxiter && m > 0; ++it) {
    const bool fp32_iteration = flt.in_fp32();
    clk.mark(PH_FILTER);
    flt.run(Q.p, m0, Y.p, m0, m);
    clk.mark(PH_ORTH);
    for (int pass = 0; pass < 2 && nlock > 0; ++pass) {  // Y -= Xlock (Xlock' Y)
      dn.gram(n, nlock, m, Xlock.p, m0, Y.p, m0, C.p, m0);
      dn.mul_small(n, nlock, m, Xlock.p, m0, C.p, m0, Y.p, m0, -1.0, 1.0);
    }
    std::swap(Q.p, Y.p);
    orthonormalize(ctx, n, m, Q.p, m0, false, 0.0, nullptr, &stats.qr_fallbacks);
    clk.mark(PH_RR);
    op_apply(op, st, Q.p, m0, Y.p, m0, m);
    dn.gram(n, m, m, Q.p, m0, Y.p, m0, Aq.p, m);
    dn.syevd(m, Aq.p, m, lam_d.p, true);
    dn.mul_small(n, m, m, Q.p, m0, Aq.p, m, X.p, m0, 1.0, 0.0);
    op_apply(op, st, X.p, m0, Y.p, m0, m);
    column_reduce(st, 1, n, m, X.p, m0, Y.p, m0, lam_d.p, res_d.p, scratch);
    clk.close();
    lam = dev_to_host(st, lam_d.p, m);
    res = dev_to_host(st, res_d.p, m);
    // convergence over locked + active pairs (chebyshev_subspace_iteration.jl:817-836)
    int64_t cnt = nlock;
    double maxres = nlock ? *std::max_element(res_lock.begin(), res_lock.end()) : -INFINITY;
    for (int64_t j = 0; j < m; ++j)
      if (lam[j] >= emin && lam[j] <= emax && res[j] < o.res_gate) {
        ++cnt;
        maxres = std::max(maxres, res[j]);
      }
    if (cnt == 0) maxres = INFINITY;
    if (o.debug) {
      printf("it=%lld inside=%lld locked=%lld maxres=%.3e\n", (long long)it, (long long)cnt,
             (long long)nlock, maxres);
      fflush(stdout);
    }
    if (o.precision == SMA_PREC_MIXED && fp32_iteration &&
        mixed.update(lam, res, emin, emax, std::max(std::fabs(smin), std::fabs(smax)),
                     it >= o.maxiter - 2))
      flt.fp64_phase = true;
    const bool ok = cnt > 0 && maxres < o.tol && !fp32_iteration;
    if (o.two_hit ? (ok && (it == 1 || prev_ok)) : ok) {
      ++it;
      break;
    }
    prev_ok = ok;
    if (fp32_iteration) continue;  // lock only pairs converged in FP64 arithmetic
    // lock the converged in-window pairs; the other Ritz vectors form the next block
    std::vector<int64_t> keep, lockj;
    for (int64_t j = 0; j < m; ++j)
      (lam[j] >= emin && lam[j] <= emax && res[j] < o.tol ? lockj : keep).push_back(j);
    if (lockj.empty()) {
      std::swap(Q.p, X.p);  // next block: the Ritz vectors
      continue;
    }
    {
      DevBuf<int64_t> d = upload_idx(st, lockj);
      launch_gather_columns_rm(st, n, (int64_t)lockj.size(), X.p, m0, d.p, Xlock.p + nlock, m0);
    }
    for (int64_t j : lockj) {
      lam_lock.push_back(lam[j]);
      res_lock.push_back(res[j]);
    }
    nlock += (int64_t)lockj.size();
    m = (int64_t)keep.size();
    if (m > 0) {
      DevBuf<int64_t> d = upload_idx(st, keep);
      launch_gather_columns_rm(st, n, m, X.p, m0, d.p, Q.p, m0);
    }
  }
  double ph[PH_COUNT] = {0, 0, 0, 0};
  clk.totals(ph);
  stats.iterations = it - 1;
  stats.basis_dim = m0;
  stats.spmm_steps = flt.total.steps;
  stats.spmm_columns = flt.columns * (int64_t)(flt.coeffs.size() > 1 ? flt.coeffs.size() - 1 : 1);
  stats.filter_bytes = flt.total.bytes;
  stats.fp32_filter_calls = flt.fp32_calls;
  stats.graph_replays = flt.w64.replays + flt.w32.replays;
  stats.locked = nlock;
  stats.filter_ms = ph[PH_FILTER];
  stats.orth_ms = ph[PH_ORTH];
  stats.rr_ms = ph[PH_RR];
  // selection over locked and active pairs, sorted by eigenvalue
  const double gate = std::max(o.res_gate, 10.0 * o.tol);
  std::vector<double> lam_all = lam_lock, res_all = res_lock;
  std::vector<int64_t> idx;
  for (int64_t j = 0; j < nlock; ++j) idx.push_back(j);
  if (m > 0)
    for (int64_t j = 0; j < (int64_t)lam.size(); ++j)
      if (lam[j] >= emin && lam[j] <= emax && res[j] < gate) {
        lam_all.push_back(lam[j]);
        res_all.push_back(res[j]);
        idx.push_back(nlock + j);
      }
  sma_result *r;
  if (idx.empty()) {
    r = empty_result(ctx, n);
  } else {
    // side by side: locked vectors, then the active Ritz vectors
    DevBuf<double> Xall(n * (nlock + std::max<int64_t>(m, 0)) + 1, st);
    const int64_t w = nlock + std::max<int64_t>(m, 0);
    if (nlock)
      SMA_CUDA(cudaMemcpy2DAsync(Xall.p, w * sizeof(double), Xlock.p, m0 * sizeof(double),
                                 nlock * sizeof(double), n, cudaMemcpyDeviceToDevice, st));
    if (m > 0)
      SMA_CUDA(cudaMemcpy2DAsync(Xall.p + nlock, w * sizeof(double), X.p, m0 * sizeof(double),
                                 m * sizeof(double), n, cudaMemcpyDeviceToDevice, st));
    std::vector<double> lsel(lam_all.size());
    for (size_t i = 0; i < lam_all.size(); ++i) lsel[i] = lam_all[i];
    const std::vector<int64_t> p = stable_argsort(lsel);
    r = make_result(ctx, n, Xall.p, w, take(idx, p), take(lam_all, p), take(res_all, p));
  }
  stats.total_ms = ms_since(t0);
  stats.kernel_launches = g_kernel_launches.load() - launches0;
  r->stats = stats;
  return r;
}

}  // namespace

// ====================================================================== Chebyshev
// chebyshev_poly_real_symm_sparse, chebyshev_subspace_iteration.jl:667-757 (sparse
// overload, matrix_free = 0) and 771-848 (matrix-free overload, matrix_free = 1).
sma_result *cheb_solve(sma_op *op, double emin, double emax, const sma_cheb_opts &o) {
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t launches0 = g_kernel_launches.load();
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  const bool mf = o.matrix_free != 0;
  const int64_t n = op->n;
  int64_t m0 = o.m0;
  const int64_t degree = o.degree;
  sma_stats stats{};
  if (!mf) {  // chebyshev_subspace_iteration.jl:669-674
    require(op->kind == OP_CSR || op->kind == OP_CSR_HALF, SMA_ERR_ARG,
            "the sparse overload needs an explicit sparse matrix");
    ensure_symmetry_known(op);
    require(op->sym_state == 1, SMA_ERR_NONSYMMETRIC,
            "Chebyshev filtered solver requires a real symmetric matrix");
    require(emin < emax, SMA_ERR_ARG, "need emin<emax");
    require(m0 > 0, SMA_ERR_ARG, "m0 must be positive");
    require(degree >= 0, SMA_ERR_ARG, "degree must be nonnegative");
  } else {
    require(m0 > 0, SMA_ERR_ARG, "m0 must be positive");
    require(degree >= 0, SMA_ERR_ARG, "degree must be nonnegative");
  }
  require(o.window_type >= 0 && o.window_type <= 2, SMA_ERR_WINDOW,
          "Unknown window type, possible are :step, :delta, and :smooth");
  m0 = std::min(m0, n);
  double smin, smax;
  if (!o.has_bounds) {  // chebyshev_subspace_iteration.jl:677-682
    require((op->kind == OP_CSR || op->kind == OP_CSR_HALF) && op->has_gersh, SMA_ERR_ARG,
            "gershgorin_bounds needs an explicit sparse matrix: pass smin and smax");
    smin = op->gersh_min;
    smax = op->gersh_max;
  } else {
    smin = o.smin;
    smax = o.smax;
  }
  if (!mf && !(emin >= smin && emax <= smax)) {  // chebyshev_subspace_iteration.jl:683
    fprintf(stderr, "Warning: target interval not contained in supplied spectral bounds; "
                    "filter quality may degrade\n");
    stats.warnings |= 1;
  }
  const double c = 0.5 * (smin + smax), d = 0.5 * (smax - smin);
  const double a = (emin - c) / d, b = (emax - c) / d;
  if (!(-1.0 <= a && a < b && b <= 1.0)) {  // chebyshev_subspace_iteration.jl:689
    char buf[256];
    snprintf(buf, sizeof buf, "mapped interval [%.17g,%.17g] not inside [-1,1]%s", a, b,
             mf ? "" : "; provide better spectral bounds");
    throw Error(SMA_ERR_INTERVAL, buf);
  }
  if (o.precision != SMA_PREC_FP64) {
    require(op->kind != OP_MATBLOCK, SMA_ERR_ARG, "FP32 filtering needs a device operator");
    ensure_fp32_values(op);
  }
  Filter flt{op, st, build_coeffs(degree, smin, smax, o.sigma, emin, emax, o.window_type, o.jackson != 0),
             smin, smax, o.precision};
  if (o.lock) return cheb_solve_locked(op, emin, emax, o, m0, smin, smax, flt, stats, t0, launches0);
  Dense dn(ctx);
  PhaseClock clk(st);
  DevBuf<double> Q(n * m0, st), Y(n * m0, st), X(n * m0, st), Aq(m0 * m0, st), lam_d(m0, st),
      res_d(m0, st), scratch;
  MixedSwitch mixed;
  launch_randn(st, n, m0, (uint64_t)o.seed, Q.p, m0);  // Random.seed!(seed); Q=randn(n,m0)
  std::vector<double> lam, res;
  bool prev_ok = false;
  int64_t it = 0;
  for (it = 1; it <= o.maxiter; ++it) {
    const bool fp32_iteration = flt.in_fp32();
    clk.mark(PH_FILTER);
    flt.run(Q.p, m0, Y.p, m0, m0);                         // Y = p(A_hat) Q
    clk.mark(PH_ORTH);
    std::swap(Q.p, Y.p);                                    // Q .= Y
    orthonormalize(ctx, n, m0, Q.p, m0, false, 0.0, nullptr, &stats.qr_fallbacks);  // thin_orth!
    clk.mark(PH_RR);
    op_apply(op, st, Q.p, m0, Y.p, m0, m0);                 // R = A Q
    dn.gram(n, m0, m0, Q.p, m0, Y.p, m0, Aq.p, m0);          // Aq = Q' R
    dn.syevd(m0, Aq.p, m0, lam_d.p, true);                   // eigen!(Symmetric(Aq)), upper
    dn.mul_small(n, m0, m0, Q.p, m0, Aq.p, m0, X.p, m0, 1.0, 0.0);  // X = Q Xq
    op_apply(op, st, X.p, m0, Y.p, m0, m0);                  // AX = A X
    column_reduce(st, 1, n, m0, X.p, m0, Y.p, m0, lam_d.p, res_d.p, scratch);  // residuals!
    clk.close();
    lam = dev_to_host(st, lam_d.p, m0);
    res = dev_to_host(st, res_d.p, m0);
    int64_t cnt = 0;
    double maxres = -INFINITY;
    std::vector<double> rin;
    for (int64_t j = 0; j < m0; ++j) {
      if (lam[j] >= emin && lam[j] <= emax && res[j] < o.res_gate) {
        ++cnt;
        maxres = std::max(maxres, res[j]);
        rin.push_back(res[j]);
      }
    }
    if (cnt == 0) maxres = INFINITY;
    if (o.debug) {
      if (mf) {  // chebyshev_subspace_iteration.jl:826 also prints the 0.9 quantile
        double r90 = INFINITY;
        if (!rin.empty()) {
          std::sort(rin.begin(), rin.end());
          const double h = 0.9 * (double)(rin.size() - 1);
          const size_t lo = (size_t)std::floor(h);
          const size_t hi = std::min(rin.size() - 1, lo + 1);
          r90 = rin[lo] + (h - (double)lo) * (rin[hi] - rin[lo]);
        }
        printf("it=%lld inside=%lld maxres=%.3e r90=%.3e\n", (long long)it, (long long)cnt, maxres, r90);
      } else {
        printf("it=%lld inside=%lld maxres=%.3e\n", (long long)it, (long long)cnt, maxres);
      }
      fflush(stdout);
    }
    if (o.precision == SMA_PREC_MIXED && fp32_iteration &&
        mixed.update(lam, res, emin, emax, std::max(std::fabs(smin), std::fabs(smax)),
                     it >= o.maxiter - 2))
      flt.fp64_phase = true;
    if (mf) {  // chebyshev_subspace_iteration.jl:827-836
      const bool ok = cnt > 0 && maxres < o.tol && !fp32_iteration;
      if (o.two_hit) {
        if (ok && (it == 1 || prev_ok)) {
          if (o.debug) { printf("converged\n"); fflush(stdout); }
          ++it;
          break;
        }
        prev_ok = ok;
      } else if (ok) {
        ++it;
        break;
      }
    }
  }
  double ph[PH_COUNT] = {0, 0, 0, 0};
  clk.totals(ph);
  stats.iterations = it - 1;
  stats.basis_dim = m0;
  stats.spmm_steps = flt.total.steps;
  stats.spmm_columns = flt.total.steps * m0;
  stats.filter_bytes = flt.total.bytes;
  stats.fp32_filter_calls = flt.fp32_calls;
  stats.graph_replays = flt.w64.replays + flt.w32.replays;
  stats.filter_ms = ph[PH_FILTER];
  stats.orth_ms = ph[PH_ORTH];
  stats.rr_ms = ph[PH_RR];
  // selection, chebyshev_subspace_iteration.jl:750-756
  std::vector<int64_t> idx;
  const double gate = std::max(o.res_gate, 10.0 * o.tol);
  for (int64_t j = 0; j < (int64_t)lam.size(); ++j)
    if (lam[j] >= emin && lam[j] <= emax && res[j] < gate) idx.push_back(j);
  sma_result *r;
  if (idx.empty()) {
    r = empty_result(ctx, n);
  } else {
    std::vector<double> lsel = take(lam, idx);
    const std::vector<int64_t> p = stable_argsort(lsel);
    idx = take(idx, p);
    r = make_result(ctx, n, X.p, m0, idx, take(lam, idx), take(res, idx));
  }
  stats.total_ms = ms_since(t0);
  stats.kernel_launches = g_kernel_launches.load() - launches0;
  r->stats = stats;
  return r;
}

}  // namespace sma
