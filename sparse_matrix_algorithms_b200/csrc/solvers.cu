// Solver drivers: chebyshev_poly_real_symm_sparse and polfed on one GPU.
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
  double ph[PH_COUNT] = {0, 0, 0};
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
  double ph[PH_COUNT] = {0, 0, 0};
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

// ====================================================================== POLFED
namespace {

struct RitzSet {
  std::vector<double> lam, res;
};

// rayleigh!, polfed.jl:791-830: lam_j = x_j' A x_j, res_j = ||A x_j - lam_j x_j||
RitzSet rayleigh(const sma_op *op, cudaStream_t st, int64_t n, int64_t k, const double *X,
                 int64_t ldx, double *AX, DevBuf<double> &lam_d, DevBuf<double> &res_d,
                 DevBuf<double> &scratch) {
  if (lam_d.count < (size_t)k) lam_d.alloc(k, st);
  if (res_d.count < (size_t)k) res_d.alloc(k, st);
  op_apply(op, st, X, ldx, AX, ldx, k);
  column_reduce(st, 0, n, k, X, ldx, AX, ldx, nullptr, lam_d.p, scratch);
  column_reduce(st, 1, n, k, X, ldx, AX, ldx, lam_d.p, res_d.p, scratch);
  RitzSet s;
  s.lam = dev_to_host(st, lam_d.p, k);
  s.res = dev_to_host(st, res_d.p, k);
  return s;
}

}  // namespace

// polfed(A::MatrixFreeRealSymOp, nev, degree; ...), polfed.jl:1128-1158, with
// build_full_basis! (polfed.jl:1022-1099) and extract_pairs (polfed.jl:892-984).
sma_result *polfed_solve(sma_op *op, int64_t nev, int64_t degree, const sma_polfed_opts &o) {
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t launches0 = g_kernel_launches.load();
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  const int64_t n = op->n;
  sma_stats stats{};
  require(o.has_bounds != 0, SMA_ERR_BOUNDS, "Matrix-free POLFED requires spectral bounds smin and smax");
  require(o.window_type >= 0 && o.window_type <= 2, SMA_ERR_WINDOW,
          "Unknown window type: " + std::to_string(o.window_type));
  require(nev > 0, SMA_ERR_ARG, "nev must be positive");
  require(degree >= 0, SMA_ERR_ARG, "degree must be nonnegative");
  require(o.s > 0 && o.s <= n, SMA_ERR_ARG, "block size s must be in 1..n");
  require(o.overextract >= 0 && o.extra_keep >= 0, SMA_ERR_ARG, "overextract and extra_keep must be nonnegative");
  const double smin = o.smin, smax = o.smax;
  if (o.precision != SMA_PREC_FP64) {
    require(op->kind != OP_MATBLOCK, SMA_ERR_ARG, "FP32 filtering needs a device operator");
    ensure_fp32_values(op);
  }
  Filter flt{op, st, build_coeffs(degree, smin, smax, o.sigma, o.emin, o.emax, o.window_type, o.jackson != 0),
             smin, smax, o.precision};
  const int64_t s = o.s;
  const int64_t mmax = o.mmax > 0 ? o.mmax : (int64_t)std::ceil(2.8 * (double)nev / (double)s);
  const int64_t Mcap = std::max<int64_t>(mmax * s, 1);
  Dense dn(ctx);
  PhaseClock clk(st);

  // ---- basis storage V = [Q_1 ... Q_m], row-major n x Mcap
  DevBuf<double> V(n * Mcap, st), W(n * s, st), C(Mcap * s, st), G(s * s, st), Aj(s * s, st),
      Bcur(s * s, st), Bprev(s * s, st), T(Mcap * Mcap, st), scratch;
  SMA_CUDA(cudaMemsetAsync(T.p, 0, Mcap * Mcap * sizeof(double), st));
  // Q1 = orth_block_polfed!(randn(n,s); rtol)   (polfed.jl:1133-1134)
  launch_randn(st, n, s, (uint64_t)o.seed, W.p, s);
  const int64_t r1 = orthonormalize(ctx, n, s, W.p, s, true, o.rtol, nullptr, &stats.qr_fallbacks);
  std::vector<int64_t> offs{0}, ranks{r1};
  if (r1 > 0)
    SMA_CUDA(cudaMemcpy2DAsync(V.p, Mcap * sizeof(double), W.p, s * sizeof(double),
                               r1 * sizeof(double), n, cudaMemcpyDeviceToDevice, st));
  int64_t nb = 0;  // blocks stored (length(Qhist))
  int64_t rprev = 0;
  for (int64_t it = 1; it <= mmax; ++it) {
    const int64_t j = it - 1;
    const int64_t o_j = offs[j], r = ranks[j];
    nb = it;  // push!(Qhist, copy(Q))
    double *Qj = V.p + o_j;
    clk.mark(PH_FILTER);
    flt.run(Qj, Mcap, W.p, r, r);  // W = p(A_hat) Q_j
    clk.mark(PH_ORTH);
    if (j > 0 && rprev > 0 && r > 0)  // W -= Q_{j-1} B_{j-1}'
      dn.mul_small(n, rprev, r, V.p + offs[j - 1], Mcap, Bprev.p, s, W.p, r, -1.0, 1.0, true);
    dn.gram(n, r, r, Qj, Mcap, W.p, r, G.p, s);        // Q_j' W
    launch_symmetrize(st, r, G.p, s, Aj.p, s);           // A_j = sym(Q_j' W)
    launch_place_blocks(st, T.p, Mcap, o_j, r, Aj.p, s, nullptr, s, 0);
    dn.mul_small(n, r, r, Qj, Mcap, Aj.p, s, W.p, r, -1.0, 1.0);  // W -= Q_j A_j
    if (it == mmax) {
      // The reference goes on to reorthogonalize and factor W, but the resulting
      // Q_{mmax+1} and B_mmax are never used (assemble_T reads B_1..B_{m-1}).
      clk.close();
      break;
    }
    const int64_t Mcur = o_j + r;
    for (int64_t p = 0; p < o.reorth_passes; ++p) {  // reorth_full!: all blocks, then Q_j
      dn.gram(n, Mcur, r, V.p, Mcap, W.p, r, C.p, Mcap);
      dn.mul_small(n, Mcur, r, V.p, Mcap, C.p, Mcap, W.p, r, -1.0, 1.0);
      dn.gram(n, r, r, Qj, Mcap, W.p, r, C.p, Mcap);
      dn.mul_small(n, r, r, Qj, Mcap, C.p, Mcap, W.p, r, -1.0, 1.0);
    }
    std::vector<double> Rh;
    const int64_t rn = orthonormalize(ctx, n, r, W.p, r, true, o.rtol, &Rh, &stats.qr_fallbacks);
    clk.close();
    if (rn == 0) break;  // rank collapsed (polfed.jl:1091)
    // B_j = R[1:rn, :] (rn x r), column-major with ld s
    std::vector<double> Bh(s * s, 0.0);
    for (int64_t cc = 0; cc < r; ++cc)
      for (int64_t rr = 0; rr < rn; ++rr) Bh[rr + cc * s] = Rh[rr + cc * r];
    SMA_CUDA(cudaMemcpyAsync(Bcur.p, Bh.data(), s * s * sizeof(double), cudaMemcpyHostToDevice, st));
    launch_place_blocks(st, T.p, Mcap, o_j, r, nullptr, s, Bcur.p, s, rn);
    SMA_CUDA(cudaMemcpy2DAsync(V.p + Mcur, Mcap * sizeof(double), W.p, r * sizeof(double),
                               rn * sizeof(double), n, cudaMemcpyDeviceToDevice, st));
    std::swap(Bcur.p, Bprev.p);
    rprev = r;
    offs.push_back(Mcur);
    ranks.push_back(rn);
  }
  const int64_t M = offs[nb - 1] + ranks[nb - 1];
  stats.iterations = nb;
  stats.basis_dim = M;

  // ---- extract_pairs (polfed.jl:892-984)
  clk.mark(PH_RR);
  DevBuf<double> theta_d(std::max<int64_t>(M, 1), st);
  dn.syevd(M, T.p, Mcap, theta_d.p, true);  // eigen(T), ascending
  const std::vector<double> theta = dev_to_host(st, theta_d.p, M);
  const int64_t m = std::min<int64_t>(M, std::max<int64_t>(o.overextract * nev, nev + o.extra_keep));
  // p = sortperm(theta; rev=true)[1:m]
  std::vector<int64_t> order(M);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return theta[a] > theta[b]; });
  order.resize(m);
  DevBuf<double> Usel(std::max<int64_t>(M * m, 1), st);
  {
    DevBuf<int64_t> d = upload_idx(st, order);
    launch_gather_columns_cm(st, M, m, T.p, Mcap, d.p, Usel.p, M);
  }
  // X = V Usel (build_X!), all m columns at once: chunking does not change the values
  DevBuf<double> X(n * std::max<int64_t>(m, 1), st), AX(n * std::max<int64_t>(m, 1), st), lam_d, res_d;
  dn.mul_small(n, M, m, V.p, Mcap, Usel.p, M, X.p, m, 1.0, 0.0);
  RitzSet rs = rayleigh(op, st, n, m, X.p, m, AX.p, lam_d, res_d, scratch);
  std::vector<double> lam_keep, res_keep;
  std::vector<int64_t> idx_keep;
  for (int64_t jj = 0; jj < m; ++jj)
    if (o.emin <= rs.lam[jj] && rs.lam[jj] <= o.emax) {
      lam_keep.push_back(rs.lam[jj]);
      res_keep.push_back(rs.res[jj]);
      idx_keep.push_back(jj);
    }
  auto finish = [&](sma_result *r) {
    clk.close();
    double ph[PH_COUNT] = {0, 0, 0};
    clk.totals(ph);
    stats.spmm_steps = flt.total.steps;
    stats.spmm_columns = flt.columns * (int64_t)(flt.coeffs.size() > 1 ? flt.coeffs.size() - 1 : 1);
    stats.filter_bytes = flt.total.bytes;
    stats.fp32_filter_calls = flt.fp32_calls;
    stats.graph_replays = flt.w64.replays + flt.w32.replays;
    stats.filter_ms = ph[PH_FILTER];
    stats.orth_ms = ph[PH_ORTH];
    stats.rr_ms = ph[PH_RR];
    stats.total_ms = ms_since(t0);
    stats.kernel_launches = g_kernel_launches.load() - launches0;
    r->stats = stats;
    return r;
  };
  if (idx_keep.empty()) {
    if (o.show_progress) { printf("m=%lld  inside=0  maxres=Inf\n", (long long)nb); fflush(stdout); }
    return finish(empty_result(ctx, n));
  }
  // MIXED: guard Ritz vectors for the FP64 polish, taken in theta order from the
  // out-of-window columns of X before the refinement reuses X's storage. Without guards
  // the polish converges at the ratio p(first outside)/p(window edge), which is close to 1.
  DevBuf<double> guard;
  int64_t ng = 0;
  if (o.precision == SMA_PREC_MIXED) {
    std::vector<int64_t> out;
    const int64_t want = std::max<int64_t>(1, ((int64_t)idx_keep.size() + 1) / 2);
    for (int64_t jj = 0; jj < m && (int64_t)out.size() < want; ++jj)
      if (!(o.emin <= rs.lam[jj] && rs.lam[jj] <= o.emax)) out.push_back(jj);
    ng = (int64_t)out.size();
    if (ng > 0) {
      guard.alloc(n * ng, st);
      DevBuf<int64_t> d = upload_idx(st, out);
      launch_gather_columns_rm(st, n, ng, X.p, m, d.p, guard.p, ng);
    }
  }
  const int64_t npre = std::min<int64_t>((int64_t)res_keep.size(), nev + o.extra_keep);
  std::vector<int64_t> ps0 = stable_argsort(res_keep);
  ps0.resize(npre);
  std::vector<double> lamc = take(lam_keep, ps0), resc = take(res_keep, ps0);
  const std::vector<int64_t> idxc = take(idx_keep, ps0);
  // Xc = build_X!(Qhist, Usel[:, idxc]) = the columns idxc of X
  DevBuf<double> Xc(n * npre, st);
  {
    DevBuf<int64_t> d = upload_idx(st, idxc);
    launch_gather_columns_rm(st, n, npre, X.p, m, d.p, Xc.p, npre);
  }
  const double *Xfin = Xc.p;
  int64_t ldfin = npre;
  std::vector<int64_t> colmap(npre);
  std::iota(colmap.begin(), colmap.end(), 0);
  if (o.refine) {
    // refine_original_rr (polfed.jl:837-880); orth_block_polfed! at its default rtol=1e-12
    const int64_t k = orthonormalize(ctx, n, npre, Xc.p, npre, true, 1e-12, nullptr, &stats.qr_fallbacks);
    if (k == 0) {
      if (o.show_progress) { printf("m=%lld  inside=0  maxres=Inf\n", (long long)nb); fflush(stdout); }
      return finish(empty_result(ctx, n));
    }
    // AQ = A Q; H = sym(Q' AQ); eigen(H); Y = Q E
    op_apply(op, st, Xc.p, npre, AX.p, npre, k);
    DevBuf<double> H(k * k, st), Hs(k * k, st), mu(k, st);
    dn.gram(n, k, k, Xc.p, npre, AX.p, npre, H.p, k);
    launch_symmetrize(st, k, H.p, k, Hs.p, k);
    dn.syevd(k, Hs.p, k, mu.p, true);
    dn.mul_small(n, k, k, Xc.p, npre, Hs.p, k, X.p, k, 1.0, 0.0);  // Y into X's storage
    RitzSet rr = rayleigh(op, st, n, k, X.p, k, AX.p, lam_d, res_d, scratch);
    const std::vector<int64_t> pl = stable_argsort(rr.lam);
    lamc.clear();
    resc.clear();
    colmap.clear();
    for (int64_t t : pl)
      if (o.emin <= rr.lam[t] && rr.lam[t] <= o.emax) {  // interval filter after refinement
        lamc.push_back(rr.lam[t]);
        resc.push_back(rr.res[t]);
        colmap.push_back(t);
      }
    if (colmap.empty()) {
      if (o.show_progress) { printf("m=%lld  inside=0  maxres=Inf\n", (long long)nb); fflush(stdout); }
      return finish(empty_result(ctx, n));
    }
    Xfin = X.p;
    ldfin = k;
  }
  DevBuf<double> Xpol;
  if (o.precision == SMA_PREC_MIXED) {
    // FP64 polish of an FP32-filtered basis: Chebyshev subspace iterations with the same
    // filter in FP64 on the in-window candidates plus the guard vectors (orthonormalize,
    // Rayleigh-Ritz with A, residuals), until the best min(nev, in-window) residuals are
    // below tol; at most three passes.
    flt.fp64_phase = true;
    const int64_t kin = (int64_t)colmap.size();
    const int64_t k = kin + ng;
    Xpol.alloc(n * k, st);
    DevBuf<double> Yp(n * k, st), Hp(k * k, st), mup(k, st), AXp(n * k, st);
    {
      DevBuf<int64_t> d = upload_idx(st, colmap);
      launch_gather_columns_rm(st, n, kin, Xfin, ldfin, d.p, Yp.p, kin);
      launch_copy_block<double, double>(st, n, kin, Yp.p, kin, Xpol.p, k);
      if (ng > 0) launch_copy_block<double, double>(st, n, ng, guard.p, ng, Xpol.p + kin, k);
    }
    auto converged = [&] {
      std::vector<double> r;
      for (size_t i = 0; i < lamc.size(); ++i)
        if (o.emin <= lamc[i] && lamc[i] <= o.emax) r.push_back(resc[i]);
      if (r.empty()) return false;
      std::sort(r.begin(), r.end());
      return r[std::min<size_t>(nev, r.size()) - 1] < o.tol;
    };
    for (int pol = 0; pol < 3 && !converged(); ++pol) {
      clk.mark(PH_FILTER);
      flt.run(Xpol.p, k, Yp.p, k, k);
      clk.mark(PH_RR);
      orthonormalize(ctx, n, k, Yp.p, k, false, 0.0, nullptr, &stats.qr_fallbacks);
      op_apply(op, st, Yp.p, k, AXp.p, k, k);
      dn.gram(n, k, k, Yp.p, k, AXp.p, k, Hp.p, k);
      dn.syevd(k, Hp.p, k, mup.p, true);
      dn.mul_small(n, k, k, Yp.p, k, Hp.p, k, Xpol.p, k, 1.0, 0.0);
      RitzSet rp = rayleigh(op, st, n, k, Xpol.p, k, AXp.p, lam_d, res_d, scratch);
      clk.close();
      lamc = rp.lam;
      resc = rp.res;
      stats.polish_iterations += 1;
    }
    // keep the in-window pairs, as the refinement does; without a polish pass lamc still
    // describes the first kin columns of Xpol (the refined candidates)
    std::vector<int64_t> in;
    for (int64_t i = 0; i < (int64_t)lamc.size(); ++i)
      if (o.emin <= lamc[i] && lamc[i] <= o.emax) in.push_back(i);
    lamc = take(lamc, in);
    resc = take(resc, in);
    colmap = in;
    Xfin = Xpol.p;
    ldfin = k;
  }
  const int64_t nkeep = std::min<int64_t>((int64_t)resc.size(), nev + o.extra_keep);
  std::vector<int64_t> ps = stable_argsort(resc);
  ps.resize(nkeep);
  std::vector<double> lamf = take(lamc, ps), rf = take(resc, ps);
  std::vector<int64_t> cf = take(colmap, ps);
  const std::vector<int64_t> pe = stable_argsort(lamf);
  lamf = take(lamf, pe);
  rf = take(rf, pe);
  cf = take(cf, pe);
  if (o.show_progress) {  // _progress_line, polfed.jl:991-1000
    std::vector<double> srt = rf;
    std::sort(srt.begin(), srt.end());
    const int64_t L = (int64_t)srt.size();
    auto q = [&](double f) {
      int64_t i = (int64_t)std::nearbyint(f * (double)L);
      i = std::min(std::max<int64_t>(i, 1), L);
      return srt[i - 1];
    };
    printf("m=%lld  inside=%lld  r90=%.16g  r95=%.16g  maxres=%.16g\n", (long long)nb,
           (long long)lamf.size(), q(0.9), q(0.95), srt[L - 1]);
    fflush(stdout);
  }
  // return rule, polfed.jl:1148-1157
  std::vector<int64_t> sel;
  const int64_t L = (int64_t)rf.size();
  bool by_lambda = false;
  if (L >= nev) {
    std::vector<double> srt = rf;
    std::sort(srt.begin(), srt.end());
    by_lambda = srt[nev - 1] < o.tol;
  }
  if (by_lambda) {
    for (int64_t t = 0; t < nev; ++t) sel.push_back(t);
  } else {
    sel = stable_argsort(rf);
    sel.resize(std::min<int64_t>(nev, L));
  }
  std::vector<int64_t> cols = take(cf, sel);
  sma_result *res = make_result(ctx, n, Xfin, ldfin, cols, take(lamf, sel), take(rf, sel));
  return finish(res);
}

}  // namespace sma
