// POLFED: block Lanczos on the Chebyshev-filtered operator p(A_hat), polfed.jl:1128-1158,
// with build_full_basis! (polfed.jl:1022-1099) and extract_pairs (polfed.jl:892-984).
//
// One window's state is a PolfedWindow: the basis V = [Q_1 ... Q_m] (row-major n x Mcap on
// the device), the block tridiagonal T assembled on the device, and the block factors.
// A block step is split at the filter: the driver filters the window's current block Q_j
// into W = p(A_hat) Q_j, then absorb() runs the rest of the step (three-term recurrence,
// T assembly, full reorthogonalization, rank-revealing QR).  So the same window code runs
//   * alone (polfed_solve): the filter of filter.cu per block, graph-replayed; and
//   * batched (polfed_batch_solve): every active window's Q_j side by side in one
//     segmented recurrence (slice_batch.h) -- the sparse matrix read once per step for all
//     windows, each column with its own window's coefficients, each window's filtered
//     block bit-identical to its single-window filter.
// extract() is extract_pairs plus, for an FP32-filtered basis (MIXED), the polish of
// polish.cu, and the reference's return rule.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <numeric>

#include "slice_batch.h"

namespace sma {

using namespace detail;

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

void validate_polfed(const sma_op *op, int64_t nev, int64_t degree, const sma_polfed_opts &o) {
  require(o.has_bounds != 0, SMA_ERR_BOUNDS, "Matrix-free POLFED requires spectral bounds smin and smax");
  require(o.window_type >= 0 && o.window_type <= 2, SMA_ERR_WINDOW,
          "Unknown window type: " + std::to_string(o.window_type));
  require(nev > 0, SMA_ERR_ARG, "nev must be positive");
  require(degree >= 0, SMA_ERR_ARG, "degree must be nonnegative");
  require(o.s > 0 && o.s <= op->n, SMA_ERR_ARG, "block size s must be in 1..n");
  require(o.overextract >= 0 && o.extra_keep >= 0, SMA_ERR_ARG,
          "overextract and extra_keep must be nonnegative");
}

// The selected pairs of one window: columns `cols` of the device block X (ld ldx).
struct WindowPairs {
  std::vector<double> lam, res;
  std::vector<int64_t> cols;
  const double *X = nullptr;
  int64_t ldx = 1;
  bool by_lambda = false;  // the return rule's first branch (the nev-th residual below tol)
};

class PolfedWindow {
 public:
  PolfedWindow(sma_op *op, int64_t nev, int64_t degree, const sma_polfed_opts &o)
      : op_(op), ctx_(op->ctx), st_(op->ctx->stream), n_(op->n), o_(o), nev_(nev), s_(o.s),
        dn_(op->ctx) {
    coeffs = build_coeffs(degree, o.smin, o.smax, o.sigma, o.emin, o.emax, o.window_type,
                          o.jackson != 0);
    mmax_ = o.mmax > 0 ? o.mmax : (int64_t)std::ceil(2.8 * (double)nev / (double)s_);
    Mcap = std::max<int64_t>(mmax_ * s_, 1);
    V_.alloc(n_ * Mcap, st_);
    W_.alloc(n_ * s_, st_);
    C_.alloc(Mcap * s_, st_);
    G_.alloc(s_ * s_, st_);
    Aj_.alloc(s_ * s_, st_);
    Bcur_.alloc(s_ * s_, st_);
    Bprev_.alloc(s_ * s_, st_);
    T_.alloc(Mcap * Mcap, st_);
    SMA_CUDA(cudaMemsetAsync(T_.p, 0, Mcap * Mcap * sizeof(double), st_));
  }

  std::vector<double> coeffs;  // the window's filter polynomial
  int64_t Mcap = 1;            // basis capacity (leading dimension of V)

  // Q1 = orth_block_polfed!(randn(n,s); rtol)   (polfed.jl:1133-1134)
  void start(sma_stats &stats) {
    launch_randn(st_, n_, s_, (uint64_t)o_.seed, W_.p, s_);
    const int64_t r1 = orthonormalize(ctx_, n_, s_, W_.p, s_, true, o_.rtol, nullptr, &stats.qr_fallbacks);
    offs_ = {0};
    ranks_ = {r1};
    if (r1 > 0)
      SMA_CUDA(cudaMemcpy2DAsync(V_.p, Mcap * sizeof(double), W_.p, s_ * sizeof(double),
                                 r1 * sizeof(double), n_, cudaMemcpyDeviceToDevice, st_));
    nb_ = 0;
    rprev_ = 0;
    finished_ = false;
  }

  bool finished() const { return finished_; }
  // the block to filter next (row-major, ld Mcap) and its width
  const double *next_block() const { return V_.p + offs_[nb_]; }
  int64_t next_rank() const { return ranks_[nb_]; }
  // where the driver writes W = p(A_hat) Q_j: n x r, ld r
  double *filter_out() { return W_.p; }
  int64_t blocks() const { return nb_; }

  // The rest of block step j once filter_out() holds p(A_hat) Q_j (polfed.jl:1034-1096).
  void absorb(PhaseClock &clk, sma_stats &stats) {
    const int64_t j = nb_;
    const int64_t o_j = offs_[j], r = ranks_[j];
    nb_ = j + 1;  // push!(Qhist, copy(Q))
    const double *Qj = V_.p + o_j;
    if (j > 0 && rprev_ > 0 && r > 0)  // W -= Q_{j-1} B_{j-1}'
      dn_.mul_small(n_, rprev_, r, V_.p + offs_[j - 1], Mcap, Bprev_.p, s_, W_.p, r, -1.0, 1.0, true);
    dn_.gram(n_, r, r, Qj, Mcap, W_.p, r, G_.p, s_);   // Q_j' W
    launch_symmetrize(st_, r, G_.p, s_, Aj_.p, s_);     // A_j = sym(Q_j' W)
    launch_place_blocks(st_, T_.p, Mcap, o_j, r, Aj_.p, s_, nullptr, s_, 0);
    dn_.mul_small(n_, r, r, Qj, Mcap, Aj_.p, s_, W_.p, r, -1.0, 1.0);  // W -= Q_j A_j
    if (nb_ == mmax_) {
      // The reference goes on to reorthogonalize and factor W, but the resulting
      // Q_{mmax+1} and B_mmax are never used (assemble_T reads B_1..B_{m-1}).
      clk.close();
      finished_ = true;
      return;
    }
    const int64_t Mcur = o_j + r;
    for (int64_t p = 0; p < o_.reorth_passes; ++p) {  // reorth_full!: all blocks, then Q_j
      dn_.gram(n_, Mcur, r, V_.p, Mcap, W_.p, r, C_.p, Mcap);
      dn_.mul_small(n_, Mcur, r, V_.p, Mcap, C_.p, Mcap, W_.p, r, -1.0, 1.0);
      dn_.gram(n_, r, r, Qj, Mcap, W_.p, r, C_.p, Mcap);
      dn_.mul_small(n_, r, r, Qj, Mcap, C_.p, Mcap, W_.p, r, -1.0, 1.0);
    }
    std::vector<double> Rh;
    const int64_t rn = orthonormalize(ctx_, n_, r, W_.p, r, true, o_.rtol, &Rh, &stats.qr_fallbacks);
    clk.close();
    if (rn == 0) {  // rank collapsed (polfed.jl:1091)
      finished_ = true;
      return;
    }
    // B_j = R[1:rn, :] (rn x r), column-major with ld s
    std::vector<double> Bh(s_ * s_, 0.0);
    for (int64_t cc = 0; cc < r; ++cc)
      for (int64_t rr = 0; rr < rn; ++rr) Bh[rr + cc * s_] = Rh[rr + cc * r];
    SMA_CUDA(cudaMemcpyAsync(Bcur_.p, Bh.data(), s_ * s_ * sizeof(double), cudaMemcpyHostToDevice, st_));
    launch_place_blocks(st_, T_.p, Mcap, o_j, r, nullptr, s_, Bcur_.p, s_, rn);
    SMA_CUDA(cudaMemcpy2DAsync(V_.p + Mcur, Mcap * sizeof(double), W_.p, r * sizeof(double),
                               rn * sizeof(double), n_, cudaMemcpyDeviceToDevice, st_));
    SMA_CUDA(cudaStreamSynchronize(st_));  // Bh must outlive its copy
    std::swap(Bcur_.p, Bprev_.p);
    rprev_ = r;
    offs_.push_back(Mcur);
    ranks_.push_back(rn);
  }

  int64_t basis_dim() const { return nb_ == 0 ? 0 : offs_[nb_ - 1] + ranks_[nb_ - 1]; }

  // extract_pairs (polfed.jl:892-984), the MIXED polish, and the return rule
  // (polfed.jl:1148-1157).  The pairs' vectors stay in this window's storage.
  WindowPairs extract(PhaseClock &clk, sma_stats &stats, FilterCount &polish) {
    WindowPairs out;
    const int64_t n = n_, nev = nev_;
    const sma_polfed_opts &o = o_;
    const int64_t M = basis_dim();
    clk.mark(PH_RR);
    auto empty = [&]() {
      if (o.show_progress) { printf("m=%lld  inside=0  maxres=Inf\n", (long long)nb_); fflush(stdout); }
      clk.close();
      return WindowPairs{};
    };
    if (M == 0) return empty();
    DevBuf<double> theta_d(M, st_);
    dn_.syevd(M, T_.p, Mcap, theta_d.p, true);  // eigen(T), ascending
    const std::vector<double> theta = dev_to_host(st_, theta_d.p, M);
    // m0 candidates (polfed.jl:901); MIXED with unfiltered guards lifts up to
    // guard_fraction * nev more Ritz vectors, further out in theta, as guards only
    const PolishConfig pc = polish_config();
    const int64_t m0 = std::min<int64_t>(M, std::max<int64_t>(o.overextract * nev, nev + o.extra_keep));
    const int64_t m =
        (o.precision == SMA_PREC_MIXED && !pc.filter_guards)
            ? std::min<int64_t>(M, m0 + (int64_t)std::ceil(pc.guard_fraction * (double)nev))
            : m0;
    // p = sortperm(theta; rev=true)[1:m]
    std::vector<int64_t> order(M);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return theta[a] > theta[b]; });
    order.resize(m);
    DevBuf<double> Usel(std::max<int64_t>(M * m, 1), st_);
    {
      DevBuf<int64_t> d = upload_idx(st_, order);
      launch_gather_columns_cm(st_, M, m, T_.p, Mcap, d.p, Usel.p, M);
    }
    // X = V Usel (build_X!): the m0 candidates first (chunking does not change the values);
    // the further Ritz vectors only as far as the guard search below needs them
    X_.alloc(n * std::max<int64_t>(m, 1), st_);
    AX_.alloc(n * std::max<int64_t>(m, 1), st_);
    dn_.mul_small(n, M, m0, V_.p, Mcap, Usel.p, M, X_.p, m, 1.0, 0.0);
    RitzSet rs = rayleigh(op_, st_, n, m0, X_.p, m, AX_.p, lam_d_, res_d_, scratch_);
    int64_t mdone = m0;
    auto lift_more = [&](int64_t cnt) {
      cnt = std::min(cnt, m - mdone);
      if (cnt <= 0) return false;
      dn_.mul_small(n, M, cnt, V_.p, Mcap, Usel.p + mdone * M, M, X_.p + mdone, m, 1.0, 0.0);
      const RitzSet r2 = rayleigh(op_, st_, n, cnt, X_.p + mdone, m, AX_.p + mdone, lam_d_,
                                  res_d_, scratch_);
      rs.lam.insert(rs.lam.end(), r2.lam.begin(), r2.lam.end());
      rs.res.insert(rs.res.end(), r2.res.begin(), r2.res.end());
      mdone += cnt;
      return true;
    };
    auto drop_basis = [&]() {  // the basis is dead once the Ritz vectors are lifted
      V_.release();            // (stream-ordered frees)
      T_.release();
    };
    std::vector<double> lam_keep, res_keep;
    std::vector<int64_t> idx_keep;
    for (int64_t jj = 0; jj < m0; ++jj)
      if (o.emin <= rs.lam[jj] && rs.lam[jj] <= o.emax) {
        lam_keep.push_back(rs.lam[jj]);
        res_keep.push_back(rs.res[jj]);
        idx_keep.push_back(jj);
      }
    if (idx_keep.empty()) {
      drop_basis();
      return empty();
    }
    // MIXED: guard Ritz vectors for the polish, taken in theta order from the out-of-window
    // columns of X before the refinement reuses X's storage.  Without guards the polish
    // converges at the ratio p(first outside)/p(window edge), which is close to 1.
    DevBuf<double> guard;
    int64_t ng = 0;
    double guard_lo = o.emin, guard_hi = o.emax;  // the span of the guards' Ritz values
    std::vector<double> guard_lam, guard_res;      // their Rayleigh quotients and residuals
    if (o.precision == SMA_PREC_MIXED) {
      std::vector<int64_t> outw;
      const int64_t want =
          std::max<int64_t>(1, (int64_t)std::ceil(pc.guard_fraction * (double)idx_keep.size()));
      // Unfiltered guards must be converged about as far as the candidates: a guard that
      // mixes eigenvectors from both sides of the window has a part, orthogonal to the
      // candidates, whose Rayleigh quotient may fall inside the window -- a spurious
      // in-window Ritz pair.  Guards are therefore the out-of-window Ritz vectors, in theta
      // order, with residual at most 10x the largest in-window candidate residual.
      double gmax = INFINITY;
      if (!pc.filter_guards) {
        gmax = 0.0;
        for (double r : res_keep) gmax = std::max(gmax, r);
        gmax *= 10.0;
      }
      for (int64_t jj = 0; (int64_t)outw.size() < want; ++jj) {
        if (jj >= mdone && !lift_more(5 * (want - (int64_t)outw.size()) / 4 + 64)) break;
        if (!(o.emin <= rs.lam[jj] && rs.lam[jj] <= o.emax) && rs.res[jj] <= gmax) {
          outw.push_back(jj);
          guard_lo = std::min(guard_lo, rs.lam[jj]);
          guard_hi = std::max(guard_hi, rs.lam[jj]);
          guard_lam.push_back(rs.lam[jj]);
          guard_res.push_back(rs.res[jj]);
        }
      }
      ng = (int64_t)outw.size();
      if (ng > 0) {
        guard.alloc(n * ng, st_);
        DevBuf<int64_t> d = upload_idx(st_, outw);
        launch_gather_columns_rm(st_, n, ng, X_.p, m, d.p, guard.p, ng);
      }
    }
    drop_basis();
    const int64_t npre = std::min<int64_t>((int64_t)res_keep.size(), nev + o.extra_keep);
    std::vector<int64_t> ps0 = stable_argsort(res_keep);
    ps0.resize(npre);
    std::vector<double> lamc = take(lam_keep, ps0), resc = take(res_keep, ps0);
    const std::vector<int64_t> idxc = take(idx_keep, ps0);
    // Xc = build_X!(Qhist, Usel[:, idxc]) = the columns idxc of X
    Xc_.alloc(n * npre, st_);
    {
      DevBuf<int64_t> d = upload_idx(st_, idxc);
      launch_gather_columns_rm(st_, n, npre, X_.p, m, d.p, Xc_.p, npre);
    }
    const double *Xfin = Xc_.p;
    int64_t ldfin = npre;
    std::vector<int64_t> colmap(npre);
    std::iota(colmap.begin(), colmap.end(), 0);
    // MIXED with unfiltered guards: the polish's Rayleigh-Ritz (on the candidates, filtered,
    // and the guards) takes the place of the refinement, which would only rotate the
    // candidates among themselves first
    if (o.refine && !(o.precision == SMA_PREC_MIXED && !pc.filter_guards && !pc.refine)) {
      // refine_original_rr (polfed.jl:837-880); orth_block_polfed! at its default rtol=1e-12
      const int64_t k = orthonormalize(ctx_, n, npre, Xc_.p, npre, true, 1e-12, nullptr, &stats.qr_fallbacks);
      if (k == 0) return empty();
      // AQ = A Q; H = sym(Q' AQ); eigen(H); Y = Q E
      op_apply(op_, st_, Xc_.p, npre, AX_.p, npre, k);
      DevBuf<double> H(k * k, st_), Hs(k * k, st_), mu(k, st_);
      dn_.gram(n, k, k, Xc_.p, npre, AX_.p, npre, H.p, k);
      launch_symmetrize(st_, k, H.p, k, Hs.p, k);
      dn_.syevd(k, Hs.p, k, mu.p, true);
      dn_.mul_small(n, k, k, Xc_.p, npre, Hs.p, k, X_.p, k, 1.0, 0.0);  // Y into X's storage
      RitzSet rr = rayleigh(op_, st_, n, k, X_.p, k, AX_.p, lam_d_, res_d_, scratch_);
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
      if (colmap.empty()) return empty();
      Xfin = X_.p;
      ldfin = k;
      Xc_.release();  // the refined vectors live in X_ now
    }
    AX_.release();
    clk.close();
    if (o.precision == SMA_PREC_MIXED) {
      // FP64 polish of the FP32-filtered basis (polish.cu): filtered subspace iterations
      // with the same polynomial on the in-window candidates plus the guard vectors, each
      // pass applying p as p(theta) x + q_theta(A_hat) r / d with the divided difference q
      // in FP32, then FP64 orthonormalization and Rayleigh-Ritz with A; until the best
      // min(nev, in-window) residuals are below tol, at most max_passes passes.
      const int64_t kin = (int64_t)colmap.size();
      const int64_t k = kin + ng;
      Xpol_.alloc(n * k, st_);
      {
        DevBuf<double> Yp(n * kin, st_);
        DevBuf<int64_t> d = upload_idx(st_, colmap);
        launch_gather_columns_rm(st_, n, kin, Xfin, ldfin, d.p, Yp.p, kin);
        launch_copy_block<double, double>(st_, n, kin, Yp.p, kin, Xpol_.p, k);
        if (ng > 0) launch_copy_block<double, double>(st_, n, ng, guard.p, ng, Xpol_.p + kin, k);
      }
      guard.release();
      X_.release();  // the candidates live in Xpol_ now (X_ held the refined vectors)
      Xc_.release();
      auto done = [&](const std::vector<double> &lam, const std::vector<double> &res) {
        std::vector<double> r;
        for (size_t i = 0; i < lam.size(); ++i)
          if (o.emin <= lam[i] && lam[i] <= o.emax) r.push_back(res[i]);
        if (r.empty()) return false;
        std::sort(r.begin(), r.end());
        return r[std::min<size_t>(nev, r.size()) - 1] < o.tol;
      };
      // the polish polynomial of degree K: the basis filter's window, or an undamped step
      // over the window widened to the guards' span (sharper edges: the guards take the
      // transition); it starts at the basis degree (times SMA_POLISH_DEGREE) and may double
      // twice when a pass stalls
      auto coeffs_of = [&](int64_t K) {
        if (pc.step_filter)
          return build_coeffs(K, o.smin, o.smax, 0.5 * (guard_lo + guard_hi), guard_lo, guard_hi,
                              SMA_WINDOW_STEP, false);
        return build_coeffs(K, o.smin, o.smax, o.sigma, o.emin, o.emax, o.window_type,
                            o.jackson != 0);
      };
      const int64_t Kp = std::max<int64_t>(
          1, (int64_t)std::llround(pc.degree_scale * (double)(coeffs.size() - 1)));
      // after the first pass only unconverged in-window pairs are filtered again: what is
      // left of their error lies beyond the guards' span, where re-filtering the guards
      // does not reach; the guards keep their first-pass vectors in the Rayleigh-Ritz
      auto needs = [&](double lam, double res) {
        return o.emin <= lam && lam <= o.emax && res >= 0.5 * o.tol;
      };
      PolishTrace trace;
      if (pc.verbose)
        trace = [&](int64_t pass, const std::vector<double> &lam, const std::vector<double> &res) {
          int64_t in = 0, ok = 0;
          double mx = 0.0;
          for (size_t i = 0; i < lam.size(); ++i)
            if (o.emin <= lam[i] && lam[i] <= o.emax) {
              ++in;
              ok += res[i] < o.tol;
              mx = std::max(mx, res[i]);
            }
          fprintf(stderr, "polish pass %lld: k=%lld in-window=%lld converged=%lld max-res=%.3e\n",
                  (long long)pass, (long long)k, (long long)in, (long long)ok, mx);
        };
      clk.mark(PH_POLISH);
      // each column's Rayleigh quotient and residual on entry: the candidates' from the
      // refinement (or extraction), the guards' from the extraction
      std::vector<double> lam0 = lamc, res0 = resc;
      lam0.insert(lam0.end(), guard_lam.begin(), guard_lam.end());
      res0.insert(res0.end(), guard_res.begin(), guard_res.end());
      const PolishOut po = polish_mixed(op_, coeffs_of, Kp, 4 * Kp, o.smin, o.smax, Xpol_.p, k,
                                        done, needs, pc.max_passes, polish, &stats.qr_fallbacks,
                                        lam0, res0, o.emin, o.emax, pc.filter_guards,
                                        pc.verbose, trace);
      clk.close();
      stats.polish_iterations += po.passes;
      // keep the in-window pairs, as the refinement does
      std::vector<int64_t> in;
      for (int64_t i = 0; i < k; ++i)
        if (o.emin <= po.lam[i] && po.lam[i] <= o.emax) in.push_back(i);
      lamc = take(po.lam, in);
      resc = take(po.res, in);
      colmap = in;
      Xfin = Xpol_.p;
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
    if (o.show_progress && !rf.empty()) {  // _progress_line, polfed.jl:991-1000
      std::vector<double> srt = rf;
      std::sort(srt.begin(), srt.end());
      const int64_t L = (int64_t)srt.size();
      auto q = [&](double f) {
        int64_t i = (int64_t)std::nearbyint(f * (double)L);
        i = std::min(std::max<int64_t>(i, 1), L);
        return srt[i - 1];
      };
      printf("m=%lld  inside=%lld  r90=%.16g  r95=%.16g  maxres=%.16g\n", (long long)nb_,
             (long long)lamf.size(), q(0.9), q(0.95), srt[L - 1]);
      fflush(stdout);
    }
    // return rule, polfed.jl:1148-1157
    std::vector<int64_t> sel;
    const int64_t L = (int64_t)rf.size();
    if (L >= nev) {
      std::vector<double> srt = rf;
      std::sort(srt.begin(), srt.end());
      out.by_lambda = srt[nev - 1] < o.tol;
    }
    if (out.by_lambda) {
      for (int64_t t = 0; t < nev; ++t) sel.push_back(t);
    } else {
      sel = stable_argsort(rf);
      sel.resize(std::min<int64_t>(nev, L));
    }
    out.cols = take(cf, sel);
    out.lam = take(lamf, sel);
    out.res = take(rf, sel);
    out.X = Xfin;
    out.ldx = ldfin;
    return out;
  }

 private:
  sma_op *op_;
  sma_ctx *ctx_;
  cudaStream_t st_;
  int64_t n_;
  sma_polfed_opts o_;
  int64_t nev_, s_, mmax_ = 0;
  Dense dn_;
  DevBuf<double> V_, W_, C_, G_, Aj_, Bcur_, Bprev_, T_;
  DevBuf<double> X_, AX_, Xc_, Xpol_, lam_d_, res_d_, scratch_;
  std::vector<int64_t> offs_, ranks_;
  int64_t nb_ = 0, rprev_ = 0;
  bool finished_ = false;
};

// spmm_steps counts the basis filter's and the polish's products; filter_* and polish_*
// keep the two apart (the basis filter runs one block shape, the polish ragged widths).
void fill_stats(sma_stats &stats, PhaseClock &clk, const FilterCount &fc,
                const FilterCount &polish, int64_t columns,
                std::chrono::steady_clock::time_point t0, int64_t launches0) {
  double ph[PH_COUNT] = {0, 0, 0, 0};
  clk.totals(ph);
  stats.spmm_steps = fc.steps + polish.steps;
  stats.spmm_columns = columns;
  stats.filter_bytes = fc.bytes;
  stats.filter_ms = ph[PH_FILTER];
  stats.orth_ms = ph[PH_ORTH];
  stats.rr_ms = ph[PH_RR];
  stats.polish_ms = ph[PH_POLISH];
  stats.polish_bytes = polish.bytes;
  stats.total_ms = ms_since(t0);
  stats.kernel_launches = g_kernel_launches.load() - launches0;
}

}  // namespace

// polfed(A::MatrixFreeRealSymOp, nev, degree; ...), polfed.jl:1128-1158.
sma_result *polfed_solve(sma_op *op, int64_t nev, int64_t degree, const sma_polfed_opts &o) {
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t launches0 = g_kernel_launches.load();
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  sma_stats stats{};
  validate_polfed(op, nev, degree, o);
  if (o.precision != SMA_PREC_FP64) {
    require(op->kind != OP_MATBLOCK, SMA_ERR_ARG, "FP32 filtering needs a device operator");
    ensure_fp32_values(op);
  }
  PhaseClock clk(st);
  PolfedWindow win(op, nev, degree, o);
  Filter flt{op, st, win.coeffs, o.smin, o.smax, o.precision};
  win.start(stats);
  while (!win.finished()) {
    const int64_t r = win.next_rank();
    clk.mark(PH_FILTER);
    flt.run(win.next_block(), win.Mcap, win.filter_out(), r, r);  // W = p(A_hat) Q_j
    clk.mark(PH_ORTH);
    win.absorb(clk, stats);
  }
  stats.iterations = win.blocks();
  stats.basis_dim = win.basis_dim();
  FilterCount polish;
  const WindowPairs wp = win.extract(clk, stats, polish);
  sma_result *r = wp.cols.empty() ? empty_result(ctx, op->n)
                                  : make_result(ctx, op->n, wp.X, wp.ldx, wp.cols, wp.lam, wp.res);
  const int64_t K = (int64_t)win.coeffs.size() - 1;
  fill_stats(stats, clk, flt.total, polish, flt.columns * std::max<int64_t>(K, 1), t0,
             launches0);
  stats.fp32_filter_calls = flt.fp32_calls + stats.polish_iterations;
  stats.graph_replays = flt.w64.replays + flt.w32.replays;
  r->stats = stats;
  return r;
}

namespace {

// One batched filter of every active window's current block, in element type T: blocks in
// (FP64, the windows' bases) -> batch.q, the segmented recurrence, batch.y -> each
// window's filter_out() (FP64).  A window whose block has rank r < s pads its columns with
// zeros (they filter to zeros and are not read back).
template <typename T>
void batch_filter(const sma_op *op, cudaStream_t st, std::vector<std::unique_ptr<PolfedWindow>> &wins,
                  const std::vector<int64_t> &ids, int64_t s, const std::vector<int64_t> &degree,
                  double smin, double smax, bool use_graph, std::unique_ptr<SliceBatch<T>> &batch,
                  std::vector<int64_t> &key, FilterCount &total, int64_t &columns,
                  int64_t &replays) {
  const int64_t n = op->n;
  if (!batch || key != ids) {
    batch.reset(new SliceBatch<T>());
    std::vector<int64_t> m0(wins.size(), s);
    std::vector<std::vector<double>> coeffs(wins.size());
    for (size_t w = 0; w < wins.size(); ++w) coeffs[w] = wins[w]->coeffs;
    batch->setup(op, st, ids, m0, degree, coeffs, smin, smax);
    key = ids;
  }
  SliceBatch<T> &b = *batch;
  for (size_t sg = 0; sg < b.wins.size(); ++sg) {
    PolfedWindow &w = *wins[b.wins[sg]];
    const int64_t r = w.next_rank();
    launch_copy_block<double, T>(st, n, r, w.next_block(), w.Mcap, b.q.p + b.off[sg], b.W);
    if (r < s)
      SMA_CUDA(cudaMemset2DAsync(b.q.p + b.off[sg] + r, b.W * sizeof(T), 0, (s - r) * sizeof(T), n, st));
    columns += r * (int64_t)(w.coeffs.size() > 1 ? w.coeffs.size() - 1 : 1);
  }
  replays += b.run(use_graph);
  check_bulk_error(op, st);
  const FilterCount fc = b.count();
  total.steps += fc.steps;
  total.bytes += fc.bytes;
  for (size_t sg = 0; sg < b.wins.size(); ++sg) {
    PolfedWindow &w = *wins[b.wins[sg]];
    const int64_t r = w.next_rank();
    launch_copy_block<T, double>(st, n, r, b.y.p + b.off[sg], b.W, w.filter_out(), r);
  }
}

}  // namespace

// Batched POLFED (no counterpart in the reference, which solves one window per call).
sma_result *polfed_batch_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                               const int64_t *nev, const int64_t *degree, const int64_t *mmax,
                               const sma_polfed_opts &o) {
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t launches0 = g_kernel_launches.load();
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  const int64_t n = op->n;
  sma_stats stats{};
  require(nwin >= 1, SMA_ERR_ARG, "need at least one window");
  require(emin && emax && nev && degree && mmax, SMA_ERR_ARG, "null window array");
  require(op->kind == OP_CSR, SMA_ERR_ARG, "batched POLFED needs an explicit sparse matrix");
  require(o.has_bounds != 0, SMA_ERR_BOUNDS, "Matrix-free POLFED requires spectral bounds smin and smax");
  if (o.precision != SMA_PREC_FP64) ensure_fp32_values(op);
  std::vector<std::unique_ptr<PolfedWindow>> wins;
  std::vector<int64_t> deg(nwin);
  for (int64_t w = 0; w < nwin; ++w) {
    require(emin[w] < emax[w] && std::isfinite(emin[w]) && std::isfinite(emax[w]), SMA_ERR_ARG,
            "window " + std::to_string(w) + ": need finite emin < emax");
    require(degree[w] >= 1, SMA_ERR_ARG, "window degrees must be >= 1");
    sma_polfed_opts ow = o;
    ow.emin = emin[w];
    ow.emax = emax[w];
    ow.sigma = 0.5 * (emin[w] + emax[w]);
    ow.mmax = mmax[w];
    ow.seed = o.seed + w;
    validate_polfed(op, nev[w], degree[w], ow);
    deg[w] = degree[w];
    wins.emplace_back(new PolfedWindow(op, nev[w], degree[w], ow));
  }
  PhaseClock clk(st);
  for (auto &w : wins) w->start(stats);
  const bool fp32 = o.precision != SMA_PREC_FP64;
  std::unique_ptr<SliceBatch<double>> b64;
  std::unique_ptr<SliceBatch<float>> b32;
  std::vector<int64_t> key;
  FilterCount total;
  int64_t columns = 0, replays = 0, calls = 0;
  for (;;) {
    std::vector<int64_t> ids;
    for (int64_t w = 0; w < nwin; ++w)
      if (!wins[w]->finished()) ids.push_back(w);
    if (ids.empty()) break;
    clk.mark(PH_FILTER);
    if (fp32)
      batch_filter<float>(op, st, wins, ids, o.s, deg, o.smin, o.smax, true, b32, key, total,
                          columns, replays);
    else
      batch_filter<double>(op, st, wins, ids, o.s, deg, o.smin, o.smax, true, b64, key, total,
                           columns, replays);
    ++calls;
    for (int64_t w : ids) {
      clk.mark(PH_ORTH);
      wins[w]->absorb(clk, stats);
    }
  }
  // extraction per window; the result holds window 0's pairs, then window 1's, ...
  std::vector<WindowPairs> pairs;
  FilterCount polish;
  int64_t k = 0, blocks_max = 0, mdim = 0;
  for (auto &w : wins) {
    blocks_max = std::max(blocks_max, w->blocks());
    mdim += w->basis_dim();
    pairs.push_back(w->extract(clk, stats, polish));
    k += (int64_t)pairs.back().cols.size();
  }
  sma_result *r;
  if (k == 0) {
    r = empty_result(ctx, n);
  } else {
    r = new sma_result();
    r->ctx = ctx;
    r->n = n;
    r->k = k;
    r->ldx = k;
    SMA_CUDA(cudaMalloc((void **)&r->X_dev, n * k * sizeof(double)));
    int64_t j0 = 0;
    for (int64_t w = 0; w < nwin; ++w) {
      const WindowPairs &p = pairs[w];
      if (p.cols.empty()) continue;
      DevBuf<int64_t> d = upload_idx(st, p.cols);
      launch_gather_columns_rm(st, n, (int64_t)p.cols.size(), p.X, p.ldx, d.p, r->X_dev + j0, k);
      for (size_t t = 0; t < p.cols.size(); ++t) {
        r->lam.push_back(p.lam[t]);
        r->res.push_back(p.res[t]);
        r->win.push_back(w);
      }
      j0 += (int64_t)p.cols.size();
    }
    SMA_CUDA(cudaStreamSynchronize(st));
  }
  for (int64_t w = 0; w < nwin; ++w) {
    r->win_iters.push_back(wins[w]->blocks());
    r->win_done.push_back(pairs[w].by_lambda ? 1 : 0);
  }
  stats.iterations = blocks_max;
  stats.basis_dim = mdim;
  fill_stats(stats, clk, total, polish, columns, t0, launches0);
  stats.fp32_filter_calls = (fp32 ? calls : 0) + stats.polish_iterations;
  stats.graph_replays = replays;
  r->stats = stats;
  return r;
}

}  // namespace sma
