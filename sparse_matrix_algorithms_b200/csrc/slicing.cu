// Batched spectrum slicing: many windows [emin_w, emax_w] over one sparse matrix, solved
// together by Chebyshev subspace iteration with one batched filter per iteration (the
// segmented, graph-captured recurrence of slice_batch.h).
//
// Per window, everything outside the filter is the Chebyshev iteration of solvers.cu
// (matrix-free overload's termination, chebyshev_subspace_iteration.jl:771-848) on that
// window's own n x m0_w blocks.
#include <memory>

#include "slice_batch.h"

namespace sma {

using namespace detail;

namespace {

struct Window {
  int64_t id = 0, m0 = 0, degree = 0;
  double emin = 0, emax = 0;
  std::vector<double> coeffs;
  DevBuf<double> Q, Y, X, Aq, lam_d, res_d, scratch;
  std::vector<double> lam, res;
  bool prev_ok = false, done = false, fp64_phase = false;
  MixedSwitch mixed;
  int64_t iterations = 0;
};

template <typename T>
struct BatchSlot {
  std::vector<int64_t> key;  // window ids of the cached batch
  std::unique_ptr<SliceBatch<T>> batch;
};

// Filters the blocks Q of the windows `ids` into their Y (FP64 in and out), in element
// type T, through the cached batch when the window set is unchanged.
template <typename T>
void batched_filter(const sma_op *op, cudaStream_t st, std::vector<Window> &win,
                    const std::vector<int64_t> &ids, double smin, double smax, bool use_graph,
                    BatchSlot<T> &slot, FilterCount &total, sma_stats &stats) {
  if (ids.empty()) return;
  if (!slot.batch || slot.key != ids) {
    slot.batch.reset(new SliceBatch<T>());
    std::vector<int64_t> m0(win.size()), degree(win.size());
    std::vector<std::vector<double>> coeffs(win.size());
    for (size_t w = 0; w < win.size(); ++w) {
      m0[w] = win[w].m0;
      degree[w] = win[w].degree;
      coeffs[w] = win[w].coeffs;
    }
    slot.batch->setup(op, st, ids, m0, degree, coeffs, smin, smax);
    slot.key = ids;
  }
  SliceBatch<T> &b = *slot.batch;
  const int64_t n = op->n;
  for (size_t s = 0; s < b.wins.size(); ++s) {
    Window &w = win[b.wins[s]];
    launch_copy_block<double, T>(st, n, w.m0, w.Q.p, w.m0, b.q.p + b.off[s], b.W);
  }
  stats.graph_replays += b.run(use_graph);
  for (size_t s = 0; s < b.wins.size(); ++s) {
    Window &w = win[b.wins[s]];
    launch_copy_block<T, double>(st, n, w.m0, b.y.p + b.off[s], b.W, w.Y.p, w.m0);
  }
  const FilterCount fc = b.count();
  total.steps += fc.steps;
  total.bytes += fc.bytes;
  for (int64_t k = b.Kmax; k >= 0; --k) stats.spmm_columns += b.active[k];
}

}  // namespace

sma_result *slice_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                        const int64_t *degree, const int64_t *m0, const sma_slice_opts &o) {
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t launches0 = g_kernel_launches.load();
  sma_ctx *ctx = op->ctx;
  cudaStream_t st = ctx->stream;
  const int64_t n = op->n;
  require(op->kind == OP_CSR, SMA_ERR_ARG, "batched spectrum slicing needs an explicit sparse matrix");
  require(nwin >= 1, SMA_ERR_ARG, "need at least one window");
  require(emin && emax && degree && m0, SMA_ERR_ARG, "null window array");
  require(o.window_type >= 0 && o.window_type <= 2, SMA_ERR_WINDOW,
          "Unknown window type, possible are :step, :delta, and :smooth");
  require(o.precision == SMA_PREC_FP64 || o.precision == SMA_PREC_FP32 ||
              o.precision == SMA_PREC_MIXED, SMA_ERR_ARG, "unknown precision");
  ensure_symmetry_known(op);
  require(op->sym_state == 1, SMA_ERR_NONSYMMETRIC,
          "Chebyshev filtered solver requires a real symmetric matrix");
  double smin, smax;
  if (o.has_bounds) {
    smin = o.smin;
    smax = o.smax;
  } else {
    require(op->has_gersh, SMA_ERR_ARG, "no spectral bounds");
    smin = op->gersh_min;
    smax = op->gersh_max;
  }
  const double c = 0.5 * (smin + smax), d = 0.5 * (smax - smin);
  std::vector<Window> win(nwin);
  sma_stats stats{};
  for (int64_t w = 0; w < nwin; ++w) {
    require(emin[w] < emax[w], SMA_ERR_ARG, "need emin<emax");
    require(m0[w] > 0, SMA_ERR_ARG, "m0 must be positive");
    require(degree[w] >= 0, SMA_ERR_ARG, "degree must be nonnegative");
    const double a = (emin[w] - c) / d, b = (emax[w] - c) / d;
    if (!(-1.0 <= a && a < b && b <= 1.0)) {
      char buf[256];
      snprintf(buf, sizeof buf, "window %lld: mapped interval [%.17g,%.17g] not inside [-1,1]",
               (long long)w, a, b);
      throw Error(SMA_ERR_INTERVAL, buf);
    }
    Window &x = win[w];
    x.id = w;
    x.m0 = std::min<int64_t>((m0[w] + 7) / 8 * 8, n / 8 * 8);
    require(x.m0 > 0, SMA_ERR_ARG, "the matrix is too small for batched slicing (n < 8)");
    x.degree = degree[w];
    x.emin = emin[w];
    x.emax = emax[w];
    x.coeffs = build_coeffs(x.degree, smin, smax, 0.5 * (x.emin + x.emax), x.emin, x.emax,
                            o.window_type, o.jackson != 0);
    x.fp64_phase = o.precision == SMA_PREC_FP64;
    x.Q.alloc(n * x.m0, st);
    x.Y.alloc(n * x.m0, st);
    x.X.alloc(n * x.m0, st);
    x.Aq.alloc(x.m0 * x.m0, st);
    x.lam_d.alloc(x.m0, st);
    x.res_d.alloc(x.m0, st);
    launch_randn(st, n, x.m0, (uint64_t)(o.seed + w), x.Q.p, x.m0);
  }
  if (o.precision != SMA_PREC_FP64) ensure_fp32_values(op);
  Dense dn(ctx);
  PhaseClock clk(st);
  BatchSlot<double> slot64;
  BatchSlot<float> slot32;
  FilterCount total;
  const double scale = std::max(std::fabs(smin), std::fabs(smax));
  int64_t it = 0;
  for (it = 1; it <= o.maxiter; ++it) {
    std::vector<int64_t> ids32, ids64;
    for (Window &x : win)
      if (!x.done) (x.fp64_phase ? ids64 : ids32).push_back(x.id);
    if (ids32.empty() && ids64.empty()) break;
    clk.mark(PH_FILTER);
    batched_filter<float>(op, st, win, ids32, smin, smax, o.graph != 0, slot32, total, stats);
    batched_filter<double>(op, st, win, ids64, smin, smax, o.graph != 0, slot64, total, stats);
    if (!ids32.empty()) stats.fp32_filter_calls += 1;
    clk.close();
    std::vector<int64_t> ids = ids32;
    ids.insert(ids.end(), ids64.begin(), ids64.end());
    std::sort(ids.begin(), ids.end());
    for (int64_t id : ids) {
      Window &x = win[id];
      const int64_t m = x.m0;
      const bool fp32_iteration = !x.fp64_phase;
      clk.mark(PH_ORTH);
      std::swap(x.Q.p, x.Y.p);
      orthonormalize(ctx, n, m, x.Q.p, m, false, 0.0, nullptr, &stats.qr_fallbacks);
      clk.mark(PH_RR);
      op_apply(op, st, x.Q.p, m, x.Y.p, m, m);
      dn.gram(n, m, m, x.Q.p, m, x.Y.p, m, x.Aq.p, m);
      dn.syevd(m, x.Aq.p, m, x.lam_d.p, true);
      dn.mul_small(n, m, m, x.Q.p, m, x.Aq.p, m, x.X.p, m, 1.0, 0.0);
      op_apply(op, st, x.X.p, m, x.Y.p, m, m);
      column_reduce(st, 1, n, m, x.X.p, m, x.Y.p, m, x.lam_d.p, x.res_d.p, x.scratch);
      clk.close();
      x.lam = dev_to_host(st, x.lam_d.p, m);
      x.res = dev_to_host(st, x.res_d.p, m);
      x.iterations = it;
      int64_t cnt = 0;
      double maxres = -INFINITY;
      for (int64_t j = 0; j < m; ++j)
        if (x.lam[j] >= x.emin && x.lam[j] <= x.emax && x.res[j] < o.res_gate) {
          ++cnt;
          maxres = std::max(maxres, x.res[j]);
        }
      if (cnt == 0) maxres = INFINITY;
      if (o.debug) {
        printf("window=%lld it=%lld inside=%lld maxres=%.3e%s\n", (long long)id, (long long)it,
               (long long)cnt, maxres, fp32_iteration ? " fp32" : "");
        fflush(stdout);
      }
      if (o.precision == SMA_PREC_MIXED && fp32_iteration &&
          x.mixed.update(x.lam, x.res, x.emin, x.emax, scale, it >= o.maxiter - 2))
        x.fp64_phase = true;
      const bool ok = cnt > 0 && maxres < o.tol && !fp32_iteration;
      if (o.two_hit ? (ok && (it == 1 || x.prev_ok)) : ok) x.done = true;
      x.prev_ok = ok;
    }
  }
  double ph[PH_COUNT] = {0, 0, 0, 0};
  clk.totals(ph);
  // selection per window (chebyshev_subspace_iteration.jl:750-756), windows in order
  const double gate = std::max(o.res_gate, 10.0 * o.tol);
  std::vector<double> lam_all, res_all;
  std::vector<int64_t> win_all;
  std::vector<std::pair<int64_t, int64_t>> cols;  // (window, column)
  int64_t itmax = 0;
  for (Window &x : win) {
    itmax = std::max(itmax, x.iterations);
    std::vector<int64_t> idx;
    std::vector<double> l;
    for (int64_t j = 0; j < (int64_t)x.lam.size(); ++j)
      if (x.lam[j] >= x.emin && x.lam[j] <= x.emax && x.res[j] < gate) {
        idx.push_back(j);
        l.push_back(x.lam[j]);
      }
    const std::vector<int64_t> p = stable_argsort(l);
    for (int64_t t : p) {
      lam_all.push_back(x.lam[idx[t]]);
      res_all.push_back(x.res[idx[t]]);
      win_all.push_back(x.id);
      cols.push_back({x.id, idx[t]});
    }
  }
  sma_result *r;
  const int64_t k = (int64_t)lam_all.size();
  if (k == 0) {
    r = empty_result(ctx, n);
  } else {
    r = new sma_result();
    r->ctx = ctx;
    r->n = n;
    r->k = k;
    r->lam = lam_all;
    r->res = res_all;
    r->ldx = k;
    r->win = win_all;
    SMA_CUDA(cudaMalloc((void **)&r->X_dev, n * k * sizeof(double)));
    int64_t j0 = 0;
    while (j0 < k) {  // one gather per window
      const int64_t w = cols[j0].first;
      std::vector<int64_t> sel;
      int64_t j1 = j0;
      for (; j1 < k && cols[j1].first == w; ++j1) sel.push_back(cols[j1].second);
      DevBuf<int64_t> dsel = upload_idx(st, sel);
      launch_gather_columns_rm(st, n, (int64_t)sel.size(), win[w].X.p, win[w].m0, dsel.p,
                               r->X_dev + j0, k);
      SMA_CUDA(cudaStreamSynchronize(st));
      j0 = j1;
    }
  }
  int64_t wsum = 0;
  for (Window &x : win) {
    wsum += x.m0;
    r->win_iters.push_back(x.iterations);
    r->win_done.push_back(x.done ? 1 : 0);
  }
  stats.iterations = itmax;
  stats.basis_dim = wsum;
  stats.spmm_steps = total.steps;
  stats.filter_bytes = total.bytes;
  stats.filter_ms = ph[PH_FILTER];
  stats.orth_ms = ph[PH_ORTH];
  stats.rr_ms = ph[PH_RR];
  stats.total_ms = ms_since(t0);
  stats.kernel_launches = g_kernel_launches.load() - launches0;
  r->stats = stats;
  return r;
}

}  // namespace sma
