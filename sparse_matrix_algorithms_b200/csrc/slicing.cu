// Batched spectrum slicing: many windows [emin_w, emax_w] over one sparse matrix, solved
// together by Chebyshev subspace iteration with one batched filter per iteration.
//
// The batched filter.  The windows' blocks are concatenated side by side into one
// row-major n x W block, windows sorted by filter degree (highest first).  The Clenshaw
// recurrence runs from the highest degree down; window w's columns join at index K_w, so
// at every index the active columns are a prefix of the block and one launch of the
// segmented CSR step (csr_clenshaw.cuh) updates all of them, each column with its own
// window's coefficient.  The three recurrence blocks start zeroed, which makes a joining
// window's first step exactly its B1 = c_K Q and its second step exactly the one without
// B2: every window's filtered block is bit-identical to the single-window filter of
// filter.cu, while the sparse matrix is read once per index for all windows.  After one
// eager call (during which the kernel autotuner measures the widths it meets) the whole
// recurrence is recorded into a CUDA graph and replayed for as long as the set of active
// windows does not change.
//
// Per window, everything outside the filter is the Chebyshev iteration of solvers.cu
// (matrix-free overload's termination, chebyshev_subspace_iteration.jl:771-848) on that
// window's own n x m0_w blocks.
#include <memory>

#include "solver_common.h"

namespace sma {

using namespace detail;

namespace {

template <typename T>
struct SliceBatch {
  const sma_op *op = nullptr;
  cudaStream_t st = nullptr;
  std::vector<int64_t> wins;             // window ids, in segment order
  std::vector<int64_t> off, width, deg;  // per segment
  int64_t n = 0, W = 0, Kmax = 0;
  double smin = 0, smax = 0;
  DevBuf<T> coef;       // (Kmax + 1) x nseg: coef[k * nseg + s] = c_k of segment s (0 above K_s)
  DevBuf<int> colseg8;  // W / 8
  DevBuf<T> q, y, b1, b2, tmp;
  std::vector<int64_t> active;  // active[k] = width of the columns taking part at index k
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t recorded_launches = 0;
  int64_t calls = 0;

  SliceBatch() = default;
  SliceBatch(const SliceBatch &) = delete;
  SliceBatch &operator=(const SliceBatch &) = delete;
  ~SliceBatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }

  void setup(const sma_op *op_, cudaStream_t st_, const std::vector<int64_t> &ids,
             const std::vector<int64_t> &m0, const std::vector<int64_t> &degree,
             const std::vector<std::vector<double>> &coeffs, double smin_, double smax_) {
    op = op_;
    st = st_;
    n = op->n;
    smin = smin_;
    smax = smax_;
    wins = ids;
    std::stable_sort(wins.begin(), wins.end(),
                     [&](int64_t a, int64_t b) { return degree[a] > degree[b]; });
    const int64_t nseg = (int64_t)wins.size();
    W = 0;
    for (int64_t w : wins) {
      off.push_back(W);
      width.push_back(m0[w]);
      deg.push_back(degree[w]);
      W += m0[w];
    }
    Kmax = deg.empty() ? 0 : deg[0];
    std::vector<T> ch((size_t)(Kmax + 1) * nseg, T(0));
    for (int64_t s = 0; s < nseg; ++s)
      for (int64_t k = 0; k <= deg[s]; ++k) ch[k * nseg + s] = (T)coeffs[wins[s]][k];
    std::vector<int> cs(W / 8);
    for (int64_t s = 0; s < nseg; ++s)
      for (int64_t c = off[s]; c < off[s] + width[s]; c += 8) cs[c / 8] = (int)s;
    active.assign(Kmax + 1, 0);
    for (int64_t k = 0; k <= Kmax; ++k)
      for (int64_t s = 0; s < nseg; ++s)
        if (deg[s] >= k) active[k] = off[s] + width[s];
    coef.alloc(ch.size(), st);
    colseg8.alloc(cs.size(), st);
    SMA_CUDA(cudaMemcpyAsync(coef.p, ch.data(), ch.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(colseg8.p, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    q.alloc(n * W, st);
    y.alloc(n * W, st);
    b1.alloc(n * W, st);
    b2.alloc(n * W, st);
    tmp.alloc(n * W, st);
    SMA_CUDA(cudaStreamSynchronize(st));  // the host tables above must outlive their copies
  }

  // The whole recurrence on q -> y.  tuned = false for graph recording.
  void record(bool tuned) {
    const int64_t nseg = (int64_t)wins.size();
    const double c = 0.5 * (smin + smax), invd = 2.0 / (smax - smin);
    const double alpha = 2.0 * invd, beta = -2.0 * c * invd;
    const size_t bytes = (size_t)(n * W) * sizeof(T);
    SMA_CUDA(cudaMemsetAsync(b1.p, 0, bytes, st));
    SMA_CUDA(cudaMemsetAsync(b2.p, 0, bytes, st));
    SMA_CUDA(cudaMemsetAsync(tmp.p, 0, bytes, st));
    T *B1 = b1.p, *B2 = b2.p, *TMP = tmp.p;
    for (int64_t k = Kmax; k >= 1; --k) {
      csr_clenshaw_step_seg<T>(op, st, active[k], q.p, W, B1, B2, W, TMP, W, coef.p + k * nseg,
                               colseg8.p, alpha, beta, tuned);
      T *t = B2;
      B2 = B1;
      B1 = TMP;
      TMP = t;
    }
    csr_clenshaw_step_seg<T>(op, st, W, q.p, W, B1, B2, W, y.p, W, coef.p, colseg8.p, invd,
                             -(c * invd), tuned);
  }

  // Algorithmic bytes of one batched filter: every step reads the matrix once and Q, B1,
  // B2 of its active columns, and writes them.
  FilterCount count() const {
    FilterCount fc;
    const double mat = clenshaw_step_bytes(op, 0, sizeof(T));
    for (int64_t k = Kmax; k >= 0; --k) {
      fc.steps += 1;
      fc.bytes += mat + 4.0 * (double)n * (double)active[k] * sizeof(T);
    }
    return fc;
  }

  // One batched filter; returns the graph launches it made (0 or 1).
  int64_t run(bool use_graph) {
    ++calls;
    if (use_graph && !exec && calls >= 2) {
      const int64_t l0 = g_kernel_launches.load();
      SMA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        record(false);
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      SMA_CUDA(cudaStreamEndCapture(st, &graph));
      SMA_CUDA(cudaGraphInstantiate(&exec, graph, 0));
      recorded_launches = g_kernel_launches.load() - l0;
      g_kernel_launches.fetch_sub(recorded_launches);  // counted when the graph runs
    }
    if (exec) {
      SMA_CUDA(cudaGraphLaunch(exec, st));
      g_kernel_launches.fetch_add(recorded_launches);
      return 1;
    }
    record(true);
    return 0;
  }
};

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
  double ph[PH_COUNT] = {0, 0, 0};
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
