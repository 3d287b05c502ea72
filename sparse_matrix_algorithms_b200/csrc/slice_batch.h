// The batched (segmented) block Clenshaw filter shared by batched spectrum slicing
// (slicing.cu) and batched POLFED (polfed_batch.cu).
//
// The windows' blocks are concatenated side by side into one row-major n x W block,
// windows sorted by filter degree (highest first).  The Clenshaw recurrence runs from the
// highest degree down; window w's columns join at index K_w, so at every index the active
// columns are a prefix of the block and one launch of the segmented CSR step
// (csr_clenshaw.cuh) updates all of them, each column with its own window's coefficient.
// The three recurrence blocks start zeroed, which makes a joining window's first step
// exactly its B1 = c_K Q and its second step exactly the one without B2: every window's
// filtered block is bit-identical to the single-window filter of filter.cu, while the
// sparse matrix is read once per index for all windows.  After one eager call (during
// which the kernel autotuner measures the widths it meets) the whole recurrence is
// recorded into a CUDA graph and replayed for as long as the set of windows is unchanged.
#pragma once

#include "solver_common.h"

namespace sma {
namespace detail {

template <typename T>
struct SliceBatch {
  const sma_op *op = nullptr;
  cudaStream_t st = nullptr;
  std::vector<int64_t> wins;             // window ids, in segment order
  std::vector<int64_t> off, width, deg;  // per segment
  int64_t n = 0, W = 0, Kmax = 0;
  double smin = 0, smax = 0;
  DevBuf<T> coef;       // (Kmax + 1) x nseg: coef[k * nseg + s] = c_k of segment s (0 above K_s)
  std::vector<double> coef1;  // one segment: its coefficients, for the unsegmented step
  DevBuf<int> colseg;  // W: the segment of every column
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
    std::vector<int> cs(W);
    for (int64_t s = 0; s < nseg; ++s)
      for (int64_t c = off[s]; c < off[s] + width[s]; ++c) cs[c] = (int)s;
    active.assign(Kmax + 1, 0);
    for (int64_t k = 0; k <= Kmax; ++k)
      for (int64_t s = 0; s < nseg; ++s)
        if (deg[s] >= k) active[k] = off[s] + width[s];
    coef1.clear();
    if (nseg == 1)
      for (int64_t k = 0; k <= Kmax; ++k) coef1.push_back((double)ch[k]);
    coef.alloc(ch.size(), st);
    colseg.alloc(cs.size(), st);
    SMA_CUDA(cudaMemcpyAsync(coef.p, ch.data(), ch.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    SMA_CUDA(cudaMemcpyAsync(colseg.p, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    q.alloc(n * W, st);
    y.alloc(n * W, st);
    b1.alloc(n * W, st);
    b2.alloc(n * W, st);
    tmp.alloc(n * W, st);
    SMA_CUDA(cudaStreamSynchronize(st));  // the host tables above must outlive their copies
  }

  // One step at index k over the first b columns.  One segment: the unsegmented step with
  // the scalar c_k (the same arithmetic on the same values -- (T) c_k either way -- without
  // the per-column coefficient lookups); several: the segmented step.
  void step(int64_t k, int64_t b, const T *B1, const T *B2, T *out, double al, double be,
            bool tuned) {
    const int64_t nseg = (int64_t)wins.size();
    if (nseg == 1) {
      if (tuned)
        csr_clenshaw_step<T>(op, st, b, q.p, W, B1, B2, W, out, W, coef1[k], al, be, true);
      else
        csr_clenshaw_step_untuned<T>(op, st, b, q.p, W, B1, B2, W, out, W, coef1[k], al, be, true);
      return;
    }
    csr_clenshaw_step_seg<T>(op, st, b, q.p, W, B1, B2, W, out, W, coef.p + k * nseg, colseg.p,
                             al, be, tuned);
  }

  // The whole recurrence on q -> y.  tuned = false for graph recording.
  void record(bool tuned) {
    const double c = 0.5 * (smin + smax), invd = 2.0 / (smax - smin);
    const double alpha = 2.0 * invd, beta = -2.0 * c * invd;
    const size_t bytes = (size_t)(n * W) * sizeof(T);
    SMA_CUDA(cudaMemsetAsync(b1.p, 0, bytes, st));
    SMA_CUDA(cudaMemsetAsync(b2.p, 0, bytes, st));
    SMA_CUDA(cudaMemsetAsync(tmp.p, 0, bytes, st));
    T *B1 = b1.p, *B2 = b2.p, *TMP = tmp.p;
    for (int64_t k = Kmax; k >= 1; --k) {
      step(k, active[k], B1, B2, TMP, alpha, beta, tuned);
      T *t = B2;
      B2 = B1;
      B1 = TMP;
      TMP = t;
    }
    step(0, W, B1, B2, y.p, invd, -(c * invd), tuned);
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

}  // namespace detail
}  // namespace sma
