// Block Clenshaw filter Y = p(A_hat) Q (apply_poly_block!,
// chebyshev_subspace_iteration.jl:554-635, polfed.jl:464-545).
//
//   B_{K+1} = B_{K+2} = 0
//   B_k = c_k Q + 2 A_hat B_{k+1} - B_{k+2}       (k = K..1)
//   Y   = c_0 Q + A_hat B_1 - B_2,    A_hat = (A - cI)/d
//
// evaluated as the reference does: B_k = c_k Q + alpha*A B_{k+1} + beta*B_{k+1} - B_{k+2}
// with invd = 2/(smax-smin), alpha = 2*invd, beta = -2*c*invd
// (chebyshev_subspace_iteration.jl:562-565).
//
// The reference zero-fills B1 and B2 and runs K+1 sparse products.  The first step
// multiplies zeros, so here it is the scaling B1 = c_K Q (bit-identical: every
// dropped term is an exact zero), and the second step reads no B2.  Each remaining
// step is ONE fused kernel launch (kernels.cu) for device operators; caller-supplied
// operators get the product from their callback followed by the axpy kernel.
#include "sma_internal.h"

namespace sma {

template <typename T>
void ClenshawWork<T>::ensure(const sma_op *op, int64_t n_, int64_t b, cudaStream_t st) {
  if (n_ == n && b <= bcap && b1.p) return;
  drop_graph();  // the graph holds the old buffers' addresses
  n = n_;
  bcap = b;
  b1.alloc(n * b, st);
  b2.alloc(n * b, st);
  tmp.alloc(n * b, st);
  q.release();
  y.release();
  if (op->kind == OP_MATBLOCK || op->kind == OP_CSR_HALF) ax.alloc(n * b, st);
}

template <typename T>
void ClenshawWork<T>::drop_graph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
  g_op = nullptr;
  g_b = -1;
  g_calls = 0;
}

double clenshaw_step_bytes(const sma_op *op, int64_t b, int elem_bytes) {
  // nnz*(value + column index) + row pointers + Q, B1, B2 reads and one write
  double mat = 0.0;
  if (op->kind == OP_CSR || op->kind == OP_CSR_HALF)  // half storage: its stored entries
    mat = (double)op->nnz * (elem_bytes + 4) + 4.0 * (op->n + 1);
  return mat + 4.0 * (double)op->n * (double)b * elem_bytes;
}

void check_bulk_error(const sma_op *op, cudaStream_t st) {
  if (!op->bulk_err) return;
  int h = 0;
  SMA_CUDA(cudaMemcpyAsync(&h, op->bulk_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  if (h != 0) {
    SMA_CUDA(cudaMemsetAsync(op->bulk_err, 0, sizeof(int), st));
    SMA_CUDA(cudaStreamSynchronize(st));
    throw Error(SMA_ERR_TIMEOUT, h == 1 ? "a bulk-copy CSR step gave up waiting for its copies"
                                        : "a bulk-copy CSR step met a CTA larger than its shared memory");
  }
}

void op_apply(const sma_op *op, cudaStream_t st, const double *X, int64_t ldx, double *Y,
              int64_t ldy, int64_t b) {
  if (b == 0 || op->n == 0) return;
  if (op->kind == OP_MATBLOCK) {
    require(ldx == ldy, SMA_ERR_ARG, "matrix-free operator callbacks need equal leading dimensions");
    const int rc = op->fn(op->user, X, Y, op->n, b, ldx, (void *)st);
    if (rc != 0) throw Error(SMA_ERR_CALLBACK, "matblock callback returned " + std::to_string(rc));
    SMA_CUDA(cudaGetLastError());
    return;
  }
  if (op->kind == OP_CSR_HALF) return half_product<double>(op, st, X, ldx, Y, ldy, b);
  launch_clenshaw_step<double>(op, st, b, nullptr, 0, X, nullptr, ldx, Y, ldy, 0.0, 1.0, 0.0, false);
  check_bulk_error(op, st);
}

template <typename T>
static void matblock_apply(const sma_op *op, cudaStream_t st, const T *X, T *AX, int64_t ld,
                           int64_t b) {
  if (op->kind == OP_CSR_HALF) return half_product<T>(op, st, X, ld, AX, ld, b);
  if constexpr (sizeof(T) == 8) {
    const int rc = op->fn(op->user, (const double *)X, (double *)AX, op->n, b, ld, (void *)st);
    if (rc != 0) throw Error(SMA_ERR_CALLBACK, "matblock callback returned " + std::to_string(rc));
  } else {
    throw Error(SMA_ERR_ARG, "caller-supplied operators take FP64 blocks only");
  }
}

// One fused step for device operators: the autotuned CSR launch, or (tuned = false, for
// graph recording) the operator's cached configuration with no events.
template <typename T>
static void fused_step(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                       const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                       double alpha, double beta, bool tuned) {
  if (!tuned && op->kind == OP_CSR)
    csr_clenshaw_step_untuned<T>(op, st, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta, true);
  else
    launch_clenshaw_step<T>(op, st, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta, true);
}

// The launches of one filter (K >= 1); returns the step count and algorithmic bytes.
template <typename T>
static FilterCount record_filter(const sma_op *op, cudaStream_t st,
                                 const std::vector<double> &coeffs, double smin, double smax,
                                 const T *Q, int64_t ldq, T *Y, int64_t ldy, int64_t b,
                                 ClenshawWork<T> &work, bool tuned) {
  FilterCount fc;
  const int64_t n = op->n;
  const int64_t K = (int64_t)coeffs.size() - 1;
  const double c = 0.5 * (smin + smax);
  const double invd = 2.0 / (smax - smin);
  const double alpha = 2.0 * invd;
  const double beta = -2.0 * c * invd;
  const bool fused = op->kind != OP_MATBLOCK && op->kind != OP_CSR_HALF;
  const double blk = (double)n * (double)b * sizeof(T);
  T *B1 = work.b1.p, *B2 = work.b2.p, *TMP = work.tmp.p;
  const int64_t ld = b;
  // step K+1 of the reference: B1 = c_K Q (its product multiplies zeros)
  launch_scale_block<T>(st, n, b, Q, ldq, B1, ld, coeffs[K]);
  fc.bytes += 2 * blk;
  bool b2_zero = true;
  const double mat_bytes = clenshaw_step_bytes(op, 0, sizeof(T));
  for (int64_t ci = K - 1; ci >= 1; --ci) {
    if (fused) {
      fused_step<T>(op, st, b, Q, ldq, B1, b2_zero ? nullptr : B2, ld, TMP, ld, coeffs[ci], alpha,
                    beta, tuned);
    } else {
      matblock_apply<T>(op, st, B1, work.ax.p, ld, b);
      launch_clenshaw_axpy<T>(st, n, b, Q, ldq, work.ax.p, ld, B1, b2_zero ? nullptr : B2, ld,
                              TMP, ld, coeffs[ci], alpha, beta);
    }
    fc.steps += 1;
    fc.bytes += mat_bytes + (b2_zero ? 3 : 4) * blk;
    T *t = B2;  // B1, B2, TMP = TMP, B1, B2
    B2 = B1;
    B1 = TMP;
    TMP = t;
    b2_zero = false;
  }
  // final step: Y = c_0 Q + invd*A B1 - c*invd*B1 - B2
  if (fused) {
    fused_step<T>(op, st, b, Q, ldq, B1, b2_zero ? nullptr : B2, ld, Y, ldy, coeffs[0], invd,
                  -(c * invd), tuned);
  } else {
    matblock_apply<T>(op, st, B1, work.ax.p, ld, b);
    launch_clenshaw_axpy<T>(st, n, b, Q, ldq, work.ax.p, ld, B1, b2_zero ? nullptr : B2, ld, Y,
                            ldy, coeffs[0], invd, -(c * invd));
  }
  fc.steps += 1;
  fc.bytes += mat_bytes + (b2_zero ? 3 : 4) * blk;
  return fc;
}

// Filters of degree below this run eagerly (launch overhead is then not the question).
constexpr int64_t kGraphMinDegree = 32;

template <typename T>
static FilterCount apply_poly_block_impl(const sma_op *op, cudaStream_t st,
                                         const std::vector<double> &coeffs, double smin,
                                         double smax, const T *Q, int64_t ldq, T *Y, int64_t ldy,
                                         int64_t b, ClenshawWork<T> &work) {
  FilterCount fc;
  const int64_t n = op->n;
  const int64_t K = (int64_t)coeffs.size() - 1;
  require(K >= 0, SMA_ERR_ARG, "empty coefficient vector");
  if (n == 0 || b == 0) return fc;
  if (K == 0) {  // no loop: Y = c_0 Q
    launch_scale_block<T>(st, n, b, Q, ldq, Y, ldy, coeffs[0]);
    fc.bytes += 2.0 * (double)n * (double)b * sizeof(T);
    return fc;
  }
  work.ensure(op, n, b, st);
  if (op->kind == OP_CSR && op->ctx->persistent && K >= kGraphMinDegree) {
    if (work.coef.count < (size_t)(K + 1)) work.coef.alloc(K + 1, st);
    if (!work.barrier.p) work.barrier.alloc(3, st);
    return persistent_filter<T>(op, st, coeffs, smin, smax, Q, ldq, Y, ldy, b, work.b1.p,
                                work.b2.p, work.tmp.p, work.coef.p, work.barrier.p);
  }
  if (op->kind == OP_MATBLOCK || op->kind == OP_CSR_HALF || K < kGraphMinDegree ||
      !op->ctx->filter_graphs)
    return record_filter<T>(op, st, coeffs, smin, smax, Q, ldq, Y, ldy, b, work, true);
  // repeated filter -> CUDA graph on the staging blocks
  const bool same = work.g_op == op && work.g_b == b && work.g_smin == smin &&
                    work.g_smax == smax && work.g_coeffs == coeffs;
  if (!same) {
    work.drop_graph();
    work.g_op = op;
    work.g_b = b;
    work.g_smin = smin;
    work.g_smax = smax;
    work.g_coeffs = coeffs;
  }
  work.g_calls += 1;
  if (work.g_calls == 1)  // first call: eager, so the kernel autotuner sees real steps
    return record_filter<T>(op, st, coeffs, smin, smax, Q, ldq, Y, ldy, b, work, true);
  if (!work.q.p) {
    work.q.alloc(n * work.bcap, st);
    work.y.alloc(n * work.bcap, st);
  }
  launch_copy_block<T, T>(st, n, b, Q, ldq, work.q.p, b);
  if (!work.exec) {
    const int64_t l0 = g_kernel_launches.load();
    SMA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      fc = record_filter<T>(op, st, coeffs, smin, smax, work.q.p, b, work.y.p, b, b, work, false);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    SMA_CUDA(cudaStreamEndCapture(st, &work.graph));
    SMA_CUDA(cudaGraphInstantiate(&work.exec, work.graph, 0));
    work.g_launches = g_kernel_launches.load() - l0;
    g_kernel_launches.fetch_sub(work.g_launches);  // counted when the graph runs
  } else {
    // step and byte counts of the recorded filter
    const double blk = (double)n * (double)b * sizeof(T);
    const double mat_bytes = clenshaw_step_bytes(op, 0, sizeof(T));
    fc.steps = K;
    fc.bytes = 2 * blk + (mat_bytes + 3 * blk) + (double)(K - 1) * (mat_bytes + 4 * blk);
  }
  SMA_CUDA(cudaGraphLaunch(work.exec, st));
  g_kernel_launches.fetch_add(work.g_launches);
  work.replays += 1;
  launch_copy_block<T, T>(st, n, b, work.y.p, b, Y, ldy);
  return fc;
}

template <typename T>
FilterCount apply_poly_block(const sma_op *op, cudaStream_t st, const std::vector<double> &coeffs,
                             double smin, double smax, const T *Q, int64_t ldq, T *Y, int64_t ldy,
                             int64_t b, ClenshawWork<T> &work) {
  const FilterCount fc = apply_poly_block_impl<T>(op, st, coeffs, smin, smax, Q, ldq, Y, ldy, b, work);
  check_bulk_error(op, st);
  return fc;
}

template struct ClenshawWork<double>;
template struct ClenshawWork<float>;
template FilterCount apply_poly_block<double>(const sma_op *, cudaStream_t,
                                              const std::vector<double> &, double, double,
                                              const double *, int64_t, double *, int64_t, int64_t,
                                              ClenshawWork<double> &);
template FilterCount apply_poly_block<float>(const sma_op *, cudaStream_t,
                                             const std::vector<double> &, double, double,
                                             const float *, int64_t, float *, int64_t, int64_t,
                                             ClenshawWork<float> &);

}  // namespace sma
