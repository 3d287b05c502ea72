// Helpers shared by the solver drivers (solvers.cu, slicing.cu).
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>

#include "sma_internal.h"

namespace sma {
namespace detail {

enum Phase { PH_FILTER = 0, PH_ORTH = 1, PH_RR = 2, PH_POLISH = 3, PH_COUNT = 4 };

// Device time per phase from pairs of CUDA events on the solve's stream.
struct PhaseClock {
  cudaStream_t st;
  std::vector<cudaEvent_t> evs;
  std::vector<int> phase;
  explicit PhaseClock(cudaStream_t s) : st(s) {}
  ~PhaseClock() {
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
  }
  void mark(int ph) {
    cudaEvent_t e;
    SMA_CUDA(cudaEventCreate(&e));
    SMA_CUDA(cudaEventRecord(e, st));
    evs.push_back(e);
    phase.push_back(ph);
  }
  // mark(ph) opens a phase, close() ends it
  void close() { mark(-1); }
  void totals(double *ms) {
    SMA_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i + 1 < evs.size(); ++i) {
      if (phase[i] < 0) continue;
      float t = 0.f;
      SMA_CUDA(cudaEventElapsedTime(&t, evs[i], evs[i + 1]));
      ms[phase[i]] += t;
    }
  }
};

inline std::vector<int64_t> stable_argsort(const std::vector<double> &v) {
  std::vector<int64_t> p(v.size());
  std::iota(p.begin(), p.end(), 0);
  std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return v[a] < v[b]; });
  return p;
}

inline std::vector<double> dev_to_host(cudaStream_t st, const double *d, size_t count) {
  std::vector<double> h(count);
  if (count) {
    SMA_CUDA(cudaMemcpyAsync(h.data(), d, count * sizeof(double), cudaMemcpyDeviceToHost, st));
    SMA_CUDA(cudaStreamSynchronize(st));
  }
  return h;
}

inline DevBuf<int64_t> upload_idx(cudaStream_t st, const std::vector<int64_t> &idx) {
  DevBuf<int64_t> d(idx.size(), st);
  if (!idx.empty())
    SMA_CUDA(cudaMemcpyAsync(d.p, idx.data(), idx.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  return d;
}

template <typename T>
std::vector<T> take(const std::vector<T> &v, const std::vector<int64_t> &idx) {
  std::vector<T> out(idx.size());
  for (size_t i = 0; i < idx.size(); ++i) out[i] = v[idx[i]];
  return out;
}

// The filter in the requested precision on an FP64 input block, FP64 output.
struct Filter {
  const sma_op *op;
  cudaStream_t st;
  std::vector<double> coeffs;
  double smin, smax;
  int64_t precision;
  ClenshawWork<double> w64;
  ClenshawWork<float> w32;
  DevBuf<float> q32, y32;
  FilterCount total;
  int64_t columns = 0;     // sum of the block widths filtered
  bool fp64_phase = false;  // MIXED: set once the FP32 phase has ended

  bool in_fp32() const {
    return precision == SMA_PREC_FP32 || (precision == SMA_PREC_MIXED && !fp64_phase);
  }

  int64_t fp32_calls = 0;

  void run(const double *Q, int64_t ldq, double *Y, int64_t ldy, int64_t b) {
    FilterCount fc;
    columns += b;
    if (in_fp32()) {
      ++fp32_calls;
      const int64_t n = op->n;
      if (q32.count < (size_t)(n * b)) {
        q32.alloc(n * b, st);
        y32.alloc(n * b, st);
      }
      launch_copy_block<double, float>(st, n, b, Q, ldq, q32.p, b);
      fc = apply_poly_block<float>(op, st, coeffs, smin, smax, q32.p, b, y32.p, b, b, w32);
      launch_copy_block<float, double>(st, n, b, y32.p, b, Y, ldy);
    } else {
      fc = apply_poly_block<double>(op, st, coeffs, smin, smax, Q, ldq, Y, ldy, b, w64);
    }
    total.steps += fc.steps;
    total.bytes += fc.bytes;
  }
};

inline void ensure_fp32_values(sma_op *op) {
  if ((op->kind != OP_CSR && op->kind != OP_CSR_HALF) || op->val32) return;
  cudaStream_t st = op->ctx->stream;
  SMA_CUDA(cudaMalloc((void **)&op->val32, std::max<int64_t>(op->nnz, 1) * sizeof(float)));
  launch_copy_block<double, float>(st, op->nnz, 1, op->val64, 1, op->val32, 1);
  SMA_CUDA(cudaStreamSynchronize(st));
}

inline void ensure_symmetry_known(sma_op *op) {
  if (op->kind != OP_CSR || op->sym_state != 0) return;
  op->sym_state = check_csr_device(op) == 0 ? 1 : 2;
}

inline double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Result holding the selected columns idx of the row-major block X (ld ldx).
inline sma_result *make_result(sma_ctx *ctx, int64_t n, const double *X, int64_t ldx,
                        const std::vector<int64_t> &idx, std::vector<double> lam,
                        std::vector<double> res) {
  auto *r = new sma_result();
  r->ctx = ctx;
  r->n = n;
  r->k = (int64_t)idx.size();
  r->lam = std::move(lam);
  r->res = std::move(res);
  r->ldx = std::max<int64_t>(r->k, 1);
  if (r->k > 0 && n > 0) {
    cudaStream_t st = ctx->stream;
    SMA_CUDA(cudaMalloc((void **)&r->X_dev, n * r->ldx * sizeof(double)));
    DevBuf<int64_t> d = upload_idx(st, idx);
    launch_gather_columns_rm(st, n, r->k, X, ldx, d.p, r->X_dev, r->ldx);
    SMA_CUDA(cudaStreamSynchronize(st));
  }
  return r;
}

inline sma_result *empty_result(sma_ctx *ctx, int64_t n) {
  auto *r = new sma_result();
  r->ctx = ctx;
  r->n = n;
  r->k = 0;
  r->ldx = 1;
  return r;
}

// MIXED precision, Chebyshev iteration: the FP32 phase ends when the in-window residuals
// reach what FP32 filtering can deliver (1e-6 of the spectral scale), when they stop
// improving (less than a factor 2 over the previous iteration), or when only two
// iterations remain; later iterations filter in FP64.  The measure is the 90% quantile of
// the residuals of ALL in-window Ritz pairs (no residual gate: FP32 residuals can sit
// above the gate, and a few spurious in-window Ritz values must not decide).
struct MixedSwitch {
  double prev = INFINITY;
  // returns true when the filter should move to FP64
  bool update(const std::vector<double> &lam, const std::vector<double> &res, double emin,
              double emax, double scale, bool last_two) {
    std::vector<double> r;
    for (size_t j = 0; j < lam.size(); ++j)
      if (lam[j] >= emin && lam[j] <= emax) r.push_back(res[j]);
    double q = INFINITY;
    if (!r.empty()) {
      std::sort(r.begin(), r.end());
      q = r[std::min(r.size() - 1, (size_t)std::ceil(0.9 * (double)r.size()) - 1)];
    }
    const bool small = q < 1e-6 * scale;
    const bool stalled = std::isfinite(q) && std::isfinite(prev) && q > 0.5 * prev;
    prev = q;
    return small || stalled || last_two;
  }
};

}  // namespace detail
}  // namespace sma
