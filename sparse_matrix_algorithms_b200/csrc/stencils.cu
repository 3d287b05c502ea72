// Matrix-free model operators: the 3D Anderson model and the XXZ chain (Sz = 0) as device
// stencils (sma_op_create_anderson, sma_op_create_xxz).  They replace a stored CSR matrix
// in every solver and filter entry point and read no index arrays: the neighbours of a row
// follow from the row index (Anderson) or from the row's basis state (XXZ).  This is the
// GPU form of the reference's matrix-free interface (MatrixFreeRealSymOp with a matblock!,
// polfed.jl:148-219) for the two benchmark models.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "sma_internal.h"

namespace sma {
namespace {

template <typename F>
int guarded(F &&f) {
  try {
    f();
    return SMA_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMA_ERR_INTERNAL;
  }
}

struct CurrentDevice {
  int prev = -1;
  explicit CurrentDevice(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) SMA_CUDA(cudaSetDevice(dev));
  }
  ~CurrentDevice() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

template <typename T>
T *upload(cudaStream_t st, const T *host, size_t count) {
  T *d = nullptr;
  SMA_CUDA(cudaMalloc((void **)&d, std::max<size_t>(count, 1) * sizeof(T)));
  if (count) SMA_CUDA(cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, st));
  return d;
}

void free_stencil(sma_op *op) {
  if (op->stencil.diag) cudaFree(op->stencil.diag);
  if (op->stencil.states) cudaFree(op->stencil.states);
  if (op->stencil.binom) cudaFree(op->stencil.binom);
  op->stencil = sma_stencil{};
}

}  // namespace
}  // namespace sma

using namespace sma;

extern "C" int sma_op_create_anderson(sma_ctx *ctx, int64_t L, const double *eps, double t,
                                      sma_op **out) {
  return guarded([&] {
    require(ctx != nullptr && out != nullptr, SMA_ERR_ARG, "null argument");
    *out = nullptr;
    require(L >= 3 && L <= 1290, SMA_ERR_ARG, "Anderson stencil needs 3 <= L <= 1290");
    require(eps != nullptr, SMA_ERR_ARG, "null on-site energies");
    const int64_t n = L * L * L;
    CurrentDevice g(ctx->device);
    auto *op = new sma_op();
    op->ctx = ctx;
    op->kind = OP_ANDERSON;
    op->n = n;
    op->nnz = 7 * n;
    op->sym_state = 1;
    op->stencil.L = (int)L;
    op->stencil.hop = t;
    try {
      op->stencil.diag = upload(ctx->stream, eps, n);
      SMA_CUDA(cudaStreamSynchronize(ctx->stream));
    } catch (...) {
      free_stencil(op);
      delete op;
      throw;
    }
    // Gershgorin interval of the model: eps_i -+ 6|t|
    const auto mm = std::minmax_element(eps, eps + n);
    op->gersh_min = *mm.first - 6.0 * std::fabs(t);
    op->gersh_max = *mm.second + 6.0 * std::fabs(t);
    op->has_gersh = true;
    *out = op;
  });
}

extern "C" int sma_op_create_xxz(sma_ctx *ctx, int64_t L, double J, double Delta,
                                 const double *h, sma_op **out) {
  return guarded([&] {
    require(ctx != nullptr && out != nullptr, SMA_ERR_ARG, "null argument");
    *out = nullptr;
    require(L >= 4 && L <= 30 && L % 2 == 0, SMA_ERR_ARG, "XXZ stencil needs an even L in 4..30");
    require(h != nullptr, SMA_ERR_ARG, "null field array");
    // C(p, k) for p < 32, k <= 16
    std::vector<int> binom(32 * 17, 0);
    for (int p = 0; p < 32; ++p) {
      binom[p * 17] = 1;
      for (int k = 1; k <= std::min(p, 16); ++k)
        binom[p * 17 + k] = binom[(p - 1) * 17 + k - 1] + (k <= p - 1 ? binom[(p - 1) * 17 + k] : 0);
    }
    const int m = (int)(L / 2);
    const int64_t n = binom[L * 17 + m];
    // Sz = 0 states in ascending order (next bit permutation with the same popcount)
    std::vector<unsigned> states(n);
    std::vector<double> diag(n);
    unsigned s = (1u << m) - 1u;
    for (int64_t r = 0; r < n; ++r) {
      states[r] = s;
      // J*Delta*sum s_i s_{i+1} + sum h_i s_i with s = +-1/2, in site order
      double d = 0.0;
      for (int64_t i = 0; i < L; ++i) {
        const int64_t j = (i + 1) % L;
        const double si = ((s >> i) & 1u) ? 0.5 : -0.5, sj = ((s >> j) & 1u) ? 0.5 : -0.5;
        d += J * Delta * si * sj;
        d += h[i] * si;
      }
      diag[r] = d;
      const unsigned lo = s & (0u - s), hi = s + lo;  // Gosper's hack
      s = (((hi ^ s) >> 2) / lo) | hi;
    }
    CurrentDevice g(ctx->device);
    auto *op = new sma_op();
    op->ctx = ctx;
    op->kind = OP_XXZ;
    op->n = n;
    op->sym_state = 1;
    op->stencil.L = (int)L;
    op->stencil.hop = 0.5 * J;
    int64_t nnz = n;
    for (int64_t r = 0; r < n; ++r) {
      const unsigned st = states[r];
      const unsigned rot = (st >> 1) | ((st & 1u) << (L - 1));
      nnz += __builtin_popcount((st ^ rot) & ((1u << L) - 1u));
    }
    op->nnz = nnz;
    try {
      op->stencil.diag = upload(ctx->stream, diag.data(), n);
      op->stencil.states = upload(ctx->stream, states.data(), n);
      op->stencil.binom = upload(ctx->stream, binom.data(), binom.size());
      SMA_CUDA(cudaStreamSynchronize(ctx->stream));
    } catch (...) {
      free_stencil(op);
      delete op;
      throw;
    }
    // Gershgorin: |diag| plus at most L flips of amplitude |J|/2
    const auto mm = std::minmax_element(diag.begin(), diag.end());
    op->gersh_min = *mm.first - 0.5 * std::fabs(J) * (double)L;
    op->gersh_max = *mm.second + 0.5 * std::fabs(J) * (double)L;
    op->has_gersh = true;
    *out = op;
  });
}

namespace sma {
void free_stencil_arrays(sma_op *op) { free_stencil(op); }
}  // namespace sma
