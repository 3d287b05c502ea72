// extern "C" entry points of libsma (declared in include/sma.h).  Every entry point
// catches sma::Error and CUDA failures, records the message for sma_last_error() and
// returns a status code; nothing throws across the C boundary.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>

#include "sma_internal.h"

namespace sma {
sma_result *cheb_solve(sma_op *op, double emin, double emax, const sma_cheb_opts &o);
sma_result *polfed_solve(sma_op *op, int64_t nev, int64_t degree, const sma_polfed_opts &o);
sma_result *polfed_batch_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                               const int64_t *nev, const int64_t *degree, const int64_t *mmax,
                               const sma_polfed_opts &o);
sma_result *slice_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                        const int64_t *degree, const int64_t *m0, const sma_slice_opts &o);

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }

namespace {

template <typename F>
int guarded(F &&f) {
  try {
    f();
    return SMA_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return SMA_ERR_NOMEM;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SMA_ERR_INTERNAL;
  }
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) SMA_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

void check_ctx(const sma_ctx *ctx) { require(ctx != nullptr, SMA_ERR_ARG, "null context"); }
void check_op(const sma_op *op) { require(op != nullptr && op->ctx, SMA_ERR_ARG, "null operator"); }

void free_op(sma_op *op) {
  if (!op) return;
  if (op->rowptr) cudaFree(op->rowptr);
  if (op->colind) cudaFree(op->colind);
  if (op->val64) cudaFree(op->val64);
  if (op->val32) cudaFree(op->val32);
  if (op->bulk_err) cudaFree(op->bulk_err);
  free_stencil_arrays(op);
  delete op;
}

void copy_coeffs(const double *coeffs, int64_t K, std::vector<double> &out) {
  require(K >= 0, SMA_ERR_ARG, "K must be nonnegative");
  require(coeffs != nullptr, SMA_ERR_ARG, "null coefficient pointer");
  out.assign(coeffs, coeffs + K + 1);
}

void check_bounds(double smin, double smax) {
  require(std::isfinite(smin) && std::isfinite(smax) && smin < smax, SMA_ERR_ARG,
          "spectral bounds must satisfy smin < smax");
}

}  // namespace
}  // namespace sma

using namespace sma;

extern "C" {

int64_t sma_kernel_launch_count(void) { return g_kernel_launches.load(); }

int sma_abi_version(void) { return SMA_ABI_VERSION; }

const char *sma_last_error(void) { return g_last_error.c_str(); }

int sma_ctx_create(int device, sma_ctx **out) {
  return guarded([&] {
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    *out = nullptr;
    int count = 0;
    SMA_CUDA(cudaGetDeviceCount(&count));
    require(device >= 0 && device < count, SMA_ERR_ARG,
            "device " + std::to_string(device) + " not present (" + std::to_string(count) + " visible)");
    DeviceGuard g(device);
    auto *ctx = new sma_ctx();
    ctx->device = device;
    const char *at = std::getenv("SMA_AUTOTUNE");
    ctx->autotune = !(at && std::string(at) == "0");
    const char *fg = std::getenv("SMA_FILTER_GRAPHS");
    ctx->filter_graphs = !(fg && std::string(fg) == "0");
    const char *pe = std::getenv("SMA_PERSISTENT");
    ctx->persistent = pe && std::string(pe) == "1";
    const char *cd = std::getenv("SMA_CUBLAS_DENSE");
    ctx->cublas_dense = cd && std::string(cd) == "1";
    const char *pd = std::getenv("SMA_PDL");
    ctx->pdl = !(pd && std::string(pd) == "0");
    try {
      SMA_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
      SMA_CUBLAS(cublasCreate(&ctx->cublas));
      SMA_CUBLAS(cublasSetStream(ctx->cublas, ctx->stream));
      SMA_CUSOLVER(cusolverDnCreate(&ctx->cusolver));
      SMA_CUSOLVER(cusolverDnSetStream(ctx->cusolver, ctx->stream));
      SMA_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
      // Keep freed stream-ordered allocations in this process's pool: solves allocate
      // and free their blocks every call.
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
    } catch (...) {
      if (ctx->cusolver) cusolverDnDestroy(ctx->cusolver);
      if (ctx->cublas) cublasDestroy(ctx->cublas);
      if (ctx->stream) cudaStreamDestroy(ctx->stream);
      delete ctx;
      throw;
    }
    *out = ctx;
  });
}

int sma_ctx_destroy(sma_ctx *ctx) {
  return guarded([&] {
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->cusolver) cusolverDnDestroy(ctx->cusolver);
    if (ctx->cublas) cublasDestroy(ctx->cublas);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
  });
}

int sma_ctx_synchronize(sma_ctx *ctx) {
  return guarded([&] {
    check_ctx(ctx);
    DeviceGuard g(ctx->device);
    SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

void *sma_ctx_stream(sma_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// Validates CSC arrays on the host (so that no device kernel can index out of bounds) and
// returns them 0-based as int32 (rp: n+1 column pointers, ci: nnz row indices).
static void validate_csc(int64_t n, int64_t nnz, const int64_t *colptr, const int64_t *rowval,
                         const double *nzval, int64_t index_base, std::vector<int> &rp,
                         std::vector<int> &ci) {
  require(n >= 0 && nnz >= 0, SMA_ERR_ARG, "negative size");
  require(n < INT32_MAX && nnz < INT32_MAX, SMA_ERR_ARG, "matrix too large for 32-bit indices");
  require(index_base == 0 || index_base == 1, SMA_ERR_ARG, "index_base must be 0 or 1");
  require(colptr != nullptr && (nnz == 0 || (rowval && nzval)), SMA_ERR_ARG, "null array");
  rp.assign(n + 1, 0);
  ci.assign(nnz, 0);
  require(colptr[0] == index_base && colptr[n] == nnz + index_base, SMA_ERR_ARG,
          "colptr must start at index_base and end at nnz + index_base");
  for (int64_t j = 0; j < n; ++j) {
    const int64_t s = colptr[j] - index_base, e = colptr[j + 1] - index_base;
    require(s >= 0 && e >= s && e <= nnz, SMA_ERR_ARG, "colptr is not monotone");
    rp[j] = (int)s;
    for (int64_t t = s; t < e; ++t) {
      const int64_t i = rowval[t] - index_base;
      require(i >= 0 && i < n, SMA_ERR_ARG, "row index out of range");
      require(t == s || rowval[t] > rowval[t - 1], SMA_ERR_ARG,
              "row indices must be strictly increasing within each column");
      ci[t] = (int)i;
    }
  }
  rp[n] = (int)nnz;
}

int sma_op_create_csc(sma_ctx *ctx, int64_t n, int64_t nnz, const int64_t *colptr,
                      const int64_t *rowval, const double *nzval, int64_t index_base,
                      int64_t check_symmetric, sma_op **out) {
  return guarded([&] {
    check_ctx(ctx);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    *out = nullptr;
    std::vector<int> rp, ci;
    validate_csc(n, nnz, colptr, rowval, nzval, index_base, rp, ci);
    DeviceGuard g(ctx->device);
    auto *op = new sma_op();
    op->ctx = ctx;
    op->kind = OP_CSR;
    op->n = n;
    op->nnz = nnz;
    try {
      cudaStream_t st = ctx->stream;
      SMA_CUDA(cudaMalloc((void **)&op->rowptr, (n + 1) * sizeof(int)));
      SMA_CUDA(cudaMalloc((void **)&op->colind, std::max<int64_t>(nnz, 1) * sizeof(int)));
      SMA_CUDA(cudaMalloc((void **)&op->val64, std::max<int64_t>(nnz, 1) * sizeof(double)));
      SMA_CUDA(cudaMemcpyAsync(op->rowptr, rp.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
      if (nnz) {
        SMA_CUDA(cudaMemcpyAsync(op->colind, ci.data(), nnz * sizeof(int), cudaMemcpyHostToDevice, st));
        SMA_CUDA(cudaMemcpyAsync(op->val64, nzval, nnz * sizeof(double), cudaMemcpyHostToDevice, st));
      }
      if (n > 0) {
        gershgorin_device(op, &op->gersh_min, &op->gersh_max);
        op->has_gersh = true;
      }
      SMA_CUDA(cudaStreamSynchronize(st));
      if (check_symmetric) {
        op->sym_state = check_csr_device(op) == 0 ? 1 : 2;
        require(op->sym_state == 1, SMA_ERR_NONSYMMETRIC, "matrix is not symmetric");
      }
    } catch (...) {
      free_op(op);
      throw;
    }
    *out = op;
  });
}

int sma_op_create_csc_upper(sma_ctx *ctx, int64_t n, int64_t nnz, const int64_t *colptr,
                            const int64_t *rowval, const double *nzval, int64_t index_base,
                            int64_t check_symmetric, sma_op **out) {
  return guarded([&] {
    check_ctx(ctx);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    *out = nullptr;
    std::vector<int> rp, ci;
    validate_csc(n, nnz, colptr, rowval, nzval, index_base, rp, ci);
    // column j of a symmetric CSC is row j: optional exact symmetry check (a_ij == a_ji
    // for every stored entry), then the upper triangle.  The operator applied is
    // U + U^T - D whatever the lower triangle held, so its Gershgorin bounds come from the
    // kept entries: each off-diagonal u_ji counts in row j and in row i.
    std::vector<int> urp(n + 1, 0), uci;
    std::vector<double> uval, diag(n, 0.0), off(n, 0.0);
    for (int64_t j = 0; j < n; ++j) {
      for (int t = rp[j]; t < rp[j + 1]; ++t) {
        const int i = ci[t];
        if (check_symmetric && i != j) {
          const int *b = ci.data() + rp[i], *e = ci.data() + rp[i + 1];
          const int *p = std::lower_bound(b, e, (int)j);
          require(p != e && *p == (int)j && nzval[p - ci.data()] == nzval[t],
                  SMA_ERR_NONSYMMETRIC, "matrix is not symmetric");
        }
        if (i >= j) {
          uci.push_back(i);
          uval.push_back(nzval[t]);
          if (i == j) {
            diag[j] = nzval[t];
          } else {
            off[j] += std::fabs(nzval[t]);
            off[i] += std::fabs(nzval[t]);
          }
        }
      }
      urp[j + 1] = (int)uci.size();
    }
    double gmin = INFINITY, gmax = -INFINITY;
    for (int64_t j = 0; j < n; ++j) {
      gmin = std::min(gmin, diag[j] - off[j]);
      gmax = std::max(gmax, diag[j] + off[j]);
    }
    const int64_t unnz = (int64_t)uci.size();
    DeviceGuard g(ctx->device);
    auto *op = new sma_op();
    op->ctx = ctx;
    op->kind = OP_CSR_HALF;
    op->n = n;
    op->nnz = unnz;
    op->sym_state = 1;  // A = U + U^T - D is symmetric by construction
    try {
      cudaStream_t st = ctx->stream;
      SMA_CUDA(cudaMalloc((void **)&op->rowptr, (n + 1) * sizeof(int)));
      SMA_CUDA(cudaMalloc((void **)&op->colind, std::max<int64_t>(unnz, 1) * sizeof(int)));
      SMA_CUDA(cudaMalloc((void **)&op->val64, std::max<int64_t>(unnz, 1) * sizeof(double)));
      SMA_CUDA(cudaMemcpyAsync(op->rowptr, urp.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
      if (unnz) {
        SMA_CUDA(cudaMemcpyAsync(op->colind, uci.data(), unnz * sizeof(int), cudaMemcpyHostToDevice, st));
        SMA_CUDA(cudaMemcpyAsync(op->val64, uval.data(), unnz * sizeof(double), cudaMemcpyHostToDevice, st));
      }
      SMA_CUDA(cudaStreamSynchronize(st));
      if (n > 0) {
        op->gersh_min = gmin;
        op->gersh_max = gmax;
        op->has_gersh = true;
      }
    } catch (...) {
      free_op(op);
      throw;
    }
    *out = op;
  });
}

int sma_op_create_lap1d(sma_ctx *ctx, int64_t n, sma_op **out) {
  return guarded([&] {
    check_ctx(ctx);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    require(n >= 2, SMA_ERR_ARG, "the 1D Laplacian stencil needs n >= 2");
    auto *op = new sma_op();
    op->ctx = ctx;
    op->kind = OP_LAP1D;
    op->n = n;
    op->nnz = 3 * n - 2;
    op->sym_state = 1;
    *out = op;
  });
}

int sma_op_create_matblock(sma_ctx *ctx, int64_t n, sma_matblock_fn fn, void *user, sma_op **out) {
  return guarded([&] {
    check_ctx(ctx);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    require(n >= 1, SMA_ERR_ARG, "operator dimension must be positive");
    require(fn != nullptr, SMA_ERR_ARG,
            "a matrix-free operator needs a device block callback (host closures are not run)");
    auto *op = new sma_op();
    op->ctx = ctx;
    op->kind = OP_MATBLOCK;
    op->n = n;
    op->fn = fn;
    op->user = user;
    *out = op;
  });
}

int sma_op_destroy(sma_op *op) {
  return guarded([&] {
    if (!op) return;
    DeviceGuard g(op->ctx->device);
    cudaStreamSynchronize(op->ctx->stream);
    free_op(op);
  });
}

int sma_op_info(const sma_op *op, int64_t *n, int64_t *nnz) {
  return guarded([&] {
    check_op(op);
    if (n) *n = op->n;
    if (nnz) *nnz = op->nnz;
  });
}

int sma_gershgorin_bounds(sma_op *op, double *smin, double *smax) {
  return guarded([&] {
    check_op(op);
    require(op->kind == OP_CSR || op->kind == OP_CSR_HALF, SMA_ERR_ARG,
            "gershgorin_bounds needs an explicit sparse matrix");
    require(op->has_gersh, SMA_ERR_ARG, "empty matrix has no Gershgorin bounds");
    if (smin) *smin = op->gersh_min;
    if (smax) *smax = op->gersh_max;
  });
}

int sma_jackson_kernel(int64_t K, double *g) {
  return guarded([&] {
    require(g != nullptr, SMA_ERR_ARG, "null output");
    const auto v = jackson_kernel(K);
    std::copy(v.begin(), v.end(), g);
  });
}

int sma_cheb_delta_coeffs(double sigma_hat, int64_t K, int64_t jackson, double *c) {
  return guarded([&] {
    require(c != nullptr && K >= 0, SMA_ERR_ARG, "bad arguments");
    const auto v = cheb_delta_coeffs(sigma_hat, K, jackson != 0);
    std::copy(v.begin(), v.end(), c);
  });
}

int sma_cheb_window_coeffs(double a, double b, int64_t K, int64_t jackson, double *c) {
  return guarded([&] {
    require(c != nullptr && K >= 0, SMA_ERR_ARG, "bad arguments");
    const auto v = cheb_window_coeffs(a, b, K, jackson != 0);
    std::copy(v.begin(), v.end(), c);
  });
}

int sma_cheb_smooth_window_coeffs(double a, double b, int64_t K, int64_t jackson, int64_t nsamp,
                                  double delta, double *c) {
  return guarded([&] {
    require(c != nullptr && K >= 0, SMA_ERR_ARG, "bad arguments");
    const auto v = cheb_smooth_window_coeffs(a, b, K, jackson != 0, nsamp, delta);
    std::copy(v.begin(), v.end(), c);
  });
}

int sma_build_coeffs(int64_t degree, double smin, double smax, double sigma, double emin,
                     double emax, int64_t window_type, int64_t jackson, double *c) {
  return guarded([&] {
    require(c != nullptr, SMA_ERR_ARG, "null output");
    const auto v = build_coeffs(degree, smin, smax, sigma, emin, emax, window_type, jackson != 0);
    std::copy(v.begin(), v.end(), c);
  });
}

int sma_apply_poly_block_dev(sma_op *op, const double *coeffs, int64_t K, double smin,
                             double smax, const void *Q_dev, int64_t ldq, void *Y_dev,
                             int64_t ldy, int64_t b, int64_t precision) {
  return guarded([&] {
    check_op(op);
    std::vector<double> c;
    copy_coeffs(coeffs, K, c);
    check_bounds(smin, smax);
    require(b >= 0 && ldq >= b && ldy >= b, SMA_ERR_ARG, "leading dimensions must be >= b");
    require(precision == SMA_PREC_FP64 || precision == SMA_PREC_FP32, SMA_ERR_ARG, "unknown precision");
    if (op->n == 0 || b == 0) return;
    require(Q_dev && Y_dev, SMA_ERR_ARG, "null block pointer");
    DeviceGuard g(op->ctx->device);
    cudaStream_t st = op->ctx->stream;
    if (precision == SMA_PREC_FP64) {
      ClenshawWork<double> w;
      apply_poly_block<double>(op, st, c, smin, smax, (const double *)Q_dev, ldq, (double *)Y_dev,
                               ldy, b, w);
      SMA_CUDA(cudaStreamSynchronize(st));
    } else {
      require(op->kind != OP_MATBLOCK, SMA_ERR_ARG, "FP32 filtering needs a device operator");
      if ((op->kind == OP_CSR || op->kind == OP_CSR_HALF) && !op->val32) {
        SMA_CUDA(cudaMalloc((void **)&op->val32, std::max<int64_t>(op->nnz, 1) * sizeof(float)));
        launch_copy_block<double, float>(st, op->nnz, 1, op->val64, 1, op->val32, 1);
      }
      ClenshawWork<float> w;
      apply_poly_block<float>(op, st, c, smin, smax, (const float *)Q_dev, ldq, (float *)Y_dev, ldy,
                              b, w);
      SMA_CUDA(cudaStreamSynchronize(st));
    }
  });
}

int sma_apply_poly_block_percol_dev(sma_op *op, const double *coeffs, int64_t K, double smin,
                                    double smax, const void *Q_dev, void *Y_dev, int64_t b,
                                    int64_t precision) {
  return guarded([&] {
    check_op(op);
    require(coeffs != nullptr && K >= 0, SMA_ERR_ARG, "coefficients: need K >= 0 and (K+1) x b values");
    check_bounds(smin, smax);
    require(b >= 0, SMA_ERR_ARG, "negative block width");
    require(precision == SMA_PREC_FP64 || precision == SMA_PREC_FP32, SMA_ERR_ARG, "unknown precision");
    require(op->kind != OP_MATBLOCK, SMA_ERR_ARG, "the per-column filter needs a device operator");
    const int64_t n = op->n;
    if (n == 0 || b == 0) return;
    require(Q_dev && Y_dev, SMA_ERR_ARG, "null block pointer");
    for (int64_t i = 0; i < (K + 1) * b; ++i)
      require(std::isfinite(coeffs[i]), SMA_ERR_ARG, "non-finite coefficient");
    DeviceGuard g(op->ctx->device);
    cudaStream_t st = op->ctx->stream;
    std::vector<int> idn(b);
    for (int64_t j = 0; j < b; ++j) idn[j] = (int)j;
    DevBuf<int> colseg(b, st);
    SMA_CUDA(cudaMemcpyAsync(colseg.p, idn.data(), b * sizeof(int), cudaMemcpyHostToDevice, st));
    auto run = [&](auto zero) {
      using T = decltype(zero);
      std::vector<T> ch((K + 1) * b);
      for (int64_t i = 0; i < (K + 1) * b; ++i) ch[i] = (T)coeffs[i];
      DevBuf<T> coef(ch.size(), st), B1(n * b, st), B2(n * b, st), TMP(n * b, st), AX;
      if (op->kind != OP_CSR) AX.alloc(n * b, st);
      SMA_CUDA(cudaMemcpyAsync(coef.p, ch.data(), ch.size() * sizeof(T), cudaMemcpyHostToDevice, st));
      percol_filter<T>(op, st, coef.p, K, smin, smax, (const T *)Q_dev, (T *)Y_dev, b, colseg.p,
                       B1.p, B2.p, TMP.p, AX.p);
      SMA_CUDA(cudaStreamSynchronize(st));
    };
    if (precision == SMA_PREC_FP64) {
      run(0.0);
    } else {
      if ((op->kind == OP_CSR || op->kind == OP_CSR_HALF) && !op->val32) {
        SMA_CUDA(cudaMalloc((void **)&op->val32, std::max<int64_t>(op->nnz, 1) * sizeof(float)));
        launch_copy_block<double, float>(st, op->nnz, 1, op->val64, 1, op->val32, 1);
      }
      run(0.0f);
    }
  });
}

int sma_dense_gram_dev(sma_ctx *ctx, int64_t n, int64_t m, int64_t k, const double *X_dev,
                       int64_t ldx, const double *Y_dev, int64_t ldy, double *C_dev, int64_t ldc,
                       double alpha, double beta) {
  return guarded([&] {
    check_ctx(ctx);
    require(n >= 0 && m >= 0 && k >= 0 && ldx >= m && ldy >= k && ldc >= std::max<int64_t>(m, 1),
            SMA_ERR_ARG, "bad sizes or leading dimensions");
    if (m == 0 || k == 0) return;
    require(C_dev && (n == 0 || (X_dev && Y_dev)), SMA_ERR_ARG, "null block pointer");
    DeviceGuard g(ctx->device);
    Dense dn(ctx);
    dn.gram(n, m, k, X_dev, ldx, Y_dev, ldy, C_dev, ldc, alpha, beta);
    SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int sma_dense_update_dev(sma_ctx *ctx, int64_t n, int64_t m, int64_t p, const double *X_dev,
                         int64_t ldx, const double *C_dev, int64_t ldc, int64_t transC,
                         double *Y_dev, int64_t ldy, double alpha, double beta) {
  return guarded([&] {
    check_ctx(ctx);
    require(n >= 0 && m >= 0 && p >= 0 && ldx >= m && ldy >= p &&
                ldc >= std::max<int64_t>(transC ? p : m, 1),
            SMA_ERR_ARG, "bad sizes or leading dimensions");
    if (n == 0 || p == 0) return;
    require(Y_dev && (m == 0 || (X_dev && C_dev)), SMA_ERR_ARG, "null block pointer");
    DeviceGuard g(ctx->device);
    Dense dn(ctx);
    dn.mul_small(n, m, p, X_dev, ldx, C_dev, ldc, Y_dev, ldy, alpha, beta, transC != 0);
    SMA_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int sma_divided_difference(const double *coeffs, int64_t K, double t, double *e, double *pt) {
  return guarded([&] {
    require(coeffs != nullptr && e != nullptr && pt != nullptr && K >= 1, SMA_ERR_ARG,
            "need K >= 1, K+1 coefficients and K outputs");
    std::vector<double> c(coeffs, coeffs + K + 1);
    divided_difference(c, t, e, pt);
  });
}

int sma_apply_poly_block(sma_op *op, const double *coeffs, int64_t K, double smin, double smax,
                         const double *Q, double *Y, int64_t b, int64_t precision) {
  return guarded([&] {
    check_op(op);
    require(b >= 0, SMA_ERR_ARG, "negative block width");
    const int64_t n = op->n;
    if (n == 0 || b == 0) return;
    require(Q && Y, SMA_ERR_ARG, "null block pointer");
    DeviceGuard g(op->ctx->device);
    cudaStream_t st = op->ctx->stream;
    DevBuf<double> qc(n * b, st), qr(n * b, st), yr(n * b, st);
    SMA_CUDA(cudaMemcpyAsync(qc.p, Q, n * b * sizeof(double), cudaMemcpyHostToDevice, st));
    launch_colmajor_to_rowmajor(st, n, b, qc.p, qr.p, b);
    int rc;
    if (precision == SMA_PREC_FP32) {
      DevBuf<float> q32(n * b, st), y32(n * b, st);
      launch_copy_block<double, float>(st, n, b, qr.p, b, q32.p, b);
      SMA_CUDA(cudaStreamSynchronize(st));
      rc = sma_apply_poly_block_dev(op, coeffs, K, smin, smax, q32.p, b, y32.p, b, b, precision);
      if (rc == SMA_OK) launch_copy_block<float, double>(st, n, b, y32.p, b, yr.p, b);
      SMA_CUDA(cudaStreamSynchronize(st));
    } else {
      SMA_CUDA(cudaStreamSynchronize(st));
      rc = sma_apply_poly_block_dev(op, coeffs, K, smin, smax, qr.p, b, yr.p, b, b, precision);
    }
    if (rc != SMA_OK) throw Error(rc, g_last_error);
    launch_rowmajor_to_colmajor(st, n, b, yr.p, b, qc.p);
    SMA_CUDA(cudaMemcpyAsync(Y, qc.p, n * b * sizeof(double), cudaMemcpyDeviceToHost, st));
    SMA_CUDA(cudaStreamSynchronize(st));
  });
}

int sma_spmm_dev(sma_op *op, const double *X_dev, int64_t ldx, double *Y_dev, int64_t ldy,
                 int64_t b) {
  return guarded([&] {
    check_op(op);
    require(b >= 0 && ldx >= b && ldy >= b, SMA_ERR_ARG, "leading dimensions must be >= b");
    if (op->n == 0 || b == 0) return;
    require(X_dev && Y_dev, SMA_ERR_ARG, "null block pointer");
    DeviceGuard g(op->ctx->device);
    op_apply(op, op->ctx->stream, X_dev, ldx, Y_dev, ldy, b);
    SMA_CUDA(cudaStreamSynchronize(op->ctx->stream));
  });
}

int sma_kpm_moments(sma_op *op, int64_t M, int64_t R, int64_t seed, double smin, double smax,
                    double *mu, double *per_vec) {
  return guarded([&] {
    check_op(op);
    require(mu != nullptr, SMA_ERR_ARG, "null moment array");
    check_bounds(smin, smax);
    require(op->n > 0, SMA_ERR_ARG, "empty operator");
    DeviceGuard g(op->ctx->device);
    kpm_moments(op, M, R, (uint64_t)seed, smin, smax, mu, per_vec);
  });
}

int sma_kpm_count(const double *mu, int64_t M, int64_t n, double smin, double smax,
                  double emin, double emax, int64_t jackson, double *count) {
  return guarded([&] {
    require(mu != nullptr && count != nullptr, SMA_ERR_ARG, "null argument");
    *count = kpm_count(mu, M, n, smin, smax, emin, emax, jackson != 0);
  });
}

void sma_cheb_opts_default(sma_cheb_opts *o) {
  if (!o) return;
  *o = sma_cheb_opts{};
  o->has_bounds = 0;
  o->sigma = 0.0;
  o->m0 = 200;
  o->degree = 80;
  o->maxiter = 8;
  o->tol = 1e-10;
  o->res_gate = 1e-6;
  o->jackson = 1;
  o->debug = 0;
  o->two_hit = 1;
  o->seed = 1;
  o->window_type = SMA_WINDOW_STEP;
  o->matrix_free = 0;
  o->precision = SMA_PREC_FP64;
}

void sma_polfed_opts_default(sma_polfed_opts *o) {
  if (!o) return;
  *o = sma_polfed_opts{};
  o->s = 8;
  o->has_bounds = 0;
  o->sigma = 0.0;
  o->emin = -INFINITY;
  o->emax = INFINITY;
  o->tol = 1e-10;
  o->threaded = 1;
  o->overextract = 2;
  o->refine = 1;
  o->window_type = SMA_WINDOW_STEP;
  o->jackson = 1;
  o->mmax = 0;
  o->rtol = 1e-12;
  o->reorth_passes = 1;
  o->extra_keep = 8;
  o->seed = 1;
  o->show_progress = 0;
  o->chunk = 64;
  o->precision = SMA_PREC_FP64;
}

int sma_cheb_solve(sma_op *op, double emin, double emax, const sma_cheb_opts *opts,
                   sma_result **out) {
  return guarded([&] {
    check_op(op);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    *out = nullptr;
    sma_cheb_opts o;
    if (opts) o = *opts; else sma_cheb_opts_default(&o);
    require(o.precision == SMA_PREC_FP64 || o.precision == SMA_PREC_FP32 ||
                o.precision == SMA_PREC_MIXED, SMA_ERR_ARG, "unknown precision");
    if (o.has_bounds) check_bounds(o.smin, o.smax);
    DeviceGuard g(op->ctx->device);
    *out = cheb_solve(op, emin, emax, o);
  });
}

int sma_polfed_solve(sma_op *op, int64_t nev, int64_t degree, const sma_polfed_opts *opts,
                     sma_result **out) {
  return guarded([&] {
    check_op(op);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    *out = nullptr;
    sma_polfed_opts o;
    if (opts) o = *opts; else sma_polfed_opts_default(&o);
    require(o.precision == SMA_PREC_FP64 || o.precision == SMA_PREC_FP32 ||
                o.precision == SMA_PREC_MIXED, SMA_ERR_ARG, "unknown precision");
    if (o.has_bounds) check_bounds(o.smin, o.smax);
    DeviceGuard g(op->ctx->device);
    *out = polfed_solve(op, nev, degree, o);
  });
}

int sma_polfed_batch_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                           const int64_t *nev, const int64_t *degree, const int64_t *mmax,
                           const sma_polfed_opts *opts, sma_result **out) {
  return guarded([&] {
    check_op(op);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    *out = nullptr;
    sma_polfed_opts o;
    if (opts) o = *opts; else sma_polfed_opts_default(&o);
    require(o.precision == SMA_PREC_FP64 || o.precision == SMA_PREC_FP32 ||
                o.precision == SMA_PREC_MIXED, SMA_ERR_ARG, "unknown precision");
    if (o.has_bounds) check_bounds(o.smin, o.smax);
    require(nwin >= 1 && nwin <= 4096, SMA_ERR_ARG, "nwin must be in 1..4096");
    DeviceGuard g(op->ctx->device);
    *out = polfed_batch_solve(op, nwin, emin, emax, nev, degree, mmax, o);
  });
}

void sma_slice_opts_default(sma_slice_opts *o) {
  if (!o) return;
  *o = sma_slice_opts{};
  o->has_bounds = 0;
  o->maxiter = 8;
  o->tol = 1e-10;
  o->res_gate = 1e-6;
  o->jackson = 1;
  o->two_hit = 1;
  o->seed = 1;
  o->window_type = SMA_WINDOW_STEP;
  o->precision = SMA_PREC_FP64;
  o->graph = 1;
  o->debug = 0;
}

int sma_slice_solve(sma_op *op, int64_t nwin, const double *emin, const double *emax,
                    const int64_t *degree, const int64_t *m0, const sma_slice_opts *opts,
                    sma_result **out) {
  return guarded([&] {
    check_op(op);
    require(out != nullptr, SMA_ERR_ARG, "null output pointer");
    *out = nullptr;
    sma_slice_opts o;
    if (opts) o = *opts; else sma_slice_opts_default(&o);
    if (o.has_bounds) check_bounds(o.smin, o.smax);
    DeviceGuard g(op->ctx->device);
    *out = slice_solve(op, nwin, emin, emax, degree, m0, o);
  });
}

int sma_mlp_create(sma_ctx *ctx, int64_t in, int64_t hid, int64_t out, int64_t seed,
                   sma_mlp **net) {
  return guarded([&] {
    require(ctx != nullptr && net != nullptr, SMA_ERR_ARG, "null argument");
    require(in >= 1 && hid >= 1 && out >= 1, SMA_ERR_ARG, "layer sizes must be positive");
    *net = nullptr;
    DeviceGuard g(ctx->device);
    auto *p = new sma_mlp();
    p->ctx = ctx;
    try {
      mlp_init(p, in, hid, out, (uint64_t)seed);
    } catch (...) {
      delete p;
      throw;
    }
    *net = p;
  });
}

int sma_mlp_destroy(sma_mlp *net) {
  return guarded([&] {
    if (!net) return;
    DeviceGuard g(net->ctx->device);
    cudaStreamSynchronize(net->ctx->stream);
    delete net;
  });
}

int sma_mlp_num_params(const sma_mlp *net, int64_t *count) {
  return guarded([&] {
    require(net != nullptr && count != nullptr, SMA_ERR_ARG, "null argument");
    *count = net->nparam;
  });
}

int sma_mlp_get_params(const sma_mlp *net, float *params) {
  return guarded([&] {
    require(net != nullptr && params != nullptr, SMA_ERR_ARG, "null argument");
    DeviceGuard g(net->ctx->device);
    mlp_get_params(net, params);
  });
}

int sma_mlp_set_params(sma_mlp *net, const float *params) {
  return guarded([&] {
    require(net != nullptr && params != nullptr, SMA_ERR_ARG, "null argument");
    DeviceGuard g(net->ctx->device);
    mlp_set_params(net, params);
  });
}

int sma_mlp_forward(sma_mlp *net, const float *X, int64_t B, float *Y) {
  return guarded([&] {
    require(net != nullptr && B >= 0, SMA_ERR_ARG, "bad argument");
    if (B == 0) return;
    require(X != nullptr && Y != nullptr, SMA_ERR_ARG, "null array");
    DeviceGuard g(net->ctx->device);
    mlp_forward(net, X, B, Y);
  });
}

int sma_mlp_grad(sma_mlp *net, const float *X, const float *T, const float *w, int64_t B,
                 float *loss, float *grad) {
  return guarded([&] {
    require(net != nullptr && X != nullptr && T != nullptr && B >= 1, SMA_ERR_ARG, "bad argument");
    DeviceGuard g(net->ctx->device);
    const float l = mlp_grad(net, X, T, w, B, grad);
    if (loss) *loss = l;
  });
}

int sma_mlp_train(sma_mlp *net, const float *X, const float *T, const float *w, int64_t N,
                  int64_t steps, double lr, int64_t minibatch, int64_t seed,
                  double weight_decay, float *loss_hist) {
  return guarded([&] {
    require(net != nullptr && X != nullptr && T != nullptr, SMA_ERR_ARG, "null argument");
    require(lr > 0.0, SMA_ERR_ARG, "learning rate must be positive");
    DeviceGuard g(net->ctx->device);
    mlp_train(net, X, T, w, N, steps, lr, minibatch, (uint64_t)seed, weight_decay, loss_hist);
  });
}

int sma_selftest_barrier_timeout(sma_ctx *ctx, int64_t *observed) {
  return guarded([&] {
    require(ctx != nullptr && observed != nullptr, SMA_ERR_ARG, "null argument");
    DeviceGuard g(ctx->device);
    *observed = barrier_selftest(ctx);
    require(*observed == SMA_ERR_TIMEOUT, SMA_ERR_INTERNAL,
            "the bounded barrier did not report its timeout");
  });
}

int sma_result_count(const sma_result *r, int64_t *k, int64_t *n) {
  return guarded([&] {
    require(r != nullptr, SMA_ERR_ARG, "null result");
    if (k) *k = r->k;
    if (n) *n = r->n;
  });
}

int sma_result_copy(const sma_result *r, double *lam, double *X, double *res) {
  return guarded([&] {
    require(r != nullptr, SMA_ERR_ARG, "null result");
    if (lam) std::copy(r->lam.begin(), r->lam.end(), lam);
    if (res) std::copy(r->res.begin(), r->res.end(), res);
    if (X && r->k > 0 && r->n > 0) {
      DeviceGuard g(r->ctx->device);
      cudaStream_t st = r->ctx->stream;
      DevBuf<double> cm(r->n * r->k, st);
      launch_rowmajor_to_colmajor(st, r->n, r->k, r->X_dev, r->ldx, cm.p);
      SMA_CUDA(cudaMemcpyAsync(X, cm.p, r->n * r->k * sizeof(double), cudaMemcpyDeviceToHost, st));
      SMA_CUDA(cudaStreamSynchronize(st));
    }
  });
}

int sma_result_stats(const sma_result *r, sma_stats *stats) {
  return guarded([&] {
    require(r != nullptr && stats != nullptr, SMA_ERR_ARG, "null argument");
    *stats = r->stats;
  });
}

int sma_result_windows(const sma_result *r, int64_t *win) {
  return guarded([&] {
    require(r != nullptr && win != nullptr, SMA_ERR_ARG, "null argument");
    for (int64_t j = 0; j < r->k; ++j) win[j] = r->win.empty() ? 0 : r->win[j];
  });
}

int sma_result_window_info(const sma_result *r, int64_t nwin, int64_t *iterations,
                           int64_t *converged) {
  return guarded([&] {
    require(r != nullptr, SMA_ERR_ARG, "null result");
    const int64_t have = r->win_iters.empty() ? 1 : (int64_t)r->win_iters.size();
    require(nwin == have, SMA_ERR_ARG, "the result holds " + std::to_string(have) + " windows");
    for (int64_t w = 0; w < nwin; ++w) {
      if (iterations) iterations[w] = r->win_iters.empty() ? r->stats.iterations : r->win_iters[w];
      if (converged) converged[w] = r->win_done.empty() ? 0 : r->win_done[w];
    }
  });
}

int sma_result_free(sma_result *r) {
  return guarded([&] {
    if (!r) return;
    if (r->X_dev) {
      DeviceGuard g(r->ctx->device);
      cudaStreamSynchronize(r->ctx->stream);
      cudaFree(r->X_dev);
    }
    delete r;
  });
}

}  // extern "C"
