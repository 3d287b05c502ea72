// sma_apply_poly_block_noalloc: the block Clenshaw filter without any device allocation.
//
// The regular filter entry points allocate their three n x b recurrence blocks (B1, B2,
// TMP) for each call.  Some callers cannot allow that: processes whose device memory is
// owned by another allocator that has reserved it up front (a framework's caching
// allocator, a Julia GPU memory pool), and latency-critical loops that must not pay for
// cudaMalloc/cudaFree and the synchronization they imply.  This variant keeps the three
// blocks in one file-scope __device__ array instead, so a call allocates nothing.
//
// Limits and sharing:
//  * capacity: each block holds at most kNoAllocMaxElems = 2^21 FP64 elements, so the call
//    accepts n*b <= 2,097,152 and rejects larger sizes with SMA_ERR_ARG; the array is
//    3 * 2^21 * 8 bytes = 48 MiB, held on every device where it is loaded until the process
//    exits;
//  * every call on a device uses the same array, which keeps the contents of the last call.
//    The recurrence writes each block before reading it (B1 = c_K Q first; B2 is first read
//    after being written), so nothing has to start at zero.  Calls whose work overlaps on
//    the GPU -- different streams, contexts or threads on the same device -- race on the
//    array; callers serialize them;
//  * the first call on a device looks the array's device address up (cudaGetSymbolAddress
//    with that device current) and caches it; make that first call before any stream
//    capture.  cudaDeviceReset ends every context of this library on that device, this
//    cached address included.
#include <cmath>
#include <mutex>
#include <string>

#include "sma_internal.h"

namespace sma {

template <typename T>
void csr_clenshaw_step_untuned(const sma_op *op, cudaStream_t st, int64_t b, const T *Q,
                               int64_t ldq, const T *B1, const T *B2, int64_t ldb, T *out,
                               int64_t ldo, double ck, double alpha, double beta, bool has_self);

namespace {

constexpr int64_t kNoAllocMaxElems = int64_t(1) << 21;
static __device__ __align__(256) double g_noalloc_scratch[3 * kNoAllocMaxElems];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device`, which must be current.  In host code
// `g_noalloc_scratch` names a host-side stand-in, never the device memory itself.
double *scratch_on(int device) {
  require(device >= 0 && device < kMaxDevices, SMA_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_ptr[device] == nullptr) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      throw Error(SMA_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") +
                                    cudaGetErrorString(e));
    g_scratch_ptr[device] = static_cast<double *>(p);
  }
  return g_scratch_ptr[device];
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

// One fused step on the operator: the CSR form without the autotuner (which creates
// events), or the stencil form.
void step(const sma_op *op, cudaStream_t st, int64_t b, const double *Q, int64_t ldq,
          const double *B1, const double *B2, double *out, int64_t ldo, double ck, double alpha,
          double beta) {
  if (op->kind == OP_CSR)
    csr_clenshaw_step_untuned<double>(op, st, b, Q, ldq, B1, B2, b, out, ldo, ck, alpha, beta, true);
  else
    launch_clenshaw_step<double>(op, st, b, Q, ldq, B1, B2, b, out, ldo, ck, alpha, beta, true);
}

void filter_noalloc(sma_op *op, const double *coeffs, int64_t K, double smin, double smax,
                    const double *Q, int64_t ldq, double *Y, int64_t ldy, int64_t b) {
  require(op != nullptr && op->ctx != nullptr, SMA_ERR_ARG, "null operator");
  require(coeffs != nullptr && K >= 0, SMA_ERR_ARG, "coefficients: need K >= 0 and K+1 values");
  require(std::isfinite(smin) && std::isfinite(smax) && smin < smax, SMA_ERR_ARG,
          "spectral bounds must satisfy smin < smax");
  require(b >= 0 && ldq >= b && ldy >= b, SMA_ERR_ARG, "leading dimensions must be >= b");
  require(op->kind == OP_CSR || op->kind == OP_LAP1D || op->kind == OP_ANDERSON ||
              op->kind == OP_XXZ,
          SMA_ERR_ARG,
          "the allocation-free filter takes a CSR matrix or a model stencil (1D Laplacian, "
          "Anderson, XXZ); half storage and caller callbacks are not accepted");
  const int64_t n = op->n;
  if (n == 0 || b == 0) return;
  require(Q != nullptr && Y != nullptr, SMA_ERR_ARG, "null block pointer");
  require(n <= kNoAllocMaxElems / b, SMA_ERR_ARG,
          "n*b = " + std::to_string(n) + "*" + std::to_string(b) +
              " exceeds the allocation-free scratch capacity of " +
              std::to_string(kNoAllocMaxElems) + " elements per block");
  CurrentDevice guard(op->ctx->device);
  double *s = scratch_on(op->ctx->device);
  double *B1 = s, *B2 = s + kNoAllocMaxElems, *TMP = s + 2 * kNoAllocMaxElems;
  cudaStream_t st = op->ctx->stream;
  // the recurrence of apply_poly_block! (chebyshev_subspace_iteration.jl:554-591)
  const double c = 0.5 * (smin + smax), invd = 2.0 / (smax - smin);
  const double alpha = 2.0 * invd, beta = -2.0 * c * invd;
  if (K == 0) {
    launch_scale_block<double>(st, n, b, Q, ldq, Y, ldy, coeffs[0]);
  } else {
    launch_scale_block<double>(st, n, b, Q, ldq, B1, b, coeffs[K]);
    bool b2_zero = true;
    for (int64_t ci = K - 1; ci >= 1; --ci) {
      step(op, st, b, Q, ldq, B1, b2_zero ? nullptr : B2, TMP, b, coeffs[ci], alpha, beta);
      double *t = B2;
      B2 = B1;
      B1 = TMP;
      TMP = t;
      b2_zero = false;
    }
    step(op, st, b, Q, ldq, B1, b2_zero ? nullptr : B2, Y, ldy, coeffs[0], invd, -(c * invd));
  }
  SMA_CUDA(cudaStreamSynchronize(st));
  check_bulk_error(op, st);  // a tuned bulk-copy step reports a wait that gave up
}

}  // namespace
}  // namespace sma

extern "C" int sma_apply_poly_block_noalloc(sma_op *op, const double *coeffs, int64_t K,
                                            double smin, double smax, const double *Q_dev,
                                            int64_t ldq, double *Y_dev, int64_t ldy, int64_t b) {
  try {
    sma::filter_noalloc(op, coeffs, K, smin, smax, Q_dev, ldq, Y_dev, ldy, b);
    return SMA_OK;
  } catch (const sma::Error &e) {
    sma::set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    sma::set_last_error(e.what());
    return SMA_ERR_INTERNAL;
  }
}
