// Symmetric half storage: only the upper triangle U (diagonal included) of a symmetric
// matrix is kept, as CSR, and
//
//   Y = A X = U X + (U - D)^T X
//
// is two launches: a row pass writes y_i = sum_{j >= i} u_ij x_j, then a scatter pass adds
// u_ij x_i into y_j for every stored off-diagonal entry (atomic adds).  It stores about half
// of the matrix's entries and indices; the atomic adds make the summation order of the
// transposed half nondeterministic, so products agree with the full-storage kernel to
// rounding, not bit for bit.  The Clenshaw filter uses it like a caller-supplied operator:
// the product into a scratch block, then the recurrence's axpy kernel.
#include "sma_internal.h"

namespace sma {

namespace {

template <typename T>
__global__ void half_rows_kernel(int64_t n, int64_t b, const int *__restrict__ rowptr,
                                 const int *__restrict__ colind, const T *__restrict__ val,
                                 const T *__restrict__ X, int64_t ldx, T *__restrict__ Y,
                                 int64_t ldy) {
  const int64_t total = n * b;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / b, c = t % b;
    T acc = T(0);
    for (int k = __ldg(rowptr + i); k < __ldg(rowptr + i + 1); ++k)
      acc = fma(__ldg(val + k), X[(int64_t)__ldg(colind + k) * ldx + c], acc);
    Y[i * ldy + c] = acc;
  }
}

template <typename T>
__global__ void half_scatter_kernel(int64_t n, int64_t b, const int *__restrict__ rowptr,
                                    const int *__restrict__ colind, const T *__restrict__ val,
                                    const T *__restrict__ X, int64_t ldx, T *Y, int64_t ldy) {
  const int64_t total = n * b;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / b, c = t % b;
    const T xi = X[i * ldx + c];
    for (int k = __ldg(rowptr + i); k < __ldg(rowptr + i + 1); ++k) {
      const int64_t j = __ldg(colind + k);
      if (j != i) atomicAdd(Y + j * ldy + c, __ldg(val + k) * xi);
    }
  }
}

unsigned grid_of(int64_t total, int num_sms) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)num_sms * 32));
}

}  // namespace

template <typename T>
void half_product(const sma_op *op, cudaStream_t st, const T *X, int64_t ldx, T *Y, int64_t ldy,
                  int64_t b) {
  require(op->kind == OP_CSR_HALF, SMA_ERR_INTERNAL, "half_product needs a half-storage operator");
  const int64_t n = op->n;
  if (n == 0 || b == 0) return;
  const T *val;
  if constexpr (sizeof(T) == 8) val = (const T *)op->val64;
  else val = (const T *)op->val32;
  require(val != nullptr, SMA_ERR_INTERNAL, "half-storage values missing for this precision");
  const unsigned grid = grid_of(n * b, op->ctx->num_sms);
  half_rows_kernel<T><<<grid, 256, 0, st>>>(n, b, op->rowptr, op->colind, val, X, ldx, Y, ldy);
  SMA_CHECK_LAUNCH();
  half_scatter_kernel<T><<<grid, 256, 0, st>>>(n, b, op->rowptr, op->colind, val, X, ldx, Y, ldy);
  SMA_CHECK_LAUNCH();
}

template void half_product<double>(const sma_op *, cudaStream_t, const double *, int64_t, double *,
                                   int64_t, int64_t);
template void half_product<float>(const sma_op *, cudaStream_t, const float *, int64_t, float *,
                                  int64_t, int64_t);

}  // namespace sma
