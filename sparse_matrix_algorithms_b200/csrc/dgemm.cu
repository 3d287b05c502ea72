// FP64 tensor-core products for the dense part of the solvers (DMMA: mma.sync f64 on the
// B200's FP64 tensor pipe).  Two shapes cover every tall-skinny product of the block
// orthogonalization, reorthogonalization and Rayleigh-Ritz lift (n >> m, k, p):
//
//   gram    C (m x k, column-major, ldc) = alpha X^T Y + beta C
//           X: n x m, Y: n x k, row-major (ldx, ldy) -- the reduction runs over n;
//   update  Y (n x p, row-major, ldy)    = alpha X B + beta Y
//           X: n x m row-major (ldx); B: m x p given as a column-major C (B = C, ldc) or as
//           the transpose of one (B = C^T, C p x m column-major, ldc).
//
// Both stage their operand tiles in shared memory with cp.async (16-byte copies, double
// buffered) and run mma.sync.aligned.m8n8k4.row.col.f64 on the tiles: a warp owns a 32 x 32
// (update) or 32 x 16 (gram) piece of the CTA's 64 x 64 / 128 x 64 output tile and keeps its
// accumulators in registers.  The gram splits n over the grid; every CTA writes its 64 x 64
// partial product to a workspace and a second kernel sums the partials in a fixed order,
// so results are deterministic (the same bits every run).  The update owns whole rows of Y:
// with beta = 0 it may write in place over X when p <= 64 (X <- X B, the triangular solve of
// CholQR written as a product with R^-1), since a CTA reads all of its rows of X before it
// writes them.
//
// DMMA fragment layout of m8n8k4 (PTX ISA, "Matrix Fragments for mma.m8n8k4 with .f64"):
// lane = 4 g + t (g = groupID 0..7, t = thread in group 0..3);
//   A (8 x 4, row):  a0 = A[g][t];   B (4 x 8, col): b0 = B[t][g];
//   C/D (8 x 8):     c0 = C[g][2t], c1 = C[g][2t + 1].
#include <algorithm>

#include "sma_internal.h"

namespace sma {
namespace dmma {

__device__ __forceinline__ void mma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ------------------------------------------------------------------ update
// CTA tile: 128 rows x 64 columns of Y; 8 warps as 4 (rows) x 2 (columns), warp tile
// 32 x 32 = 4 x 4 fragments.  K chunk 16 (four k-steps of 4), two stages.
constexpr int UM = 128, UN = 64, UK = 16;
constexpr int UA = UK + 4;  // padded row of the A stage (doubles)
constexpr int UB = UK + 4;  // padded row of the B stage, stored [column][k]
constexpr int kUpdateThreads = 256;

struct UpdateSmem {
  double a[2][UM][UA];
  double b[2][UN][UB];
};

// B(i, j) for the update: TB = false -> C[i + j ldc] (column-major m x p);
// TB = true -> C[j + i ldc] (the transpose of a column-major p x m).
template <bool TB>
__global__ void __launch_bounds__(kUpdateThreads)
update_kernel(int64_t n, int m, int p, const double *X, int64_t ldx,  // Y may alias X
              const double *__restrict__ C, int64_t ldc, double *Y, int64_t ldy, double alpha,
              double beta, bool vec16) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  UpdateSmem &sm = *reinterpret_cast<UpdateSmem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = (warp & 3) * 32, wc = (warp >> 2) * 32;
  const int64_t row0 = (int64_t)blockIdx.x * UM;
  const int col0 = blockIdx.y * UN;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nk = (m + UK - 1) / UK;  // m = 0: Y = beta Y
  // stage loader: A rows row0.., k chunk kc; B k chunk kc, columns col0..
  auto load = [&](int stage, int kc) {
    const int k0 = kc * UK;
    // A: 128 x 16 doubles; with 16-byte copies 8 per row
    if (vec16 && k0 + UK <= m) {
      for (int e = tid; e < UM * (UK / 2); e += kUpdateThreads) {
        const int r = e / (UK / 2), c2 = (e % (UK / 2)) * 2;
        const int64_t gr = row0 + r;
        double *dst = &sm.a[stage][r][c2];
        if (gr < n) cp_async16(dst, X + gr * ldx + k0 + c2);
        else { dst[0] = 0.0; dst[1] = 0.0; }
      }
    } else {
      for (int e = tid; e < UM * UK; e += kUpdateThreads) {
        const int r = e / UK, c = e % UK;
        const int64_t gr = row0 + r;
        double *dst = &sm.a[stage][r][c];
        if (gr < n && k0 + c < m) cp_async8(dst, X + gr * ldx + k0 + c);
        else *dst = 0.0;
      }
    }
    // B: 16 (k) x 64 (columns), stored [column][k]
    for (int e = tid; e < UN * UK; e += kUpdateThreads) {
      int j, kk;
      if (TB) { kk = e / UN; j = e % UN; }   // consecutive threads: consecutive columns
      else { j = e / UK; kk = e % UK; }      // consecutive threads: consecutive k
      const int gk = k0 + kk, gj = col0 + j;
      double *dst = &sm.b[stage][j][kk];
      if (gk < m && gj < p) cp_async8(dst, TB ? C + gj + (int64_t)gk * ldc : C + gk + (int64_t)gj * ldc);
      else *dst = 0.0;
    }
    cp_async_commit();
  };
  if (nk > 0) load(0, 0);
  for (int kc = 0; kc < nk; ++kc) {
    const int stage = kc & 1;
    if (kc + 1 < nk) {
      load(stage ^ 1, kc + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < UK; ks += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sm.a[stage][wr + i * 8 + g][ks + t];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sm.b[stage][wc + j * 8 + g][ks + t];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_8x8x4(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
  // epilogue: Y = alpha acc + beta Y (Y not read when beta == 0)
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t r = row0 + wr + i * 8 + g;
    if (r >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = col0 + wc + j * 8 + 2 * t;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (c + h < p) {
          double *y = Y + r * ldy + c + h;
          *y = beta == 0.0 ? alpha * acc[i][j][h] : alpha * acc[i][j][h] + beta * *y;
        }
      }
    }
  }
}

// ------------------------------------------------------------------ gram
// Output tile 64 (m) x 64 (k) per CTA; the CTA sums rows [r0, r1) of n in chunks of 16.
// 8 warps as 2 (m) x 4 (k): warp tile 32 x 16 = 4 x 2 fragments.
constexpr int GM = 64, GN = 64, GK = 16;
constexpr int GP = 64 + 4;  // padded stage rows (doubles)
constexpr int kGramThreads = 256;

struct GramSmem {
  double x[2][GK][GP];
  double y[2][GK][GP];
};

__global__ void __launch_bounds__(kGramThreads)
gram_partial_kernel(int64_t n, int m, int k, const double *__restrict__ X, int64_t ldx,
                    const double *__restrict__ Y, int64_t ldy, int64_t rows_per_split,
                    double *__restrict__ part, bool vec16, bool upper) {
  if (upper && blockIdx.x > blockIdx.y) return;  // a tile below the diagonal (no barrier yet)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GramSmem &sm = *reinterpret_cast<GramSmem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 32, wk = (warp >> 1) * 16;
  const int m0 = blockIdx.x * GM, k0 = blockIdx.y * GN;
  const int64_t r0 = (int64_t)blockIdx.z * rows_per_split;
  const int64_t r1 = min(n, r0 + rows_per_split);
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int64_t nrows = r1 > r0 ? r1 - r0 : 0;
  const int nc = (int)((nrows + GK - 1) / GK);
  auto load = [&](int stage, int c) {
    const int64_t rb = r0 + (int64_t)c * GK;
    if (vec16 && m0 + GM <= m && k0 + GN <= k) {
      for (int e = tid; e < GK * (GM / 2); e += kGramThreads) {
        const int r = e / (GM / 2), c2 = (e % (GM / 2)) * 2;
        const int64_t gr = rb + r;
        double *dx = &sm.x[stage][r][c2];
        double *dy = &sm.y[stage][r][c2];
        if (gr < r1) {
          cp_async16(dx, X + gr * ldx + m0 + c2);
          cp_async16(dy, Y + gr * ldy + k0 + c2);
        } else {
          dx[0] = dx[1] = 0.0;
          dy[0] = dy[1] = 0.0;
        }
      }
    } else {
      for (int e = tid; e < GK * GM; e += kGramThreads) {
        const int r = e / GM, c1 = e % GM;
        const int64_t gr = rb + r;
        double *dx = &sm.x[stage][r][c1];
        double *dy = &sm.y[stage][r][c1];
        if (gr < r1 && m0 + c1 < m) cp_async8(dx, X + gr * ldx + m0 + c1);
        else *dx = 0.0;
        if (gr < r1 && k0 + c1 < k) cp_async8(dy, Y + gr * ldy + k0 + c1);
        else *dy = 0.0;
      }
    }
    cp_async_commit();
  };
  if (nc > 0) load(0, 0);
  for (int c = 0; c < nc; ++c) {
    const int stage = c & 1;
    if (c + 1 < nc) {
      load(stage ^ 1, c + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < GK; ks += 4) {
      double a[4], b[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sm.x[stage][ks + t][wm + i * 8 + g];  // A = X^T
#pragma unroll
      for (int j = 0; j < 2; ++j) b[j] = sm.y[stage][ks + t][wk + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) mma_8x8x4(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
  // partial tile, column-major 64 x 64 within this CTA's slot
  double *pt = part + (((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * (GM * GN);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ii = wm + i * 8 + g, jj = wk + j * 8 + 2 * t + h;
        pt[ii + jj * GM] = acc[i][j][h];
      }
}

// C[i + j ldc] = alpha * sum_s part_s(i, j) + beta * C[i + j ldc], splits summed in order.
__global__ void gram_reduce_kernel(int m, int k, int tiles_m, int tiles_k, int splits,
                                   const double *__restrict__ part, double *C, int64_t ldc,
                                   double alpha, double beta, bool upper) {
  const int64_t total = (int64_t)m * k;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    const int bx = i / GM, by = j / GN, ii = i % GM, jj = j % GN;
    if (upper && bx > by) continue;  // its partials were never written
    double s = 0.0;
    for (int z = 0; z < splits; ++z)
      s += part[(((int64_t)z * tiles_k + by) * tiles_m + bx) * (GM * GN) + ii + jj * GM];
    double *c = C + i + (int64_t)j * ldc;
    *c = beta == 0.0 ? alpha * s : alpha * s + beta * *c;
  }
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

}  // namespace dmma

void dgemm_update(cudaStream_t st, int num_sms, int64_t n, int64_t m, int64_t p, const double *X,
                  int64_t ldx, const double *C, int64_t ldc, bool transC, double *Y, int64_t ldy,
                  double alpha, double beta) {
  using namespace dmma;
  if (n == 0 || p == 0) return;
  require(m <= INT32_MAX && p <= INT32_MAX, SMA_ERR_ARG, "product too wide");
  const bool vec16 = aligned16(X) && ldx % 2 == 0;
  const dim3 grid((unsigned)((n + UM - 1) / UM), (unsigned)((p + UN - 1) / UN));
  const size_t smem = sizeof(UpdateSmem);
  if (transC) {
    SMA_CUDA(cudaFuncSetAttribute(update_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    update_kernel<true><<<grid, kUpdateThreads, smem, st>>>(n, (int)m, (int)p, X, ldx, C, ldc, Y,
                                                           ldy, alpha, beta, vec16);
  } else {
    SMA_CUDA(cudaFuncSetAttribute(update_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    update_kernel<false><<<grid, kUpdateThreads, smem, st>>>(n, (int)m, (int)p, X, ldx, C, ldc, Y,
                                                            ldy, alpha, beta, vec16);
  }
  SMA_CHECK_LAUNCH();
  (void)num_sms;
}

void dgemm_gram(cudaStream_t st, int num_sms, int64_t n, int64_t m, int64_t k, const double *X,
                int64_t ldx, const double *Y, int64_t ldy, double *C, int64_t ldc, double alpha,
                double beta, DevBuf<double> &work, bool upper) {
  using namespace dmma;
  if (m == 0 || k == 0) return;
  require(m <= INT32_MAX && k <= INT32_MAX, SMA_ERR_ARG, "product too wide");
  const int tm = (int)((m + GM - 1) / GM), tk = (int)((k + GN - 1) / GN);
  // about two CTAs per SM over the whole grid, each summing at least 256 rows
  const int64_t want = std::max<int64_t>(1, (2LL * num_sms) / ((int64_t)tm * tk));
  const int64_t splits = std::max<int64_t>(1, std::min<int64_t>(want, (n + 255) / 256));
  const int64_t rows = (n + splits - 1) / splits;
  const size_t need = (size_t)splits * tm * tk * GM * GN;
  if (work.count < need) work.alloc(need, st);
  const bool vec16 = aligned16(X) && aligned16(Y) && ldx % 2 == 0 && ldy % 2 == 0;
  const size_t smem = sizeof(GramSmem);
  SMA_CUDA(cudaFuncSetAttribute(gram_partial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gram_partial_kernel<<<dim3(tm, tk, (unsigned)splits), kGramThreads, smem, st>>>(
      n, (int)m, (int)k, X, ldx, Y, ldy, rows, work.p, vec16, upper && m == k);
  SMA_CHECK_LAUNCH();
  const int64_t total = m * k;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4LL * num_sms);
  gram_reduce_kernel<<<blocks, 256, 0, st>>>((int)m, (int)k, tm, tk, (int)splits, work.p, C, ldc,
                                             alpha, beta, upper && m == k);
  SMA_CHECK_LAUNCH();
}

}  // namespace sma
