// The whole block Clenshaw recurrence in ONE cooperative launch (persistent kernel).
//
// Every CTA stays resident for all K+1 steps and owns the row tiles blockIdx.x,
// blockIdx.x + gridDim.x, ...; between steps all CTAs meet at a grid barrier.  This removes
// the per-step launch and the drain/fill of a kernel boundary, which dominate when a step
// is short (a matrix and block that live in L2: the C2 configuration's steps take
// ~17 us).  Each step computes exactly what the fused step kernel of csr_clenshaw.cuh
// computes, with the same FMA order, so the results are bit-identical to the step-by-step
// filter.
//
// Coherence.  The three rotating recurrence blocks are written by other CTAs during the
// launch, and L1 is not coherent across SMs, so every read of them goes through L2
// (ld.global.cg); Q and the CSR arrays are read-only during the launch (ld.global.nc).
//
// The grid barrier is a counter plus a generation word.  Its wait is bounded by elapsed
// time, read from the %globaltimer nanosecond clock: a CTA that has waited longer than the
// limit (one second for the filter), or sees another CTA's error flag, sets the error flag
// and returns; the host reads the flag after the launch and reports SMA_ERR_TIMEOUT.  A
// spin count far beyond any real wait backs the clock up, so the loop ends even if the
// clock stood still.  The launch is cooperative (cudaLaunchCooperativeKernel), so all CTAs
// are co-resident or the launch fails without running.
#include <cuda_runtime.h>

#include <algorithm>

#include "sma_internal.h"
#include "vec.cuh"

namespace sma {
namespace persist {

constexpr int kThreads = 256;

// ---- L2-only vector loads for the blocks written during the launch
template <typename T, int V>
__device__ __forceinline__ void ldcg1(const T *p, T *f) {
  using VT = typename Vec<T, V>::type;
  const VT x = __ldcg(reinterpret_cast<const VT *>(p));
  if constexpr (V == 1) {
    f[0] = x;
  } else if constexpr (V == 2) {
    f[0] = x.x; f[1] = x.y;
  } else {
    f[0] = x.x; f[1] = x.y; f[2] = x.z; f[3] = x.w;
  }
}

template <typename T, int V>
__device__ __forceinline__ void ldcg(const T *p, T (&f)[V]) {
  constexpr int kPer = (V * (int)sizeof(T) <= 16) ? V : 16 / (int)sizeof(T);
#pragma unroll
  for (int k = 0; k < V / kPer; ++k) ldcg1<T, kPer>(p + k * kPer, f + k * kPer);
}

// R consecutive CSR entries from j, all gathers in flight before the FMAs (ascending order)
template <typename T, int V, int R>
__device__ __forceinline__ void chunk(const int *__restrict__ cols, const T *__restrict__ vals,
                                      int j, const T *B1c, int64_t ldb, T (&acc)[V]) {
  int c[R];
  T x[R][V], a[R];
#pragma unroll
  for (int u = 0; u < R; ++u) c[u] = __ldg(cols + j + u);
#pragma unroll
  for (int u = 0; u < R; ++u) ldcg<T, V>(B1c + (int64_t)c[u] * ldb, x[u]);
#pragma unroll
  for (int u = 0; u < R; ++u) a[u] = __ldg(vals + j + u);
#pragma unroll
  for (int u = 0; u < R; ++u)
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = fma(a[u], x[u][v], acc[v]);
}

template <typename T, int V, int U>
__device__ __forceinline__ void row_product(const int *__restrict__ cols, const T *__restrict__ vals,
                                            int start, int end, const T *B1c, int64_t ldb,
                                            T (&acc)[V]) {
  int j = start;
  for (; j + U <= end; j += U) chunk<T, V, U>(cols, vals, j, B1c, ldb, acc);
  switch (end - j) {
    case 7: if constexpr (U > 7) chunk<T, V, 7>(cols, vals, j, B1c, ldb, acc); break;
    case 6: if constexpr (U > 6) chunk<T, V, 6>(cols, vals, j, B1c, ldb, acc); break;
    case 5: if constexpr (U > 5) chunk<T, V, 5>(cols, vals, j, B1c, ldb, acc); break;
    case 4: if constexpr (U > 4) chunk<T, V, 4>(cols, vals, j, B1c, ldb, acc); break;
    case 3: chunk<T, V, 3>(cols, vals, j, B1c, ldb, acc); break;
    case 2: chunk<T, V, 2>(cols, vals, j, B1c, ldb, acc); break;
    case 1: chunk<T, V, 1>(cols, vals, j, B1c, ldb, acc); break;
    default: break;
  }
}

struct Barrier {
  unsigned *count;
  unsigned *gen;
  int *err;
  unsigned nblocks;
  unsigned long long max_wait_ns;  // give up after this much elapsed time
};

// Spins of 100 ns sleeps after which a wait gives up whatever the clock says (2^34 spins
// take far longer than any wait limit used here).
constexpr unsigned long long kSpinBackstop = 1ull << 34;

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// All CTAs meet; returns false (in every thread of the CTA) when the wait gave up.
__device__ __forceinline__ bool grid_sync(const Barrier &bar) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = *reinterpret_cast<volatile unsigned *>(bar.gen);
    __threadfence();  // this CTA's writes of the step are visible before it arrives
    const unsigned arrived = atomicAdd(bar.count, 1u) + 1u;
    if (arrived == bar.nblocks) {
      atomicExch(bar.count, 0u);
      __threadfence();
      atomicAdd(bar.gen, 1u);
    } else {
      unsigned long long spins = 0;
      const unsigned long long t0 = globaltimer_ns();
      while (*reinterpret_cast<volatile unsigned *>(bar.gen) == g) {
        if (globaltimer_ns() - t0 > bar.max_wait_ns || ++spins > kSpinBackstop ||
            *reinterpret_cast<volatile int *>(bar.err) != 0) {
          atomicExch(bar.err, 1);
          ok = 0;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <typename T, int V, int G, int U>
__global__ void __launch_bounds__(kThreads)
clenshaw_persistent_kernel(const int *__restrict__ rowptr, const int *__restrict__ colind,
                           const T *__restrict__ val, int n, int b, const T *__restrict__ Q,
                           int64_t ldq, T *buf0, T *buf1, T *buf2, T *Y, int64_t ldy,
                           const T *__restrict__ coeffs, int K, T alpha, T beta, T invd,
                           T beta_last, Barrier bar) {
  constexpr int kRows = kThreads / G;
  const int ntiles = (n + kRows - 1) / kRows;
  const int lane = threadIdx.x % G;
  const int64_t ldb = b;
  T *B1 = buf0, *B2 = buf1, *TMP = buf2;
  {  // index K+1 of the reference: B1 = c_K Q
    const T ck = coeffs[K];
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      const int row = tile * kRows + (int)threadIdx.x / G;
      if (row >= n) continue;
      for (int c0 = lane * V; c0 < b; c0 += G * V) {
        T q[V], r[V];
        ldv<T, V>(Q + (int64_t)row * ldq + c0, q);
#pragma unroll
        for (int v = 0; v < V; ++v) r[v] = mul_rn(ck, q[v]);
        stv<T, V>(B1 + (int64_t)row * ldb + c0, r);
      }
    }
  }
  if (!grid_sync(bar)) return;
  for (int ci = K - 1; ci >= 0; --ci) {
    const bool last = ci == 0;
    const bool has_b2 = ci != K - 1;
    T *out = last ? Y : TMP;
    const int64_t ldo = last ? ldy : ldb;
    const T a = last ? invd : alpha;
    const T bt = last ? beta_last : beta;
    const T ck = coeffs[ci];
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      const int row = tile * kRows + (int)threadIdx.x / G;
      if (row >= n) continue;
      const int start = __ldg(rowptr + row), end = __ldg(rowptr + row + 1);
      for (int c0 = lane * V; c0 < b; c0 += G * V) {
        T q[V], s[V], t[V], acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = T(0);
        ldv<T, V>(Q + (int64_t)row * ldq + c0, q);
        ldcg<T, V>(B1 + (int64_t)row * ldb + c0, s);
        if (has_b2) ldcg<T, V>(B2 + (int64_t)row * ldb + c0, t);
        row_product<T, V, U>(colind, val, start, end, B1 + c0, ldb, acc);
        T r[V];
#pragma unroll
        for (int v = 0; v < V; ++v)
          r[v] = has_b2 ? clenshaw_combine<true, true, true>(acc[v], q[v], s[v], t[v], ck, a, bt)
                        : clenshaw_combine<true, true, false>(acc[v], q[v], s[v], T(0), ck, a, bt);
        stv<T, V>(out + (int64_t)row * ldo + c0, r);
      }
    }
    if (last) break;
    if (!grid_sync(bar)) return;
    T *tt = B2;  // B1, B2, TMP = TMP, B1, B2
    B2 = B1;
    B1 = TMP;
    TMP = tt;
  }
}

template <typename T, int V, int G>
int launch(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq, T *buf0,
           T *buf1, T *buf2, T *Y, int64_t ldy, const T *coeffs, int K, double alpha,
           double beta, double invd, double beta_last, unsigned *barrier_words, int *err) {
  auto kern = clenshaw_persistent_kernel<T, V, G, 8>;
  int per_sm = 0;
  SMA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0));
  require(per_sm >= 1, SMA_ERR_INTERNAL, "persistent filter kernel cannot be resident");
  constexpr int kRows = kThreads / G;
  const int64_t ntiles = (op->n + kRows - 1) / kRows;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)per_sm * op->ctx->num_sms));
  const T *val;
  if constexpr (sizeof(T) == 8) val = (const T *)op->val64;
  else val = (const T *)op->val32;
  int n = (int)op->n, bi = (int)b, Ki = K;
  T a = (T)alpha, bt = (T)beta, id = (T)invd, bl = (T)beta_last;
  Barrier bar{barrier_words, barrier_words + 1, err, grid, 1000000000ull};  // 1 s
  void *args[] = {(void *)&op->rowptr, (void *)&op->colind, (void *)&val, &n, &bi, (void *)&Q,
                  &ldq, &buf0, &buf1, &buf2, &Y, &ldy, (void *)&coeffs, &Ki, &a, &bt, &id, &bl,
                  &bar};
  SMA_CUDA(cudaLaunchCooperativeKernel((const void *)kern, dim3(grid), dim3(kThreads), args, 0, st));
  SMA_CHECK_LAUNCH();
  return (int)grid;
}

template <typename T, int V>
int launch_g(int G, const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq, T *b0,
             T *b1, T *b2, T *Y, int64_t ldy, const T *c, int K, double al, double be,
             double id, double bl, unsigned *w, int *e) {
  switch (G) {
    case 4: return launch<T, V, 4>(op, st, b, Q, ldq, b0, b1, b2, Y, ldy, c, K, al, be, id, bl, w, e);
    case 8: return launch<T, V, 8>(op, st, b, Q, ldq, b0, b1, b2, Y, ldy, c, K, al, be, id, bl, w, e);
    case 16: return launch<T, V, 16>(op, st, b, Q, ldq, b0, b1, b2, Y, ldy, c, K, al, be, id, bl, w, e);
    default: return launch<T, V, 32>(op, st, b, Q, ldq, b0, b1, b2, Y, ldy, c, K, al, be, id, bl, w, e);
  }
}

}  // namespace persist

// Y = p(A_hat) Q for a CSR operator in one persistent launch (K >= 1).  All blocks are
// row-major with ld = b except Q (ldq) and Y (ldy).  Synchronizes the stream to read the
// barrier's error flag.
template <typename T>
FilterCount persistent_filter(const sma_op *op, cudaStream_t st, const std::vector<double> &coeffs,
                              double smin, double smax, const T *Q, int64_t ldq, T *Y, int64_t ldy,
                              int64_t b, T *buf0, T *buf1, T *buf2, T *coeff_dev,
                              unsigned *barrier_words) {
  FilterCount fc;
  const int64_t n = op->n;
  const int K = (int)coeffs.size() - 1;
  require(op->kind == OP_CSR && K >= 1, SMA_ERR_INTERNAL, "persistent filter needs CSR and K >= 1");
  const double c = 0.5 * (smin + smax), invd = 2.0 / (smax - smin);
  std::vector<T> ch(coeffs.size());
  for (size_t i = 0; i < coeffs.size(); ++i) ch[i] = (T)coeffs[i];
  SMA_CUDA(cudaMemcpyAsync(coeff_dev, ch.data(), ch.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  SMA_CUDA(cudaMemsetAsync(barrier_words, 0, 3 * sizeof(unsigned), st));
  auto aligned = [](const void *p, int bytes) { return ((uintptr_t)p % bytes) == 0; };
  int V = 1;
  for (int v : {2, 4}) {
    const int bytes = v * (int)sizeof(T);
    if (bytes <= 16 && b % v == 0 && ldq % v == 0 && ldy % v == 0 && aligned(Q, bytes) &&
        aligned(Y, bytes) && aligned(buf0, bytes) && aligned(buf1, bytes) && aligned(buf2, bytes))
      V = v;
  }
  const int64_t lanes = (b + V - 1) / V;
  const int G = lanes <= 4 ? 4 : lanes <= 8 ? 8 : lanes <= 16 ? 16 : 32;
  int *err = reinterpret_cast<int *>(barrier_words + 2);
  const double al = 2.0 * invd, be = -2.0 * c * invd, bl = -(c * invd);
  if (V == 1)
    persist::launch_g<T, 1>(G, op, st, b, Q, ldq, buf0, buf1, buf2, Y, ldy, coeff_dev, K, al, be, invd, bl, barrier_words, err);
  else if (V == 2)
    persist::launch_g<T, 2>(G, op, st, b, Q, ldq, buf0, buf1, buf2, Y, ldy, coeff_dev, K, al, be, invd, bl, barrier_words, err);
  else if constexpr (sizeof(T) == 4)
    persist::launch_g<T, 4>(G, op, st, b, Q, ldq, buf0, buf1, buf2, Y, ldy, coeff_dev, K, al, be, invd, bl, barrier_words, err);
  else
    throw Error(SMA_ERR_INTERNAL, "bad persistent vector width");
  int herr = 0;
  SMA_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  if (herr) throw Error(SMA_ERR_TIMEOUT, "persistent filter: a grid barrier wait gave up");
  const double blk = (double)n * (double)b * sizeof(T);
  const double mat = clenshaw_step_bytes(op, 0, sizeof(T));
  fc.steps = K;
  fc.bytes = 2 * blk + (mat + 3 * blk) + (double)(K - 1) * (mat + 4 * blk);
  return fc;
}

namespace persist {
// A grid barrier that can never complete: `expected` CTAs are awaited, fewer are launched.
__global__ void barrier_selftest_kernel(Barrier bar) {
  grid_sync(bar);
}
}  // namespace persist

// Runs the barrier with one CTA missing and a 10 ms wait limit; returns SMA_ERR_TIMEOUT
// when the wait gave up and reported it through the error flag (the expected outcome).
int barrier_selftest(sma_ctx *ctx) {
  cudaStream_t st = ctx->stream;
  DevBuf<unsigned> words(3, st);
  SMA_CUDA(cudaMemsetAsync(words.p, 0, 3 * sizeof(unsigned), st));
  const unsigned launched = 2;
  persist::Barrier bar{words.p, words.p + 1, reinterpret_cast<int *>(words.p + 2), launched + 1,
                       10000000ull};  // 10 ms
  void *args[] = {&bar};
  SMA_CUDA(cudaLaunchCooperativeKernel((const void *)persist::barrier_selftest_kernel,
                                       dim3(launched), dim3(persist::kThreads), args, 0, st));
  SMA_CHECK_LAUNCH();
  int herr = 0;
  SMA_CUDA(cudaMemcpyAsync(&herr, words.p + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  return herr ? SMA_ERR_TIMEOUT : SMA_OK;
}

template FilterCount persistent_filter<double>(const sma_op *, cudaStream_t, const std::vector<double> &,
                                               double, double, const double *, int64_t, double *,
                                               int64_t, int64_t, double *, double *, double *,
                                               double *, unsigned *);
template FilterCount persistent_filter<float>(const sma_op *, cudaStream_t, const std::vector<double> &,
                                              double, double, const float *, int64_t, float *,
                                              int64_t, int64_t, float *, float *, float *, float *,
                                              unsigned *);

}  // namespace sma
