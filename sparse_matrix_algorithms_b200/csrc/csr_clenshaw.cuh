// The fused CSR Clenshaw step and its online autotuner (included by csr_clenshaw_f64.cu and
// csr_clenshaw_f32.cu, one translation unit per element type).
//
//   out[i, :] = ck*Q[i, :] + alpha * sum_j A[i,j] B1[j, :] + beta*B1[i, :] - B2[i, :]
//
// One CTA of 256 threads owns 256/G consecutive rows; a group of G threads owns one row and
// each thread covers V consecutive columns of every G*V-wide column pass (V*sizeof(T) is
// 8..32 bytes: one or two 16-byte loads per neighbour row).  Gathers are issued U at a
// time so that U neighbour rows are in flight per thread, and the epilogue operands (the
// row of Q, B1, B2) are requested before the gathers.  Two families differ in how a
// thread obtains its row's (column, value) pairs:
//   DIRECT  every thread reads them itself; the G lanes of a group read the same
//           addresses, which the L1 cache serves as one broadcast;
//   STAGED  the CTA first copies the pairs of all its rows (one contiguous CSR range)
//           into shared memory with coalesced loads, then reads them from there.
// Both families are launched as programmatic dependents of the previous step (when the
// context allows it): a CTA first lets the next step's grid be scheduled, reads what no
// step writes (its CSR rows and the row of Q), and only then waits for the previous grid
// to complete (griddepcontrol.wait) before it reads B1 or B2 or writes anything -- so the
// next step's CTAs fill the SMs that this step's last wave leaves idle.  Launched without
// the attribute, both instructions are no-ops.
// Every configuration accumulates with FMA in ascending column order -- the order of the
// reference's CSC product on a symmetric matrix -- so all configurations write
// bit-identical results, and the autotuner may run real recurrence steps with different
// configurations while it measures them.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "sma_internal.h"
#include "vec.cuh"

namespace sma {
namespace csr {

constexpr int kThreads = 256;
constexpr int kStage = 1024;  // CSR entries a STAGED CTA keeps in shared memory

template <typename T, int V, bool HQ, bool HS, bool HB>
__device__ __forceinline__ void epilogue(T *__restrict__ out, const T (&acc)[V], const T (&q)[V],
                                         const T (&s)[V], const T (&t)[V], const T (&ck)[V],
                                         T alpha, T beta) {
  T r[V];
#pragma unroll
  for (int v = 0; v < V; ++v)
    r[v] = clenshaw_combine<HQ, HS, HB>(acc[v], q[v], s[v], t[v], ck[v], alpha, beta);
  stv<T, V>(out, r);
}

// The Q coefficient of each of a thread's V columns c0 .. c0+V-1: the step's scalar ck, or
// (PC) the coefficient of the column's segment, cseg[colseg[c]].
template <typename T, int V, bool PC>
__device__ __forceinline__ void coeffs_of(T (&ckv)[V], T ck, const T *__restrict__ cseg,
                                          const int *__restrict__ colseg, int c0) {
#pragma unroll
  for (int v = 0; v < V; ++v) {
    if constexpr (PC) ckv[v] = __ldg(cseg + __ldg(colseg + c0 + v));
    else ckv[v] = ck;
  }
}

// R consecutive entries from j: all R gathers are issued before the first FMA, so R
// neighbour rows are in flight at once; FMAs in ascending entry order.
template <typename T, int V, int R>
__device__ __forceinline__ void chunk(const int *__restrict__ cols, const T *__restrict__ vals,
                                      int off, int j, const T *__restrict__ B1c, int64_t ldb,
                                      T (&acc)[V]) {
  int c[R];
  T x[R][V], a[R];
#pragma unroll
  for (int u = 0; u < R; ++u) c[u] = cols[j + u - off];
#pragma unroll
  for (int u = 0; u < R; ++u) ldv<T, V>(B1c + (int64_t)c[u] * ldb, x[u]);
#pragma unroll
  for (int u = 0; u < R; ++u) a[u] = vals[j + u - off];
#pragma unroll
  for (int u = 0; u < R; ++u)
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = fma(a[u], x[u][v], acc[v]);
}

// acc += sum over the row's entries j in [start, end) of vals[j-off] * B1c[cols[j-off] * ldb]:
// chunks of U, then the r < U remaining entries as ONE chunk of exactly r (a switch over
// r), so that a row shorter than U -- the 7-entry rows of the Anderson lattice under
// U = 8 -- still has all its gathers in flight together.
template <typename T, int V, int U>
__device__ __forceinline__ void row_product(const int *__restrict__ cols, const T *__restrict__ vals,
                                            int off, int start, int end, const T *__restrict__ B1c,
                                            int64_t ldb, T (&acc)[V]) {
  int j = start;
  for (; j + U <= end; j += U) chunk<T, V, U>(cols, vals, off, j, B1c, ldb, acc);
  switch (end - j) {
    case 7: if constexpr (U > 7) chunk<T, V, 7>(cols, vals, off, j, B1c, ldb, acc); break;
    case 6: if constexpr (U > 6) chunk<T, V, 6>(cols, vals, off, j, B1c, ldb, acc); break;
    case 5: if constexpr (U > 5) chunk<T, V, 5>(cols, vals, off, j, B1c, ldb, acc); break;
    case 4: if constexpr (U > 4) chunk<T, V, 4>(cols, vals, off, j, B1c, ldb, acc); break;
    case 3: chunk<T, V, 3>(cols, vals, off, j, B1c, ldb, acc); break;
    case 2: chunk<T, V, 2>(cols, vals, off, j, B1c, ldb, acc); break;
    case 1: chunk<T, V, 1>(cols, vals, off, j, B1c, ldb, acc); break;
    default: break;
  }
}

// Programmatic dependent launch: let the next grid in the stream be scheduled; wait until
// the grids this one depends on have completed and their writes are visible.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename T, int V, int G, int U, bool HQ, bool HS, bool HB, bool PC>
__global__ void __launch_bounds__(kThreads)
direct_kernel(const int *__restrict__ rowptr, const int *__restrict__ colind,
              const T *__restrict__ val, int64_t n, int b, const T *__restrict__ Q, int64_t ldq,
              const T *__restrict__ B1, const T *__restrict__ B2, int64_t ldb,
              T *__restrict__ out, int64_t ldo, T ck, T alpha, T beta,
              const T *__restrict__ cseg, const int *__restrict__ colseg) {
  constexpr int kRows = kThreads / G;
  pdl_trigger();
  const int64_t row = (int64_t)blockIdx.x * kRows + threadIdx.x / G;
  const bool live = row < n;
  const int lane = threadIdx.x % G;
  int start = 0, end = 0;
  T q[V], s[V], t[V];
  if (live) {  // what no step writes: the CSR row and the first pass's row of Q
    start = __ldg(rowptr + row);
    end = __ldg(rowptr + row + 1);
    if constexpr (HQ) if (lane * V < b) ldv<T, V>(Q + row * ldq + lane * V, q);
  }
  pdl_wait();
  if (!live) return;
  for (int c0 = lane * V; c0 < b; c0 += G * V) {
    T acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = T(0);
    if constexpr (HQ) if (c0 != lane * V) ldv<T, V>(Q + row * ldq + c0, q);
    if constexpr (HS) ldv<T, V>(B1 + row * ldb + c0, s);
    if constexpr (HB) ldv<T, V>(B2 + row * ldb + c0, t);
    row_product<T, V, U>(colind, val, 0, start, end, B1 + c0, ldb, acc);
    T ckv[V];
    coeffs_of<T, V, PC>(ckv, ck, cseg, colseg, c0);
    epilogue<T, V, HQ, HS, HB>(out + row * ldo + c0, acc, q, s, t, ckv, alpha, beta);
  }
}

template <typename T, int V, int G, int U, bool HQ, bool HS, bool HB, bool PC>
__global__ void __launch_bounds__(kThreads)
staged_kernel(const int *__restrict__ rowptr, const int *__restrict__ colind,
              const T *__restrict__ val, int64_t n, int b, const T *__restrict__ Q, int64_t ldq,
              const T *__restrict__ B1, const T *__restrict__ B2, int64_t ldb,
              T *__restrict__ out, int64_t ldo, T ck, T alpha, T beta,
              const T *__restrict__ cseg, const int *__restrict__ colseg) {
  constexpr int kRows = kThreads / G;
  __shared__ int s_col[kStage];
  __shared__ T s_val[kStage];
  pdl_trigger();
  const int64_t row0 = (int64_t)blockIdx.x * kRows;
  const int64_t row = row0 + threadIdx.x / G;
  const int lane = threadIdx.x % G;
  const bool live = row < n;
  T q[V], s[V], t[V];
  if constexpr (HQ) if (live && lane * V < b) ldv<T, V>(Q + row * ldq + lane * V, q);
  const int64_t rlast = min(n, row0 + kRows);
  const int base = __ldg(rowptr + row0);
  const int top = __ldg(rowptr + rlast);
  const bool staged = top - base <= kStage;
  if (staged) {
    for (int i = threadIdx.x; i < top - base; i += kThreads) {
      s_col[i] = __ldg(colind + base + i);
      s_val[i] = __ldg(val + base + i);
    }
  }
  __syncthreads();
  pdl_wait();  // B1 and B2 come from the previous steps
  if (!live) return;  // no barrier follows
  const int start = __ldg(rowptr + row);
  const int end = __ldg(rowptr + row + 1);
  for (int c0 = lane * V; c0 < b; c0 += G * V) {
    T acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = T(0);
    if constexpr (HQ) if (c0 != lane * V) ldv<T, V>(Q + row * ldq + c0, q);
    if constexpr (HS) ldv<T, V>(B1 + row * ldb + c0, s);
    if constexpr (HB) ldv<T, V>(B2 + row * ldb + c0, t);
    if (staged) row_product<T, V, U>(s_col, s_val, base, start, end, B1 + c0, ldb, acc);
    else row_product<T, V, U>(colind, val, 0, start, end, B1 + c0, ldb, acc);
    T ckv[V];
    coeffs_of<T, V, PC>(ckv, ck, cseg, colseg, c0);
    epilogue<T, V, HQ, HS, HB>(out + row * ldo + c0, acc, q, s, t, ckv, alpha, beta);
  }
}

// ASYNC family: every thread moves exactly 16 bytes (V = 16/sizeof(T) elements) of each
// neighbour row it needs with cp.async (global -> shared, asynchronous), for up to NB
// neighbours at a time plus the epilogue rows of Q, B1 and B2, then waits for its own
// copies only and computes from shared memory.  All of a row's gathers are in flight at
// once without holding registers, so a row costs one memory latency.  Each thread reads
// back only the chunks it copied itself, so no barrier is needed.  CTAs are 128 threads;
// shared memory per CTA is (NB + 3) * 128 * 16 bytes (22.5 KB for NB = 8, 38.9 KB for 16).
constexpr int kAsyncThreads = 128;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <typename T, int G, int NB, bool HQ, bool HS, bool HB>
__global__ void __launch_bounds__(kAsyncThreads)
async_kernel(const int *__restrict__ rowptr, const int *__restrict__ colind,
             const T *__restrict__ val, int64_t n, int b, const T *__restrict__ Q, int64_t ldq,
             const T *__restrict__ B1, const T *__restrict__ B2, int64_t ldb,
             T *__restrict__ out, int64_t ldo, T ck, T alpha, T beta) {
  constexpr int V = 16 / (int)sizeof(T);
  constexpr int kRows = kAsyncThreads / G;
  __shared__ uint4 buf[NB + 3][kAsyncThreads];  // slot-major: a warp's copies are contiguous
  const int64_t row = (int64_t)blockIdx.x * kRows + threadIdx.x / G;
  if (row >= n) return;
  const int tid = threadIdx.x;
  const int lane = tid % G;
  const int start = __ldg(rowptr + row);
  const int end = __ldg(rowptr + row + 1);
  for (int c0 = lane * V; c0 < b; c0 += G * V) {
    if constexpr (HQ) cp_async16(&buf[NB][tid], Q + row * ldq + c0);
    if constexpr (HS) cp_async16(&buf[NB + 1][tid], B1 + row * ldb + c0);
    if constexpr (HB) cp_async16(&buf[NB + 2][tid], B2 + row * ldb + c0);
    T acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = T(0);
    for (int j0 = start; j0 < end; j0 += NB) {
      const int cnt = min(NB, end - j0);
      for (int u = 0; u < cnt; ++u)
        cp_async16(&buf[u][tid], B1 + (int64_t)__ldg(colind + j0 + u) * ldb + c0);
      cp_async_wait_all();
      for (int u = 0; u < cnt; ++u) {
        const T a = __ldg(val + j0 + u);
        const T *x = reinterpret_cast<const T *>(&buf[u][tid]);
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = fma(a, x[v], acc[v]);
      }
    }
    cp_async_wait_all();  // epilogue rows of an empty row
    T q[V], s[V], t[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if constexpr (HQ) q[v] = reinterpret_cast<const T *>(&buf[NB][tid])[v];
      if constexpr (HS) s[v] = reinterpret_cast<const T *>(&buf[NB + 1][tid])[v];
      if constexpr (HB) t[v] = reinterpret_cast<const T *>(&buf[NB + 2][tid])[v];
    }
    T ckv[V];
    coeffs_of<T, V, false>(ckv, ck, nullptr, nullptr, c0);
    epilogue<T, V, HQ, HS, HB>(out + row * ldo + c0, acc, q, s, t, ckv, alpha, beta);
  }
}

// BULK family: a CTA of kBulkThreads threads owns RC = kBulkThreads / G rows (G threads of V
// elements each cover a row in ONE pass, b = G V) and first stages everything its step
// reads into shared memory: its CSR pairs (plain coalesced loads), then with 1D bulk copies
// (cp.async.bulk global -> this CTA's shared memory; no multicast, local memory only) the
// rows of Q, B1 and B2 it updates and every neighbour row of B1 its pairs name, all
// completing on one mbarrier.  Every row a CTA needs is in flight at once without holding
// registers, and the arithmetic reads shared memory only, in the same order as the other
// families (bit-identical results).  Whole rows move, so rows must be 16..512 bytes and all
// leading dimensions multiples of 16 bytes.  The host sizes the shared memory for the
// largest CTA of the operator.  The wait on the mbarrier is bounded by elapsed time
// (%globaltimer, one second): a CTA that gives up sets *err, waits (bounded again) for its
// copies, and returns without writing; the host then reports SMA_ERR_TIMEOUT.
constexpr int kBulkThreads = 256;
constexpr unsigned long long kBulkWaitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long bulk_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void bulk_copy(void *smem_dst, const void *gsrc, unsigned bytes,
                                          unsigned mbar) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
      ::"r"(d), "l"(gsrc), "r"(bytes), "r"(mbar) : "memory");
}

// Waits for phase 0 of the mbarrier; false when `limit_ns` of elapsed time passed first.
__device__ __forceinline__ bool bulk_wait(unsigned mbar, unsigned long long limit_ns) {
  const unsigned long long t0 = bulk_clock_ns();
  for (unsigned long long spin = 0;; ++spin) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(mbar) : "memory");
    if (done) return true;
    if (bulk_clock_ns() - t0 > limit_ns || spin > (1ull << 34)) return false;
  }
}

template <typename T, int V, int G, bool HQ, bool HS, bool HB>
__global__ void __launch_bounds__(kBulkThreads)
bulk_kernel(const int *__restrict__ rowptr, const int *__restrict__ colind,
            const T *__restrict__ val, int64_t n, int b, const T *__restrict__ Q, int64_t ldq,
            const T *__restrict__ B1, const T *__restrict__ B2, int64_t ldb,
            T *__restrict__ out, int64_t ldo, T ck, T alpha, T beta, int cap, int *err) {
  constexpr int RC = kBulkThreads / G;
  constexpr int NR = (HQ ? 1 : 0) + (HS ? 1 : 0) + (HB ? 1 : 0);
  extern __shared__ __align__(16) unsigned char bulk_smem[];
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(bulk_smem);
  T *rows = reinterpret_cast<T *>(bulk_smem + 16);  // NR x RC rows: Q, B1, B2 (those present)
  T *nbr = rows + (size_t)NR * RC * b;               // cap neighbour rows
  T *sval = nbr + (size_t)cap * b;
  int *scol = reinterpret_cast<int *>(sval + cap);
  const unsigned mbar = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  const unsigned rb = (unsigned)b * sizeof(T);
  const int64_t row0 = (int64_t)blockIdx.x * RC;
  const int nrows = (int)min((int64_t)RC, n - row0);
  const int base = __ldg(rowptr + row0);
  const int cnt = __ldg(rowptr + row0 + nrows) - base;
  if (cnt > cap) {  // the host sized shared memory for the largest CTA: never taken
    if (threadIdx.x == 0) atomicExch(err, 2);
    return;
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int i = threadIdx.x; i < cnt; i += kBulkThreads) {
    scol[i] = __ldg(colind + base + i);
    sval[i] = __ldg(val + base + i);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned bytes = ((unsigned)cnt + (unsigned)(NR * nrows)) * rb;
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
                 ::"r"(mbar), "r"(bytes) : "memory");
  }
  __syncthreads();
  for (int i = threadIdx.x; i < cnt; i += kBulkThreads)
    bulk_copy(nbr + (size_t)i * b, B1 + (int64_t)scol[i] * ldb, rb, mbar);
  {
    int slot = 0;
    const T *src[3];
    int64_t ld[3];
    if constexpr (HQ) { src[slot] = Q; ld[slot] = ldq; ++slot; }
    if constexpr (HS) { src[slot] = B1; ld[slot] = ldb; ++slot; }
    if constexpr (HB) { src[slot] = B2; ld[slot] = ldb; ++slot; }
    for (int e = threadIdx.x; e < NR * nrows; e += kBulkThreads) {
      const int k = e / nrows, r = e % nrows;
      bulk_copy(rows + ((size_t)k * RC + r) * b, src[k] + (row0 + r) * ld[k], rb, mbar);
    }
  }
  if (!bulk_wait(mbar, kBulkWaitNs)) {
    if (threadIdx.x == 0) atomicExch(err, 1);
    bulk_wait(mbar, kBulkWaitNs);  // let the copies in flight land before the CTA exits
    return;
  }
  const int r = threadIdx.x / G;
  if (r >= nrows) return;
  const int c0 = (threadIdx.x % G) * V;
  const int64_t row = row0 + r;
  const int start = __ldg(rowptr + row) - base, end = __ldg(rowptr + row + 1) - base;
  T acc[V], q[V], sv[V], t[V], ckv[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = T(0);
    ckv[v] = ck;
  }
  for (int e = start; e < end; ++e) {
    const T a = sval[e];
    const T *x = nbr + (size_t)e * b + c0;
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = fma(a, x[v], acc[v]);
  }
  int slot = 0;
  if constexpr (HQ) {
#pragma unroll
    for (int v = 0; v < V; ++v) q[v] = rows[((size_t)slot * RC + r) * b + c0 + v];
    ++slot;
  }
  if constexpr (HS) {
#pragma unroll
    for (int v = 0; v < V; ++v) sv[v] = rows[((size_t)slot * RC + r) * b + c0 + v];
    ++slot;
  }
  if constexpr (HB) {
#pragma unroll
    for (int v = 0; v < V; ++v) t[v] = rows[((size_t)slot * RC + r) * b + c0 + v];
  }
  epilogue<T, V, HQ, HS, HB>(out + row * ldo + c0, acc, q, sv, t, ckv, alpha, beta);
}

// ------------------------------------------------------------------ configurations
// Encoded as fam | V << 4 | G << 8 | U << 16 (for the ASYNC family U is NB).
inline int enc(int fam, int V, int G, int U) { return fam | (V << 4) | (G << 8) | (U << 16); }
inline int fam_of(int c) { return c & 15; }
inline int v_of(int c) { return (c >> 4) & 15; }
inline int g_of(int c) { return (c >> 8) & 255; }
inline int u_of(int c) { return c >> 16; }

template <typename T>
struct Args {
  const sma_op *op;
  cudaStream_t st;
  int64_t b;
  const T *Q;
  int64_t ldq;
  const T *B1, *B2;
  int64_t ldb;
  T *out;
  int64_t ldo;
  double ck, alpha, beta;
  // per-segment coefficients of this step (cseg[segment]) and the segment of every column
  // (colseg[column]); null for one coefficient.  Batched spectrum slicing maps a window's
  // columns to its segment; the POLFED polish gives every column its own polynomial.
  const T *cseg = nullptr;
  const int *colseg = nullptr;
};

// Launch of a DIRECT or STAGED step: as a programmatic dependent of the previous launch in
// the stream when the context allows it (the kernels wait for their predecessor before
// they touch B1, B2 or the output), else an ordinary launch.
template <typename... KArgs, typename... Args>
void launch_step(const sma_op *op, void (*kernel)(KArgs...), unsigned grid, cudaStream_t st,
                 Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = op->ctx->pdl ? 1 : 0;
  SMA_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
  SMA_CHECK_LAUNCH();
}

template <typename T, int V, int G, int U, bool HQ, bool HS, bool HB>
void launch_one(int fam, const Args<T> &a) {
  const T *val;
  if constexpr (sizeof(T) == 8) val = (const T *)a.op->val64;
  else val = (const T *)a.op->val32;
  constexpr int kRows = kThreads / G;
  const unsigned grid = (unsigned)((a.op->n + kRows - 1) / kRows);
  const sma_op *op = a.op;
  if constexpr (HQ && HS && HB) {
    if (a.cseg) {
      auto k = fam == 0 ? direct_kernel<T, V, G, U, true, true, true, true>
                        : staged_kernel<T, V, G, U, true, true, true, true>;
      return launch_step(op, k, grid, a.st, op->rowptr, op->colind, val, op->n, (int)a.b, a.Q,
                         a.ldq, a.B1, a.B2, a.ldb, a.out, a.ldo, T(0), (T)a.alpha, (T)a.beta,
                         a.cseg, a.colseg);
    }
  }
  if (a.cseg) throw Error(SMA_ERR_INTERNAL, "segmented Clenshaw step needs the full variant");
  auto k = fam == 0 ? direct_kernel<T, V, G, U, HQ, HS, HB, false>
                    : staged_kernel<T, V, G, U, HQ, HS, HB, false>;
  launch_step(op, k, grid, a.st, op->rowptr, op->colind, val, op->n, (int)a.b, a.Q, a.ldq, a.B1,
              a.B2, a.ldb, a.out, a.ldo, (T)a.ck, (T)a.alpha, (T)a.beta, (const T *)nullptr,
              (const int *)nullptr);
}

template <typename T, int G, int NB, bool HQ, bool HS, bool HB>
void launch_async(const Args<T> &a) {
  if (a.cseg) throw Error(SMA_ERR_INTERNAL, "the asynchronous family has no segmented variant");
  const T *val;
  if constexpr (sizeof(T) == 8) val = (const T *)a.op->val64;
  else val = (const T *)a.op->val32;
  constexpr int kRows = kAsyncThreads / G;
  const unsigned grid = (unsigned)((a.op->n + kRows - 1) / kRows);
  async_kernel<T, G, NB, HQ, HS, HB><<<grid, kAsyncThreads, 0, a.st>>>(
      a.op->rowptr, a.op->colind, val, a.op->n, (int)a.b, a.Q, a.ldq, a.B1, a.B2, a.ldb, a.out,
      a.ldo, (T)a.ck, (T)a.alpha, (T)a.beta);
  SMA_CHECK_LAUNCH();
}

// The most CSR entries held by any CTA of RC consecutive rows (cached per RC).
inline int bulk_max_pairs(const sma_op *op, int RC) {
  sma_op *o = const_cast<sma_op *>(op);
  const auto it = o->bulk_pairs.find(RC);
  if (it != o->bulk_pairs.end()) return it->second;
  if (o->host_rowptr.empty()) {
    o->host_rowptr.resize(op->n + 1);
    SMA_CUDA(cudaMemcpy(o->host_rowptr.data(), op->rowptr, (op->n + 1) * sizeof(int),
                        cudaMemcpyDeviceToHost));
  }
  int mx = 0;
  for (int64_t r = 0; r < op->n; r += RC) {
    const int64_t e = std::min<int64_t>(op->n, r + RC);
    mx = std::max(mx, o->host_rowptr[e] - o->host_rowptr[r]);
  }
  o->bulk_pairs[RC] = mx;
  return mx;
}

inline size_t bulk_smem_bytes(int RC, int nr, int b, int cap, size_t elem) {
  return 16 + (size_t)nr * RC * b * elem + (size_t)cap * (b * elem + elem + sizeof(int));
}

template <typename T, int V, int G, bool HQ, bool HS, bool HB>
void launch_bulk(const Args<T> &a) {
  if (a.cseg) throw Error(SMA_ERR_INTERNAL, "the bulk family has no segmented variant");
  const sma_op *op = a.op;
  if (a.b != (int64_t)G * V) throw Error(SMA_ERR_INTERNAL, "bulk family: b != G V");
  const T *val;
  if constexpr (sizeof(T) == 8) val = (const T *)op->val64;
  else val = (const T *)op->val32;
  constexpr int RC = kBulkThreads / G;
  constexpr int NR = (HQ ? 1 : 0) + (HS ? 1 : 0) + (HB ? 1 : 0);
  const int cap = std::max(1, bulk_max_pairs(op, RC));
  const size_t smem = bulk_smem_bytes(RC, NR, (int)a.b, cap, sizeof(T));
  require(op->bulk_err != nullptr, SMA_ERR_INTERNAL, "bulk family without its error flag");
  SMA_CUDA(cudaFuncSetAttribute(bulk_kernel<T, V, G, HQ, HS, HB>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const unsigned grid = (unsigned)((op->n + RC - 1) / RC);
  bulk_kernel<T, V, G, HQ, HS, HB><<<grid, kBulkThreads, smem, a.st>>>(
      op->rowptr, op->colind, val, op->n, (int)a.b, a.Q, a.ldq, a.B1, a.B2, a.ldb, a.out, a.ldo,
      (T)a.ck, (T)a.alpha, (T)a.beta, cap, op->bulk_err);
  SMA_CHECK_LAUNCH();
}

// Whether the BULK family can take this step: whole rows of 16..512 bytes, every leading
// dimension and base address on 16 bytes, and the largest CTA's rows within shared memory.
template <typename T, bool HQ, bool HS, bool HB>
bool bulk_fits(const Args<T> &a, int V) {
  const int64_t rb = a.b * (int64_t)sizeof(T);
  if (a.cseg || rb < 16 || rb > 512 || rb % 16 || a.b % V) return false;
  const int64_t G = a.b / V;
  if (G != 4 && G != 8 && G != 16 && G != 32) return false;
  auto al = [](const void *p) { return p == nullptr || ((uintptr_t)p & 15) == 0; };
  if ((a.ldb * sizeof(T)) % 16 || (HQ && (a.ldq * sizeof(T)) % 16) || !al(a.Q) || !al(a.B1) ||
      !al(a.B2))
    return false;
  const int RC = kBulkThreads / (int)G;
  const int nr = (HQ ? 1 : 0) + (HS ? 1 : 0) + (HB ? 1 : 0);
  const int cap = std::max(1, bulk_max_pairs(a.op, RC));
  return bulk_smem_bytes(RC, nr, (int)a.b, cap, sizeof(T)) <= 200 * 1024;
}

template <typename T, int V, bool HQ, bool HS, bool HB>
void launch_v(int c, const Args<T> &a) {
  const int fam = fam_of(c);
  if (fam == 3) {
    switch (g_of(c)) {
      case 4: return launch_bulk<T, V, 4, HQ, HS, HB>(a);
      case 8: return launch_bulk<T, V, 8, HQ, HS, HB>(a);
      case 16: return launch_bulk<T, V, 16, HQ, HS, HB>(a);
      case 32: return launch_bulk<T, V, 32, HQ, HS, HB>(a);
      default: throw Error(SMA_ERR_INTERNAL, "bad bulk CSR kernel configuration");
    }
  }
  if (fam == 2) {
    if constexpr (V * sizeof(T) == 16) {
      switch (g_of(c) * 100 + u_of(c)) {
        case 408: return launch_async<T, 4, 8, HQ, HS, HB>(a);
        case 416: return launch_async<T, 4, 16, HQ, HS, HB>(a);
        case 808: return launch_async<T, 8, 8, HQ, HS, HB>(a);
        case 816: return launch_async<T, 8, 16, HQ, HS, HB>(a);
        case 1608: return launch_async<T, 16, 8, HQ, HS, HB>(a);
        case 1616: return launch_async<T, 16, 16, HQ, HS, HB>(a);
        case 3208: return launch_async<T, 32, 8, HQ, HS, HB>(a);
        case 3216: return launch_async<T, 32, 16, HQ, HS, HB>(a);
        default: break;
      }
    }
    throw Error(SMA_ERR_INTERNAL, "bad asynchronous CSR kernel configuration");
  }
  switch (g_of(c) * 100 + u_of(c)) {
    case 404: return launch_one<T, V, 4, 4, HQ, HS, HB>(fam, a);
    case 408: return launch_one<T, V, 4, 8, HQ, HS, HB>(fam, a);
    case 804: return launch_one<T, V, 8, 4, HQ, HS, HB>(fam, a);
    case 808: return launch_one<T, V, 8, 8, HQ, HS, HB>(fam, a);
    case 1604: return launch_one<T, V, 16, 4, HQ, HS, HB>(fam, a);
    case 1608: return launch_one<T, V, 16, 8, HQ, HS, HB>(fam, a);
    case 3204: return launch_one<T, V, 32, 4, HQ, HS, HB>(fam, a);
    case 3208: return launch_one<T, V, 32, 8, HQ, HS, HB>(fam, a);
    default: throw Error(SMA_ERR_INTERNAL, "bad CSR kernel configuration");
  }
}

template <typename T, bool HQ, bool HS, bool HB>
void launch_cfg(int c, const Args<T> &a) {
  switch (v_of(c)) {
    case 1: return launch_v<T, 1, HQ, HS, HB>(c, a);
    case 2: return launch_v<T, 2, HQ, HS, HB>(c, a);
    case 4: return launch_v<T, 4, HQ, HS, HB>(c, a);
    default:
      if constexpr (sizeof(T) == 4) {
        if (v_of(c) == 8) return launch_v<T, 8, HQ, HS, HB>(c, a);
      }
      throw Error(SMA_ERR_INTERNAL, "bad CSR vector width");
  }
}

inline bool aligned(const void *p, int bytes) { return p == nullptr || ((uintptr_t)p % bytes) == 0; }

// Online autotuner.  The first 2 x (number of candidates) launches for a given operator,
// element type, variant, width and leading dimension run the candidates in turn on the
// real recurrence steps, bracketed by CUDA events; after the last of them one event
// synchronization reads the times, and the four fastest candidates (best of two runs) run
// four times more each, in turn; the fastest of those (best of its four runs) is kept for
// the operator's lifetime.  Single runs of a 50-100 us step vary by 10 % or more with
// clocks and neighbouring launches, so the second round guards the choice against a
// lucky or unlucky trial.  Candidates: both families; the widest vector the
// alignment allows, and half of it when that is 32 bytes; the narrowest power-of-two
// group covering the block in one column pass, and the half-width group; U = 4 and 8.
// Small operators (n < 20000) and contexts with autotuning off use the first candidate.
template <typename T, bool HQ, bool HS, bool HB>
void step(const Args<T> &a) {
  const sma_op *op = a.op;
  auto ok = [&](int v) {
    const int bytes = std::min(16, v * (int)sizeof(T));
    return a.b % v == 0 && a.ldb % v == 0 && a.ldo % v == 0 && (!HQ || a.ldq % v == 0) &&
           aligned(a.Q, bytes) && aligned(a.B1, bytes) && aligned(a.B2, bytes) &&
           aligned(a.out, bytes);
  };
  int vmax = 1;
  for (int v : {2, 4, 8})
    if (v * (int)sizeof(T) <= 32 && ok(v)) vmax = v;
  const uint64_t key = ((uint64_t)sizeof(T) << 56) | ((uint64_t)vmax << 52) |
                       ((uint64_t)((HQ ? 4 : 0) | (HS ? 2 : 0) | (HB ? 1 : 0)) << 48) |
                       (a.cseg ? (1ull << 51) : 0ull) | ((uint64_t)a.b << 24) |
                       (uint64_t)std::min<int64_t>(a.ldb, 0xFFFFFF);
  CsrTune &tu = const_cast<sma_op *>(op)->tuned[key];
  if (tu.chosen >= 0) return launch_cfg<T, HQ, HS, HB>(tu.chosen, a);
  if (tu.cands.empty()) {
    for (int fam : {1, 0})
      for (int V : {vmax, vmax / 2}) {
        if (V < 1 || (V != vmax && vmax * (int)sizeof(T) < 32)) continue;
        const int64_t lanes = (a.b + V - 1) / V;
        const int g0 = lanes <= 4 ? 4 : lanes <= 8 ? 8 : lanes <= 16 ? 16 : 32;
        for (int G : {g0, g0 / 2}) {
          if (G < 4) continue;
          tu.cands.push_back(enc(fam, V, G, 8));
          tu.cands.push_back(enc(fam, V, G, 4));
        }
      }
    for (int V : {vmax, vmax / 2}) {  // the BULK family: whole rows staged by bulk copies
      // (a key with 16-byte vectors guarantees 16-byte pointers and leading dimensions)
      if (V >= 1 && vmax * (int)sizeof(T) >= 16 && bulk_fits<T, HQ, HS, HB>(a, V)) {
        if (!op->bulk_err) {
          SMA_CUDA(cudaMalloc((void **)&const_cast<sma_op *>(op)->bulk_err, sizeof(int)));
          SMA_CUDA(cudaMemset(op->bulk_err, 0, sizeof(int)));
        }
        tu.cands.push_back(enc(3, V, (int)(a.b / V), 0));
      }
    }
    if (vmax * (int)sizeof(T) >= 16 && !a.cseg) {  // the ASYNC family moves 16-byte chunks
      const int V = 16 / (int)sizeof(T);
      const int64_t lanes = (a.b + V - 1) / V;
      const int g0 = lanes <= 4 ? 4 : lanes <= 8 ? 8 : lanes <= 16 ? 16 : 32;
      tu.cands.push_back(enc(2, V, g0, 8));
      tu.cands.push_back(enc(2, V, g0, 16));
      if (g0 >= 8) tu.cands.push_back(enc(2, V, g0 / 2, 8));
    }
    if (!op->ctx->autotune || op->n < 20000) {
      tu.chosen = tu.cands[0];
      return launch_cfg<T, HQ, HS, HB>(tu.chosen, a);
    }
  }
  const int kReps = tu.round == 0 ? 2 : 4;
  const size_t ncand = tu.cands.size();
  const size_t idx = tu.trial.size();
  const int c = tu.cands[idx % ncand];
  cudaEvent_t e0, e1;
  SMA_CUDA(cudaEventCreate(&e0));
  SMA_CUDA(cudaEventCreate(&e1));
  tu.events.push_back(e0);
  tu.events.push_back(e1);
  tu.trial.push_back(c);
  SMA_CUDA(cudaEventRecord(e0, a.st));
  launch_cfg<T, HQ, HS, HB>(c, a);
  SMA_CUDA(cudaEventRecord(e1, a.st));
  if (idx + 1 < kReps * ncand) return;
  SMA_CUDA(cudaEventSynchronize(e1));
  std::vector<float> best(ncand, INFINITY);
  for (size_t i = 0; i < tu.trial.size(); ++i) {
    float ms = 0.f;
    SMA_CUDA(cudaEventElapsedTime(&ms, tu.events[2 * i], tu.events[2 * i + 1]));
    best[i % ncand] = std::min(best[i % ncand], ms);
  }
  if (tu.round == 0 && ncand > 4) {  // the four best run again
    std::vector<size_t> order(ncand);
    for (size_t i = 0; i < ncand; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return best[x] < best[y]; });
    std::vector<int> top;
    for (size_t i = 0; i < 4; ++i) top.push_back(tu.cands[order[i]]);
    if (const char *vb = std::getenv("SMA_AUTOTUNE_VERBOSE"); vb && vb[0] == '1') {
      fprintf(stderr, "sma autotune round 1: %s n=%lld b=%lld ld=%lld ->", sizeof(T) == 8 ? "fp64" : "fp32",
              (long long)op->n, (long long)a.b, (long long)a.ldb);
      for (size_t i = 0; i < ncand; ++i)
        fprintf(stderr, " %s/V%d/G%d/U%d=%.1fus",
                fam_of(tu.cands[i]) == 3   ? "bulk"
                : fam_of(tu.cands[i]) == 2 ? "async"
                : fam_of(tu.cands[i])      ? "staged"
                                           : "direct",
                v_of(tu.cands[i]), g_of(tu.cands[i]), u_of(tu.cands[i]), 1e3 * best[i]);
      fprintf(stderr, "\n");
    }
    tu.release();
    tu.cands = top;
    tu.round = 1;
    return;
  }
  const size_t w = std::min_element(best.begin(), best.end()) - best.begin();
  tu.chosen = tu.cands[w];
  tu.release();
  if (const char *vb = std::getenv("SMA_AUTOTUNE_VERBOSE"); vb && vb[0] == '1') {
    fprintf(stderr, "sma autotune: %s n=%lld b=%lld ld=%lld variant=%d%d%d ->", sizeof(T) == 8 ? "fp64" : "fp32",
            (long long)op->n, (long long)a.b, (long long)a.ldb, (int)HQ, (int)HS, (int)HB);
    for (size_t i = 0; i < ncand; ++i)
      fprintf(stderr, " %s%s/V%d/G%d/U%d=%.1fus", i == w ? "*" : "",
              fam_of(tu.cands[i]) == 3   ? "bulk"
              : fam_of(tu.cands[i]) == 2 ? "async"
              : fam_of(tu.cands[i])      ? "staged"
                                         : "direct",
              v_of(tu.cands[i]), g_of(tu.cands[i]), u_of(tu.cands[i]), 1e3 * best[i]);
    fprintf(stderr, "\n");
  }
}

template <typename T>
void clenshaw_step(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                   const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                   double alpha, double beta, bool has_self) {
  const Args<T> a{op, st, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta};
  if (Q && has_self && B2) return step<T, true, true, true>(a);
  if (Q && has_self && !B2) return step<T, true, true, false>(a);
  if (!Q && !has_self && !B2) return step<T, false, false, false>(a);
  throw Error(SMA_ERR_INTERNAL, "unsupported Clenshaw step variant");
}

}  // namespace csr
}  // namespace sma

namespace sma {
template <typename T>
void csr_clenshaw_step(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                       const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                       double alpha, double beta, bool has_self) {
  csr::clenshaw_step<T>(op, st, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta, has_self);
}
}  // namespace sma

namespace sma {
namespace csr {

// The CSR step without the autotuner: the operator's tuned configuration for this key when
// one has been chosen, else the autotuner's first candidate.  Creates no events and never
// inserts into the tuning cache (used by the allocation-free entry point).
template <typename T, bool HQ, bool HS, bool HB>
void step_untuned(const Args<T> &a) {
  auto ok = [&](int v) {
    const int bytes = std::min(16, v * (int)sizeof(T));
    return a.b % v == 0 && a.ldb % v == 0 && a.ldo % v == 0 && (!HQ || a.ldq % v == 0) &&
           aligned(a.Q, bytes) && aligned(a.B1, bytes) && aligned(a.B2, bytes) &&
           aligned(a.out, bytes);
  };
  int vmax = 1;
  for (int v : {2, 4, 8})
    if (v * (int)sizeof(T) <= 32 && ok(v)) vmax = v;
  const uint64_t key = ((uint64_t)sizeof(T) << 56) | ((uint64_t)vmax << 52) |
                       ((uint64_t)((HQ ? 4 : 0) | (HS ? 2 : 0) | (HB ? 1 : 0)) << 48) |
                       (a.cseg ? (1ull << 51) : 0ull) | ((uint64_t)a.b << 24) |
                       (uint64_t)std::min<int64_t>(a.ldb, 0xFFFFFF);
  const auto it = a.op->tuned.find(key);
  if (it != a.op->tuned.end() && it->second.chosen >= 0)
    return launch_cfg<T, HQ, HS, HB>(it->second.chosen, a);
  const int64_t lanes = (a.b + vmax - 1) / vmax;
  const int g0 = lanes <= 4 ? 4 : lanes <= 8 ? 8 : lanes <= 16 ? 16 : 32;
  launch_cfg<T, HQ, HS, HB>(enc(1, vmax, g0, 8), a);
}

}  // namespace csr

template <typename T>
void csr_clenshaw_step_untuned(const sma_op *op, cudaStream_t st, int64_t b, const T *Q,
                               int64_t ldq, const T *B1, const T *B2, int64_t ldb, T *out,
                               int64_t ldo, double ck, double alpha, double beta, bool has_self) {
  const csr::Args<T> a{op, st, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta};
  if (Q && has_self && B2) return csr::step_untuned<T, true, true, true>(a);
  if (Q && has_self && !B2) return csr::step_untuned<T, true, true, false>(a);
  throw Error(SMA_ERR_INTERNAL, "unsupported Clenshaw step variant");
}

// The segmented step: column c takes the coefficient cseg[colseg[c]]; Q, B1 and B2 are all
// read.  tuned = false uses the operator's cached configuration (or the default one) and
// creates no events, so that it may be recorded into a CUDA graph.
template <typename T>
void csr_clenshaw_step_seg(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                           const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo,
                           const T *cseg, const int *colseg, double alpha, double beta,
                           bool tuned) {
  csr::Args<T> a{op, st, b, Q, ldq, B1, B2, ldb, out, ldo, 0.0, alpha, beta};
  a.cseg = cseg;
  a.colseg = colseg;
  if (tuned) return csr::step<T, true, true, true>(a);
  csr::step_untuned<T, true, true, true>(a);
}
}  // namespace sma
