// CUDA kernels of libsma (sm_100a).
//
// The hot one, the fused block Clenshaw step
//
//     out[i,:] = ck*Q[i,:] + alpha*sum_j A[i,j]*B1[j,:] + beta*B1[i,:] - B2[i,:],
//
// replaces the reference's `mul!(AX,A,B1)` followed by a separate 4-array axpy sweep
// (chebyshev_subspace_iteration.jl:573-582, polfed.jl:483-492); AX never reaches memory.
// Its CSR form lives in csr_clenshaw.cuh; this file holds the stencil form (the matrix-
// free 1D Laplacian), the dispatcher, and the small kernels around the solvers.
#include "sma_internal.h"
#include "vec.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>

namespace sma {

std::atomic<int64_t> g_kernel_launches{0};

namespace {

constexpr int kThreads = 256;

// Each stencil functor has prepare(row), the per-row work done once, and product(prep, ...)
// for one column pass: acc += (A B1)[row, c0:c0+V].
//
// tridiag(-1,2,-1) stencil, evaluated as the reference's lap1d_matblock!
// (polfed.jl:1209-1219): Y[1]=2X[1]-X[2]; Y[i]=-X[i-1]+2X[i]-X[i+1]; Y[n]=-X[n-1]+2X[n].
template <typename T>
struct Lap1dRows {
  int64_t n;
  struct Prep {
    int64_t row;
  };
  __device__ __forceinline__ Prep prepare(int64_t row) const { return {row}; }
  template <int V>
  __device__ __forceinline__ void product(const Prep &p, const T *__restrict__ B1, int64_t ldb,
                                          int c0, T (&acc)[V]) const {
    const int64_t row = p.row;
    T xm[V], x0[V], xp[V];
    ldv<T, V>(B1 + row * ldb + c0, x0);
    if (row == 0) {
      ldv<T, V>(B1 + (row + 1) * ldb + c0, xp);
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = T(2) * x0[v] - xp[v];
    } else if (row == n - 1) {
      ldv<T, V>(B1 + (row - 1) * ldb + c0, xm);
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = -xm[v] + T(2) * x0[v];
    } else {
      ldv<T, V>(B1 + (row - 1) * ldb + c0, xm);
      ldv<T, V>(B1 + (row + 1) * ldb + c0, xp);
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = -xm[v] + T(2) * x0[v] - xp[v];
    }
  }
};

// 3D Anderson model on an L^3 periodic lattice, row i = x + L*(y + L*z): diag[i] on the
// diagonal and `hop` at the six neighbours x+-1, y+-1, z+-1.  The seven terms are sorted by
// column with a 16-comparator sorting network and accumulated in that order -- the order
// of the stored matrix's CSR row -- so the stencil and the CSR kernel give bit-identical
// products.  Needs L >= 3 (six distinct neighbours).
template <typename T>
struct AndersonRows {
  int64_t L;
  const double *__restrict__ diag;
  T hop;
  // sorted columns (int32: n < 2^31) and the sorted position of the diagonal entry
  struct Prep {
    int c[7];
    int dpos;
    T d;
  };
  __device__ __forceinline__ Prep prepare(int64_t row64) const {
    const int row = (int)row64, l = (int)L, l2 = l * l;
    const int x = row % l, y = (row / l) % l, z = row / l2;
    int r0 = row, r1 = x + 1 == l ? row - (l - 1) : row + 1, r2 = x == 0 ? row + (l - 1) : row - 1;
    int r3 = y + 1 == l ? row - (l - 1) * l : row + l, r4 = y == 0 ? row + (l - 1) * l : row - l;
    int r5 = z + 1 == l ? row - (l - 1) * l2 : row + l2, r6 = z == 0 ? row + (l - 1) * l2 : row - l2;
#define SMA_CS(i, j)         \
  if (r##i > r##j) {         \
    const int tr = r##i;     \
    r##i = r##j;             \
    r##j = tr;               \
  }
    SMA_CS(0, 6) SMA_CS(2, 3) SMA_CS(4, 5) SMA_CS(0, 2) SMA_CS(1, 4) SMA_CS(3, 6)
    SMA_CS(0, 1) SMA_CS(2, 5) SMA_CS(3, 4) SMA_CS(1, 2) SMA_CS(4, 6) SMA_CS(2, 3)
    SMA_CS(4, 5) SMA_CS(1, 2) SMA_CS(3, 4) SMA_CS(5, 6)
#undef SMA_CS
    Prep p{{r0, r1, r2, r3, r4, r5, r6}, 0, (T)__ldg(diag + row64)};
#pragma unroll
    for (int u = 0; u < 7; ++u)
      if (p.c[u] == row) p.dpos = u;
    return p;
  }
  template <int V>
  __device__ __forceinline__ void product(const Prep &p, const T *__restrict__ B1, int64_t ldb,
                                          int c0, T (&acc)[V]) const {
    T xs[7][V];
#pragma unroll
    for (int u = 0; u < 7; ++u) ldv<T, V>(B1 + (int64_t)p.c[u] * ldb + c0, xs[u]);
#pragma unroll
    for (int u = 0; u < 7; ++u) {
      const T a = u == p.dpos ? p.d : hop;
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = fma(a, xs[u][v], acc[v]);
    }
  }
};

// Random-field XXZ chain of length L in the Sz = 0 sector.  Row r is the basis state
// s = states[r] (bit i = site i up); its index is its combinatorial rank
// sum_j C(p_j, j) over its set bits p_1 < p_2 < ... .  Flipping the antiparallel bond
// (i, i+1) moves one set bit by one position, which changes the rank by +-C(i, k), k the
// number of set bits below i; the periodic bond (L-1, 0) re-ranks the flipped state.
// Terms: diag[r] x_r, then `hop` (J/2) times each neighbour in bond order.
template <typename T>
struct XxzRows {
  int L;
  const double *__restrict__ diag;
  const unsigned *__restrict__ states;
  const int *__restrict__ binom;  // C(p, k) at binom[p*17 + k]
  T hop;
  struct Prep {
    int64_t row, pcol;  // pcol: neighbour across the periodic bond, or -1
    unsigned s;
    T d;
  };
  __device__ __forceinline__ Prep prepare(int64_t row) const {
    Prep p{row, -1, __ldg(states + row), (T)__ldg(diag + row)};
    if (((p.s >> (L - 1)) ^ p.s) & 1u) {
      unsigned t = p.s ^ (1u | (1u << (L - 1)));
      int64_t col = 0;
      for (int j = 1; t; ++j) {
        col += __ldg(binom + (__ffs(t) - 1) * 17 + j);
        t &= t - 1;
      }
      p.pcol = col;
    }
    return p;
  }
  template <int V>
  __device__ __forceinline__ void product(const Prep &p, const T *__restrict__ B1, int64_t ldb,
                                          int c0, T (&acc)[V]) const {
    const int64_t row = p.row;
    const unsigned s = p.s;
    T x[V];
    ldv<T, V>(B1 + row * ldb + c0, x);
    const T d = p.d;
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = fma(d, x[v], acc[v]);
    int k = 0;
    for (int i = 0; i + 1 < L; ++i) {
      const unsigned bi = (s >> i) & 1u;
      if (bi != ((s >> (i + 1)) & 1u)) {
        const int delta = __ldg(binom + i * 17 + k);
        const int64_t col = bi ? row + delta : row - delta;
        ldv<T, V>(B1 + col * ldb + c0, x);
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = fma(hop, x[v], acc[v]);
      }
      k += (int)bi;
    }
    if (p.pcol >= 0) {
      ldv<T, V>(B1 + p.pcol * ldb + c0, x);
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = fma(hop, x[v], acc[v]);
    }
  }
};

// ------------------------------------------------------------------ stencil Clenshaw step
template <typename T, int V, int G, bool HAS_Q, bool HAS_SELF, bool HAS_B2, typename Rows>
__global__ void __launch_bounds__(kThreads)
stencil_step_kernel(Rows rows, int64_t n, int b, const T *__restrict__ Q, int64_t ldq,
                     const T *__restrict__ B1, const T *__restrict__ B2, int64_t ldb,
                     T *__restrict__ out, int64_t ldo, T ck, T alpha, T beta) {
  constexpr int kRows = kThreads / G;
  const int lane = threadIdx.x % G;
  for (int64_t row = (int64_t)blockIdx.x * kRows + threadIdx.x / G; row < n;
       row += (int64_t)gridDim.x * kRows) {
    const auto prep = rows.prepare(row);
    for (int c0 = lane * V; c0 < b; c0 += G * V) {
      T acc[V], q[V], s[V], t[V], r[V];
      // epilogue operands first, so that their latency overlaps the neighbour gathers
      if constexpr (HAS_Q) ldv<T, V>(Q + row * ldq + c0, q);
      if constexpr (HAS_SELF) ldv<T, V>(B1 + row * ldb + c0, s);
      if constexpr (HAS_B2) ldv<T, V>(B2 + row * ldb + c0, t);
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = T(0);
      rows.template product<V>(prep, B1, ldb, c0, acc);
#pragma unroll
      for (int v = 0; v < V; ++v)
        r[v] = clenshaw_combine<HAS_Q, HAS_SELF, HAS_B2>(acc[v], q[v], s[v], t[v], ck, alpha, beta);
      stv<T, V>(out + row * ldo + c0, r);
    }
  }
}

template <typename T, int V, int G, bool HQ, bool HS, bool HB, typename Rows>
void launch_cfg(const Rows &rows, cudaStream_t st, int64_t n, int64_t b, const T *Q, int64_t ldq,
                const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                double alpha, double beta) {
  constexpr int kRows = kThreads / G;
  const int64_t need = (n + kRows - 1) / kRows;
  const int grid = (int)std::min<int64_t>(need, 148LL * 256);
  stencil_step_kernel<T, V, G, HQ, HS, HB, Rows><<<grid, kThreads, 0, st>>>(
      rows, n, (int)b, Q, ldq, B1, B2, ldb, out, ldo, (T)ck, (T)alpha, (T)beta);
}

template <typename T, int V, bool HQ, bool HS, bool HB, typename Rows>
void pick_group(const Rows &rows, cudaStream_t st, int64_t n, int64_t b, const T *Q, int64_t ldq,
                const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                double alpha, double beta) {
  const int64_t lanes = (b + V - 1) / V;
  if (lanes <= 4)
    launch_cfg<T, V, 4, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  else if (lanes <= 8)
    launch_cfg<T, V, 8, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  else if (lanes <= 16)
    launch_cfg<T, V, 16, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  else
    launch_cfg<T, V, 32, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
}

inline bool aligned(const void *p, int bytes) { return p == nullptr || ((uintptr_t)p % bytes) == 0; }

template <typename T, bool HQ, bool HS, bool HB, typename Rows>
void pick_vec(const Rows &rows, cudaStream_t st, int64_t n, int64_t b, const T *Q, int64_t ldq,
              const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck, double alpha,
              double beta) {
  auto ok = [&](int v) {
    const int bytes = v * (int)sizeof(T);
    return b % v == 0 && ldb % v == 0 && ldo % v == 0 && (!HQ || ldq % v == 0) &&
           aligned(Q, bytes) && aligned(B1, bytes) && aligned(B2, bytes) && aligned(out, bytes);
  };
  if constexpr (sizeof(T) == 4) {
    if (ok(4)) return pick_group<T, 4, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
    if (ok(2)) return pick_group<T, 2, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  } else {
    if (ok(2)) return pick_group<T, 2, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  }
  pick_group<T, 1, HQ, HS, HB>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
}

template <typename T, typename Rows>
void dispatch_flags(const Rows &rows, cudaStream_t st, int64_t n, int64_t b, const T *Q,
                    int64_t ldq, const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo,
                    double ck, double alpha, double beta, bool has_self) {
  if (Q && has_self && B2)
    pick_vec<T, true, true, true>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  else if (Q && has_self && !B2)
    pick_vec<T, true, true, false>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  else if (!Q && !has_self && !B2)
    pick_vec<T, false, false, false>(rows, st, n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta);
  else
    throw Error(SMA_ERR_INTERNAL, "unsupported Clenshaw step variant");
}

// ------------------------------------------------------------------ elementwise block ops
template <typename T>
__global__ void scale_block_kernel(int64_t n, int64_t b, const T *__restrict__ Q, int64_t ldq,
                                   T *__restrict__ out, int64_t ldo, T ck) {
  const int64_t total = n * b;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / b, j = t % b;
    out[i * ldo + j] = mul_rn(ck, Q[i * ldq + j]);
  }
}

template <typename T>
__global__ void clenshaw_axpy_kernel(int64_t n, int64_t b, const T *__restrict__ Q, int64_t ldq,
                                     const T *__restrict__ AX, int64_t ldax,
                                     const T *__restrict__ B1, const T *__restrict__ B2,
                                     int64_t ldb, T *__restrict__ out, int64_t ldo, T ck, T alpha,
                                     T beta) {
  const int64_t total = n * b;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / b, j = t % b;
    const T q = Q[i * ldq + j], a = AX[i * ldax + j], s = B1[i * ldb + j];
    out[i * ldo + j] = B2 ? clenshaw_combine<true, true, true>(a, q, s, B2[i * ldb + j], ck, alpha, beta)
                          : clenshaw_combine<true, true, false>(a, q, s, T(0), ck, alpha, beta);
  }
}

template <typename TS, typename TD>
__global__ void copy_block_kernel(int64_t n, int64_t b, const TS *__restrict__ src, int64_t lds,
                                  TD *__restrict__ dst, int64_t ldd) {
  const int64_t total = n * b;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / b, j = t % b;
    dst[i * ldd + j] = (TD)src[i * lds + j];
  }
}

inline int grid_for(int64_t total) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148LL * 32));
}

// ------------------------------------------------------------------ random start blocks
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Element (i, j) of an n x m standard-normal block: flat index k = i + j*n (Julia's
// column-major randn fill order), uniforms 2k and 2k+1 of the SplitMix64 counter
// stream seed ^ 0x5DEECE66D, Box-Muller z = sqrt(-2 ln(1-u0)) cos(2 pi u1).
__global__ void randn_kernel(int64_t n, int64_t m, uint64_t seed, double *__restrict__ out,
                             int64_t ld) {
  const uint64_t s = seed ^ 0x5DEECE66DULL;
  const uint64_t golden = 0x9E3779B97F4A7C15ULL;
  const int64_t total = n * m;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / m, j = t % m;
    const uint64_t k = (uint64_t)i + (uint64_t)j * (uint64_t)n;
    const uint64_t x0 = mix64(s + (2 * k + 1) * golden);
    const uint64_t x1 = mix64(s + (2 * k + 2) * golden);
    const double u0 = (double)(x0 >> 11) * (1.0 / 9007199254740992.0);
    const double u1 = (double)(x1 >> 11) * (1.0 / 9007199254740992.0);
    out[i * ld + j] = sqrt(-2.0 * log1p(-u0)) * cos(2.0 * 3.141592653589793 * u1);
  }
}

// ------------------------------------------------------------------ column reductions
__global__ void colred_stage1(int mode, int64_t n, int64_t k, const double *__restrict__ X,
                              int64_t ldx, const double *__restrict__ Y, int64_t ldy,
                              const double *__restrict__ lam, double *__restrict__ partial,
                              int64_t rows_per_chunk) {
  __shared__ double sh[8][33];
  const int cl = threadIdx.x % 32, rl = threadIdx.x / 32;
  const int64_t col = (int64_t)blockIdx.y * 32 + cl;
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_chunk;
  const int64_t r1 = min(n, r0 + rows_per_chunk);
  double s = 0.0;
  if (col < k) {
    const double l = mode == 1 ? lam[col] : 0.0;
    for (int64_t i = r0 + rl; i < r1; i += 8) {
      const double x = X[i * ldx + col];
      const double y = Y[i * ldy + col];
      if (mode == 0) {
        s = fma(x, y, s);
      } else {
        const double d = y - l * x;
        s = fma(d, d, s);
      }
    }
  }
  sh[rl][cl] = s;
  __syncthreads();
  if (rl == 0 && col < k) {
    double t = 0.0;
#pragma unroll
    for (int r = 0; r < 8; ++r) t += sh[r][cl];
    partial[(int64_t)blockIdx.x * k + col] = t;
  }
}

__global__ void colred_stage2(int mode, int64_t chunks, int64_t k, const double *__restrict__ partial,
                              double *__restrict__ out) {
  for (int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; col < k;
       col += (int64_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int64_t c = 0; c < chunks; ++c) t += partial[c * k + col];
    out[col] = mode == 1 ? sqrt(t) : t;
  }
}

// ------------------------------------------------------------------ layout helpers
// out (row-major C x R, ldo) = in^T where in is row-major R x C (ldi)
__global__ void transpose_kernel(int64_t R, int64_t C, const double *__restrict__ in, int64_t ldi,
                                 double *__restrict__ out, int64_t ldo) {
  __shared__ double tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t r = r0 + dy, c = c0 + threadIdx.x;
    if (r < R && c < C) tile[dy][threadIdx.x] = in[r * ldi + c];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t c = c0 + dy, r = r0 + threadIdx.x;
    if (r < R && c < C) out[c * ldo + r] = tile[threadIdx.x][dy];
  }
}

__global__ void symmetrize_kernel(int64_t k, const double *__restrict__ G, int64_t ldg,
                                  double *__restrict__ H, int64_t ldh) {
  const int64_t total = k * k;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % k, j = t / k;
    H[i + j * ldh] = 0.5 * (G[i + j * ldg] + G[j + i * ldg]);
  }
}

__global__ void place_blocks_kernel(double *__restrict__ T, int64_t ldt, int64_t o, int64_t r,
                                    const double *__restrict__ Aj, int64_t lda,
                                    const double *__restrict__ Bj, int64_t ldbj, int64_t r2) {
  // column-major T; Aj r x r, Bj r2 x r (column-major); a null block is skipped
  const int64_t totalA = Aj ? r * r : 0, totalB = Bj ? r2 * r : 0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < totalA + totalB;
       t += (int64_t)gridDim.x * blockDim.x) {
    if (t < totalA) {
      const int64_t i = t % r, j = t / r;
      T[(o + i) + (o + j) * ldt] = Aj[i + j * lda];
    } else {
      const int64_t u = t - totalA;
      const int64_t i = u % r2, j = u / r2;
      const double v = Bj[i + j * ldbj];
      T[(o + r + i) + (o + j) * ldt] = v;
      T[(o + j) + (o + r + i) * ldt] = v;
    }
  }
}

__global__ void gather_cols_cm_kernel(int64_t M, int64_t k, const double *__restrict__ src,
                                      int64_t lds, const int64_t *__restrict__ idx,
                                      double *__restrict__ dst, int64_t ldd) {
  const int64_t total = M * k;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % M, j = t / M;
    dst[i + j * ldd] = src[i + idx[j] * lds];
  }
}

__global__ void gather_cols_rm_kernel(int64_t n, int64_t k, const double *__restrict__ src,
                                      int64_t lds, const int64_t *__restrict__ idx,
                                      double *__restrict__ dst, int64_t ldd) {
  const int64_t total = n * k;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / k, j = t % k;
    dst[i * ldd + j] = src[i * lds + idx[j]];
  }
}

__global__ void add_diag_kernel(int64_t k, double *G, int64_t ld, double shift) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k;
       i += (int64_t)gridDim.x * blockDim.x)
    G[i + i * ld] += shift;
}

__global__ void zero_lower_kernel(int64_t k, double *G, int64_t ld) {
  const int64_t total = k * k;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % k, j = t / k;
    if (i > j) G[i + j * ld] = 0.0;
  }
}

__global__ void identity_kernel(int64_t k, double *G, int64_t ld) {
  const int64_t total = k * k;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % k, j = t / k;
    G[i + j * ld] = i == j ? 1.0 : 0.0;
  }
}

// ------------------------------------------------------------------ CSR checks
__global__ void gershgorin_kernel(int64_t n, const int *__restrict__ rowptr,
                                  const int *__restrict__ colind, const double *__restrict__ val,
                                  double *__restrict__ pmin, double *__restrict__ pmax) {
  __shared__ double smin[256], smax[256];
  double lo = INFINITY, hi = -INFINITY;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double d = 0.0, r = 0.0;
    for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) {
      if (colind[j] == i) d = val[j];
      else r += fabs(val[j]);
    }
    lo = fmin(lo, d - r);
    hi = fmax(hi, d + r);
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pmin[blockIdx.x] = smin[0];
    pmax[blockIdx.x] = smax[0];
  }
}

// flags bit 0: columns not strictly increasing in a row; bit 1: A != A^T
__global__ void check_csr_kernel(int64_t n, const int *__restrict__ rowptr,
                                 const int *__restrict__ colind, const double *__restrict__ val,
                                 int *__restrict__ flags) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int s = rowptr[i], e = rowptr[i + 1];
    for (int t = s; t < e; ++t) {
      const int j = colind[t];
      if (t + 1 < e && colind[t + 1] <= j) atomicOr(flags, 1);
      if (j < 0 || j >= n) { atomicOr(flags, 1); continue; }
      const double v = val[t];
      // find (j, i) in row j by binary search
      int lo = rowptr[j], hi = rowptr[j + 1] - 1;
      bool found = false;
      double w = 0.0;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int c = colind[mid];
        if (c == i) { found = true; w = val[mid]; break; }
        if (c < i) lo = mid + 1; else hi = mid - 1;
      }
      if (found ? !(w == v) : (v != 0.0)) atomicOr(flags, 2);
    }
  }
}

}  // namespace

// ------------------------------------------------------------------ public launchers
template <typename T>
void launch_clenshaw_step(const sma_op *op, cudaStream_t st, int64_t b, const T *Q, int64_t ldq,
                          const T *B1, const T *B2, int64_t ldb, T *out, int64_t ldo, double ck,
                          double alpha, double beta, bool has_self) {
  if (op->n == 0 || b == 0) return;
  if (op->kind == OP_CSR) {
    csr_clenshaw_step<T>(op, st, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta, has_self);
  } else if (op->kind == OP_LAP1D) {
    Lap1dRows<T> rows{op->n};
    dispatch_flags<T>(rows, st, op->n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta, has_self);
    SMA_CHECK_LAUNCH();
  } else if (op->kind == OP_ANDERSON) {
    AndersonRows<T> rows{op->stencil.L, op->stencil.diag, (T)op->stencil.hop};
    dispatch_flags<T>(rows, st, op->n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta, has_self);
    SMA_CHECK_LAUNCH();
  } else if (op->kind == OP_XXZ) {
    XxzRows<T> rows{op->stencil.L, op->stencil.diag, op->stencil.states, op->stencil.binom,
                    (T)op->stencil.hop};
    dispatch_flags<T>(rows, st, op->n, b, Q, ldq, B1, B2, ldb, out, ldo, ck, alpha, beta, has_self);
    SMA_CHECK_LAUNCH();
  } else {
    throw Error(SMA_ERR_INTERNAL, "fused Clenshaw step needs a device operator");
  }
}

template <typename T>
void launch_scale_block(cudaStream_t st, int64_t n, int64_t b, const T *Q, int64_t ldq, T *out,
                        int64_t ldo, double ck) {
  if (n * b == 0) return;
  scale_block_kernel<T><<<grid_for(n * b), 256, 0, st>>>(n, b, Q, ldq, out, ldo, (T)ck);
  SMA_CHECK_LAUNCH();
}

template <typename T>
void launch_clenshaw_axpy(cudaStream_t st, int64_t n, int64_t b, const T *Q, int64_t ldq,
                          const T *AX, int64_t ldax, const T *B1, const T *B2, int64_t ldb,
                          T *out, int64_t ldo, double ck, double alpha, double beta) {
  if (n * b == 0) return;
  clenshaw_axpy_kernel<T><<<grid_for(n * b), 256, 0, st>>>(n, b, Q, ldq, AX, ldax, B1, B2, ldb,
                                                           out, ldo, (T)ck, (T)alpha, (T)beta);
  SMA_CHECK_LAUNCH();
}

template <typename TS, typename TD>
void launch_copy_block(cudaStream_t st, int64_t n, int64_t b, const TS *src, int64_t lds, TD *dst,
                       int64_t ldd) {
  if (n * b == 0) return;
  copy_block_kernel<TS, TD><<<grid_for(n * b), 256, 0, st>>>(n, b, src, lds, dst, ldd);
  SMA_CHECK_LAUNCH();
}

template void launch_clenshaw_step<double>(const sma_op *, cudaStream_t, int64_t, const double *,
                                           int64_t, const double *, const double *, int64_t,
                                           double *, int64_t, double, double, double, bool);
template void launch_clenshaw_step<float>(const sma_op *, cudaStream_t, int64_t, const float *,
                                          int64_t, const float *, const float *, int64_t, float *,
                                          int64_t, double, double, double, bool);
template void launch_scale_block<double>(cudaStream_t, int64_t, int64_t, const double *, int64_t,
                                         double *, int64_t, double);
template void launch_scale_block<float>(cudaStream_t, int64_t, int64_t, const float *, int64_t,
                                        float *, int64_t, double);
template void launch_clenshaw_axpy<double>(cudaStream_t, int64_t, int64_t, const double *, int64_t,
                                           const double *, int64_t, const double *, const double *,
                                           int64_t, double *, int64_t, double, double, double);
template void launch_clenshaw_axpy<float>(cudaStream_t, int64_t, int64_t, const float *, int64_t,
                                          const float *, int64_t, const float *, const float *,
                                          int64_t, float *, int64_t, double, double, double);
template void launch_copy_block<double, double>(cudaStream_t, int64_t, int64_t, const double *,
                                                int64_t, double *, int64_t);
template void launch_copy_block<double, float>(cudaStream_t, int64_t, int64_t, const double *,
                                               int64_t, float *, int64_t);
template void launch_copy_block<float, double>(cudaStream_t, int64_t, int64_t, const float *,
                                               int64_t, double *, int64_t);
template void launch_copy_block<float, float>(cudaStream_t, int64_t, int64_t, const float *,
                                              int64_t, float *, int64_t);

void launch_randn(cudaStream_t st, int64_t n, int64_t m, uint64_t seed, double *out, int64_t ld) {
  if (n * m == 0) return;
  randn_kernel<<<grid_for(n * m), 256, 0, st>>>(n, m, seed, out, ld);
  SMA_CHECK_LAUNCH();
}

void column_reduce(cudaStream_t st, int mode, int64_t n, int64_t k, const double *X, int64_t ldx,
                   const double *Y, int64_t ldy, const double *lam, double *out,
                   DevBuf<double> &scratch) {
  if (k == 0) return;
  const int64_t ctiles = (k + 31) / 32;
  int64_t chunks = std::max<int64_t>(1, std::min<int64_t>((n + 63) / 64, (148 * 8 + ctiles - 1) / ctiles));
  const int64_t rows_per_chunk = (n + chunks - 1) / chunks;
  chunks = std::max<int64_t>(1, (n + rows_per_chunk - 1) / rows_per_chunk);
  if (scratch.count < (size_t)(chunks * k)) scratch.alloc(chunks * k, st);
  dim3 grid((unsigned)chunks, (unsigned)ctiles);
  colred_stage1<<<grid, 256, 0, st>>>(mode, n, k, X, ldx, Y, ldy, lam, scratch.p, rows_per_chunk);
  SMA_CHECK_LAUNCH();
  colred_stage2<<<(unsigned)std::max<int64_t>(1, (k + 255) / 256), 256, 0, st>>>(mode, chunks, k,
                                                                                scratch.p, out);
  SMA_CHECK_LAUNCH();
}

static void transpose(cudaStream_t st, int64_t R, int64_t C, const double *in, int64_t ldi,
                      double *out, int64_t ldo) {
  if (R * C == 0) return;
  dim3 grid((unsigned)((C + 31) / 32), (unsigned)((R + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(R, C, in, ldi, out, ldo);
  SMA_CHECK_LAUNCH();
}

void launch_rowmajor_to_colmajor(cudaStream_t st, int64_t n, int64_t k, const double *src,
                                 int64_t lds, double *dst) {
  transpose(st, n, k, src, lds, dst, n);
}

void launch_colmajor_to_rowmajor(cudaStream_t st, int64_t n, int64_t k, const double *src,
                                 double *dst, int64_t ldd) {
  // column-major n x k (ld n) is row-major k x n (ld n)
  transpose(st, k, n, src, n, dst, ldd);
}

void launch_symmetrize(cudaStream_t st, int64_t k, const double *G, int64_t ldg, double *H,
                       int64_t ldh) {
  if (k == 0) return;
  symmetrize_kernel<<<grid_for(k * k), 256, 0, st>>>(k, G, ldg, H, ldh);
  SMA_CHECK_LAUNCH();
}

void launch_place_blocks(cudaStream_t st, double *T, int64_t ldt, int64_t o, int64_t r,
                         const double *Aj, int64_t lda, const double *Bj, int64_t ldbj,
                         int64_t r2) {
  const int64_t total = (Aj ? r * r : 0) + (Bj ? r2 * r : 0);
  if (total == 0) return;
  place_blocks_kernel<<<grid_for(total), 256, 0, st>>>(T, ldt, o, r, Aj, lda, Bj, ldbj, r2);
  SMA_CHECK_LAUNCH();
}

void launch_gather_columns_cm(cudaStream_t st, int64_t M, int64_t k, const double *src,
                              int64_t lds, const int64_t *idx, double *dst, int64_t ldd) {
  if (M * k == 0) return;
  gather_cols_cm_kernel<<<grid_for(M * k), 256, 0, st>>>(M, k, src, lds, idx, dst, ldd);
  SMA_CHECK_LAUNCH();
}

void launch_gather_columns_rm(cudaStream_t st, int64_t n, int64_t k, const double *src,
                              int64_t lds, const int64_t *idx, double *dst, int64_t ldd) {
  if (n * k == 0) return;
  gather_cols_rm_kernel<<<grid_for(n * k), 256, 0, st>>>(n, k, src, lds, idx, dst, ldd);
  SMA_CHECK_LAUNCH();
}

void launch_add_diagonal(cudaStream_t st, int64_t k, double *G, int64_t ld, double shift) {
  if (k == 0) return;
  add_diag_kernel<<<grid_for(k), 256, 0, st>>>(k, G, ld, shift);
  SMA_CHECK_LAUNCH();
}

void launch_zero_lower(cudaStream_t st, int64_t k, double *G, int64_t ld) {
  if (k == 0) return;
  zero_lower_kernel<<<grid_for(k * k), 256, 0, st>>>(k, G, ld);
  SMA_CHECK_LAUNCH();
}

void launch_identity(cudaStream_t st, int64_t k, double *G, int64_t ld) {
  if (k == 0) return;
  identity_kernel<<<grid_for(k * k), 256, 0, st>>>(k, G, ld);
  SMA_CHECK_LAUNCH();
}

void gershgorin_device(const sma_op *op, double *smin, double *smax) {
  cudaStream_t st = op->ctx->stream;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((op->n + 255) / 256, 1024));
  DevBuf<double> part(2 * grid, st);
  gershgorin_kernel<<<grid, 256, 0, st>>>(op->n, op->rowptr, op->colind, op->val64, part.p,
                                          part.p + grid);
  SMA_CHECK_LAUNCH();
  std::vector<double> h(2 * grid);
  SMA_CUDA(cudaMemcpyAsync(h.data(), part.p, 2 * grid * sizeof(double), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  double lo = INFINITY, hi = -INFINITY;
  for (int i = 0; i < grid; ++i) {
    lo = std::min(lo, h[i]);
    hi = std::max(hi, h[grid + i]);
  }
  *smin = lo;
  *smax = hi;
}

int check_csr_device(const sma_op *op) {
  cudaStream_t st = op->ctx->stream;
  DevBuf<int> flag(1, st);
  SMA_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((op->n + 255) / 256, 4096));
  check_csr_kernel<<<grid, 256, 0, st>>>(op->n, op->rowptr, op->colind, op->val64, flag.p);
  SMA_CHECK_LAUNCH();
  int h = 0;
  SMA_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SMA_CUDA(cudaStreamSynchronize(st));
  if (h & 1) return 1;
  if (h & 2) return 2;
  return 0;
}

}  // namespace sma
