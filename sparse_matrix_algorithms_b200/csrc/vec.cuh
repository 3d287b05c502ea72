// Vector loads/stores of V consecutive elements (V*sizeof(T) <= 32 bytes, issued as one
// or two accesses of at most 16 bytes).  Read-only data goes through the non-coherent
// path (__ldg); it is written only by earlier kernel launches.
#pragma once

#include <cuda_runtime.h>

namespace sma {

template <typename T, int V>
struct Vec;
template <> struct Vec<double, 1> { using type = double; };
template <> struct Vec<double, 2> { using type = double2; };
template <> struct Vec<float, 1> { using type = float; };
template <> struct Vec<float, 2> { using type = float2; };
template <> struct Vec<float, 4> { using type = float4; };

template <typename T, int V>
__device__ __forceinline__ void ldv1(const T *__restrict__ p, T *f) {
  using VT = typename Vec<T, V>::type;
  const VT x = __ldg(reinterpret_cast<const VT *>(p));
  if constexpr (V == 1) {
    f[0] = x;
  } else if constexpr (V == 2) {
    f[0] = x.x; f[1] = x.y;
  } else {
    f[0] = x.x; f[1] = x.y; f[2] = x.z; f[3] = x.w;
  }
}

template <typename T, int V>
__device__ __forceinline__ void stv1(T *__restrict__ p, const T *f) {
  using VT = typename Vec<T, V>::type;
  VT x;
  if constexpr (V == 1) {
    x = f[0];
  } else if constexpr (V == 2) {
    x.x = f[0]; x.y = f[1];
  } else {
    x.x = f[0]; x.y = f[1]; x.z = f[2]; x.w = f[3];
  }
  *reinterpret_cast<VT *>(p) = x;
}

template <typename T, int V>
__device__ __forceinline__ void ldv(const T *__restrict__ p, T (&f)[V]) {
  constexpr int kPer = (V * (int)sizeof(T) <= 16) ? V : 16 / (int)sizeof(T);
#pragma unroll
  for (int k = 0; k < V / kPer; ++k) ldv1<T, kPer>(p + k * kPer, f + k * kPer);
}

template <typename T, int V>
__device__ __forceinline__ void stv(T *__restrict__ p, const T (&f)[V]) {
  constexpr int kPer = (V * (int)sizeof(T) <= 16) ? V : 16 / (int)sizeof(T);
#pragma unroll
  for (int k = 0; k < V / kPer; ++k) stv1<T, kPer>(p + k * kPer, f + k * kPer);
}

}  // namespace sma

namespace sma {

// Round-to-nearest products and sums that the compiler never contracts into FMAs.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// One element of a Clenshaw step's epilogue, ck*q + alpha*acc + beta*s - t, evaluated left
// to right as the reference's broadcast TMP .= c_k .* Q .+ alpha .* AX .+ beta .* B1 .- B2
// (chebyshev_subspace_iteration.jl:576-580) with every product and sum rounded on its own.
// Left to the compiler, ck*q + alpha*acc may be fused either way round into an FMA, and
// different kernels would then round differently; with this form every kernel that takes a
// step -- CSR, segmented, stencil, persistent, matrix-free axpy -- writes the same bits.
// HQ, HS, HB: whether the q, s and t terms are present.
template <bool HQ, bool HS, bool HB, typename T>
__device__ __forceinline__ T clenshaw_combine(T acc, T q, T s, T t, T ck, T alpha, T beta) {
  T x = mul_rn(alpha, acc);
  if constexpr (HQ) x = add_rn(mul_rn(ck, q), x);
  if constexpr (HS) x = add_rn(x, mul_rn(beta, s));
  if constexpr (HB) x = sub_rn(x, t);
  return x;
}

}  // namespace sma
