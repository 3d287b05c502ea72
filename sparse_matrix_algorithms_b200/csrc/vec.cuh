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
