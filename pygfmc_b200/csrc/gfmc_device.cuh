// Device-side helpers of the GFMC engine: the Threefry-2x32 random stream
// with JAX's key semantics, uniform draws, and warp primitives.
//
// Key semantics (PyGFMC runs on jax.random with the partitionable Threefry):
//   split(key, n)[i] == fold_in(key, i) == threefry2x32(key, (0, i))
//   uniform(key) draws the bits of threefry2x32(key, (0, 0)):
//     float64: (y0 << 32 | y1) >> 12 as the mantissa of [1, 2), minus 1
//     float32: (y0 ^ y1) >> 9 as the mantissa of [1, 2), minus 1
// These are what engine/evolution.py:687-689,840 and
// walkers/reconfiguration.py:53 consume.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gfmc {

struct Key {
  uint32_t a, b;
};

__host__ __device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) {
  return (x << r) | (x >> (32 - r));
}

// Threefry-2x32, 20 rounds (Salmon et al., SC'11; Random123 constants).
__host__ __device__ __forceinline__ void threefry2x32(uint32_t k0, uint32_t k1, uint32_t c0,
                                                      uint32_t c1, uint32_t &o0, uint32_t &o1) {
  const uint32_t k2 = k0 ^ k1 ^ 0x1BD11BDAu;
  uint32_t x0 = c0 + k0, x1 = c1 + k1;
#define GFMC_TF_ROUND(r) { x0 += x1; x1 = rotl32(x1, r); x1 ^= x0; }
  GFMC_TF_ROUND(13) GFMC_TF_ROUND(15) GFMC_TF_ROUND(26) GFMC_TF_ROUND(6)
  x0 += k1; x1 += k2 + 1u;
  GFMC_TF_ROUND(17) GFMC_TF_ROUND(29) GFMC_TF_ROUND(16) GFMC_TF_ROUND(24)
  x0 += k2; x1 += k0 + 2u;
  GFMC_TF_ROUND(13) GFMC_TF_ROUND(15) GFMC_TF_ROUND(26) GFMC_TF_ROUND(6)
  x0 += k0; x1 += k1 + 3u;
  GFMC_TF_ROUND(17) GFMC_TF_ROUND(29) GFMC_TF_ROUND(16) GFMC_TF_ROUND(24)
  x0 += k1; x1 += k2 + 4u;
  GFMC_TF_ROUND(13) GFMC_TF_ROUND(15) GFMC_TF_ROUND(26) GFMC_TF_ROUND(6)
  x0 += k2; x1 += k0 + 5u;
#undef GFMC_TF_ROUND
  o0 = x0;
  o1 = x1;
}

__host__ __device__ __forceinline__ Key fold(Key k, uint32_t d) {
  Key r;
  threefry2x32(k.a, k.b, 0u, d, r.a, r.b);
  return r;
}

__host__ __device__ __forceinline__ double uniform_f64(Key k) {
  uint32_t y0, y1;
  threefry2x32(k.a, k.b, 0u, 0u, y0, y1);
  uint64_t bits = ((((uint64_t)y0) << 32) | (uint64_t)y1) >> 12;
  bits |= 0x3FF0000000000000ull;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)bits) - 1.0;
#else
  double f;
  __builtin_memcpy(&f, &bits, 8);
  return f - 1.0;
#endif
}

__host__ __device__ __forceinline__ float uniform_f32(Key k) {
  uint32_t y0, y1;
  threefry2x32(k.a, k.b, 0u, 0u, y0, y1);
  uint32_t bits = ((y0 ^ y1) >> 9) | 0x3F800000u;
#ifdef __CUDA_ARCH__
  return __uint_as_float(bits) - 1.0f;
#else
  float f;
  __builtin_memcpy(&f, &bits, 4);
  return f - 1.0f;
#endif
}

template <typename T> __device__ __forceinline__ T uniform(Key k);
template <> __device__ __forceinline__ double uniform<double>(Key k) { return uniform_f64(k); }
template <> __device__ __forceinline__ float uniform<float>(Key k) { return uniform_f32(k); }

// ---- warp primitives ------------------------------------------------------
template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T> __device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T u = __shfl_xor_sync(0xffffffffu, v, o);
    v = u > v ? u : v;
  }
  return v;
}

// Inclusive scan across the 32 lanes (Hillis-Steele order, fixed).
template <typename T> __device__ __forceinline__ T warp_inclusive_scan(T v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

template <typename T> __device__ __forceinline__ T math_exp(T x);
template <> __device__ __forceinline__ double math_exp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float math_exp<float>(float x) { return __expf(x); }

template <typename T> __device__ __forceinline__ T math_log(T x);
template <> __device__ __forceinline__ double math_log<double>(double x) { return log(x); }
template <> __device__ __forceinline__ float math_log<float>(float x) { return __logf(x); }

template <typename T> __device__ __forceinline__ T math_min(T x, T y);
template <> __device__ __forceinline__ double math_min<double>(double x, double y) { return fmin(x, y); }
template <> __device__ __forceinline__ float math_min<float>(float x, float y) { return fminf(x, y); }

// Correctly rounded reciprocal: the value of 1 / x under IEEE division.
template <typename T> __device__ __forceinline__ T math_rcp(T x);
template <> __device__ __forceinline__ double math_rcp<double>(double x) { return __drcp_rn(x); }
template <> __device__ __forceinline__ float math_rcp<float>(float x) { return __frcp_rn(x); }

template <typename T> __device__ __forceinline__ T math_log1p(T x);
template <> __device__ __forceinline__ double math_log1p<double>(double x) { return log1p(x); }
template <> __device__ __forceinline__ float math_log1p<float>(float x) { return log1pf(x); }

template <typename T> __device__ __forceinline__ T math_sqrt(T x);
template <> __device__ __forceinline__ double math_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float math_sqrt<float>(float x) { return sqrtf(x); }

template <typename T> __device__ __forceinline__ T next_below(T x);
template <> __device__ __forceinline__ double next_below<double>(double x) { return nextafter(x, 0.0); }
template <> __device__ __forceinline__ float next_below<float>(float x) { return nextafterf(x, 0.0f); }

template <typename T> __device__ __forceinline__ T pos_inf();
template <> __device__ __forceinline__ double pos_inf<double>() { return __longlong_as_double(0x7FF0000000000000ll); }
template <> __device__ __forceinline__ float pos_inf<float>() { return __int_as_float(0x7F800000); }

}  // namespace gfmc
