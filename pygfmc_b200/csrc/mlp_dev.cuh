// Device helpers of the MLP guide shared by its step kernel (mlp.cu) and
// its trainer (mlp_train.cu): the tanh form, the Bose-Hubbard move decode
// and the W1 columns a move exchanges.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

#include "bose_moves.cuh"
#include "engine.cuh"

namespace gfmc {
namespace mlpdev {

// tanh y = 1 - 2 / (1 + e^{2y}) with e^{2y} = 2^{K y}, K = 2 log2(e): one
// ex2 and one rcp (absolute error about 1e-7; e^{2y} overflowing to inf
// gives 1, underflowing to 0 gives -1).
constexpr float KT = 2.8853900817779268f;

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// 1 / (1 + e^{2y}) from Ky = K y: tanh y = 1 - 2 of it.
__device__ __forceinline__ float sig2(float Ky) { return rcp_approx(1.0f + ex2_approx(Ky)); }
// First-layer activation before its bf16 rounding: the hardware tanh (one
// special-function operation; its error is below the bf16 step).
__device__ __forceinline__ float tanh_h1(float z) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(z));
  return y;
}

// A move of the Bose-Hubbard layout (bose_decode) with its unguided element
// (bose_element); b == a, db = 0 for the single-site h_pm moves.
struct Mv {
  int a, b, da, db;
  float v;
};

__device__ __forceinline__ Mv mlp_move(const DevModel<float> &m, const uint8_t *occ, int o) {
  const BoseMove bm = bose_decode(m, o);
  Mv mv;
  mv.a = bm.a; mv.b = bm.b; mv.da = bm.da; mv.db = bm.db;
  mv.v = bose_element<float>(m, occ, bm);
  // a move that leaves [0, n_max] has no element (and reads no W1 column),
  // whatever the couplings hold
  const int a1 = (int)occ[mv.a] + mv.da, b1 = (int)occ[mv.b] + mv.db;
  if (a1 < 0 || a1 > m.n_max || b1 < 0 || b1 > m.n_max) mv.v = 0.0f;
  return mv;
}

// W1 columns a move exchanges: (old a, new a, old b, new b); x < 0 for none
// (the current configuration), z < 0 for a single-site move.
__device__ __forceinline__ int4 move_cols(const Mv &mv, const uint8_t *occ, int np1) {
  const int ca0 = mv.a * np1 + occ[mv.a];
  int4 c = make_int4(ca0, ca0 + mv.da, -1, -1);
  if (mv.b != mv.a) {
    const int cb0 = mv.b * np1 + occ[mv.b];
    c.z = cb0;
    c.w = cb0 + mv.db;
  }
  return c;
}

__device__ __forceinline__ void bf8(const uint4 &u, float (&f)[8]) {
  const __nv_bfloat162 *p = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    f[2 * i] = __low2float(p[i]);
    f[2 * i + 1] = __high2float(p[i]);
  }
}

}  // namespace mlpdev
}  // namespace gfmc
