// Guide state of a whole population at once, for dense Jastrow couplings:
//   F[w, k] = sum_p Jd[p, k] x_p(w)       (x = +-1 spins or occupations)
// and, for spin-1/2, the signed ratio factors s_k = x_k exp(-2 x_k (F_k + h_k))
// the step kernel carries (JastrowSpinHalf; jastrow_spin_half.py:290-353).
//
// The step kernel rebuilds this state per walker when it has none to carry
// (a fresh population, every refresh); with a dense coupling matrix that is
// N^2 multiply-adds per walker through L2.  Here the population's fields are
// one (walkers x N) x (N x N) product: a block takes 64 walkers and 128
// output sites, stages x (64 x 16) and J (16 x 128) chunks in shared memory,
// and each thread accumulates 4 walkers x 8 sites in registers, adding the
// sites p = 0 .. N-1 in order with one fused multiply-add each -- the order
// and rounding of the step kernel's own rebuild, so the carried state is
// bit-identical to it.  Rows are indexed like the configurations (the step
// reads them through the parent map).
#include "engine.cuh"

namespace gfmc {
namespace {

constexpr int FW = 64;    // walkers per block
constexpr int FS = 128;   // output sites per pass
constexpr int FK = 16;    // sites p per shared-memory chunk

template <typename T, int FAM>
__device__ __forceinline__ T x_of(const void *cfg, int NW, int CB, int w, int p) {
  if (FAM == SPIN_HALF) {
    const uint64_t *b = reinterpret_cast<const uint64_t *>(cfg) + (size_t)w * NW;
    return ((b[p >> 6] >> (p & 63)) & 1ull) ? T(1) : T(-1);
  }
  return T(reinterpret_cast<const uint8_t *>(cfg)[(size_t)w * CB + p]);
}

template <typename T, int FAM>
__global__ void __launch_bounds__(256) fields_kernel(DevModel<T> m, DevGuide<T> g, int n,
                                                     const void *cfg, T *out) {
  __shared__ T Xs[FK][FW];
  __shared__ T Js[FK][FS];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int N = m.N, NW = (N + 63) / 64, CB = ((N + 15) / 16) * 16;
  const int w0 = blockIdx.x * FW;
  for (int s0 = 0; s0 < N; s0 += FS) {
    T acc[4][8];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) acc[a][b] = T(0);
    for (int p0 = 0; p0 < N; p0 += FK) {
      for (int i = tid; i < FK * FW; i += 256) {
        const int kk = i / FW, ww = i % FW, p = p0 + kk, w = w0 + ww;
        Xs[kk][ww] = (p < N && w < n) ? x_of<T, FAM>(cfg, NW, CB, w, p) : T(0);
      }
      for (int i = tid; i < FK * FS; i += 256) {
        const int kk = i / FS, ss = i % FS, p = p0 + kk, k = s0 + ss;
        Js[kk][ss] = (p < N && k < N) ? g.Jd[(size_t)p * N + k] : T(0);
      }
      __syncthreads();
      const int kmax = N - p0 < FK ? N - p0 : FK;
      for (int kk = 0; kk < kmax; ++kk) {
        T xv[4], jv[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) xv[a] = Xs[kk][4 * ty + a];
#pragma unroll
        for (int b = 0; b < 8; ++b) jv[b] = Js[kk][tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = fma(jv[b], xv[a], acc[a][b]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int w = w0 + 4 * ty + a;
      if (w >= n) continue;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int k = s0 + tx + 16 * b;
        if (k >= N) continue;
        T v = acc[a][b];
        if (FAM == SPIN_HALF) {
          const T x = x_of<T, FAM>(cfg, NW, CB, w, k);
          v = x * math_exp(T(-2) * x * (g.has_h ? v + g.h[k] : v));
        }
        out[(size_t)w * N + k] = v;
      }
    }
  }
}

}  // namespace

template <typename T>
cudaError_t launch_fields(const DevModel<T> &m, const DevGuide<T> &g, int n, const void *cfg,
                          T *out, cudaStream_t s) {
  if (!g.dense || !g.Jd || g.kind == GUIDE_NONE) return cudaErrorInvalidValue;
  const int blocks = (n + FW - 1) / FW;
  if (m.family == SPIN_HALF)
    fields_kernel<T, SPIN_HALF><<<blocks, 256, 0, s>>>(m, g, n, cfg, out);
  else
    fields_kernel<T, BOSE_HUBBARD><<<blocks, 256, 0, s>>>(m, g, n, cfg, out);
  return cudaGetLastError();
}

template cudaError_t launch_fields<double>(const DevModel<double> &, const DevGuide<double> &, int,
                                           const void *, double *, cudaStream_t);
template cudaError_t launch_fields<float>(const DevModel<float> &, const DevGuide<float> &, int,
                                          const void *, float *, cudaStream_t);

}  // namespace gfmc
