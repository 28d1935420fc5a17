// Value bookkeeping of the off-diagonal forward walk (float64).
//
// engine/evolution.py forward_walk_operator:891-1101: the operator values of
// the shadow walkers follow every shadow reconfiguration (v = v[indices],
// :1061), the estimate after m shadow steps is mean(v) and the norm the sum
// of the shadow's log G_t (:1063, accumulated in order from 0).
//
// fw_remap: one thread per walker, v_out[i] = v_in[parents[i]]; when the
//   step is recorded, per-block sums of v_out (warp shuffles, then the
//   block's warps in a fixed order).
// fw_finish: one thread per window, the block sums in a fixed order divided
//   by N, and the sequential running sum of log G up to m.
#include "engine.cuh"
#include "fw.cuh"

namespace gfmc {
namespace {

constexpr int FT = 256;

__device__ __forceinline__ void block_sum_store(double v, double *dst) {
  __shared__ double sh[FT / 32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[wi] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < FT / 32; ++i) s += sh[i];
    *dst = s;
  }
}

__global__ void __launch_bounds__(FT) fw_remap_kernel(int n, const int *parents,
                                                      const double *v_in, double *v_out,
                                                      double *partial) {
  const int i = blockIdx.x * FT + threadIdx.x;
  double v = 0.0;
  if (i < n) {
    v = parents ? v_in[parents[i]] : v_in[i];
    if (v_out) v_out[i] = v;
  }
  if (partial) block_sum_store(v, partial + blockIdx.x);
}

__global__ void fw_finish_kernel(const double *partial, int nb, int n, const double *logG,
                                 FwRows rows, double *val_out, double *norm_out) {
  const int j = threadIdx.x;
  if (j >= rows.n_m) return;
  const int m = rows.m[j];
  const double *p = partial + (size_t)m * nb;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += p[b];
  double lg = 0.0;
  for (int t = 0; t < m; ++t) lg = lg + logG[t];
  val_out[j] = s / (double)n;
  norm_out[j] = lg;
}

}  // namespace

int fw_blocks(int n) { return (n + FT - 1) / FT; }

cudaError_t launch_fw_remap(int n, const int *parents, const double *v_in, double *v_out,
                            double *partial, cudaStream_t s) {
  fw_remap_kernel<<<fw_blocks(n), FT, 0, s>>>(n, parents, v_in, v_out, partial);
  return cudaGetLastError();
}

cudaError_t launch_fw_finish(const double *partial, int nb, int n, const double *logG,
                             const FwRows &rows, double *val_out, double *norm_out,
                             cudaStream_t s) {
  fw_finish_kernel<<<1, 32, 0, s>>>(partial, nb, n, logG, rows, val_out, norm_out);
  return cudaGetLastError();
}

}  // namespace gfmc
